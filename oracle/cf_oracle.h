/*
 * cf_oracle.h -- CPU oracle for the cuckoo filter batch path (test
 * infrastructure; never linked by the CUDA library).  See cf_oracle.c for the
 * reference lines each function restates.
 */
#ifndef CF_ORACLE_H
#define CF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { CFO_POLICY_BFS = 0, CFO_POLICY_DFS = 1 };
/* Alternate-bucket policy (reference include/bucket_policies.cuh). */
enum { CFO_ALT_XOR = 0, CFO_ALT_ADDSUB = 1, CFO_ALT_OFFSET = 2 };
enum { CFO_MODE_REFERENCE = 0, CFO_MODE_CONSERVING = 1 };
enum {
    CFO_STAT_PRIMARY = 0,
    CFO_STAT_SECONDARY = 1,
    CFO_STAT_EVICTED_INSERTS = 2,
    CFO_STAT_EVICTIONS = 3,
    CFO_STAT_FAILED = 4,
    CFO_STAT_COUNT = 5
};

typedef struct cfo_params {
    uint32_t key_bytes;     /* 4 or 8 */
    uint32_t bits;          /* 8, 16 or 32 */
    uint32_t bucket_size;   /* slots per bucket, power of two */
    uint32_t word_bytes;    /* 4 or 8 */
    uint32_t policy;        /* CFO_POLICY_* */
    uint32_t max_evictions;
    uint64_t num_buckets;   /* power of two for CFO_ALT_XOR; even for CFO_ALT_ADDSUB */
    uint32_t alt_policy;    /* CFO_ALT_* */
} cfo_params;

uint64_t cfo_xxhash64(const void* data, size_t len);
uint64_t cfo_num_buckets(uint64_t capacity, uint32_t bucket_size);
uint64_t cfo_num_buckets_policy(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy);
uint32_t cfo_alt_tag(const cfo_params* P, uint32_t tag);
uint64_t cfo_alt_bucket(const cfo_params* P, uint64_t bucket, uint32_t tag);
void cfo_candidates(const cfo_params* P, const void* keys, size_t n, uint64_t* i1, uint64_t* i2,
                    uint32_t* fp);

size_t cfo_insert_seq(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out,
                      int mode, uint64_t* stats);
size_t cfo_delete_seq(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out);
size_t cfo_count_occupied(const cfo_params* P, const uint8_t* table);
uint64_t cfo_probe_count(const cfo_params* P, const uint8_t* table, const void* keys, size_t n);

size_t cfo_insert_mt(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out,
                     int threads);
size_t cfo_contains_mt(const cfo_params* P, const uint8_t* table, const void* keys, size_t n, uint8_t* out,
                       int threads);
size_t cfo_delete_mt(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out,
                     int threads);

void cfo_splitmix64(uint64_t seed, uint64_t first, size_t n, uint64_t* out);

#ifdef __cplusplus
}
#endif

#endif
