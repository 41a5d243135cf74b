/*
 * cuckoo_b200.h -- C ABI of the B200 cuckoo filter (libcuckoo_b200.so).
 *
 * This is the drop-in boundary for the batch path of the reference's
 * header-only CuckooFilter<Config> (reference include/CuckooFilter.cuh).  Every
 * entry point takes plain pointers and sizes; device pointers are CUDA device
 * (or managed) memory on the device the filter was created on; `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * All functions return CF_OK (0) or a negative cf_status; on error a message is
 * available from cf_last_error() on the calling thread.  Nothing here exits the
 * process (the reference's CUDA_CALL prints and calls exit(), helpers.cuh:202-210).
 *
 * Table image: identical to the reference's (CuckooFilter.cuh:224-237): bucket b
 * is bucket_bytes = bucket_size*bits_per_tag/8 contiguous bytes at offset
 * b*bucket_bytes; slot s holds its tag at byte s*bits_per_tag/8 of the bucket,
 * 0 means empty.  num_buckets is a power of two under the XOR policy.
 */
#ifndef CUCKOO_B200_H
#define CUCKOO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CF_ABI_VERSION 1

typedef enum cf_status {
    CF_OK = 0,
    CF_ERR_INVALID = -1,     /* bad argument or configuration */
    CF_ERR_UNSUPPORTED = -2, /* configuration not compiled into this library */
    CF_ERR_CUDA = -3,        /* CUDA runtime error (see cf_last_error) */
    CF_ERR_NO_MEMORY = -4,   /* device or pinned allocation failed */
    CF_ERR_DEVICE = -5,      /* a device-side retry bound was hit; table is consistent */
    CF_ERR_NOT_LOADED = -6   /* no usable CUDA device */
} cf_status;

/* Eviction policy (reference enum class EvictionPolicy, CuckooFilter.cuh:19-22). */
typedef enum cf_eviction { CF_EVICT_BFS = 0, CF_EVICT_DFS = 1 } cf_eviction;

/* Alternate-bucket policy (reference bucket_policies.cuh): XorAltBucketPolicy
 * (:15-84; power-of-two bucket count), AddSubAltBucketPolicy (:95-177; even
 * bucket count, primary buckets in the first half, alternates in the second)
 * and OffsetAltBucketPolicy (:179-350; any bucket count, the tag's top bit is
 * a choice bit: 0 in the primary bucket, 1 in the alternate).  AddSub and
 * Offset are built for 16-bit tags in 16-slot buckets (the reference's
 * bucket_policy_benchmark.cu:16-17 geometry), on every execution path and in
 * filter sets. */
typedef enum cf_alt_policy { CF_ALT_XOR = 0, CF_ALT_ADDSUB = 1, CF_ALT_OFFSET = 2 } cf_alt_policy;

/*
 * Runtime form of CuckooConfig<T, bitsPerTag, maxEvictions, blockSize,
 * bucketSize, AltBucketPolicy, evictionPolicy, WordType>
 * (reference include/CuckooFilter.cuh:44-74).
 */
typedef struct cf_config {
    uint32_t key_bytes;       /* sizeof(T): 4 (uint32_t) or 8 (uint64_t) */
    uint32_t bits_per_tag;    /* bitsPerTag: 8, 16 or 32 */
    uint32_t bucket_size;     /* bucketSize: slots per bucket, power of two, 8..256 bytes per bucket */
    uint32_t word_bytes;      /* sizeof(WordType): 8, or 4 for the (8, 16), (16, 16) and (32, 8) tag/bucket geometries */
    uint32_t eviction_policy; /* cf_eviction */
    uint32_t max_evictions;   /* maxEvictions: 1..512 */
    uint32_t block_size;      /* blockSize: threads per block, multiple of 32, <= 512; 0 = tuned */
    uint32_t alt_policy;      /* cf_alt_policy */
} cf_config;

typedef struct cf_filter cf_filter;

/* Geometry of a created filter. */
typedef struct cf_info {
    uint64_t num_buckets;   /* getNumBuckets() (CuckooFilter.cuh:740) */
    uint64_t capacity;      /* capacity() = num_buckets * bucket_size (:732) */
    uint64_t size_in_bytes; /* sizeInBytes() = num_buckets * bucket_bytes (:748) */
    uint32_t bucket_bytes;
    int32_t device;
} cf_info;

/* Cumulative device counters since creation or cf_reset_stats(). */
typedef struct cf_stats {
    uint64_t occupied;        /* occupiedSlots() (:699-704) */
    uint64_t primary;         /* inserts stored in their primary bucket */
    uint64_t secondary;       /* inserts stored in their alternate bucket */
    uint64_t evicted_inserts; /* inserts that needed eviction */
    uint64_t evictions;       /* slot exchanges performed (the reference's evictionCount(), :714) */
    uint64_t failed;          /* inserts that failed (table unchanged for that key) */
    uint64_t lost;            /* stored tags dropped by crossing eviction walks (expected 0) */
    uint64_t removed;         /* successful deletes */
    uint64_t duplicates;      /* BFS copies left behind by racing walks (an extra entry; expected 0) */
} cf_stats;

/* Library ABI version (CF_ABI_VERSION). */
int cf_abi_version(void);

/* Kernels this library has launched since it was loaded (all filters, all
 * devices; a diagnostic counter). */
uint64_t cf_launch_count(void);

/* Message for the last failed call on this thread ("" if none). */
const char* cf_last_error(void);

/* Name of a status code. */
const char* cf_status_string(int status);

/* 1 if (key_bytes, bits_per_tag, bucket_size, word_bytes) is compiled in. */
int cf_config_supported(const cf_config* cfg);

/* Number of buckets the filter would use for `capacity` slots:
 * nextPowerOfTwo(ceil(capacity / bucket_size)) (XorAltBucketPolicy::calculateNumBuckets,
 * bucket_policies.cuh:80-83). */
uint64_t cf_num_buckets_for(uint64_t capacity, uint32_t bucket_size);

/* calculateNumBuckets of an alternate-bucket policy (cf_alt_policy): XOR as
 * cf_num_buckets_for; AddSub ceil(capacity / bucket_size) rounded up to even
 * (bucket_policies.cuh:166-176); Offset ceil(capacity / bucket_size) (:346-349). */
uint64_t cf_num_buckets_for_policy(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy);

/* explicit CuckooFilter(size_t capacity) (CuckooFilter.cuh:420-428): allocates
 * and zeroes the table on the current device. */
int cf_create(const cf_config* cfg, uint64_t capacity, cf_filter** out);

/* ~CuckooFilter() (CuckooFilter.cuh:435-447). NULL is accepted. */
int cf_destroy(cf_filter* f);

int cf_get_info(const cf_filter* f, cf_info* out);

/*
 * size_t insertMany(const T* d_keys, size_t n, cudaStream_t) (CuckooFilter.cuh:457-464).
 * Synchronous on `stream`; *occupied_out (optional) receives occupiedSlots()
 * after the batch.  d_out (optional, n bytes) receives 1 for each key stored,
 * 0 for each key whose insert failed (extension: the reference reports only the
 * count).  A failed insert leaves every previously stored tag in place.
 */
int cf_insert(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream,
              uint64_t* occupied_out);

/*
 * size_t insertManySorted(const T* d_keys, size_t n, cudaStream_t)
 * (CuckooFilter.cuh:475-508).  Same contract as cf_insert; keys are first
 * partitioned by primary bucket so that table writes are coalesced.
 */
int cf_insert_sorted(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream,
                     uint64_t* occupied_out);

/*
 * void containsMany(const T* d_keys, size_t n, bool* d_output, cudaStream_t)
 * (CuckooFilter.cuh:518-523).  d_out: n bytes, 1 = maybe present, 0 = absent.
 * Synchronous on `stream`.
 */
int cf_contains(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream);

/*
 * size_t deleteMany(const T* d_keys, size_t n, bool* d_output, cudaStream_t)
 * (CuckooFilter.cuh:536-548).  Removes one copy per key; d_out (optional)
 * receives 1 per removed key.  Synchronous; *occupied_out (optional) as above.
 */
int cf_delete(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream,
              uint64_t* occupied_out);

/* Asynchronous forms: enqueue on `stream` and return; counters stay on the
 * device (read them with cf_occupied / cf_get_stats, which synchronize). */
int cf_insert_async(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream);
int cf_contains_async(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream);
int cf_delete_async(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream);

/* void clear() (CuckooFilter.cuh:675-682): zero the table and the counters. */
int cf_clear(cf_filter* f, void* stream);

/* size_t occupiedSlots() (CuckooFilter.cuh:699-704). Synchronizes the device. */
int cf_occupied(cf_filter* f, uint64_t* out);

/* size_t countOccupiedSlots() (CuckooFilter.cuh:759-785): counts non-empty
 * slots of the table image (on the device). */
int cf_count_occupied_slots(cf_filter* f, uint64_t* out);

int cf_get_stats(cf_filter* f, cf_stats* out);
/* Zero all counters except `occupied` (resetEvictionCount(), CuckooFilter.cuh:723). */
int cf_reset_stats(cf_filter* f);

/* Device pointer to the table image and its size (the reference's d_buckets, :350).
 * The caller may write through the pointer at any time: from this call on, the
 * library no longer assumes that the table is empty after cf_clear (an insert
 * into a table it knows to be empty skips loading it). */
int cf_table(cf_filter* f, void** d_table, uint64_t* bytes);

/* Replace the table image with `bytes` bytes from `src` (device or host memory)
 * and recount the occupancy.  Synchronous. */
int cf_load_table(cf_filter* f, const void* src, uint64_t bytes, void* stream);

/* Tunables of a filter (cf_set_option / cf_get_option). */
typedef enum cf_option {
    /* Upper bound on the device workspace of the staged paths, in bytes.
     * 0 (default) = automatic: a batch gets a workspace for all of it (16
     * bytes per key, about 24 with per-key results, up to 2^31 keys per chunk) when
     * the device's free memory, less a reserve of 1/16 of the device, allows,
     * else the largest chunk that fits.  The reference allocates the sorted
     * insert's buffers inside every call (CuckooFilter.cuh:475-508); here the
     * workspace is kept for later calls and freed with the filter.  Larger
     * batches than the limit are processed in chunks that fit. */
    CF_OPT_WORKSPACE_LIMIT = 1,
    /* Batch size from which insertMany, containsMany and deleteMany stream
     * table segments through shared memory instead of probing at random
     * (insertManySorted always does).  0 = automatic: one key per bucket for
     * inserts, eight per bucket for lookups and deletes; UINT64_MAX = never. */
    CF_OPT_SEGMENTED_MIN_KEYS = 2,
    /* Read-only: bytes of workspace currently allocated. */
    CF_OPT_WORKSPACE_BYTES = 3,
    /* Inside a segment-staged batch: number of keys that missed their primary
     * bucket from which the alternate-bucket round is segment-staged too
     * (otherwise those keys are probed at random).  0 = automatic (table bytes
     * / 64 for inserts, eight keys per bucket for lookups and deletes). */
    CF_OPT_ROUND2_SEGMENTED_MIN_KEYS = 4,
    /* Batch size from which every operation is region-staged: the batch is
     * partitioned by ~16 MiB table region in one pass and applied region by
     * region, so probes hit L2.  0 = automatic, which never picks this path
     * (measured slower than the others on B200); UINT64_MAX = never. */
    CF_OPT_REGION_MIN_KEYS = 5,
    /* Force one execution path for every batch (cf_staging); CF_STAGING_AUTO
     * (default) picks by batch size as described above. */
    CF_OPT_STAGING = 6,
    /* Table bytes per region of the region-staged path: a power of two,
     * 0 = default (16 MiB).  The table is cut into at most 256 regions, so
     * tables above 4 GiB get larger regions. */
    CF_OPT_REGION_BYTES = 7,
    /* Read-only: number of regions of the region-staged path. */
    CF_OPT_REGION_COUNT = 8,
    /* Random-probe lookups: keys per thread (1, 2 or 4; 0 = default). */
    CF_OPT_LOOKUP_KPT = 9,
    /* Random-probe kernels (lookups, deletes, inserts): 0 = one tile of keys
     * per CTA, the grid sized by the batch (default: measured fastest on B200);
     * 1 = a persistent grid of one wave of CTAs striding over the batch. */
    CF_OPT_PERSISTENT = 10,
    /* 1 = record the eviction-chain-length histogram of inserts
     * (cf_get_chain_histogram); 0 = off (default; one atomic per evicting
     * insert when on). */
    CF_OPT_CHAIN_HISTOGRAM = 11,
    /* Segment-staged inserts of at least one key per bucket: tags the first
     * round (primary buckets) may leave in a bucket.  0 = automatic: 13 of
     * 16 slots (bucket_size minus 3/16 of it), the keys that miss their
     * primary and then their alternate bucket get a third round at the
     * primary bucket before eviction; bucket_size = no limit and no third
     * round (the reference's primary-first order: a key goes to its
     * alternate bucket only when its primary is full).  1..bucket_size. */
    CF_OPT_ROUND1_CAP = 12,
    /* Lanes per key of the random-probe lookups and deletes
     * (containsMany / deleteMany, CuckooFilter.cuh:1143-1183).  0 or 1
     * (default): one lane per key, which loads the whole bucket as one 16- or
     * 32-byte vector.  W in {2, 4, 8, 16, 32} with bucket_bytes / W equal to 4
     * or 8 and at most 64 slots per bucket (otherwise CF_ERR_INVALID): W
     * consecutive lanes share a key, each loading its 4- or 8-byte piece of
     * the bucket; a lookup votes by ballot, and a delete assembles the
     * bucket's slot mask by shuffles and clears the reference's slot with one
     * compare-and-swap on the piece that holds it.  Results are the same for
     * every width. */
    CF_OPT_PROBE_WIDTH = 13
} cf_option;

/* Eviction-chain-length histogram since creation, cf_clear or cf_reset_stats,
 * recorded while CF_OPT_CHAIN_HISTOGRAM is on: bins[0] = inserts that needed
 * eviction but found a free slot without moving a tag, bins[b] for b >= 1 =
 * stored inserts whose chain moved L tags with 2^(b-1) <= L < 2^b (the last
 * bin holds every L >= 256).  Failed inserts are counted in cf_stats.failed. */
#define CF_CHAIN_BINS 10
int cf_get_chain_histogram(cf_filter* f, uint64_t* bins);

/* Execution paths (CF_OPT_STAGING).  All give the same per-key results. */
typedef enum cf_staging {
    CF_STAGING_AUTO = 0,
    CF_STAGING_RANDOM = 1,  /* probe buckets at random, any batch size (insertManySorted: segment-staged) */
    CF_STAGING_SEGMENT = 2, /* sort by 64 KiB segment, stage segments in shared memory */
    CF_STAGING_REGION = 3   /* partition by ~16 MiB region, apply in region order through L2 */
} cf_staging;

int cf_set_option(cf_filter* f, int option, uint64_t value);
int cf_get_option(cf_filter* f, int option, uint64_t* value);

/* Copy the table image to `dst` (device or host memory, `bytes` == table size). Synchronous. */
int cf_store_table(cf_filter* f, void* dst, uint64_t bytes, void* stream);

/* static getCandidateBuckets(key, numBuckets) (CuckooFilter.cuh:366-369 ->
 * the policy's getCandidateBuckets, bucket_policies.cuh:46-61, :125-140,
 * :232-256) for n HOST keys: the kernels' hashing evaluated on the CPU.  fp is
 * the tag as stored in the primary bucket i1.  Any of i1/i2/fp may be NULL. */
int cf_hash_candidates(const cf_config* cfg, uint64_t num_buckets, const void* h_keys, uint64_t n, uint64_t* i1,
                       uint64_t* i2, uint32_t* fp);

/* static hash64(key) (CuckooFilter.cuh:362-364 -> xxhash::xxhash64, hashutil.cuh:71-161,
 * seed 0) of n HOST values of value_bytes = 1, 2, 4 or 8 bytes each. */
int cf_hash64(uint32_t value_bytes, const void* h_values, uint64_t n, uint64_t* out);

/* static getAlternateBucket(bucket, fp, numBuckets) (CuckooFilter.cuh:378-381 ->
 * the policy's getAlternateBucket, bucket_policies.cuh:72-74, :150-160, :300-323)
 * for n HOST (bucket, tag) pairs of cfg's alternate-bucket policy.  XOR:
 * out[i] = buckets[i] ^ (xxHash64(tag as TagType) & (num_buckets - 1)).  Under
 * the Offset policy the tag is stored in the alternate bucket with its choice
 * bit (1 << (bits_per_tag - 1)) flipped. */
int cf_alt_buckets(const cf_config* cfg, uint64_t num_buckets, const uint64_t* buckets, const uint32_t* tags,
                   uint64_t n, uint64_t* out);

/*
 * insertManySorted for callers that cannot allocate device memory.  No
 * counterpart in the reference (whose insertManySorted calls cudaMalloc and
 * cudaFree inside every call, CuckooFilter.cuh:475-508).
 *
 * cf_insert_sorted grows a workspace with cudaMalloc and may free it again.
 * A process that serves many streams cannot let a call do that (cudaMalloc
 * and cudaFree can synchronize the whole device and stall every other
 * stream), and a host whose device memory is reserved by another allocator
 * has none to give.  This entry point runs the same segment-staged insert on
 * a fixed scratch area built into the library (cf_noalloc_scratch_bytes(),
 * about 27 MiB), which every GPU that loads the library's device code holds
 * until the process exits.  It calls no cudaMalloc, cudaFree or allocating
 * routine; each call looks up the scratch's device address on the filter's
 * device with cudaGetSymbolAddress, which allocates nothing.
 *
 * Limits: at most CF_NOALLOC_MAX_KEYS keys per call (larger n returns
 * CF_ERR_INVALID; split the batch), tables of at most 2^18 segments of 64 KiB
 * (16 GiB; else CF_ERR_UNSUPPORTED).  All calls share the one scratch area
 * and each call leaves its contents behind (every call rewrites what it
 * reads before reading it): calls that overlap on the GPU (other streams,
 * other threads, other filters) race and must be serialized by the caller.
 * Contract otherwise as cf_insert_sorted: d_out and occupied_out optional,
 * and the call synchronizes `stream` before it returns.
 */
#define CF_NOALLOC_MAX_KEYS (1u << 20)
int cf_insert_sorted_noalloc(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream,
                             uint64_t* occupied_out);

/* Bytes of the fixed scratch area used by cf_insert_sorted_noalloc. */
uint64_t cf_noalloc_scratch_bytes(void);

/* Lookups of this batch whose tag is in the primary bucket (one probe); the
 * rest take two probes.  Diagnostic for sector accounting. */
int cf_probe_count(cf_filter* f, const void* d_keys, uint64_t n, uint64_t* primary_hits, void* stream);

/*
 * ------------------------------------------------------------- filter sets
 *
 * Batched form over many filters (an extension; the reference runs one filter
 * per object and one launch per batch, CuckooFilter.cuh:457-548).  A set holds
 * n_filters independent filters of one configuration (64-bit keys; 8/16, 16/16
 * or 32/8 bits per tag / bucket size with the XOR policy, 16/16 with AddSub or
 * Offset), each with its own capacity and its own
 * counters, tables in one device pool.  A batched call takes a device work
 * list: item j covers keys [d_offsets[j], d_offsets[j+1]) of the concatenated
 * key buffer and targets filter d_filters[j]; d_offsets has n_items + 1
 * monotonic entries with d_offsets[n_items] = n, and d_out (when given) is
 * aligned with the keys.  All items run in ONE persistent kernel.  The
 * *_async calls only launch (no allocation, no synchronization), so they can
 * be captured into a CUDA graph and replayed; cf_set_sync synchronizes and
 * reports device-side errors (an item naming a filter outside the set: its
 * keys are skipped, CF_ERR_INVALID).
 */
typedef struct cf_set cf_set;

typedef enum cf_set_op { CF_SET_OP_INSERT = 0, CF_SET_OP_CONTAINS = 1, CF_SET_OP_DELETE = 2 } cf_set_op;

int cf_set_create(const cf_config* cfg, uint32_t n_filters, const uint64_t* capacities, cf_set** out);
int cf_set_destroy(cf_set* s);
/* Number of filters and bytes of the table pool. */
int cf_set_size(const cf_set* s, uint32_t* n_filters, uint64_t* pool_bytes);
int cf_set_get_info(const cf_set* s, uint32_t i, cf_info* out);
/* Device pointer and size of filter i's table image (layout as cf_table). */
int cf_set_table(cf_set* s, uint32_t i, void** d_table, uint64_t* bytes);

/* insertMany / containsMany / deleteMany of every item, one launch each. */
int cf_set_insert_async(cf_set* s, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                        const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream);
int cf_set_contains_async(cf_set* s, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                          const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream);
int cf_set_delete_async(cf_set* s, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                        const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream);
int cf_set_sync(cf_set* s, void* stream);

/* Zero every table and counter (synchronous). */
int cf_set_clear(cf_set* s, void* stream);
/* occupiedSlots() of every filter into out[n_filters]. */
int cf_set_occupied(cf_set* s, uint64_t* out);
int cf_set_get_stats(cf_set* s, uint32_t i, cf_stats* out);

/* Launch shape of an operation: threads per block (multiple of 32, <= 512),
 * keys per thread (1, 2, 4, 8) and, for lookups, the probe width (1 = one
 * thread per key; 4 or 8 lanes per key, each loading a 4- or 8-byte piece of
 * the bucket, where the bucket splits that way). */
int cf_set_set_launch(cf_set* s, int op, uint32_t block, uint32_t kpt, uint32_t width);
int cf_set_get_launch(const cf_set* s, int op, uint32_t* block, uint32_t* kpt, uint32_t* width);

/* Autotuner: times every launch shape (blocks {128, 256, 512} x keys per
 * thread {1, 2, 4, 8} x probe widths {1, 4, 8} for lookups) on the given batch
 * and keeps the fastest for `op`.  Lookups leave the set unchanged; tuning
 * inserts or deletes clears the set (each trial starts from an empty set) and
 * leaves it empty.  *best_ms (optional) receives the best trial's time. */
int cf_set_autotune(cf_set* s, int op, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                    const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream, float* best_ms);

/* ------------------------------------------------------------ key sharding
 *
 * The exchange step of the hash-partitioned multi-GPU form (replaces the
 * reference's Partitioner and gossip multisplit, CuckooFilterMultiGPU.cuh:44-50
 * and :226-234, and the placement of results, :292-312).  Key k belongs to
 * shard hash64(k) % num_shards, hash64 being the filter's own 64-bit xxHash of
 * the key (4- or 8-byte keys).
 *
 * Routing CF_SHARD_REFERENCE is the reference's: hash64(k) % num_shards.  With
 * the XOR policy and a power-of-two shard count it ties the shard to the low
 * bits of the primary bucket (both come from the low bits of hash64(k)), so a
 * shard's keys use only 1/num_shards of its buckets as primary buckets (more
 * evictions, and failed inserts near full load).  CF_SHARD_REMIXED routes by
 * remix64(hash64(k)) % num_shards instead, remix64 being splitmix64's
 * bijective output mixer, which keeps shard and buckets independent.
 *
 * cf_shard_partition groups a device batch of n keys by shard: d_out_keys
 * holds shard 0's keys, then shard 1's, and so on; d_out_pos[i] is the batch
 * position of d_out_keys[i]; d_counts (num_shards uint64 values, device
 * memory) receives the keys per shard.  The order inside a shard's group is
 * unspecified.  n < 2^32; num_shards 1..256; d_workspace is device memory of
 * at least cf_shard_workspace_bytes(n, num_shards) bytes.
 *
 * cf_shard_unpartition writes d_out[d_pos[i]] = d_grouped[i] for i < n: per-key
 * results that come back in group order land at their batch positions.  It
 * reads the run starts that cf_shard_partition of the same batch (same n and
 * num_shards) left in d_workspace, so the workspace must be untouched in
 * between; otherwise the results are undefined (no access leaves the arrays).
 *
 * Both calls only launch on `stream` (no allocation, no synchronization). */
typedef enum cf_shard_routing { CF_SHARD_REFERENCE = 0, CF_SHARD_REMIXED = 1 } cf_shard_routing;

uint64_t cf_shard_workspace_bytes(uint64_t n, uint32_t num_shards);
int cf_shard_partition(const void* d_keys, uint64_t n, uint32_t key_bytes, uint32_t num_shards, uint32_t routing,
                       void* d_out_keys, uint32_t* d_out_pos, uint64_t* d_counts, void* d_workspace,
                       uint64_t workspace_bytes, void* stream);
int cf_shard_unpartition(const uint8_t* d_grouped, const uint32_t* d_pos, uint64_t n, uint32_t num_shards,
                         const void* d_workspace, uint64_t workspace_bytes, uint8_t* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUCKOO_B200_H */
