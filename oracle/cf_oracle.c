/*
 * cf_oracle.c -- CPU restatement of the reference cuckoo filter's batch path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the CPU
 * baseline ("port").  Only the test suite, the smoke check and the benchmark's
 * CPU-baseline / reference legs load it.  The product path (the CUDA library)
 * never links or calls it.
 *
 * What it restates (all paths relative to the reference project root):
 *   - xxHash64 with seed 0 over the raw bytes of a 1/2/4/8-byte value:
 *       include/hashutil.cuh:44-48 (primes), :61-68 (finalize), :71-161 (xxhash64).
 *     Inputs here are always shorter than 32 bytes, so only the short-input
 *     branch (:127-158) is reachable; the 32-byte stripe loop is not restated.
 *   - XorAltBucketPolicy: include/bucket_policies.cuh:46-61 (candidates),
 *     :72-74 (alternate bucket), :80-83 (bucket count) + include/helpers.cuh:31-45.
 *   - AddSubAltBucketPolicy :95-177 (two halves; the alternate of a bucket in
 *     the first half is (b + h(tag) mod half) mod half + half, of one in the
 *     second (b - h(tag) mod half) mod half; an even bucket count) and
 *     OffsetAltBucketPolicy :179-350 (the tag's top bit is a choice bit: 0 in
 *     the primary bucket, 1 in the alternate; the alternate is b + off or
 *     b - off mod nB with off = h(tag without the choice bit) mod nB, never 0;
 *     moving a tag flips its choice bit), as the filter uses them at
 *     CuckooFilter.cuh:1033-1059 (insert), :1091-1094 (contains),
 *     :1109-1112 (remove) and :945, :988 (evictions).
 *   - Bucket layout: include/CuckooFilter.cuh:224-237 (slot s of bucket b lives at
 *     byte b*bucketBytes + s*(bits/8), little-endian packed words).
 *   - tryInsertAtBucket :859-904, tryRemoveAtBucket :805-848,
 *     insertWithEvictionDFS :917-954, insertWithEvictionBFS :967-1018,
 *     insert :1029-1080, contains :1088-1098, remove :1106-1116.
 *
 * Two insert failure modes are provided:
 *   CFO_MODE_REFERENCE  - exactly the reference: a DFS chain that runs out of
 *                         evictions drops the tag it is holding (:953).
 *   CFO_MODE_CONSERVING - the CUDA library's semantics: a failed DFS chain is
 *                         undone step by step, so the table is left exactly as
 *                         before the failed insert and no stored tag is lost.
 * Both modes make identical choices up to the first failed chain.
 *
 * Word-granular scanning: the reference scans a bucket word by word starting at
 * word (tag & (bs-1)) / tagsPerWord and takes the lowest matching lane of a
 * word.  That is the same as scanning slots circularly from
 * align_down(tag & (bs-1), tagsPerWord), which is how it is written here, so
 * the same code serves 64-bit and 32-bit words.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "cf_oracle.h"

/* ---------------------------------------------------------------- xxHash64 */

static const uint64_t XP1 = 11400714785074694791ULL;
static const uint64_t XP2 = 14029467366897019727ULL;
static const uint64_t XP3 = 1609587929392839161ULL;
static const uint64_t XP4 = 9650029242287828579ULL;
static const uint64_t XP5 = 2870177450012600261ULL;

static inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

static inline uint64_t xxh_avalanche(uint64_t h) {
    h ^= h >> 33;
    h *= XP2;
    h ^= h >> 29;
    h *= XP3;
    h ^= h >> 32;
    return h;
}

/* XXH64(seed = 0) of len < 32 little-endian bytes. */
uint64_t cfo_xxhash64(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    uint64_t h = XP5 + (uint64_t)len;
    size_t off = 0;
    while (len - off >= 8) {
        uint64_t k;
        memcpy(&k, p + off, 8);
        k *= XP2;
        k = rotl64(k, 31) * XP1;
        h ^= k;
        h = rotl64(h, 27) * XP1 + XP4;
        off += 8;
    }
    if (len - off >= 4) {
        uint32_t k;
        memcpy(&k, p + off, 4);
        h ^= (uint64_t)k * XP1;
        h = rotl64(h, 23) * XP2 + XP3;
        off += 4;
    }
    while (off < len) {
        h ^= (uint64_t)p[off] * XP5;
        h = rotl64(h, 11) * XP1;
        ++off;
    }
    return xxh_avalanche(h);
}

/* ------------------------------------------------------------ bucket policy */

uint64_t cfo_num_buckets(uint64_t capacity, uint32_t bucket_size) {
    /* std::ceil((double)capacity / bucketSize), then nextPowerOfTwo. */
    double req = (double)capacity / (double)bucket_size;
    uint64_t r = (uint64_t)req;
    if ((double)r < req) r += 1;
    if (r != 0 && (r & (r - 1)) == 0) return r;
    uint64_t n = r - 1;
    n |= n >> 1;
    n |= n >> 2;
    n |= n >> 4;
    n |= n >> 8;
    n |= n >> 16;
    n |= n >> 32;
    return n + 1;
}

static inline uint64_t tag_hash(uint32_t tag, uint32_t bits) {
    uint8_t b[4];
    memcpy(b, &tag, 4);
    return cfo_xxhash64(b, bits / 8);
}

uint64_t cfo_num_buckets_policy(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy) {
    if (alt_policy == CFO_ALT_XOR) return cfo_num_buckets(capacity, bucket_size);
    double req = (double)capacity / (double)bucket_size;
    uint64_t r = (uint64_t)req;
    if ((double)r < req) r += 1;
    if (alt_policy == CFO_ALT_ADDSUB && (r % 2) != 0) r += 1;
    return r;
}

static inline uint32_t choice_bit(const cfo_params* P) { return 1u << (P->bits - 1); }

/* Non-zero offset of a tag without its choice bit (computeOffset, :245-249). */
static inline uint64_t tag_offset(const cfo_params* P, uint32_t pure) {
    const uint64_t off = tag_hash(pure, P->bits) % P->num_buckets;
    return off == 0 ? 1 : off;
}

static inline uint64_t alt_bucket(const cfo_params* P, uint64_t b, uint32_t tag) {
    const uint64_t nb = P->num_buckets;
    switch (P->alt_policy) {
        case CFO_ALT_ADDSUB: {
            const uint64_t half = nb / 2;
            const uint64_t fh = tag_hash(tag, P->bits) % half;
            return b < half ? ((b + fh) % half) + half : (b - fh) % half;
        }
        case CFO_ALT_OFFSET: {
            const uint32_t pure = tag & (choice_bit(P) - 1);
            const uint64_t off = tag_offset(P, pure);
            return (tag & choice_bit(P)) == 0 ? (b + off) % nb : (b + nb - off) % nb;
        }
        default:
            return b ^ (tag_hash(tag, P->bits) & (nb - 1));
    }
}

/* The tag as stored after it moves to its alternate bucket
 * (getAlternateBucketWithNewFp, CuckooFilter.cuh:394-401): the Offset
 * policy flips the choice bit, the others keep the tag. */
static inline uint32_t alt_tag(const cfo_params* P, uint32_t tag) {
    return P->alt_policy == CFO_ALT_OFFSET ? (tag ^ choice_bit(P)) : tag;
}

uint32_t cfo_alt_tag(const cfo_params* P, uint32_t tag) { return alt_tag(P, tag); }

static inline uint64_t key_at(const cfo_params* P, const void* keys, size_t i) {
    if (P->key_bytes == 8) return ((const uint64_t*)keys)[i];
    return ((const uint32_t*)keys)[i];
}

static inline void candidates(const cfo_params* P, uint64_t key, uint64_t* i1, uint64_t* i2,
                              uint32_t* fp) {
    uint8_t kb[8];
    memcpy(kb, &key, 8);
    const uint64_t h = cfo_xxhash64(kb, P->key_bytes);
    uint32_t mask = P->bits == 32 ? 0xFFFFFFFFu : ((1u << P->bits) - 1u);
    if (P->alt_policy == CFO_ALT_OFFSET) mask = choice_bit(P) - 1; /* choice bit 0 */
    uint32_t f = (uint32_t)(h >> 32) & mask;
    if (f == 0) f = 1;
    const uint32_t hb = (uint32_t)(h & 0xFFFFFFFFu);
    switch (P->alt_policy) {
        case CFO_ALT_ADDSUB: *i1 = (uint64_t)hb % (P->num_buckets / 2); break;
        case CFO_ALT_OFFSET: *i1 = (uint64_t)hb % P->num_buckets; break;
        default: *i1 = (uint64_t)hb & (P->num_buckets - 1); break;
    }
    *i2 = alt_bucket(P, *i1, f);
    *fp = f;
}

void cfo_candidates(const cfo_params* P, const void* keys, size_t n, uint64_t* i1, uint64_t* i2,
                    uint32_t* fp) {
    for (size_t i = 0; i < n; ++i) {
        uint64_t a, b;
        uint32_t f;
        candidates(P, key_at(P, keys, i), &a, &b, &f);
        if (i1) i1[i] = a;
        if (i2) i2[i] = b;
        if (fp) fp[i] = f;
    }
}

uint64_t cfo_alt_bucket(const cfo_params* P, uint64_t bucket, uint32_t tag) {
    return alt_bucket(P, bucket, tag);
}

/* -------------------------------------------------------------- table access */

static inline size_t bucket_bytes(const cfo_params* P) { return (size_t)P->bucket_size * P->bits / 8; }
static inline uint32_t tags_per_word(const cfo_params* P) { return P->word_bytes * 8 / P->bits; }

static inline uint32_t get_slot(const cfo_params* P, const uint8_t* t, uint64_t b, uint32_t s) {
    const uint8_t* q = t + b * bucket_bytes(P) + (size_t)s * (P->bits / 8);
    switch (P->bits) {
        case 8: return q[0];
        case 16: { uint16_t v; memcpy(&v, q, 2); return v; }
        default: { uint32_t v; memcpy(&v, q, 4); return v; }
    }
}

static inline void set_slot(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t s, uint32_t v) {
    uint8_t* q = t + b * bucket_bytes(P) + (size_t)s * (P->bits / 8);
    switch (P->bits) {
        case 8: q[0] = (uint8_t)v; break;
        case 16: { uint16_t w = (uint16_t)v; memcpy(q, &w, 2); break; }
        default: memcpy(q, &v, 4); break;
    }
}

static inline uint32_t scan_start(const cfo_params* P, uint32_t tag) {
    const uint32_t tpw = tags_per_word(P);
    return ((tag & (P->bucket_size - 1)) / tpw) * tpw;
}

static int bucket_has(const cfo_params* P, const uint8_t* t, uint64_t b, uint32_t tag) {
    for (uint32_t s = 0; s < P->bucket_size; ++s)
        if (get_slot(P, t, b, s) == tag) return 1;
    return 0;
}

/* tryInsertAtBucket (CuckooFilter.cuh:859-904), sequential. */
static int try_insert(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t tag) {
    const uint32_t s0 = scan_start(P, tag);
    for (uint32_t i = 0; i < P->bucket_size; ++i) {
        const uint32_t s = (s0 + i) & (P->bucket_size - 1);
        if (get_slot(P, t, b, s) == 0) {
            set_slot(P, t, b, s, tag);
            return 1;
        }
    }
    return 0;
}

/* tryRemoveAtBucket (CuckooFilter.cuh:805-848), sequential. */
static int try_remove(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t tag) {
    const uint32_t s0 = scan_start(P, tag);
    for (uint32_t i = 0; i < P->bucket_size; ++i) {
        const uint32_t s = (s0 + i) & (P->bucket_size - 1);
        if (get_slot(P, t, b, s) == tag) {
            set_slot(P, t, b, s, 0);
            return 1;
        }
    }
    return 0;
}

/* insertWithEvictionDFS (CuckooFilter.cuh:917-954).  In conserving mode a
 * failed chain is undone in reverse order. */
static int evict_dfs(const cfo_params* P, uint8_t* t, uint32_t fp, uint64_t start, int mode,
                     uint64_t* n_evictions) {
    uint32_t cur = fp;
    uint64_t cb = start;
    const uint32_t maxe = P->max_evictions;
    uint8_t* path = (uint8_t*)malloc(maxe ? maxe : 1);
    for (uint32_t e = 0; e < maxe; ++e) {
        const uint32_t slot = (uint32_t)(((uint64_t)cur + (uint64_t)e * 7u) & (P->bucket_size - 1));
        path[e] = (uint8_t)slot;
        const uint32_t victim = get_slot(P, t, cb, slot);
        set_slot(P, t, cb, slot, cur);
        if (n_evictions) ++*n_evictions;
        cb = alt_bucket(P, cb, victim);
        cur = alt_tag(P, victim);
        if (try_insert(P, t, cb, cur)) {
            free(path);
            return 1;
        }
    }
    if (mode == CFO_MODE_CONSERVING) {
        /* Walk back: the held tag returns to the bucket it came from, which
         * is alt(cb, held) because the alternate map is an involution (with
         * the tag in that bucket's form). */
        for (uint32_t e = maxe; e-- > 0;) {
            cb = alt_bucket(P, cb, cur);
            const uint32_t back = get_slot(P, t, cb, path[e]);
            set_slot(P, t, cb, path[e], alt_tag(P, cur));
            cur = back;
        }
        /* cur is now fp again and cb == start; fp is discarded. */
    }
    free(path);
    return 0;
}

/* insertWithEvictionBFS (CuckooFilter.cuh:967-1018), sequential. */
static int evict_bfs(const cfo_params* P, uint8_t* t, uint32_t fp, uint64_t start, int mode,
                     uint64_t* n_evictions) {
    const uint32_t half = P->bucket_size / 2;
    const uint32_t nc = half < 8 ? half : 8;
    for (uint32_t i = 0; i < nc; ++i) {
        const uint32_t slot = (uint32_t)(((uint64_t)fp + (uint64_t)i * 7u) & (P->bucket_size - 1));
        const uint32_t cand = get_slot(P, t, start, slot);
        if (cand == 0) {
            if (try_insert(P, t, start, fp)) return 1;
            continue;
        }
        const uint64_t alt = alt_bucket(P, start, cand);
        if (try_insert(P, t, alt, alt_tag(P, cand))) {
            if (get_slot(P, t, start, slot) == cand) {
                set_slot(P, t, start, slot, fp);
                if (n_evictions) ++*n_evictions;
                return 1;
            }
            try_remove(P, t, alt, alt_tag(P, cand));
        }
    }
    return evict_dfs(P, t, fp, start, mode, n_evictions);
}

/* CuckooFilter::insert (CuckooFilter.cuh:1029-1080): the tag goes to its
 * primary bucket, else (in its alternate form) to its alternate, else eviction
 * starts at i1 for an even tag and i2 for an odd one. */
static int insert_one(const cfo_params* P, uint8_t* t, uint64_t key, int mode, uint64_t* stats) {
    uint64_t i1, i2;
    uint32_t fp;
    candidates(P, key, &i1, &i2, &fp);
    const uint32_t fp2 = alt_tag(P, fp);
    if (try_insert(P, t, i1, fp)) {
        if (stats) stats[CFO_STAT_PRIMARY]++;
        return 1;
    }
    if (try_insert(P, t, i2, fp2)) {
        if (stats) stats[CFO_STAT_SECONDARY]++;
        return 1;
    }
    const uint64_t start = (fp & 1) == 0 ? i1 : i2;
    const uint32_t sfp = (fp & 1) == 0 ? fp : fp2;
    uint64_t ev = 0;
    int ok = P->policy == CFO_POLICY_BFS ? evict_bfs(P, t, sfp, start, mode, &ev)
                                         : evict_dfs(P, t, sfp, start, mode, &ev);
    if (stats) {
        stats[CFO_STAT_EVICTED_INSERTS]++;
        stats[CFO_STAT_EVICTIONS] += ev;
        if (!ok) stats[CFO_STAT_FAILED]++;
    }
    return ok;
}

size_t cfo_insert_seq(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out,
                      int mode, uint64_t* stats) {
    size_t ok = 0;
    for (size_t i = 0; i < n; ++i) {
        int r = insert_one(P, table, key_at(P, keys, i), mode, stats);
        if (out) out[i] = (uint8_t)r;
        ok += (size_t)r;
    }
    return ok;
}

size_t cfo_delete_seq(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out) {
    size_t ok = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t i1, i2;
        uint32_t fp;
        candidates(P, key_at(P, keys, i), &i1, &i2, &fp);
        int r = try_remove(P, table, i1, fp) || try_remove(P, table, i2, alt_tag(P, fp));
        if (out) out[i] = (uint8_t)r;
        ok += (size_t)r;
    }
    return ok;
}

size_t cfo_count_occupied(const cfo_params* P, const uint8_t* table) {
    size_t c = 0;
    for (uint64_t b = 0; b < P->num_buckets; ++b)
        for (uint32_t s = 0; s < P->bucket_size; ++s) c += get_slot(P, table, b, s) != 0;
    return c;
}

/* Number of bucket probes a lookup makes with the reference's short-circuit
 * order (CuckooFilter.cuh:1096): 1 if the tag is in the primary bucket, else 2. */
uint64_t cfo_probe_count(const cfo_params* P, const uint8_t* table, const void* keys, size_t n) {
    uint64_t total = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t i1, i2;
        uint32_t fp;
        candidates(P, key_at(P, keys, i), &i1, &i2, &fp);
        (void)i2;
        total += bucket_has(P, table, i1, fp) ? 1 : 2;
    }
    return total;
}

/* ----------------------------------------------------- multithreaded (port) */

/* The concurrent CPU port follows the same algorithm as the CUDA library:
 * per-word compare-and-swap, BFS copy-then-swap, DFS exchange walk with undo. */

static inline int lane_shift(const cfo_params* P, uint32_t s) {
    return (int)((s & (tags_per_word(P) - 1)) * P->bits);
}

static inline uint64_t* word_ptr64(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t s) {
    return (uint64_t*)(t + b * bucket_bytes(P) + (size_t)(s / tags_per_word(P)) * 8);
}
static inline uint32_t* word_ptr32(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t s) {
    return (uint32_t*)(t + b * bucket_bytes(P) + (size_t)(s / tags_per_word(P)) * 4);
}

static inline uint64_t load_word(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t s) {
    if (P->word_bytes == 8) return __atomic_load_n(word_ptr64(P, t, b, s), __ATOMIC_RELAXED);
    return __atomic_load_n(word_ptr32(P, t, b, s), __ATOMIC_RELAXED);
}

static inline int cas_word(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t s, uint64_t* expected,
                           uint64_t desired) {
    if (P->word_bytes == 8)
        return __atomic_compare_exchange_n(word_ptr64(P, t, b, s), expected, desired, 0, __ATOMIC_RELAXED,
                                           __ATOMIC_RELAXED);
    uint32_t e = (uint32_t)*expected;
    int r = __atomic_compare_exchange_n(word_ptr32(P, t, b, s), &e, (uint32_t)desired, 0, __ATOMIC_RELAXED,
                                        __ATOMIC_RELAXED);
    *expected = e;
    return r;
}

static inline uint64_t tag_mask64(const cfo_params* P) {
    return P->bits == 32 ? 0xFFFFFFFFull : ((1ull << P->bits) - 1ull);
}

static int mt_try_insert(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t tag) {
    const uint32_t tpw = tags_per_word(P), s0 = scan_start(P, tag);
    const uint64_t m = tag_mask64(P);
    for (uint32_t i = 0; i < P->bucket_size; i += tpw) {
        const uint32_t ws = (s0 + i) & (P->bucket_size - 1);
        uint64_t w = load_word(P, t, b, ws);
        for (;;) {
            int lane = -1;
            for (uint32_t j = 0; j < tpw; ++j)
                if (((w >> (j * P->bits)) & m) == 0) { lane = (int)j; break; }
            if (lane < 0) break;
            const uint64_t d = w | ((uint64_t)tag << (lane * P->bits));
            if (cas_word(P, t, b, ws, &w, d)) return 1;
        }
    }
    return 0;
}

static int mt_try_remove(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t tag) {
    const uint32_t tpw = tags_per_word(P), s0 = scan_start(P, tag);
    const uint64_t m = tag_mask64(P);
    for (uint32_t i = 0; i < P->bucket_size; i += tpw) {
        const uint32_t ws = (s0 + i) & (P->bucket_size - 1);
        uint64_t w = load_word(P, t, b, ws);
        for (;;) {
            int lane = -1;
            for (uint32_t j = 0; j < tpw; ++j)
                if (((w >> (j * P->bits)) & m) == tag) { lane = (int)j; break; }
            if (lane < 0) break;
            const uint64_t d = w & ~(m << (lane * P->bits));
            if (cas_word(P, t, b, ws, &w, d)) return 1;
        }
    }
    return 0;
}

/* Atomically replace slot s of bucket b with v; returns the previous tag. */
static uint32_t mt_exchange_slot(const cfo_params* P, uint8_t* t, uint64_t b, uint32_t s, uint32_t v) {
    const uint64_t m = tag_mask64(P);
    const int sh = lane_shift(P, s);
    uint64_t w = load_word(P, t, b, s);
    for (;;) {
        const uint64_t d = (w & ~(m << sh)) | ((uint64_t)v << sh);
        if (cas_word(P, t, b, s, &w, d)) return (uint32_t)((w >> sh) & m);
    }
}

static int mt_evict_dfs(const cfo_params* P, uint8_t* t, uint32_t fp, uint64_t start, uint8_t* path) {
    uint32_t cur = fp;
    uint64_t cb = start;
    for (uint32_t e = 0; e < P->max_evictions; ++e) {
        const uint32_t slot = (uint32_t)(((uint64_t)cur + (uint64_t)e * 7u) & (P->bucket_size - 1));
        path[e] = (uint8_t)slot;
        const uint32_t victim = mt_exchange_slot(P, t, cb, slot, cur);
        if (victim == 0) return 1;
        cb = alt_bucket(P, cb, victim);
        cur = alt_tag(P, victim);
        if (mt_try_insert(P, t, cb, cur)) return 1;
    }
    for (uint32_t e = P->max_evictions; e-- > 0;) {
        cb = alt_bucket(P, cb, cur);
        cur = mt_exchange_slot(P, t, cb, path[e], alt_tag(P, cur));
        /* A slot emptied concurrently absorbed the held tag: every tag,
         * including fp, is now stored. */
        if (cur == 0) return 1;
    }
    return 0;
}

static int mt_evict_bfs(const cfo_params* P, uint8_t* t, uint32_t fp, uint64_t start, uint8_t* path) {
    const uint32_t half = P->bucket_size / 2;
    const uint32_t nc = half < 8 ? half : 8;
    const uint64_t m = tag_mask64(P);
    for (uint32_t i = 0; i < nc; ++i) {
        const uint32_t slot = (uint32_t)(((uint64_t)fp + (uint64_t)i * 7u) & (P->bucket_size - 1));
        const int sh = lane_shift(P, slot);
        uint64_t w = load_word(P, t, start, slot);
        const uint32_t cand = (uint32_t)((w >> sh) & m);
        if (cand == 0) {
            if (mt_try_insert(P, t, start, fp)) return 1;
            continue;
        }
        const uint64_t alt = alt_bucket(P, start, cand);
        if (mt_try_insert(P, t, alt, alt_tag(P, cand))) {
            w = load_word(P, t, start, slot);
            if (((w >> sh) & m) == cand) {
                const uint64_t d = (w & ~(m << sh)) | ((uint64_t)fp << sh);
                if (cas_word(P, t, start, slot, &w, d)) return 1;
            }
            mt_try_remove(P, t, alt, alt_tag(P, cand));
        }
    }
    return mt_evict_dfs(P, t, fp, start, path);
}

typedef struct {
    const cfo_params* P;
    uint8_t* table;
    const void* keys;
    uint8_t* out;
    size_t lo, hi;
    int op;
    size_t ok;
} mt_job;

static void* mt_worker(void* arg) {
    mt_job* J = (mt_job*)arg;
    const cfo_params* P = J->P;
    uint8_t* path = J->op == 0 ? (uint8_t*)malloc(P->max_evictions ? P->max_evictions : 1) : NULL;
    size_t ok = 0;
    for (size_t i = J->lo; i < J->hi; ++i) {
        uint64_t i1, i2;
        uint32_t fp;
        candidates(P, key_at(P, J->keys, i), &i1, &i2, &fp);
        int r;
        const uint32_t fp2 = alt_tag(P, fp);
        if (J->op == 0) {
            r = mt_try_insert(P, J->table, i1, fp) || mt_try_insert(P, J->table, i2, fp2);
            if (!r) {
                const uint64_t start = (fp & 1) == 0 ? i1 : i2;
                const uint32_t sfp = (fp & 1) == 0 ? fp : fp2;
                r = P->policy == CFO_POLICY_BFS ? mt_evict_bfs(P, J->table, sfp, start, path)
                                                : mt_evict_dfs(P, J->table, sfp, start, path);
            }
        } else if (J->op == 1) {
            r = bucket_has(P, J->table, i1, fp) || bucket_has(P, J->table, i2, fp2);
        } else {
            r = mt_try_remove(P, J->table, i1, fp) || mt_try_remove(P, J->table, i2, fp2);
        }
        if (J->out) J->out[i] = (uint8_t)r;
        ok += (size_t)r;
    }
    free(path);
    J->ok = ok;
    return NULL;
}

static size_t run_mt(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out, int op,
                     int threads) {
    if (threads < 1) threads = 1;
    if ((size_t)threads > n) threads = n ? (int)n : 1;
    mt_job* jobs = (mt_job*)calloc((size_t)threads, sizeof(mt_job));
    pthread_t* tids = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int i = 0; i < threads; ++i) {
        jobs[i].P = P;
        jobs[i].table = table;
        jobs[i].keys = keys;
        jobs[i].out = out;
        jobs[i].lo = n * (size_t)i / (size_t)threads;
        jobs[i].hi = n * (size_t)(i + 1) / (size_t)threads;
        jobs[i].op = op;
        if (threads == 1)
            mt_worker(&jobs[i]);
        else
            pthread_create(&tids[i], NULL, mt_worker, &jobs[i]);
    }
    size_t ok = 0;
    for (int i = 0; i < threads; ++i) {
        if (threads > 1) pthread_join(tids[i], NULL);
        ok += jobs[i].ok;
    }
    free(jobs);
    free(tids);
    return ok;
}

size_t cfo_insert_mt(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out,
                     int threads) {
    return run_mt(P, table, keys, n, out, 0, threads);
}

size_t cfo_contains_mt(const cfo_params* P, const uint8_t* table, const void* keys, size_t n, uint8_t* out,
                       int threads) {
    return run_mt(P, (uint8_t*)table, keys, n, out, 1, threads);
}

size_t cfo_delete_mt(const cfo_params* P, uint8_t* table, const void* keys, size_t n, uint8_t* out,
                     int threads) {
    return run_mt(P, table, keys, n, out, 2, threads);
}

/* --------------------------------------------------------------- generators */

/* splitmix64 (Steele, Lea, Flood 2014): state += 0x9E3779B97F4A7C15, then the
 * published output mix.  Output i uses state seed + (i+1)*gamma.  The mix is a
 * bijection of the state, so one seed never repeats a value within 2^64
 * outputs. */
void cfo_splitmix64(uint64_t seed, uint64_t first, size_t n, uint64_t* out) {
    uint64_t s = seed + first * 0x9E3779B97F4A7C15ULL;
    for (size_t i = 0; i < n; ++i) {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        out[i] = z ^ (z >> 31);
    }
}
