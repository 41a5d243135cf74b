// cf_kernels.cuh -- batch kernels of the B200 cuckoo filter.
//
// One thread owns KPT consecutive keys of a tile; a persistent grid strides
// over tiles.  A thread issues the KPT primary-bucket loads back to back, then
// the KPT secondary-bucket loads for the keys that missed, so each thread keeps
// several independent 32-byte sector requests in flight (the reference keeps
// one key per thread, CuckooFilter.cuh:1119-1183).
//
// Semantics follow the reference's device code:
//   contains : tag in bucket i1 or i2                         (CuckooFilter.cuh:1088-1098)
//   remove   : clear the first matching slot of i1, else i2   (:805-848, :1106-1116)
//   insert   : first empty slot of i1, else i2, else evict    (:859-904, :1029-1080)
//   BFS      : copy a candidate to its alternate bucket, then swap fp in (:967-1018)
//   DFS      : exchange walk of at most maxEvictions steps    (:917-954)
// "First slot" means: scan CAS words circularly from word (tag & (bs-1)) / tagsPerWord,
// lowest lane of a word first.
//
// Differences from the reference, all deliberate:
//   * a DFS walk that runs out of evictions is undone step by step, so a failed
//     insert leaves every previously stored tag in place (the reference drops the
//     tag in hand, CuckooFilter.cuh:953, which makes an earlier key a false
//     negative);
//   * every compare-and-swap retry loop is bounded; hitting the bound sets an
//     error flag that the host turns into a status code;
//   * counters are accumulated per thread and flushed once per warp.
#pragma once

#include <cstdint>

#include "cf_device.cuh"

namespace cfb {

// Hard cap on maxEvictions: the DFS undo log lives in a per-thread local array.
constexpr uint32_t kMaxEvictionsCap = 512;
// Bound on compare-and-swap retries of one bucket operation.
constexpr int kCasRetryLimit = 1 << 16;

// Device counter slots (64-bit each).
enum Counter : int {
    CTR_OCCUPIED = 0,
    CTR_PRIMARY = 1,
    CTR_SECONDARY = 2,
    CTR_EVICTED_INSERTS = 3,
    CTR_EVICTIONS = 4,
    CTR_FAILED = 5,
    CTR_LOST = 6,
    CTR_ERROR = 7,
    CTR_REMOVED = 8,
    CTR_DUP = 9,
    CTR_HIST0 = 16,  // eviction-chain-length histogram, kChainBins counters
    CTR_COUNT = 32
};
// Chain-length bins: 0 evictions (a slot freed up), 1, 2-3, 4-7, ..., >= 256.
constexpr int kChainBins = 10;
constexpr uint64_t ERR_CAS_LIMIT = 1;   // a compare-and-swap retry bound was hit
constexpr uint64_t ERR_WAIT_LIMIT = 2;  // a bulk copy did not complete within its poll bound

struct DevTable {
    uint8_t* buckets;
    uint64_t nb_mask;
    unsigned long long* ctr;
    unsigned long long* hist = nullptr;  // chain-length histogram (kChainBins), or null when not recorded
};

// Records the eviction chain of one stored key (L slot exchanges).
__device__ __forceinline__ void record_chain(const DevTable& t, uint32_t L) {
    if (!t.hist) return;
    const int bin = L == 0 ? 0 : (32 - __clz(L)) < kChainBins - 1 ? (32 - __clz(L)) : kChainBins - 1;
    atomicAdd(&t.hist[bin], 1ull);
}

template <class C>
__device__ __forceinline__ uint64_t* bucket_words(const DevTable& t, uint64_t b) {
    return reinterpret_cast<uint64_t*>(t.buckets + b * static_cast<uint64_t>(C::bucket_bytes));
}

// Select element w of a register array without dynamic indexing.
template <int N>
__device__ __forceinline__ uint64_t pick(const uint64_t (&c)[N], int w) {
    uint64_t r = c[0];
#pragma unroll
    for (int j = 1; j < N; ++j) r = (j == w) ? c[j] : r;
    return r;
}
template <int N>
__device__ __forceinline__ void put(uint64_t (&c)[N], int w, uint64_t v) {
#pragma unroll
    for (int j = 0; j < N; ++j)
        if (j == w) c[j] = v;
}

// First word, in circular order from sw, whose bit is set in `words` (wc bits).
template <int WC>
__device__ __forceinline__ int first_word(uint32_t words, int sw) {
    if constexpr (WC == 1) {
        return 0;
    } else {
        constexpr uint32_t full = WC == 32 ? ~0u : ((1u << (WC % 32)) - 1u);
        const uint32_t rot = sw ? (((words >> sw) | (words << (WC - sw))) & full) : words;
        return (sw + __ffs(rot) - 1) & (WC - 1);
    }
}

// Per-bucket slot mask type: one bit per slot.
template <class C>
using SlotMask = typename std::conditional<(C::bs > 32), unsigned long long, unsigned int>::type;

// Bit s set when slot s of bucket image c holds `tag` (0: the empty slots).
template <class C>
__device__ __forceinline__ SlotMask<C> slots_holding(const uint64_t (&c)[C::nchunks], uint32_t tag) {
    static_assert(C::bs <= 64, "slot masks hold at most 64 slots");
    const uint64_t rep = replicate<C::bits>(tag);
    SlotMask<C> m = 0;
#pragma unroll
    for (int j = 0; j < C::nchunks; ++j) {
        const uint64_t z = zero_lanes<C::bits>(c[j] ^ rep);
#pragma unroll
        for (int l = 0; l < C::lanes_per_chunk; ++l)
            m |= static_cast<SlotMask<C>>((z >> (l * C::bits + C::bits - 1)) & 1u) << (j * C::lanes_per_chunk + l);
    }
    return m;
}

// First slot set in m, circularly from slot s0 (m != 0).
template <class C>
__device__ __forceinline__ uint32_t first_slot_from(SlotMask<C> m, uint32_t s0) {
    constexpr int kBits = 8 * sizeof(SlotMask<C>);
    constexpr SlotMask<C> full = C::bs == kBits ? ~static_cast<SlotMask<C>>(0)
                                                : ((static_cast<SlotMask<C>>(1) << (C::bs % kBits)) - 1);
    const SlotMask<C> rot = s0 ? (((m >> s0) | (m << (C::bs - s0))) & full) : m;
    uint32_t off;
    if constexpr (sizeof(SlotMask<C>) == 8)
        off = __ffsll(static_cast<long long>(rot)) - 1;
    else
        off = __ffs(static_cast<int>(rot)) - 1;
    return (s0 + off) & (C::bs - 1);
}

// First slot of the reference's word-by-word scan (start word
// (tag & (bs-1)) / tpw, lowest lane first) among the slots set in m.
template <class C>
__device__ __forceinline__ uint32_t scan_slot(SlotMask<C> m, uint32_t tag) {
    return first_slot_from<C>(m, ((tag & (C::bs - 1)) / C::tpw) * C::tpw);
}

// tryInsertAtBucket on a bucket whose current image is in c (refreshed on
// compare-and-swap failure).  Returns true when fp was stored.
template <class C>
__device__ bool try_insert(uint64_t* bw, uint64_t (&c)[C::nchunks], uint32_t fp, bool& err) {
    if constexpr (!C::chunk_scan) {
        for (int it = 0; it < kCasRetryLimit; ++it) {
            const SlotMask<C> m = slots_holding<C>(c, 0);
            if (!m) return false;
            const uint32_t slot = scan_slot<C>(m, fp);
            const int w = static_cast<int>(slot / C::lanes_per_chunk);
            const uint64_t cur = pick(c, w);
            const uint64_t desired = cur | (static_cast<uint64_t>(fp) << ((slot % C::lanes_per_chunk) * C::bits));
            const uint64_t old = cas64(bw + w, cur, desired);
            if (old == cur) return true;
            put(c, w, old);
        }
        err = true;
        return false;
    }
    const int sw = static_cast<int>((fp & (C::bs - 1)) / C::tpw);
    for (int it = 0; it < kCasRetryLimit; ++it) {
        uint32_t words = 0;
#pragma unroll
        for (int j = 0; j < C::nchunks; ++j) words |= (zero_lanes<C::bits>(c[j]) != 0 ? 1u : 0u) << j;
        if (!words) return false;
        const int w = first_word<C::wc>(words, sw);
        const uint64_t cur = pick(c, w);
        const int lane = lowest_lane<C::bits>(zero_lanes<C::bits>(cur));
        const uint64_t desired = cur | (static_cast<uint64_t>(fp) << (lane * C::bits));
        const uint64_t old = cas64(bw + w, cur, desired);
        if (old == cur) return true;
        put(c, w, old);
    }
    err = true;
    return false;
}

// One step of tryInsertAtBucket: the word index and the compare-and-swap
// values that store fp in the first empty slot of bucket image c, scanning
// words from fp's start word.  False when c has no empty slot.
template <class C>
__device__ __forceinline__ bool plan_insert(const uint64_t (&c)[C::nchunks], uint32_t fp, int& w, uint64_t& cur,
                                            uint64_t& desired) {
    if constexpr (!C::chunk_scan) {
        const SlotMask<C> m = slots_holding<C>(c, 0);
        if (!m) return false;
        const uint32_t slot = scan_slot<C>(m, fp);
        w = static_cast<int>(slot / C::lanes_per_chunk);
        cur = pick(c, w);
        desired = cur | (static_cast<uint64_t>(fp) << ((slot % C::lanes_per_chunk) * C::bits));
        return true;
    }
    const int sw = static_cast<int>((fp & (C::bs - 1)) / C::tpw);
    uint32_t words = 0;
#pragma unroll
    for (int j = 0; j < C::nchunks; ++j) words |= (zero_lanes<C::bits>(c[j]) != 0 ? 1u : 0u) << j;
    if (!words) return false;
    w = first_word<C::wc>(words, sw);
    cur = pick(c, w);
    const int lane = lowest_lane<C::bits>(zero_lanes<C::bits>(cur));
    desired = cur | (static_cast<uint64_t>(fp) << (lane * C::bits));
    return true;
}

// The compare-and-swap that tryRemoveAtBucket would try first: clear the
// first slot holding fp, in the reference's scan order, of bucket image c.
// False when c does not hold fp.
template <class C>
__device__ __forceinline__ bool plan_remove(const uint64_t (&c)[C::nchunks], uint32_t fp, int& w, uint64_t& cur,
                                            uint64_t& desired) {
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
    if constexpr (!C::chunk_scan) {
        const SlotMask<C> m = slots_holding<C>(c, fp);
        if (!m) return false;
        const uint32_t slot = scan_slot<C>(m, fp);
        w = static_cast<int>(slot / C::lanes_per_chunk);
        cur = pick(c, w);
        desired = cur & ~(lane_mask << ((slot % C::lanes_per_chunk) * C::bits));
        return true;
    }
    const int sw = static_cast<int>((fp & (C::bs - 1)) / C::tpw);
    const uint64_t rep = replicate<C::bits>(fp);
    uint32_t words = 0;
#pragma unroll
    for (int j = 0; j < C::nchunks; ++j) words |= (zero_lanes<C::bits>(c[j] ^ rep) != 0 ? 1u : 0u) << j;
    if (!words) return false;
    w = first_word<C::wc>(words, sw);
    cur = pick(c, w);
    const int lane = lowest_lane<C::bits>(zero_lanes<C::bits>(cur ^ rep));
    desired = cur & ~(lane_mask << (lane * C::bits));
    return true;
}

// tryRemoveAtBucket: clear the first slot holding fp.
template <class C>
__device__ bool try_remove(uint64_t* bw, uint64_t (&c)[C::nchunks], uint32_t fp, bool& err) {
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
    if constexpr (!C::chunk_scan) {
        for (int it = 0; it < kCasRetryLimit; ++it) {
            const SlotMask<C> m = slots_holding<C>(c, fp);
            if (!m) return false;
            const uint32_t slot = scan_slot<C>(m, fp);
            const int w = static_cast<int>(slot / C::lanes_per_chunk);
            const uint64_t cur = pick(c, w);
            const uint64_t desired = cur & ~(lane_mask << ((slot % C::lanes_per_chunk) * C::bits));
            const uint64_t old = cas64(bw + w, cur, desired);
            if (old == cur) return true;
            put(c, w, old);
        }
        err = true;
        return false;
    }
    const int sw = static_cast<int>((fp & (C::bs - 1)) / C::tpw);
    const uint64_t rep = replicate<C::bits>(fp);
    for (int it = 0; it < kCasRetryLimit; ++it) {
        uint32_t words = 0;
#pragma unroll
        for (int j = 0; j < C::nchunks; ++j) words |= (zero_lanes<C::bits>(c[j] ^ rep) != 0 ? 1u : 0u) << j;
        if (!words) return false;
        const int w = first_word<C::wc>(words, sw);
        const uint64_t cur = pick(c, w);
        const int lane = lowest_lane<C::bits>(zero_lanes<C::bits>(cur ^ rep));
        const uint64_t desired = cur & ~(lane_mask << (lane * C::bits));
        const uint64_t old = cas64(bw + w, cur, desired);
        if (old == cur) return true;
        put(c, w, old);
    }
    err = true;
    return false;
}

template <class C>
__device__ __forceinline__ bool has_tag(const uint64_t (&c)[C::nchunks], uint32_t fp) {
    const uint64_t rep = replicate<C::bits>(fp);
    uint64_t any = 0;
#pragma unroll
    for (int j = 0; j < C::nchunks; ++j) any |= zero_lanes<C::bits>(c[j] ^ rep);
    return any != 0;
}

// Atomically replace the tag in `slot`; returns the tag that was there.
template <class C>
__device__ uint32_t exchange_slot(uint64_t* bw, uint32_t slot, uint32_t v, bool& err) {
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
    const int w = static_cast<int>(slot / C::lanes_per_chunk);
    const int sh = static_cast<int>(slot % C::lanes_per_chunk) * C::bits;
    uint64_t cur = load_word_rlx(bw + w);
    for (int it = 0; it < kCasRetryLimit; ++it) {
        const uint64_t desired = (cur & ~(lane_mask << sh)) | (static_cast<uint64_t>(v) << sh);
        const uint64_t old = cas64(bw + w, cur, desired);
        if (old == cur) return static_cast<uint32_t>((cur >> sh) & lane_mask);
        cur = old;
    }
    err = true;
    return v;  // treated as "slot already held v": nothing moved
}

struct EvictStats {
    uint32_t evictions = 0;
    uint32_t lost = 0;  // stored tags dropped when eviction walks crossed
    uint32_t dup = 0;   // BFS copies that could not be taken back (an extra entry)
};

// Undo of a BFS copy (reference CuckooFilter.cuh:1011-1012): remove one instance
// of a tag from its bucket pair {a, b}, where it is stored as `tag_a` in a and
// as alt_tag(tag_a) in b.  While the copy was in place another walk may have
// moved it to the other bucket of the pair, or be carrying an instance between
// the two, so both buckets are tried, a bounded number of times.  Any instance
// will do: equal tags of one pair are interchangeable.  (The reference removes
// the candidate's old form from the alternate bucket; under the Offset policy
// that is not the form it copied there.)
template <class C>
__device__ bool remove_from_pair(const DevTable& t, uint64_t a, uint64_t b, uint32_t tag_a, bool& err) {
    for (int it = 0; it < 1024; ++it) {
        uint64_t c[C::nchunks];
        uint64_t* aw = bucket_words<C>(t, a);
        load_rlx<C::bucket_bytes>(aw, c);
        if (try_remove<C>(aw, c, tag_a, err)) return true;
        uint64_t* bw = bucket_words<C>(t, b);
        load_rlx<C::bucket_bytes>(bw, c);
        if (try_remove<C>(bw, c, alt_tag<C>(tag_a), err)) return true;
        if (err) return false;
        __nanosleep(100);
    }
    return false;
}

// insertWithEvictionDFS with undo.  Returns true when fp is stored.
template <class C>
__device__ __noinline__ bool evict_dfs(DevTable t, uint32_t fp, uint64_t start, uint64_t other, uint32_t max_ev,
                                       EvictStats& st, bool& err) {
    uint8_t path[kMaxEvictionsCap];
    uint32_t cur = fp;
    uint64_t cb = start;
    for (uint32_t e = 0; e < max_ev; ++e) {
        const uint32_t slot = static_cast<uint32_t>((static_cast<uint64_t>(cur) + 7ull * e) & (C::bs - 1));
        path[e] = static_cast<uint8_t>(slot);
        const uint32_t victim = exchange_slot<C>(bucket_words<C>(t, cb), slot, cur, err);
        if (err) return false;
        ++st.evictions;
        if (victim == 0) return true;  // a slot emptied concurrently took the tag
        cb = alt_bucket<C>(cb, victim, t.nb_mask);
        cur = alt_tag<C>(victim);
        uint64_t c[C::nchunks];
        uint64_t* bw = bucket_words<C>(t, cb);
        load_rlx<C::bucket_bytes>(bw, c);
        if (try_insert<C>(bw, c, cur, err)) return true;
        if (err) return false;
    }
    // Out of evictions: walk the chain back.  The held tag returns to the
    // bucket it was taken from, alt(cb, held), at the logged slot (in that
    // bucket's form).
    for (uint32_t e = max_ev; e-- > 0;) {
        cb = alt_bucket<C>(cb, cur, t.nb_mask);
        cur = exchange_slot<C>(bucket_words<C>(t, cb), path[e], alt_tag<C>(cur), err);
        if (err) return false;
        if (cur == 0) return true;
    }
    if (cur == fp && (cb == start || cb == other)) return false;  // table restored, fp not stored
    // Another walk crossed ours: the tag now in hand belongs to a different
    // key, and fp is stored.  Give the stray tag one more chance.
    {
        uint64_t c[C::nchunks];
        uint64_t* bw = bucket_words<C>(t, cb);
        load_rlx<C::bucket_bytes>(bw, c);
        if (try_insert<C>(bw, c, cur, err)) return true;
        const uint64_t ab = alt_bucket<C>(cb, cur, t.nb_mask);
        bw = bucket_words<C>(t, ab);
        load_rlx<C::bucket_bytes>(bw, c);
        if (try_insert<C>(bw, c, alt_tag<C>(cur), err)) return true;
    }
    ++st.lost;
    return true;
}

// insertWithEvictionBFS: up to min(8, bs/2) candidates of the start bucket are
// moved to their alternate bucket (copy first, then swap fp in, undo the copy
// if the candidate moved meanwhile); then DFS.
//
// The start bucket is read once (one vector load) and the candidates are taken
// from that snapshot; the swap's compare-and-swap re-validates the candidate.
template <class C>
__device__ bool evict_bfs(DevTable t, uint32_t fp, uint64_t start, uint64_t other, uint32_t max_ev,
                          EvictStats& st, bool& err) {
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
    constexpr uint32_t ncand = (C::bs / 2) < 8 ? (C::bs / 2) : 8;
    uint64_t* sbw = bucket_words<C>(t, start);
    uint64_t snap[C::nchunks];
    load_rlx<C::bucket_bytes>(sbw, snap);
    for (uint32_t i = 0; i < ncand; ++i) {
        const uint32_t slot = static_cast<uint32_t>((static_cast<uint64_t>(fp) + 7ull * i) & (C::bs - 1));
        const int w = static_cast<int>(slot / C::lanes_per_chunk);
        const int sh = static_cast<int>(slot % C::lanes_per_chunk) * C::bits;
        uint64_t word = pick(snap, w);
        const uint32_t cand = static_cast<uint32_t>((word >> sh) & lane_mask);
        uint64_t c[C::nchunks];
        if (cand == 0) {
            load_rlx<C::bucket_bytes>(sbw, c);
            if (try_insert<C>(sbw, c, fp, err)) return true;
            if (err) return false;
            continue;
        }
        const uint64_t ab = alt_bucket<C>(start, cand, t.nb_mask);
        uint64_t* abw = bucket_words<C>(t, ab);
        load_rlx<C::bucket_bytes>(abw, c);
        if (try_insert<C>(abw, c, alt_tag<C>(cand), err)) {
            word = load_word_rlx(sbw + w);
            if (((word >> sh) & lane_mask) == cand) {
                const uint64_t desired = (word & ~(lane_mask << sh)) | (static_cast<uint64_t>(fp) << sh);
                if (cas64(sbw + w, word, desired) == word) {
                    ++st.evictions;
                    return true;
                }
            }
            if (!remove_from_pair<C>(t, ab, start, alt_tag<C>(cand), err)) ++st.dup;
            load_rlx<C::bucket_bytes>(sbw, snap);  // the start bucket changed under us
        }
        if (err) return false;
    }
    return evict_dfs<C>(t, fp, start, other, max_ev, st, err);
}

// ------------------------------------------------------------ key loading

template <class C, int KPT>
__device__ __forceinline__ void load_keys(const typename C::Key* keys, uint64_t k0, uint64_t n, bool vec_ok,
                                          uint64_t (&key)[KPT]) {
    if (vec_ok && k0 + KPT <= n) {
        if constexpr (C::key_bytes == 8 && KPT % 4 == 0) {
#pragma unroll
            for (int j = 0; j < KPT; j += 4)
                ld_stream_v4u64(reinterpret_cast<const uint64_t*>(keys) + k0 + j, key[j], key[j + 1], key[j + 2],
                                key[j + 3]);
            return;
        } else if constexpr (C::key_bytes == 8 && KPT == 2) {
            asm volatile("ld.global.nc.L1::no_allocate.v2.u64 {%0,%1}, [%2];"
                         : "=l"(key[0]), "=l"(key[1])
                         : "l"(reinterpret_cast<const uint64_t*>(keys) + k0));
            return;
        } else if constexpr (C::key_bytes == 4 && KPT % 4 == 0) {
#pragma unroll
            for (int j = 0; j < KPT; j += 4) {
                uint32_t a, b, c, d;
                ld_stream_v4u32(reinterpret_cast<const uint32_t*>(keys) + k0 + j, a, b, c, d);
                key[j] = a;
                key[j + 1] = b;
                key[j + 2] = c;
                key[j + 3] = d;
            }
            return;
        }
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        key[j] = 0;
        if (k0 + j < n) {
            if constexpr (C::key_bytes == 8)
                key[j] = ld_stream_u64(reinterpret_cast<const uint64_t*>(keys) + k0 + j);
            else
                key[j] = ld_stream_u32(reinterpret_cast<const uint32_t*>(keys) + k0 + j);
        }
    }
}

// Store KPT result bytes (bit j of `bits` -> out[k0 + j]).  When the run of
// KPT bytes is aligned, one 1/2/4/8-byte streaming store writes them all.
template <int KPT>
__device__ __forceinline__ void store_results(uint8_t* out, uint64_t k0, uint64_t n, bool vec_ok, uint32_t bits) {
    if (vec_ok && k0 + KPT <= n) {
        uint64_t v = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) v |= static_cast<uint64_t>((bits >> j) & 1u) << (8 * j);
        if constexpr (KPT == 8) {
            asm volatile("st.global.cs.u64 [%0], %1;" ::"l"(out + k0), "l"(v) : "memory");
        } else if constexpr (KPT == 4) {
            asm volatile("st.global.cs.u32 [%0], %1;" ::"l"(out + k0), "r"(static_cast<uint32_t>(v)) : "memory");
        } else if constexpr (KPT == 2) {
            asm volatile("st.global.cs.u16 [%0], %1;" ::"l"(out + k0), "h"(static_cast<uint16_t>(v)) : "memory");
        } else {
            out[k0] = static_cast<uint8_t>(v);
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < KPT; ++j)
        if (k0 + j < n) out[k0 + j] = static_cast<uint8_t>((bits >> j) & 1u);
}

__device__ __forceinline__ void flush_counter(unsigned long long* ctr, uint32_t v) {
    const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(ctr, static_cast<unsigned long long>(s));
}

// ------------------------------------------------------------------ kernels

template <class C, int KPT>
__global__ void __launch_bounds__(512) k_contains(DevTable t, const typename C::Key* __restrict__ keys, uint64_t n,
                                                  uint8_t* __restrict__ out, bool keys_vec, bool out_vec) {
    const uint64_t tile = static_cast<uint64_t>(blockDim.x) * KPT;
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x) * KPT;
        if (k0 >= n) continue;
        uint64_t key[KPT];
        load_keys<C, KPT>(keys, k0, n, keys_vec, key);
        uint64_t b[KPT];
        uint32_t fp[KPT];
        uint64_t c[KPT][C::nchunks];
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            candidates<C>(key[j], t.nb_mask, b[j], fp[j]);
            if (k0 + j < n) load_nc<C::bucket_bytes>(t.buckets + b[j] * C::bucket_bytes, c[j]);
        }
        uint32_t hit = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if (k0 + j < n && has_tag<C>(c[j], fp[j])) hit |= 1u << j;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (k0 + j < n && !((hit >> j) & 1u)) {
                b[j] = alt_bucket<C>(b[j], fp[j], t.nb_mask);
                load_nc<C::bucket_bytes>(t.buckets + b[j] * C::bucket_bytes, c[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if (k0 + j < n && !((hit >> j) & 1u) && has_tag<C>(c[j], alt_tag<C>(fp[j]))) hit |= 1u << j;
        store_results<KPT>(out, k0, n, out_vec, hit);
    }
}

template <class C, int KPT>
__global__ void __launch_bounds__(512) k_delete(DevTable t, const typename C::Key* __restrict__ keys, uint64_t n,
                                                uint8_t* __restrict__ out, bool keys_vec, bool out_vec) {
    const uint64_t tile = static_cast<uint64_t>(blockDim.x) * KPT;
    uint32_t removed = 0;
    bool err = false;
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x) * KPT;
        if (k0 >= n) continue;
        uint64_t key[KPT];
        load_keys<C, KPT>(keys, k0, n, keys_vec, key);
        uint64_t b[KPT];
        uint32_t fp[KPT];
        uint64_t c[KPT][C::nchunks];
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            candidates<C>(key[j], t.nb_mask, b[j], fp[j]);
            if (k0 + j < n) load_rlx<C::bucket_bytes>(t.buckets + b[j] * C::bucket_bytes, c[j]);
        }
        uint32_t done = 0;
        // every key's first compare-and-swap is issued before any result is
        // checked, so a thread's KPT round trips overlap; a lost race falls
        // back to tryRemoveAtBucket's retry loop on the refreshed word
        auto remove_batch = [&](uint32_t live, bool alt) {
            int w[KPT];
            uint64_t exp[KPT], des[KPT], old[KPT];
            uint32_t planned = 0;
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                w[j] = 0;
                exp[j] = des[j] = 0;
                const uint32_t tag = alt ? alt_tag<C>(fp[j]) : fp[j];
                if (((live >> j) & 1u) && plan_remove<C>(c[j], tag, w[j], exp[j], des[j])) planned |= 1u << j;
            }
#pragma unroll
            for (int j = 0; j < KPT; ++j)
                if ((planned >> j) & 1u) old[j] = cas64(bucket_words<C>(t, b[j]) + w[j], exp[j], des[j]);
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                if (!((planned >> j) & 1u)) continue;
                if (old[j] == exp[j]) {
                    done |= 1u << j;
                } else {
                    put(c[j], w[j], old[j]);
                    if (try_remove<C>(bucket_words<C>(t, b[j]), c[j], alt ? alt_tag<C>(fp[j]) : fp[j], err))
                        done |= 1u << j;
                }
            }
        };
        uint32_t valid = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if (k0 + j < n) valid |= 1u << j;
        remove_batch(valid, false);
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (((valid & ~done) >> j) & 1u) {
                b[j] = alt_bucket<C>(b[j], fp[j], t.nb_mask);
                load_rlx<C::bucket_bytes>(t.buckets + b[j] * C::bucket_bytes, c[j]);
            }
        }
        remove_batch(valid & ~done, true);
        removed += __popc(done);
        if (out) store_results<KPT>(out, k0, n, out_vec, done);
    }
    const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, removed);
    if ((threadIdx.x & 31) == 0 && s) {
        atomicAdd(&t.ctr[CTR_REMOVED], static_cast<unsigned long long>(s));
        atomicAdd(&t.ctr[CTR_OCCUPIED], ~static_cast<unsigned long long>(s) + 1ull);  // -= s
    }
    if (__any_sync(0xFFFFFFFFu, err) && (threadIdx.x & 31) == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// ------------------------------------------------- warp-cooperative probing
//
// containsMany / deleteMany with W lanes per key (CF_OPT_PROBE_WIDTH): a group
// of W consecutive lanes owns KPT consecutive keys, and lane r of the group
// loads bytes [r*PB, (r+1)*PB) of each bucket (PB = bucket_bytes / W, 4 or 8).
// The group votes by ballot (lookups) or assembles the bucket's slot mask by
// shuffles (deletes), so a key's bucket is one coalesced 32-lane request
// shared by W lanes instead of one lane's 16- or 32-byte vector load.

template <class C, int W>
struct CoopGeom {
    static constexpr int PB = C::bucket_bytes / W;          // bytes of a bucket per lane
    static constexpr int spl = PB * 8 / C::bits;            // slots per lane
    static constexpr bool ok = W >= 2 && W <= 32 && C::bucket_bytes % W == 0 && (PB == 4 || PB == 8) && C::bs <= 64;
};

// Lookup piece test: does the `PB`-byte piece (zero-extended into 64 bits)
// hold tag fp?  Zero-extended lanes XOR the replicated tag are non-zero, so
// they never match.
template <class C, int PB>
__device__ __forceinline__ bool piece_has(uint64_t piece, uint32_t fp) {
    const uint64_t rep = replicate<C::bits>(fp);
    uint64_t z = zero_lanes<C::bits>(piece ^ rep);
    if constexpr (PB < 8) z &= (1ull << (8 * PB)) - 1ull;
    return z != 0;
}

// Slots of a piece holding fp, as bits 0 .. PB*8/bits - 1.
template <class C, int PB>
__device__ __forceinline__ uint32_t piece_slots(uint64_t piece, uint32_t fp) {
    constexpr int spl = PB * 8 / C::bits;
    const uint64_t z = zero_lanes<C::bits>(piece ^ replicate<C::bits>(fp));
    uint32_t m = 0;
#pragma unroll
    for (int l = 0; l < spl; ++l) m |= static_cast<uint32_t>((z >> (l * C::bits + C::bits - 1)) & 1u) << l;
    return m;
}

template <int PB>
__device__ __forceinline__ uint64_t load_piece(const uint8_t* p) {
    if constexpr (PB == 8) {
        uint64_t v;
        asm volatile("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
        return v;
    } else {
        uint32_t v;
        asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
        return v;
    }
}

// As load_piece, coherent with the compare-and-swaps of the same launch.
template <int PB>
__device__ __forceinline__ uint64_t load_piece_rlx(const uint8_t* p) {
    if constexpr (PB == 8) {
        uint64_t v;
        asm volatile("ld.relaxed.gpu.global.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
        return v;
    } else {
        uint32_t v;
        asm volatile("ld.relaxed.gpu.global.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        return v;
    }
}

// containsMany (CuckooFilter.cuh:1088-1098, :1143-1155) with W lanes per key.
template <class C, int KPT, int W>
__global__ void __launch_bounds__(512) k_contains_coop(DevTable t, const typename C::Key* __restrict__ keys,
                                                       uint64_t n, uint8_t* __restrict__ out, bool out_vec) {
    using G = CoopGeom<C, W>;
    static_assert(G::ok, "W lanes of 4 or 8 bytes each cover the bucket");
    const uint32_t lane = threadIdx.x & 31, r = lane % W;
    const uint32_t gmask = (W == 32 ? 0xFFFFFFFFu : ((1u << W) - 1u)) << (lane - r);
    const uint64_t tile = static_cast<uint64_t>(blockDim.x / W) * KPT;
    // the trip count is uniform over the block: every lane reaches every ballot
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x / W) * KPT;
        uint64_t b[KPT], piece[KPT];
        uint32_t fp[KPT];
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            b[j] = 0;
            fp[j] = 0;
            piece[j] = 0;
            if (k0 + j < n) {
                candidates<C>(static_cast<uint64_t>(keys[k0 + j]), t.nb_mask, b[j], fp[j]);
                piece[j] = load_piece<G::PB>(t.buckets + b[j] * C::bucket_bytes + r * G::PB);
            }
        }
        uint32_t hit = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const bool mine = k0 + j < n && piece_has<C, G::PB>(piece[j], fp[j]);
            if (__ballot_sync(0xFFFFFFFFu, mine) & gmask) hit |= 1u << j;
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (k0 + j < n && !((hit >> j) & 1u)) {
                b[j] = alt_bucket<C>(b[j], fp[j], t.nb_mask);
                fp[j] = alt_tag<C>(fp[j]);
                piece[j] = load_piece<G::PB>(t.buckets + b[j] * C::bucket_bytes + r * G::PB);
            }
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const bool mine = k0 + j < n && !((hit >> j) & 1u) && piece_has<C, G::PB>(piece[j], fp[j]);
            if (__ballot_sync(0xFFFFFFFFu, mine) & gmask) hit |= 1u << j;
        }
        if (r == 0 && k0 < n) store_results<KPT>(out, k0, n, out_vec, hit);
    }
}

// tryRemoveAtBucket (first slot holding fp in the reference's scan order) for
// the keys of `pend`, W lanes per key: the group assembles the bucket's slot
// mask from its pieces, and the lane holding the chosen slot clears it with a
// compare-and-swap on its own 4- or 8-byte word.  A lost race refreshes that
// lane's piece and the group chooses again.  Keys removed are set in `done`.
template <class C, int W, int KPT>
__device__ __forceinline__ void coop_remove(const DevTable& t, const uint64_t (&b)[KPT], const uint32_t (&fp)[KPT],
                                            uint64_t (&piece)[KPT], uint32_t pend, uint32_t& done, bool& err,
                                            uint32_t r, uint32_t gmask) {
    using G = CoopGeom<C, W>;
    using M = SlotMask<C>;
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        bool want = (pend >> j) & 1u;  // uniform over the group
        for (int it = 0; it < kCasRetryLimit; ++it) {
            if (!__any_sync(0xFFFFFFFFu, want)) break;
            M m = want ? static_cast<M>(static_cast<M>(piece_slots<C, G::PB>(piece[j], fp[j])) << (r * G::spl))
                       : static_cast<M>(0);
#pragma unroll
            for (int d = 1; d < W; d <<= 1) m |= __shfl_xor_sync(0xFFFFFFFFu, m, d);
            bool ok = false;
            if (want && m) {
                const uint32_t slot = scan_slot<C>(m, fp[j]);
                if (slot / G::spl == r) {
                    uint8_t* p = t.buckets + b[j] * C::bucket_bytes + r * G::PB;
                    const uint64_t cur = piece[j];
                    const uint64_t des = cur & ~(lane_mask << ((slot % G::spl) * C::bits));
                    uint64_t old;
                    if constexpr (G::PB == 8)
                        old = atomicCAS(reinterpret_cast<unsigned long long*>(p), cur, des);
                    else
                        old = atomicCAS(reinterpret_cast<unsigned int*>(p), static_cast<unsigned int>(cur),
                                        static_cast<unsigned int>(des));
                    ok = old == cur;
                    if (!ok) piece[j] = old;
                }
            }
            const uint32_t vote = __ballot_sync(0xFFFFFFFFu, ok) & gmask;
            if (want && !m) {
                want = false;  // no copy of fp in this bucket
            } else if (want && vote) {
                want = false;
                done |= 1u << j;
            }
        }
        if (want) err = true;
    }
}

// deleteMany (CuckooFilter.cuh:805-848, :1157-1183) with W lanes per key.
template <class C, int KPT, int W>
__global__ void __launch_bounds__(512) k_delete_coop(DevTable t, const typename C::Key* __restrict__ keys, uint64_t n,
                                                     uint8_t* __restrict__ out, bool out_vec) {
    using G = CoopGeom<C, W>;
    static_assert(G::ok, "W lanes of 4 or 8 bytes each cover the bucket");
    const uint32_t lane = threadIdx.x & 31, r = lane % W;
    const uint32_t gmask = (W == 32 ? 0xFFFFFFFFu : ((1u << W) - 1u)) << (lane - r);
    const uint64_t tile = static_cast<uint64_t>(blockDim.x / W) * KPT;
    uint32_t removed = 0;
    bool err = false;
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x / W) * KPT;
        uint64_t b[KPT], piece[KPT];
        uint32_t fp[KPT];
        uint32_t pend = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            b[j] = 0;
            fp[j] = 0;
            piece[j] = 0;
            if (k0 + j < n) {
                candidates<C>(static_cast<uint64_t>(keys[k0 + j]), t.nb_mask, b[j], fp[j]);
                piece[j] = load_piece_rlx<G::PB>(t.buckets + b[j] * C::bucket_bytes + r * G::PB);
                pend |= 1u << j;
            }
        }
        uint32_t done = 0;
        coop_remove<C, W, KPT>(t, b, fp, piece, pend, done, err, r, gmask);
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (((pend >> j) & 1u) && !((done >> j) & 1u)) {
                b[j] = alt_bucket<C>(b[j], fp[j], t.nb_mask);
                fp[j] = alt_tag<C>(fp[j]);
                piece[j] = load_piece_rlx<G::PB>(t.buckets + b[j] * C::bucket_bytes + r * G::PB);
            }
        }
        coop_remove<C, W, KPT>(t, b, fp, piece, pend & ~done, done, err, r, gmask);
        if (r == 0) {
            removed += __popc(done);
            if (out && k0 < n) store_results<KPT>(out, k0, n, out_vec, done);
        }
    }
    const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, removed);
    if ((threadIdx.x & 31) == 0 && s) {
        atomicAdd(&t.ctr[CTR_REMOVED], static_cast<unsigned long long>(s));
        atomicAdd(&t.ctr[CTR_OCCUPIED], ~static_cast<unsigned long long>(s) + 1ull);  // -= s
    }
    if (__any_sync(0xFFFFFFFFu, err) && (threadIdx.x & 31) == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// Eviction for one key whose two buckets were full (CuckooFilter::insert,
// CuckooFilter.cuh:1066-1071): start at i1 if the tag is even, else at i2.
template <class C>
__device__ __noinline__ bool evict_key(DevTable t, uint64_t key, uint32_t policy_bfs, uint32_t max_ev,
                                       EvictStats& st, bool& err) {
    uint64_t i1;
    uint32_t fp;
    candidates<C>(key, t.nb_mask, i1, fp);
    const uint64_t i2 = alt_bucket<C>(i1, fp, t.nb_mask);
    const uint64_t start = (fp & 1u) == 0 ? i1 : i2;
    const uint64_t other = (fp & 1u) == 0 ? i2 : i1;
    const uint32_t sfp = (fp & 1u) == 0 ? fp : alt_tag<C>(fp);  // the tag in the start bucket's form
    const uint32_t before = st.evictions;
    const bool ok = policy_bfs ? evict_bfs<C>(t, sfp, start, other, max_ev, st, err)
                               : evict_dfs<C>(t, sfp, start, other, max_ev, st, err);
    if (ok) record_chain(t, st.evictions - before);
    return ok;
}

// Inclusive prefix sum across the warp.
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, v, d);
        if (lane >= static_cast<uint32_t>(d)) v += u;
    }
    return v;
}

// insertMany.  Pass 1 per key: first empty slot of i1, else of i2.  Keys whose
// two buckets are full are not evicted in place (one evicting lane would stall
// its 31 neighbours for the whole chain); their indices are parked in a
// per-warp shared-memory buffer and evicted 32 at a time, one key per lane.
template <class C, int KPT>
__global__ void __launch_bounds__(512) k_insert(DevTable t, const typename C::Key* __restrict__ keys, uint64_t n,
                                                uint8_t* __restrict__ out, bool keys_vec, bool out_vec,
                                                uint32_t policy_bfs, uint32_t max_ev) {
    constexpr int kBuf = 32 + 32 * KPT;  // < 32 left over + one tile's worth
    __shared__ uint64_t s_defer[16 * kBuf];
    uint64_t* buf = s_defer + (threadIdx.x >> 5) * kBuf;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t pending = 0;  // warp-uniform number of parked keys
    const uint64_t tile = static_cast<uint64_t>(blockDim.x) * KPT;
    uint32_t n_prim = 0, n_sec = 0, n_evk = 0, n_fail = 0;
    EvictStats st;
    bool err = false;

    auto evict_parked = [&](uint64_t idx) {
        const uint64_t key = C::key_bytes == 8 ? static_cast<uint64_t>(reinterpret_cast<const uint64_t*>(keys)[idx])
                                               : static_cast<uint64_t>(reinterpret_cast<const uint32_t*>(keys)[idx]);
        ++n_evk;
        if (evict_key<C>(t, key, policy_bfs, max_ev, st, err)) {
            if (out) out[idx] = 1;
        } else {
            ++n_fail;
        }
    };

    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x) * KPT;
        uint32_t valid = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) valid |= (k0 + j < n ? 1u : 0u) << j;
        uint64_t key[KPT];
        uint64_t b[KPT];
        uint32_t fp[KPT];
        uint64_t c[KPT][C::nchunks];
        uint32_t done = 0;
        if (valid) {
            load_keys<C, KPT>(keys, k0, n, keys_vec, key);
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                candidates<C>(key[j], t.nb_mask, b[j], fp[j]);
                if ((valid >> j) & 1u) load_rlx<C::bucket_bytes>(t.buckets + b[j] * C::bucket_bytes, c[j]);
            }
#pragma unroll
            for (int j = 0; j < KPT; ++j)
                if (((valid >> j) & 1u) && try_insert<C>(bucket_words<C>(t, b[j]), c[j], fp[j], err)) done |= 1u << j;
            n_prim += __popc(done);
            const uint32_t miss = valid & ~done;
            if (miss) {
#pragma unroll
                for (int j = 0; j < KPT; ++j) {
                    if ((miss >> j) & 1u) {
                        b[j] = alt_bucket<C>(b[j], fp[j], t.nb_mask);
                        load_rlx<C::bucket_bytes>(t.buckets + b[j] * C::bucket_bytes, c[j]);
                    }
                }
                uint32_t sec = 0;
#pragma unroll
                for (int j = 0; j < KPT; ++j)
                    if (((miss >> j) & 1u) && try_insert<C>(bucket_words<C>(t, b[j]), c[j], alt_tag<C>(fp[j]), err))
                        sec |= 1u << j;
                n_sec += __popc(sec);
                done |= sec;
            }
            if (out) store_results<KPT>(out, k0, n, out_vec, done);
        }
        // park the keys whose buckets are both full
        const uint32_t hard = valid & ~done;
        const uint32_t cnt = __popc(hard);
        const uint32_t incl = warp_inclusive_scan(cnt);
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint32_t pos = pending + incl - cnt;
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if ((hard >> j) & 1u) buf[pos++] = k0 + j;
        pending += total;
        __syncwarp();  // parked indices and result bytes visible to the whole warp
        while (pending >= 32) {
            pending -= 32;
            const uint64_t idx = buf[pending + lane];
            __syncwarp();
            evict_parked(idx);
        }
    }
    if (lane < pending) evict_parked(buf[lane]);
    // a tag dropped by crossing eviction walks leaves the table one entry short
    flush_counter(&t.ctr[CTR_OCCUPIED], n_prim + n_sec + (n_evk - n_fail) - st.lost + st.dup);
    flush_counter(&t.ctr[CTR_DUP], st.dup);
    flush_counter(&t.ctr[CTR_PRIMARY], n_prim);
    flush_counter(&t.ctr[CTR_SECONDARY], n_sec);
    flush_counter(&t.ctr[CTR_EVICTED_INSERTS], n_evk);
    flush_counter(&t.ctr[CTR_EVICTIONS], st.evictions);
    flush_counter(&t.ctr[CTR_FAILED], n_fail);
    flush_counter(&t.ctr[CTR_LOST], st.lost);
    if (__any_sync(0xFFFFFFFFu, err) && (threadIdx.x & 31) == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// Occupied-slot count of the whole table (countOccupiedSlots, CuckooFilter.cuh:759-785).
template <class C>
__global__ void k_count_occupied(DevTable t, uint64_t nb, unsigned long long* result) {
    uint32_t cnt = 0;
    for (uint64_t b = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; b < nb;
         b += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t c[C::nchunks];
        load_nc<C::bucket_bytes>(t.buckets + b * C::bucket_bytes, c);
#pragma unroll
        for (int j = 0; j < C::nchunks; ++j) cnt += C::lanes_per_chunk - __popcll(zero_lanes<C::bits>(c[j]));
    }
    flush_counter(result, cnt);
}

// Probe accounting for the roofline: how many lookups of this batch find their
// tag in the primary bucket (1 sector) versus need the secondary (2 sectors).
template <class C>
__global__ void k_probe_count(DevTable t, const typename C::Key* __restrict__ keys, uint64_t n,
                              unsigned long long* result) {
    uint32_t prim = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t b;
        uint32_t fp;
        candidates<C>(static_cast<uint64_t>(keys[i]), t.nb_mask, b, fp);
        uint64_t c[C::nchunks];
        load_nc<C::bucket_bytes>(t.buckets + b * C::bucket_bytes, c);
        prim += has_tag<C>(c, fp) ? 1u : 0u;
    }
    flush_counter(result, prim);
}

}  // namespace cfb
