// cf_set.cuh -- batched execution over many filters (a filter set).
//
// Thousands of independent filters with uneven key batches run in ONE launch
// of a persistent kernel.  The work list lives in device memory: item j is the
// key range [offs[j], offs[j+1]) of the concatenated key buffer, destined for
// filter filt[j] (offs is monotonic, offs[n_items] = total keys).  The grid
// strides over tiles of the concatenated keys; each thread finds the item of
// its first key by binary search over offs and walks forward from there, so
// no per-item scratch or host-side tiling is needed and the launch can be
// captured in a CUDA graph and replayed with new keys in the same buffers.
//
// Per-key semantics are the single-filter kernels' (cf_kernels.cuh): the
// reference's insert / contains / remove (CuckooFilter.cuh:805-1116) applied
// to the filter the key belongs to.  Counters are per filter; a warp adds its
// lanes' counts with one atomic per distinct filter (__match_any_sync).
//
// Tunables (template parameters, picked by the set's autotuner): KPT keys per
// thread, and for lookups the probe width W: W lanes cooperate on one key,
// each loading bucket_bytes / W bytes of each bucket, and vote by ballot.
#pragma once

#include <cstdint>

#include "cf_kernels.cuh"

namespace cfb {

// Item of key k: the largest j with offs[j] <= k (empty items are skipped).
__device__ __forceinline__ uint32_t set_find_item(const uint64_t* __restrict__ offs, uint32_t n_items, uint64_t k) {
    uint32_t lo = 0, hi = n_items;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// Advance item j (an item of some key <= k) to the item of key k.
__device__ __forceinline__ uint32_t set_advance(const uint64_t* __restrict__ offs, uint32_t n_items, uint32_t j,
                                                uint64_t k) {
    while (j + 1 < n_items && offs[j + 1] <= k) ++j;
    return j;
}

constexpr uint64_t ERR_BAD_FILTER = 4;  // a work item named a filter outside the set

// Filter of item j, or n_filters (invalid) when the work list names a filter
// outside the set; such keys are skipped and flagged.
__device__ __forceinline__ uint32_t set_filter(const uint32_t* __restrict__ filt, uint32_t item, uint32_t n_filters) {
    const uint32_t f = filt[item];
    return f < n_filters ? f : n_filters;
}

// Adds v (per lane) to counter `idx` of filter f (per lane): one atomic per
// distinct filter of the warp.  All lanes of the warp must call it.
__device__ __forceinline__ void set_add_ctr(const DevTable* __restrict__ descs, uint32_t f, bool active, int idx,
                                            uint32_t v) {
    const uint32_t key = active ? f : 0xFFFFFFFFu;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
    uint32_t s = 0;
    for (uint32_t m = peers; m; m &= m - 1) s += __shfl_sync(peers, v, __ffs(m) - 1);
    const int lane = threadIdx.x & 31;
    if (active && lane == __ffs(peers) - 1 && s) {
        if (idx == CTR_REMOVED) {
            atomicAdd(&descs[f].ctr[CTR_REMOVED], static_cast<unsigned long long>(s));
            atomicAdd(&descs[f].ctr[CTR_OCCUPIED], ~static_cast<unsigned long long>(s) + 1ull);
        } else {
            atomicAdd(&descs[f].ctr[idx], static_cast<unsigned long long>(s));
        }
    }
}

// containsMany over the set, W = 1: each thread owns KPT consecutive keys.
template <class C, int KPT>
__global__ void __launch_bounds__(512) k_set_contains1(const DevTable* __restrict__ descs,
                                                       const uint32_t* __restrict__ filt,
                                                       const uint64_t* __restrict__ offs, uint32_t n_items, uint32_t n_filters,
                                                       const typename C::Key* __restrict__ keys, uint64_t n,
                                                       uint8_t* __restrict__ out, unsigned long long* err_flag) {
    const uint64_t tile = static_cast<uint64_t>(blockDim.x) * KPT;
    bool bad = false;
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x) * KPT;
        if (k0 >= n) continue;
        uint32_t item = set_find_item(offs, n_items, k0);
        uint32_t valid = 0;  // keys of this thread that exist and name a filter of the set
        DevTable t[KPT];
        uint64_t b[KPT];
        uint32_t fp[KPT];
        uint64_t c[KPT][C::nchunks];
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const uint64_t k = k0 + j;
            if (k < n) {
                item = set_advance(offs, n_items, item, k);
                const uint32_t f = set_filter(filt, item, n_filters);
                if (f == n_filters) {
                    bad = true;
                    continue;
                }
                valid |= 1u << j;
                t[j] = descs[f];
                candidates<C>(static_cast<uint64_t>(keys[k]), t[j].nb_mask, b[j], fp[j]);
                load_nc<C::bucket_bytes>(t[j].buckets + b[j] * C::bucket_bytes, c[j]);
            }
        }
        uint32_t hit = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if (((valid >> j) & 1u) && has_tag<C>(c[j], fp[j])) hit |= 1u << j;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (((valid >> j) & 1u) && !((hit >> j) & 1u)) {
                b[j] = alt_bucket<C>(b[j], fp[j], t[j].nb_mask);
                fp[j] = alt_tag<C>(fp[j]);  // the tag in the alternate bucket's form
                load_nc<C::bucket_bytes>(t[j].buckets + b[j] * C::bucket_bytes, c[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (k0 + j >= n) break;
            if (((valid >> j) & 1u) && !((hit >> j) & 1u) && has_tag<C>(c[j], fp[j])) hit |= 1u << j;
            out[k0 + j] = static_cast<uint8_t>((hit >> j) & 1u);
        }
    }
    if (bad) atomicOr(err_flag, ERR_BAD_FILTER);
}

// containsMany over the set, W lanes per key (W in {2, 4, 8}, a divisor of
// the bucket's 4-byte words): each group of W lanes owns KPT consecutive keys;
// lane r of the group loads bytes [r*PB, (r+1)*PB) of each bucket.
template <class C, int KPT, int W>
__global__ void __launch_bounds__(512) k_set_containsW(const DevTable* __restrict__ descs,
                                                       const uint32_t* __restrict__ filt,
                                                       const uint64_t* __restrict__ offs, uint32_t n_items, uint32_t n_filters,
                                                       const typename C::Key* __restrict__ keys, uint64_t n,
                                                       uint8_t* __restrict__ out, unsigned long long* err_flag) {
    constexpr int PB = C::bucket_bytes / W;
    bool bad = false;
    static_assert(PB == 4 || PB == 8, "a lane loads 4 or 8 bytes of a bucket");
    const uint32_t lane = threadIdx.x & 31, r = lane % W;
    const uint32_t gshift = lane - r;  // first lane of the group
    const uint32_t gmask = ((1u << W) - 1u) << gshift;
    const uint64_t groups = blockDim.x / W;
    const uint64_t tile = groups * KPT;
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x / W) * KPT;
        uint32_t item = k0 < n ? set_find_item(offs, n_items, k0) : 0;
        DevTable t[KPT];
        uint64_t b[KPT];
        uint32_t fp[KPT];
        uint64_t piece[KPT];
        uint32_t valid = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const uint64_t k = k0 + j;
            piece[j] = 0;
            fp[j] = 1;
            if (k < n) {
                item = set_advance(offs, n_items, item, k);
                const uint32_t f = set_filter(filt, item, n_filters);
                if (f == n_filters) {
                    bad = true;
                    continue;
                }
                valid |= 1u << j;
                t[j] = descs[f];
                candidates<C>(static_cast<uint64_t>(keys[k]), t[j].nb_mask, b[j], fp[j]);
                piece[j] = load_piece<PB>(t[j].buckets + b[j] * C::bucket_bytes + r * PB);
            }
        }
        uint32_t hit = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const bool mine = ((valid >> j) & 1u) && piece_has<C, PB>(piece[j], fp[j]);
            if (__ballot_sync(0xFFFFFFFFu, mine) & gmask) hit |= 1u << j;
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            if (((valid >> j) & 1u) && !((hit >> j) & 1u)) {
                b[j] = alt_bucket<C>(b[j], fp[j], t[j].nb_mask);
                fp[j] = alt_tag<C>(fp[j]);
                piece[j] = load_piece<PB>(t[j].buckets + b[j] * C::bucket_bytes + r * PB);
            }
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const bool mine = ((valid >> j) & 1u) && !((hit >> j) & 1u) && piece_has<C, PB>(piece[j], fp[j]);
            if (__ballot_sync(0xFFFFFFFFu, mine) & gmask) hit |= 1u << j;
            if (r == 0 && k0 + j < n) out[k0 + j] = static_cast<uint8_t>((hit >> j) & 1u);
        }
    }
    if (bad) atomicOr(err_flag, ERR_BAD_FILTER);
}

// deleteMany over the set: each thread owns KPT consecutive keys.
template <class C, int KPT>
__global__ void __launch_bounds__(512) k_set_delete(const DevTable* __restrict__ descs, const uint32_t* __restrict__ filt,
                                                    const uint64_t* __restrict__ offs, uint32_t n_items, uint32_t n_filters,
                                                    const typename C::Key* __restrict__ keys, uint64_t n,
                                                    uint8_t* __restrict__ out, unsigned long long* err_flag) {
    const uint64_t tile = static_cast<uint64_t>(blockDim.x) * KPT;
    bool err = false, bad = false;
    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x) * KPT;
        uint32_t item = k0 < n ? set_find_item(offs, n_items, k0) : 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const uint64_t k = k0 + j;
            const bool v = k < n;
            uint32_t f = 0;
            bool ok = false;
            bool live = v;
            if (v) {
                item = set_advance(offs, n_items, item, k);
                f = set_filter(filt, item, n_filters);
                live = f < n_filters;
            }
            if (v && !live) {
                bad = true;
                if (out) out[k] = 0;
            }
            if (live) {
                const DevTable t = descs[f];
                uint64_t b;
                uint32_t fp;
                candidates<C>(static_cast<uint64_t>(keys[k]), t.nb_mask, b, fp);
                uint64_t c[C::nchunks];
                load_rlx<C::bucket_bytes>(t.buckets + b * C::bucket_bytes, c);
                ok = try_remove<C>(bucket_words<C>(t, b), c, fp, err);
                if (!ok && !err) {
                    b = alt_bucket<C>(b, fp, t.nb_mask);
                    fp = alt_tag<C>(fp);
                    load_rlx<C::bucket_bytes>(t.buckets + b * C::bucket_bytes, c);
                    ok = try_remove<C>(bucket_words<C>(t, b), c, fp, err);
                }
                if (out) out[k] = ok ? 1 : 0;
            }
            set_add_ctr(descs, f, live, CTR_REMOVED, ok ? 1u : 0u);
        }
    }
    if (__any_sync(0xFFFFFFFFu, err) && (threadIdx.x & 31) == 0) atomicOr(err_flag, ERR_CAS_LIMIT);
    if (bad) atomicOr(err_flag, ERR_BAD_FILTER);
}

// insertMany over the set: each thread owns KPT consecutive keys; first empty
// slot of the primary, else of the alternate bucket; keys whose two buckets
// are full are parked per warp and evicted 32 at a time, one per lane (as
// k_insert does).
template <class C, int KPT>
__global__ void __launch_bounds__(512) k_set_insert(const DevTable* __restrict__ descs, const uint32_t* __restrict__ filt,
                                                    const uint64_t* __restrict__ offs, uint32_t n_items, uint32_t n_filters,
                                                    const typename C::Key* __restrict__ keys, uint64_t n,
                                                    uint8_t* __restrict__ out, uint32_t policy_bfs, uint32_t max_ev,
                                                    unsigned long long* err_flag) {
    constexpr int kBuf = 32 + 32 * KPT;
    __shared__ uint64_t s_defer[16 * kBuf];
    uint64_t* buf = s_defer + (threadIdx.x >> 5) * kBuf;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t pending = 0;
    bool err = false, bad = false;
    const uint64_t tile = static_cast<uint64_t>(blockDim.x) * KPT;

    // evict the parked key index idx (or nothing when !v); warp-uniform call
    auto evict_parked = [&](uint64_t idx, bool v) {
        uint32_t f = 0;
        bool ok = false;
        EvictStats st;
        if (v) {
            // parked keys passed the filter check when they were first tried
            f = set_filter(filt, set_find_item(offs, n_items, idx), n_filters);
            ok = evict_key<C>(descs[f], static_cast<uint64_t>(keys[idx]), policy_bfs, max_ev, st, err);
            if (ok && out) out[idx] = 1;
        }
        set_add_ctr(descs, f, v, CTR_EVICTED_INSERTS, 1u);
        set_add_ctr(descs, f, v, CTR_FAILED, ok ? 0u : 1u);
        set_add_ctr(descs, f, v, CTR_EVICTIONS, st.evictions);
        set_add_ctr(descs, f, v, CTR_LOST, st.lost);
        set_add_ctr(descs, f, v, CTR_DUP, st.dup);
        set_add_ctr(descs, f, v, CTR_OCCUPIED, (ok ? 1u : 0u) - st.lost + st.dup);
    };

    for (uint64_t base = blockIdx.x * tile; base < n; base += static_cast<uint64_t>(gridDim.x) * tile) {
        const uint64_t k0 = base + static_cast<uint64_t>(threadIdx.x) * KPT;
        uint32_t item = k0 < n ? set_find_item(offs, n_items, k0) : 0;
        uint32_t hard = 0;
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const uint64_t k = k0 + j;
            const bool v = k < n;
            uint32_t f = 0;
            int where = 0;  // 1 primary, 2 secondary, 0 not stored
            bool live = v;
            if (v) {
                item = set_advance(offs, n_items, item, k);
                f = set_filter(filt, item, n_filters);
                live = f < n_filters;
                if (!live) {
                    bad = true;
                    if (out) out[k] = 0;
                }
            }
            if (live) {
                const DevTable t = descs[f];
                uint64_t b;
                uint32_t fp;
                candidates<C>(static_cast<uint64_t>(keys[k]), t.nb_mask, b, fp);
                uint64_t c[C::nchunks];
                load_rlx<C::bucket_bytes>(t.buckets + b * C::bucket_bytes, c);
                if (try_insert<C>(bucket_words<C>(t, b), c, fp, err)) {
                    where = 1;
                } else if (!err) {
                    b = alt_bucket<C>(b, fp, t.nb_mask);
                    fp = alt_tag<C>(fp);
                    load_rlx<C::bucket_bytes>(t.buckets + b * C::bucket_bytes, c);
                    if (try_insert<C>(bucket_words<C>(t, b), c, fp, err)) where = 2;
                }
                if (where == 0) hard |= 1u << j;
                if (where && out) out[k] = 1;
                if (!where && out) out[k] = 0;
            }
            set_add_ctr(descs, f, live, CTR_PRIMARY, where == 1 ? 1u : 0u);
            set_add_ctr(descs, f, live, CTR_SECONDARY, where == 2 ? 1u : 0u);
            set_add_ctr(descs, f, live, CTR_OCCUPIED, where ? 1u : 0u);
        }
        // park the keys whose buckets are both full
        const uint32_t cnt = __popc(hard);
        const uint32_t incl = warp_inclusive_scan(cnt);
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint32_t pos = pending + incl - cnt;
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if ((hard >> j) & 1u) buf[pos++] = k0 + j;
        pending += total;
        __syncwarp();
        while (pending >= 32) {
            pending -= 32;
            const uint64_t idx = buf[pending + lane];
            __syncwarp();
            evict_parked(idx, true);
        }
    }
    evict_parked(lane < pending ? buf[lane] : 0, lane < pending);
    if (__any_sync(0xFFFFFFFFu, err) && lane == 0) atomicOr(err_flag, ERR_CAS_LIMIT);
    if (bad) atomicOr(err_flag, ERR_BAD_FILTER);
}

}  // namespace cfb
