// cf_region.cuh -- region-staged batch execution (L2 as the staging buffer).
//
// A random 32-byte probe of an out-of-L2 table costs one DRAM row activation,
// and the device completes only ~38 G of those per second.  The same probes
// issued region by region -- all probes of one ~16 MiB slice of the table
// before the next slice -- hit the 126 MB L2 after the slice's first touches
// and run ~5x faster.  This path therefore
//   1. partitions the batch by table region in ONE pass (hash each key, count
//      regions per CTA, scan, scatter through a shared-memory tile so that each
//      region's entries leave the tile as one contiguous run),
//   2. walks the partitioned entries in order with the whole grid, so the grid
//      works on one or two regions at a time, probing or updating buckets with
//      ordinary loads and compare-and-swap that hit L2,
//   3. for lookups, both candidate buckets of a key are partitioned in the same
//      pass (two entries per key, results OR-ed into a bitmap), so the table is
//      streamed once; deletes and inserts keep the reference's order (primary
//      bucket first), so the keys that miss are partitioned again by alternate
//      bucket for a second round, and insert misses of that round go to the
//      eviction kernels of the segment path.
// Entries are (bucket << bits) | tag with a 32-bit payload (the key's position
// in the batch), as in the segment path.  Per-key semantics are those of the
// random-access kernels (CuckooFilter.cuh:805-1116 of the reference): the
// order in which keys of one batch are applied is unspecified, as it is for
// the reference's one-thread-per-key kernels.
#pragma once

#include <cstdint>

#include "cf_segmented.cuh"

namespace cfb {

constexpr int kRgThreads = 256;
constexpr uint32_t kRgMaxRegions = 256;
constexpr int kRgTile = 2048;  // entries staged per tile
constexpr int kRgIPT = kRgTile / kRgThreads;
constexpr uint64_t kRgRegionBytes = 16ull << 20;  // target region size
static_assert(kRgThreads == static_cast<int>(kRgMaxRegions), "the scan gives one thread per region");

// Items of a partition pass.
enum RgMode : int {
    RG_KEYS = 0,       // keys; one entry (primary bucket) per key, payload = key index
    RG_KEYS_DUAL = 1,  // keys; two entries (primary and alternate bucket) per key
    RG_ENT = 2         // (entry, payload) pairs from an earlier round
};

template <int MODE>
constexpr int rg_items_per_tile() {
    return MODE == RG_KEYS_DUAL ? kRgTile / 2 : kRgTile;
}

// Contiguous share of each CTA: a whole number of tiles.
template <int MODE>
__device__ __forceinline__ uint64_t rg_chunk(uint64_t m) {
    constexpr uint64_t T = rg_items_per_tile<MODE>();
    const uint64_t per = (m + gridDim.x - 1) / gridDim.x;
    return (per + T - 1) / T * T;
}

// Keys and staged entries are read once: streaming loads, evicted from L2
// first, so the table region and the result bitmap stay resident.
template <class C>
__device__ __forceinline__ uint64_t rg_load_key(const void* keys, uint64_t i) {
    if constexpr (C::key_bytes == 8)
        return ld_once_u64(static_cast<const uint64_t*>(keys) + i);
    else
        return ld_once_u32(static_cast<const uint32_t*>(keys) + i);
}

// Per-CTA region histogram of its contiguous share: hist[region * grid + cta].
template <class C, int MODE>
__global__ void __launch_bounds__(kRgThreads) k_rg_hist(const void* src, uint64_t nb_mask, uint64_t n,
                                                        const unsigned long long* n_dev, int rl, uint32_t nreg,
                                                        uint32_t* hist) {
    __shared__ uint32_t cnt[kRgMaxRegions];
    for (uint32_t d = threadIdx.x; d < kRgMaxRegions; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    const uint64_t m = item_count(n, n_dev);
    const uint64_t chunk = rg_chunk<MODE>(m);
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < m ? lo + chunk : m;
    constexpr int U = 8;
    for (uint64_t b = lo; b < hi; b += static_cast<uint64_t>(blockDim.x) * U) {
        uint64_t x[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t i = b + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            x[j] = 0;
            if (i < hi) {
                if constexpr (MODE == RG_ENT)
                    x[j] = ld_once_u64(static_cast<const uint64_t*>(src) + i);
                else
                    x[j] = rg_load_key<C>(src, i);
            }
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t i = b + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            if (i >= hi) continue;
            if constexpr (MODE == RG_ENT) {
                atomicAdd(&cnt[static_cast<uint32_t>((x[j] >> C::bits) >> rl)], 1u);
            } else {
                uint64_t i1;
                uint32_t fp;
                candidates<C>(x[j], nb_mask, i1, fp);
                atomicAdd(&cnt[static_cast<uint32_t>(i1 >> rl)], 1u);
                if constexpr (MODE == RG_KEYS_DUAL)
                    atomicAdd(&cnt[static_cast<uint32_t>(alt_bucket<C>(i1, fp, nb_mask) >> rl)], 1u);
            }
        }
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < nreg; d += blockDim.x) hist[static_cast<uint64_t>(d) * gridDim.x + blockIdx.x] = cnt[d];
}

// Scatter of the CTA's share by region, using the scanned histogram as its
// starting offset per region.  Each tile of kRgTile entries is ranked with one
// shared-memory atomic per entry (order within a region is not kept), staged
// in region order and written out as contiguous runs.  PAY: write payloads.
template <class C, int MODE, bool PAY>
__global__ void __launch_bounds__(kRgThreads, 3) k_rg_scatter(const void* src, const uint32_t* __restrict__ src_pay,
                                                           uint64_t nb_mask, uint64_t n,
                                                           const unsigned long long* n_dev, int rl, uint32_t nreg,
                                                           const uint32_t* __restrict__ offs, uint64_t* __restrict__ dst,
                                                           uint32_t* __restrict__ dst_pay) {
    __shared__ uint64_t st_e[kRgTile];
    __shared__ uint32_t st_p[PAY ? kRgTile : 1];
    __shared__ uint32_t running[kRgMaxRegions];
    __shared__ uint32_t cnt[kRgMaxRegions];
    __shared__ uint32_t toff[kRgMaxRegions];
    __shared__ uint32_t wsum[kRgThreads / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ebits = C::bits + rl;  // entry >> ebits = region
    for (uint32_t d = tid; d < kRgMaxRegions; d += blockDim.x) {
        running[d] = d < nreg ? offs[static_cast<uint64_t>(d) * gridDim.x + blockIdx.x] : 0u;
        cnt[d] = 0;
    }
    __syncthreads();
    const uint64_t m = item_count(n, n_dev);
    const uint64_t chunk = rg_chunk<MODE>(m);
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < m ? lo + chunk : m;
    constexpr int T = rg_items_per_tile<MODE>();
    constexpr int IPT = T / kRgThreads;                  // items per thread
    constexpr int EPI = MODE == RG_KEYS_DUAL ? 2 : 1;   // entries per item
    // the next tile's items are loaded while the current tile is ranked and
    // written, so their DRAM latency overlaps this tile's shared-memory work
    uint64_t xn[IPT];
    uint32_t xpn[IPT];
    auto fetch = [&](uint64_t tb) {
        const uint32_t cnt_items = static_cast<uint32_t>(hi - tb < static_cast<uint64_t>(T) ? hi - tb : T);
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t q = j * kRgThreads + tid;
            xn[j] = 0;
            xpn[j] = 0;
            if (q < cnt_items) {
                if constexpr (MODE == RG_ENT) {
                    xn[j] = ld_once_u64(static_cast<const uint64_t*>(src) + tb + q);
                    if constexpr (PAY) xpn[j] = ld_once_u32(src_pay + tb + q);
                } else {
                    xn[j] = rg_load_key<C>(src, tb + q);
                }
            }
        }
    };
    if (lo < hi) fetch(lo);
    for (uint64_t tb = lo; tb < hi; tb += T) {
        const uint32_t count_items = static_cast<uint32_t>(hi - tb < static_cast<uint64_t>(T) ? hi - tb : T);
        uint64_t e[IPT * EPI];
        uint32_t p[IPT];            // payload per item (both entries of a key share it)
        uint32_t rd[IPT * EPI];     // rank << 16 | region (region kRgMaxRegions = no entry)
        uint64_t x[IPT];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            x[j] = xn[j];
            p[j] = MODE == RG_ENT ? xpn[j] : static_cast<uint32_t>(tb + j * kRgThreads + tid);
        }
        if (tb + T < hi) fetch(tb + T);
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const bool v = j * kRgThreads + tid < count_items;
            if constexpr (MODE == RG_ENT) {
                e[j] = x[j];
            } else {
                uint64_t i1;
                uint32_t fp;
                candidates<C>(x[j], nb_mask, i1, fp);
                e[j * EPI] = pack_entry<C>(i1, fp);
                if constexpr (MODE == RG_KEYS_DUAL)  // the alternate bucket with the tag in that bucket's form
                    e[j * EPI + 1] = pack_entry<C>(alt_bucket<C>(i1, fp, nb_mask), alt_tag<C>(fp));
            }
#pragma unroll
            for (int k = 0; k < EPI; ++k) {
                const uint32_t d = static_cast<uint32_t>(e[j * EPI + k] >> ebits);
                rd[j * EPI + k] = v ? (atomicAdd(&cnt[d], 1u) << 16) | d : kRgMaxRegions;
            }
        }
        __syncthreads();
        // exclusive scan of the tile's region counts (thread d owns region d)
        {
            const uint32_t c = cnt[tid];
            const uint32_t incl = warp_inclusive_scan(c);
            if (lane == 31) wsum[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                const uint32_t w = lane < kRgThreads / 32 ? wsum[lane] : 0u;
                const uint32_t wi = warp_inclusive_scan(w);
                if (lane < kRgThreads / 32) wsum[lane] = wi - w;
            }
            __syncthreads();
            toff[tid] = wsum[warp] + incl - c;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < IPT * EPI; ++k) {
            const uint32_t d = rd[k] & 0xFFFFu;
            if (d < kRgMaxRegions) {
                const uint32_t pos = toff[d] + (rd[k] >> 16);
                st_e[pos] = e[k];
                if constexpr (PAY) st_p[pos] = p[k / EPI];
            }
        }
        __syncthreads();
        // ordinary write-back stores: a region's run from this tile and the
        // next tile's run meet in L2 and leave for DRAM as whole lines
        const uint32_t count_e = count_items * EPI;
        for (uint32_t q = tid; q < count_e; q += kRgThreads) {
            const uint64_t v = st_e[q];
            const uint32_t d = static_cast<uint32_t>(v >> ebits);
            const uint32_t g = running[d] + (q - toff[d]);
            dst[g] = v;
            if constexpr (PAY) dst_pay[g] = st_p[q];
        }
        __syncthreads();
        running[tid] += cnt[tid];
        cnt[tid] = 0;
        __syncthreads();
    }
}

// In-order walk of region-partitioned entries.  Tile t of kRgTile/2 entries
// goes to CTA t mod grid, so the whole grid advances through the entries (and
// so through the table's regions) together.  round 1: entries carry the
// primary bucket (or, for RG_KEYS_DUAL lookups, either bucket); misses are
// appended, keyed by the alternate bucket, to `next` when it is given.
// round 2: entries carry the alternate bucket; insert misses are appended
// unchanged to `next` for eviction.  Hits set bit `payload` of `bitmap`.
template <class C, int OP>
__global__ void __launch_bounds__(kRgThreads) k_rg_probe(DevTable t, const uint64_t* __restrict__ ent,
                                                         const uint32_t* __restrict__ pay, uint64_t n,
                                                         const unsigned long long* n_dev, int round,
                                                         uint64_t* __restrict__ next, uint32_t* __restrict__ next_pay,
                                                         unsigned long long* next_count, uint32_t* bitmap) {
    __shared__ uint32_t s_warp[kRgThreads / 32];
    __shared__ unsigned long long s_base;
    constexpr int U = OP == SEG_CONTAINS ? 8 : 4;  // entries per thread in flight
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const uint64_t m = item_count(n, n_dev);
    const uint64_t tile = static_cast<uint64_t>(kRgThreads) * U;
    const uint64_t keep = l2_policy_keep();  // the result bitmap stays in L2
    uint32_t n_ok = 0;
    bool err = false;
    for (uint64_t base = blockIdx.x * tile; base < m; base += static_cast<uint64_t>(gridDim.x) * tile) {
        uint64_t ev[U];
        uint32_t pv[U];
        uint64_t c[U][C::nchunks];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = base + static_cast<uint64_t>(j) * kRgThreads + tid;
            ev[j] = 0;
            pv[j] = 0;
            if (k < m) {
                ev[j] = ld_once_u64(ent + k);
                if (pay) pv[j] = ld_once_u32(pay + k);
            }
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = base + static_cast<uint64_t>(j) * kRgThreads + tid;
            if (k < m) {
                const uint8_t* bp = t.buckets + (ev[j] >> C::bits) * C::bucket_bytes;
                if constexpr (OP == SEG_CONTAINS)
                    load_nc<C::bucket_bytes>(bp, c[j]);
                else
                    load_rlx<C::bucket_bytes>(bp, c[j]);
            }
        }
        uint32_t fwd_mask = 0;
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = base + static_cast<uint64_t>(j) * kRgThreads + tid;
            if (k >= m) continue;
            const uint32_t fp = static_cast<uint32_t>(ev[j]) & C::tag_mask;
            uint64_t* bw = bucket_words<C>(t, ev[j] >> C::bits);
            bool ok;
            if constexpr (OP == SEG_INSERT)
                ok = try_insert<C>(bw, c[j], fp, err);
            else if constexpr (OP == SEG_CONTAINS)
                ok = has_tag<C>(c[j], fp);
            else
                ok = try_remove<C>(bw, c[j], fp, err);
            if (ok && bitmap) red_or_policy(&bitmap[pv[j] >> 5], 1u << (pv[j] & 31), keep);
            n_ok += ok ? 1u : 0u;
            if (!ok && next) fwd_mask |= 1u << j;
        }
        if (next) {  // uniform: one reservation per CTA and tile
            const uint32_t cnt = __popc(fwd_mask);
            const uint32_t incl = warp_inclusive_scan(cnt);
            if (lane == 31) s_warp[tid >> 5] = incl;
            __syncthreads();
            if (tid < 32) {
                const uint32_t x = tid < kRgThreads / 32 ? s_warp[tid] : 0u;
                const uint32_t xi = warp_inclusive_scan(x);
                if (tid < kRgThreads / 32) s_warp[tid] = xi - x;
                if (tid == 31 && xi) s_base = atomicAdd(next_count, static_cast<unsigned long long>(xi));
            }
            __syncthreads();
            if (fwd_mask) {
                uint64_t o = s_base + s_warp[tid >> 5] + incl - cnt;
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    if ((fwd_mask >> j) & 1u) {
                        uint32_t fp = static_cast<uint32_t>(ev[j]) & C::tag_mask;
                        uint64_t b = ev[j] >> C::bits;
                        if (round == 1) {  // keyed by the alternate bucket, the tag in that bucket's form
                            b = alt_bucket<C>(b, fp, t.nb_mask);
                            fp = alt_tag<C>(fp);
                        }
                        next[o] = pack_entry<C>(b, fp);
                        if (next_pay) next_pay[o] = pv[j];
                        ++o;
                    }
                }
            }
            __syncthreads();
        }
    }
    if constexpr (OP == SEG_INSERT) {
        flush_counter(&t.ctr[round == 1 ? CTR_PRIMARY : CTR_SECONDARY], n_ok);
        flush_counter(&t.ctr[CTR_OCCUPIED], n_ok);
    } else if constexpr (OP == SEG_DELETE) {
        const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, n_ok);
        if (lane == 0 && s) {
            atomicAdd(&t.ctr[CTR_REMOVED], static_cast<unsigned long long>(s));
            atomicAdd(&t.ctr[CTR_OCCUPIED], ~static_cast<unsigned long long>(s) + 1ull);
        }
    }
    if (__any_sync(0xFFFFFFFFu, err) && lane == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// Lookup walk of region-partitioned entries (both buckets of every key were
// staged, RG_KEYS_DUAL).  Like k_rg_probe, but the outcome of entry k is
// written as bit k of `hits` (one ballot word per warp and step, in entry
// order), so the walk's only writes are sequential; k_rg_gather turns the
// bits into per-key results.
template <class C>
__global__ void __launch_bounds__(kRgThreads) k_rg_lookup(DevTable t, const uint64_t* __restrict__ ent, uint64_t m,
                                                            uint32_t* __restrict__ hits) {
    constexpr int U = C::bucket_bytes > 32 ? 3 : C::bucket_bytes > 16 ? 6 : 8;  // bucket loads in flight per thread
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t tile = static_cast<uint64_t>(kRgThreads) * U;
    for (uint64_t base = blockIdx.x * tile; base < m; base += static_cast<uint64_t>(gridDim.x) * tile) {
        uint64_t ev[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = base + static_cast<uint64_t>(j) * kRgThreads + threadIdx.x;
            ev[j] = k < m ? ld_once_u64(ent + k) : 0;
        }
        uint64_t c[U][C::nchunks];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = base + static_cast<uint64_t>(j) * kRgThreads + threadIdx.x;
            if (k < m) load_nc_issue<C::bucket_bytes>(t.buckets + (ev[j] >> C::bits) * C::bucket_bytes, c[j]);
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = base + static_cast<uint64_t>(j) * kRgThreads + threadIdx.x;
            const bool hit = k < m && has_tag<C>(c[j], static_cast<uint32_t>(ev[j]) & C::tag_mask);
            const uint32_t word = __ballot_sync(0xFFFFFFFFu, hit);
            const uint64_t k0 = base + static_cast<uint64_t>(j) * kRgThreads + warp * 32;  // multiple of 32
            if (lane == 0 && k0 < m) hits[k0 >> 5] = word;
        }
    }
}

// Per-key lookup results from the entry-order hit bits.  CTA c owns the keys
// of the partition pass's chunk c (same grid and chunking as k_rg_scatter) and
// reads, region by region, the run of entries that chunk c contributed to each
// region: offs (the scanned histogram, [region][cta]) gives each run's start
// and the next element its end.  The payload of an entry is its key's index;
// hits are OR-ed into a shared-memory bitmap of the chunk (dynamic shared
// memory: one bit per key of the chunk), then written out as bytes in order.
static __global__ void __launch_bounds__(kRgThreads) k_rg_gather(const uint32_t* __restrict__ pay,
                                                          const uint32_t* __restrict__ hits,
                                                          const uint32_t* __restrict__ offs, uint32_t nreg,
                                                          uint64_t m, uint64_t total, uint8_t* __restrict__ out) {
    extern __shared__ uint32_t sbm[];
    const uint64_t chunk = rg_chunk<RG_KEYS_DUAL>(m);
    const uint64_t lo = blockIdx.x * chunk;
    if (lo >= m) return;
    const uint64_t hi = lo + chunk < m ? lo + chunk : m;
    const uint32_t nwords = static_cast<uint32_t>((hi - lo + 31) / 32);
    for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) sbm[i] = 0;
    __syncthreads();
    const uint64_t nflat = static_cast<uint64_t>(nreg) * gridDim.x;
    for (uint32_t r = 0; r < nreg; ++r) {
        const uint64_t idx = static_cast<uint64_t>(r) * gridDim.x + blockIdx.x;
        const uint64_t s = offs[idx];
        const uint64_t e = idx + 1 < nflat ? offs[idx + 1] : total;
        for (uint64_t k = s + threadIdx.x; k < e; k += blockDim.x) {
            if ((hits[k >> 5] >> (k & 31)) & 1u) {
                const uint32_t q = static_cast<uint32_t>(pay[k] - lo);
                atomicOr(&sbm[q >> 5], 1u << (q & 31));
            }
        }
    }
    __syncthreads();
    const uint64_t cnt = hi - lo;
    if ((reinterpret_cast<uintptr_t>(out + lo) & 15) == 0) {
        // 16 results per thread and store
        for (uint64_t q0 = static_cast<uint64_t>(threadIdx.x) * 16; q0 < cnt; q0 += static_cast<uint64_t>(blockDim.x) * 16) {
            if (q0 + 16 <= cnt) {
                const uint32_t bits = (sbm[q0 >> 5] >> (q0 & 31)) & 0xFFFFu;
                uint64_t lo8 = 0, hi8 = 0;
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    lo8 |= static_cast<uint64_t>((bits >> b) & 1u) << (8 * b);
                    hi8 |= static_cast<uint64_t>((bits >> (b + 8)) & 1u) << (8 * b);
                }
                *reinterpret_cast<ulonglong2*>(out + lo + q0) = make_ulonglong2(lo8, hi8);
            } else {
                for (uint64_t q = q0; q < cnt; ++q) out[lo + q] = static_cast<uint8_t>((sbm[q >> 5] >> (q & 31)) & 1u);
            }
        }
    } else {
        for (uint64_t q = threadIdx.x; q < cnt; q += blockDim.x)
            out[lo + q] = static_cast<uint8_t>((sbm[q >> 5] >> (q & 31)) & 1u);
    }
}

}  // namespace cfb
