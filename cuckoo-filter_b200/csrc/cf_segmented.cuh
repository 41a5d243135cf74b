// cf_segmented.cuh -- segment-staged batch execution.
//
// Random 32-byte probes of an out-of-L2 table are capped by the number of DRAM
// transactions the memory system completes per second, not by bandwidth: on
// B200 each random probe costs one transaction (128 B fetched) and the device
// completes about 38 G of them per second, whatever the load width or path.
// For batches that are large relative to the table this path instead
//   1. radix-partitions the batch by table segment (packed (bucket << bits) |
//      tag entries, 8-bit digits, stable, shared-memory staging so every write
//      is a coalesced run),
//   2. streams each 64 KiB table segment once into shared memory, applies all of
//      the segment's operations there with shared-memory compare-and-swap, and
//      writes the segment back with coalesced stores,
//   3. repeats 1-2 for the keys that missed their primary bucket, keyed by the
//      alternate bucket,
//   4. (insert) evicts for the remaining keys with the random-access BFS/DFS.
// This is the reference's insertManySorted idea (sort by primary bucket so the
// writes coalesce, CuckooFilter.cuh:475-508 and :1209-1266) carried to its end:
// the sort is only as fine as a shared-memory segment, and lookups and deletes
// use it too.
//
// Per-key semantics are the plain path's: a key's tag goes to the first empty
// slot of its primary bucket, else of its alternate, else eviction starts at
// i1 for an even tag and i2 for an odd one.  One key alone takes exactly the
// plain path's steps.
#pragma once

#include <cstdint>

#include "cf_kernels.cuh"

namespace cfb {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
// Entries per thread of a scatter tile: 24 without payloads (a 6144-entry
// tile, two CTAs per SM in 107 KB of shared memory), 16 with payloads (the
// 4-byte payload buffers need the room).  On B200 a 2^31-entry pass took
// 7.97 ms with 24 against 8.58 ms with 16.
template <int PAY>
constexpr int rs_ipt() {
    return PAY ? 16 : 24;
}
template <int PAY>
constexpr int rs_tile() {
    return kRsThreads * rs_ipt<PAY>();
}
// Every CTA chunk of a radix pass is a multiple of this many entries, which
// both tile sizes divide.
constexpr int kRsChunkAlign = 12288;
static_assert(kRsChunkAlign % rs_tile<0>() == 0 && kRsChunkAlign % rs_tile<1>() == 0, "chunk alignment");
constexpr int kRsHistThreads = 512;
// Histogram CTAs per scatter CTA: each counts one part of the scatter CTA's
// chunk, so the histogram pass runs on three times the scatter's grid.
constexpr int kRsHistSub = 3;
static_assert(kRsThreads == kRadix, "the scatter's per-digit phases give one thread per digit");
constexpr int kSegBytes = 65536;
// Entry flag (bit 63) for the step-machine BFS: this key's BFS candidates all
// failed already, send it to DFS.  Used only where entries leave bit 63 free.
constexpr uint64_t kDfsFlag = 1ull << 63;
constexpr int kSegThreads = 256;
constexpr int kSegInsertThreads = 256;

template <class C>
__device__ __forceinline__ uint64_t pack_entry(uint64_t bucket, uint32_t fp) {
    return (bucket << C::bits) | fp;
}

template <class C>
__device__ __forceinline__ uint64_t load_key(const void* keys, uint64_t i) {
    if constexpr (C::key_bytes == 8)
        return ld_stream_u64(static_cast<const uint64_t*>(keys) + i);
    else
        return ld_stream_u32(static_cast<const uint32_t*>(keys) + i);
}

// Packed (primary bucket, tag) entry of a key.
template <class C>
__device__ __forceinline__ uint64_t entry_of_key(uint64_t key, uint64_t nb_mask) {
    uint64_t b;
    uint32_t fp;
    candidates<C>(key, nb_mask, b, fp);
    return pack_entry<C>(b, fp);
}


// Number of items of a radix pass: fixed, or read from a device counter.
__device__ __forceinline__ uint64_t item_count(uint64_t n, const unsigned long long* n_dev) {
    return n_dev ? static_cast<uint64_t>(*n_dev) : n;
}

__device__ __forceinline__ uint64_t chunk_of(uint64_t n, uint32_t parts) {
    const uint64_t per = (n + parts - 1) / parts;
    return (per + kRsChunkAlign - 1) / kRsChunkAlign * kRsChunkAlign;
}

// Digit histogram of each scatter CTA's contiguous chunk, counted by
// kRsHistSub CTAs per chunk: hist[(digit * scatter grid + cta) * kRsHistSub +
// part], so one scan gives every scatter CTA its start per digit.
// KEYS: items are keys, hashed here into packed entries that are also written
// to `ent_out` (so later passes never hash again); otherwise packed entries.
// SEGS (last pass of a sort whose earlier passes ordered the items by the
// lower `lo_bits` bits of the segment id): also counts every segment,
// seg_count[(digit << lo_bits) | lower] += 1, so the segment starts are one
// scan away.  Within a CTA's chunk the lower bits never decrease: while they
// stay the same, the run's per-digit counts are the growth of the digit
// counts since the last flush (snap), added to seg_count when the run ends;
// a step that straddles a change adds its items to seg_count one by one.
// One shared-memory atomic per item either way.
template <class C, bool KEYS, bool SEGS>
__global__ void __launch_bounds__(kRsHistThreads, 3)
    k_rs_hist(const void* src, uint64_t nb_mask, uint64_t n, const unsigned long long* n_dev, int shift,
              uint32_t* hist, uint64_t* ent_out, int lo_bits, uint32_t* seg_count) {
    __shared__ uint32_t cnt[kRadix];
    __shared__ uint32_t snap[SEGS ? kRadix : 1];
    for (int i = threadIdx.x; i < kRadix; i += blockDim.x) {
        cnt[i] = 0;
        if constexpr (SEGS) snap[i] = 0;
    }
    __syncthreads();
    const uint64_t m = item_count(n, n_dev);
    const uint32_t sgrid = gridDim.x / kRsHistSub, cta = blockIdx.x / kRsHistSub, part = blockIdx.x % kRsHistSub;
    const uint64_t chunk = chunk_of(m, sgrid);
    const uint64_t sub = (chunk / kRsHistSub + 31) / 32 * 32;
    const uint64_t c_hi = static_cast<uint64_t>(cta) * chunk + chunk < m ? static_cast<uint64_t>(cta) * chunk + chunk : m;
    const uint64_t lo0 = static_cast<uint64_t>(cta) * chunk + part * sub;
    const uint64_t lo = lo0 < c_hi ? lo0 : c_hi;
    const uint64_t hi = lo + sub < c_hi && part + 1 < kRsHistSub ? lo + sub : c_hi;
    const uint64_t* ent = static_cast<const uint64_t*>(src);
    const int lo_shift = shift - lo_bits;
    const uint32_t lo_mask = (1u << lo_bits) - 1u;
    uint32_t cur = 0;  // lower segment bits of the current run (uniform over the CTA)
    constexpr int U = 8;  // independent loads in flight per thread
    const uint64_t step = static_cast<uint64_t>(blockDim.x) * U;
    for (uint64_t b = lo; b < hi; b += step) {
        bool straddle = false;
        if constexpr (SEGS) {
            // (a first pass over keys is also the last only when there are no lower bits)
            uint32_t lf = 0, ll = 0;
            if (!KEYS && lo_bits > 0) {
                const uint64_t last = (b + step < hi ? b + step : hi) - 1;
                lf = static_cast<uint32_t>(ent[b] >> lo_shift) & lo_mask;
                ll = static_cast<uint32_t>(ent[last] >> lo_shift) & lo_mask;
            }
            if (lf != cur || lf != ll) {  // the run ends here: flush it
                __syncthreads();
                for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
                    const uint32_t c = cnt[d] - snap[d];
                    if (c) atomicAdd(&seg_count[(static_cast<uint32_t>(d) << lo_bits) | cur], c);
                    snap[d] = cnt[d];
                }
                __syncthreads();
                cur = lf;
            }
            straddle = lf != ll;
            if (straddle) cur = ll;  // the run after this step
        }
        // every load of the step is issued before any key is hashed
        uint64_t e[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t i = b + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            e[j] = 0;
            if (i < hi) e[j] = KEYS ? load_key<C>(src, i) : ent[i];
        }
        if constexpr (KEYS) {
#pragma unroll
            for (int j = 0; j < U; ++j) e[j] = entry_of_key<C>(e[j], nb_mask);
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t i = b + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            if (i < hi) {
                const uint32_t d = static_cast<uint32_t>(e[j] >> shift) & (kRadix - 1);
                atomicAdd(&cnt[d], 1u);
                if constexpr (KEYS) ent_out[i] = e[j];
                if constexpr (SEGS)
                    if (straddle)
                        atomicAdd(&seg_count[(d << lo_bits) | (static_cast<uint32_t>(e[j] >> lo_shift) & lo_mask)], 1u);
            }
        }
        if constexpr (SEGS) {
            if (straddle) {  // the step's items are in seg_count already: keep them out of the run
                __syncthreads();
                for (int d = threadIdx.x; d < kRadix; d += blockDim.x) snap[d] = cnt[d];
                __syncthreads();
            }
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
        hist[(static_cast<uint64_t>(d) * sgrid + cta) * kRsHistSub + part] = cnt[d];
        if constexpr (SEGS) {
            const uint32_t c = cnt[d] - snap[d];
            if (c) atomicAdd(&seg_count[(static_cast<uint32_t>(d) << lo_bits) | cur], c);
        }
    }
}

// Exclusive scan of `count` uint32 values in place (sums wrap modulo 2^32),
// one CTA of 1024 threads.  Each warp owns one contiguous span of whole rows
// (a row: 32 lanes x 4 values, one coalesced 16-byte load per lane when the
// array is 16-byte aligned), with eight rows in flight per lane: the warp
// sums its span, the 32 warp sums are scanned, and the warp reads its span
// again and writes it scanned row by row.  Two passes of a few dependent
// round trips each, instead of one block-synchronized step per 16K values.
static __global__ void __launch_bounds__(1024) k_scan_u32(uint32_t* v, uint32_t count) {
    constexpr uint32_t R = 8;    // rows in flight per lane
    constexpr uint32_t ROW = 128;
    __shared__ uint32_t warp_tot[32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool vec = (reinterpret_cast<uintptr_t>(v) & 15) == 0;
    const uint64_t n = count;
    const uint64_t span = ((n + 31) / 32 + ROW - 1) / ROW * ROW;
    const uint64_t b = warp * span < n ? warp * span : n;
    const uint64_t e = b + span < n ? b + span : n;
    // the four values from index i (16-byte aligned when vec; zero past e)
    auto ld4 = [&](uint64_t i) -> uint4 {
        if (vec && i + 4 <= e) return *reinterpret_cast<const uint4*>(v + i);
        uint4 x;
        x.x = i < e ? v[i] : 0u;
        x.y = i + 1 < e ? v[i + 1] : 0u;
        x.z = i + 2 < e ? v[i + 2] : 0u;
        x.w = i + 3 < e ? v[i + 3] : 0u;
        return x;
    };
    uint32_t s = 0;
    for (uint64_t row = b; row < e; row += ROW * R) {
        uint4 x[R];
#pragma unroll
        for (uint32_t q = 0; q < R; ++q) x[q] = ld4(row + q * ROW + lane * 4);
#pragma unroll
        for (uint32_t q = 0; q < R; ++q) s += x[q].x + x[q].y + x[q].z + x[q].w;
    }
    s = __reduce_add_sync(0xFFFFFFFFu, s);
    if (lane == 0) warp_tot[warp] = s;
    __syncthreads();
    if (warp == 0) {
        const uint32_t t = warp_tot[lane];
        warp_tot[lane] = warp_inclusive_scan(t) - t;
    }
    __syncthreads();
    uint32_t carry = warp_tot[warp];
    for (uint64_t row = b; row < e; row += ROW * R) {
        uint4 x[R];
#pragma unroll
        for (uint32_t q = 0; q < R; ++q) x[q] = ld4(row + q * ROW + lane * 4);
#pragma unroll
        for (uint32_t q = 0; q < R; ++q) {
            const uint32_t ls = x[q].x + x[q].y + x[q].z + x[q].w;
            const uint32_t incl = warp_inclusive_scan(ls);
            uint4 o;
            o.x = carry + incl - ls;
            o.y = o.x + x[q].x;
            o.z = o.y + x[q].y;
            o.w = o.z + x[q].z;
            const uint64_t i = row + q * ROW + lane * 4;
            if (vec && i + 4 <= e) {
                *reinterpret_cast<uint4*>(v + i) = o;
            } else {
                if (i < e) v[i] = o.x;
                if (i + 1 < e) v[i + 1] = o.y;
                if (i + 2 < e) v[i + 2] = o.z;
                if (i + 3 < e) v[i + 3] = o.w;
            }
            carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
        }
    }
}

// Shared memory of k_rs_scatter.  Each tile is staged in digit order in the
// buffer it arrived in, so one tile is in flight while the other is ranked,
// staged and written out.
template <int PAY>
struct RsScatterSmem {
    static constexpr int TILE = rs_tile<PAY>();
    uint64_t in[2][TILE];                      // bulk-copy double buffer (entries), then the staged tile
    uint32_t in_pay[2][PAY ? TILE : 1];        // payloads: bulk-copied (PAY 2), then staged
    uint32_t cnt[kRadix];                         // digit counts of the tile (ranking by atomics)
    uint16_t warp_cnt[kRsWarps][kRadix];          // stable ranking: per-warp digit counts, then their warp prefix
    uint32_t running[kRadix];                     // next output position per digit
    uint32_t tot[kRadix];                         // tile count per digit
    uint32_t tile_off[kRadix];                    // first staged position of each digit in the tile
    uint32_t out_base[kRadix];                    // output index of staged position q = out_base[digit] + q (mod 2^32)
    uint32_t grp_tot[kRadix / 32];                // tile count of each group of 32 digits
    uint64_t bar[2];
};

// One LSD pass over packed entries: scatter them to dst by digit, using the
// scanned histogram as the CTA's starting offset per digit.  Full tiles
// arrive by bulk copy into a double buffer (the copy of tile t+2 is issued
// when tile t has been written out, so tile t+1 is in flight while tile t is
// worked on).  Each tile is ranked in shared memory (rs_ipt entries per thread),
// staged in digit order in its own buffer and written out as contiguous runs.
//
// The sort only has to group entries by segment, so a pass needs to keep the
// input order only among entries whose lower `lo_bits` segment bits (the
// digits of the earlier passes) differ.  The input of a later pass is sorted
// by those bits, so a tile whose first and last entries agree on them holds a
// single value: it is ranked with one shared-memory atomic per entry (order
// within a digit unspecified).  Only a tile spanning several lower values
// (at most one per value change, so a few hundred per pass) is ranked stably
// (lanes with equal digits found by eight ballots, then warp order).
// PAY: 0 = no payload, 1 = the payload of entry i is i itself, 2 = payloads
// read from src_pay.
template <int PAY>
__global__ void __launch_bounds__(kRsThreads, 2) k_rs_scatter(const uint64_t* __restrict__ src,
                                                              const uint32_t* __restrict__ src_pay, uint64_t n,
                                                              const unsigned long long* n_dev, int shift, int lo_bits,
                                                              const uint32_t* offs, uint64_t* __restrict__ dst,
                                                              uint32_t* __restrict__ dst_pay, unsigned long long* err,
                                                              int narrow) {
    constexpr int IPT = rs_ipt<PAY>();
    constexpr int TILE = rs_tile<PAY>();
    extern __shared__ __align__(128) unsigned char rs_raw[];
    RsScatterSmem<PAY>& sm = *reinterpret_cast<RsScatterSmem<PAY>*>(rs_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t m = item_count(n, n_dev);
    const uint64_t chunk = chunk_of(m, gridDim.x);
    const uint64_t lo = blockIdx.x * chunk;
    const uint64_t hi = lo + chunk < m ? lo + chunk : m;
    const uint32_t ntile = lo < hi ? static_cast<uint32_t>((hi - lo + TILE - 1) / TILE) : 0u;
    const uint32_t nfull = lo < hi ? static_cast<uint32_t>((hi - lo) / TILE) : 0u;  // only the last can be partial
    const int lo_shift = shift - lo_bits;
    const uint64_t lo_mask = (1ull << lo_bits) - 1ull;
    for (int d = tid; d < kRadix; d += blockDim.x) {
        sm.running[d] = offs[(static_cast<uint64_t>(d) * gridDim.x + blockIdx.x) * kRsHistSub];
        sm.tot[d] = 0;
        sm.cnt[d] = 0;
    }
    for (int i = tid; i < kRsWarps * kRadix; i += blockDim.x) (&sm.warp_cnt[0][0])[i] = 0;
    if (tid == 0) {
        mbar_init(&sm.bar[0], 1);
        mbar_init(&sm.bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // thread 0: start the copy of full tile t into buffer t & 1
    auto issue = [&](uint32_t t) {
        if (t >= nfull) return;
        const uint32_t b = t & 1u;
        const uint64_t i0 = lo + static_cast<uint64_t>(t) * TILE;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&sm.bar[b], TILE * 8u + (PAY == 2 ? TILE * 4u : 0u));
        bulk_g2s(sm.in[b], src + i0, TILE * 8u, &sm.bar[b]);
        if constexpr (PAY == 2) bulk_g2s(sm.in_pay[b], src_pay + i0, TILE * 4u, &sm.bar[b]);
    };
    if (tid == 0) {
        issue(0);
        issue(1);
    }
    bool failed = false;
    for (uint32_t t = 0; t < ntile; ++t) {
        const uint32_t b = t & 1u;
        const uint64_t tb = lo + static_cast<uint64_t>(t) * TILE;
        const bool full = t < nfull;
        const uint32_t count = full ? static_cast<uint32_t>(TILE) : static_cast<uint32_t>(hi - tb);
        uint64_t e[IPT];
        uint32_t p[IPT], rank[IPT];
        uint64_t first, last;
        if (full) {
            if (!mbar_wait(&sm.bar[b], (t >> 1) & 1u, kMbarPollLimit)) failed = true;
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t idx = warp * 32 * IPT + j * 32 + lane;
                e[j] = sm.in[b][idx];
                p[j] = 0;
                if constexpr (PAY == 1) p[j] = static_cast<uint32_t>(tb + idx);
                if constexpr (PAY == 2) p[j] = sm.in_pay[b][idx];
            }
            first = sm.in[b][0];
            last = sm.in[b][TILE - 1];
        } else {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint64_t i = tb + warp * 32 * IPT + j * 32 + lane;
                e[j] = 0;
                p[j] = 0;
                if (i < hi) {
                    e[j] = __ldcs(reinterpret_cast<const unsigned long long*>(src) + i);
                    if constexpr (PAY == 1) p[j] = static_cast<uint32_t>(i);
                    if constexpr (PAY == 2) p[j] = __ldcs(reinterpret_cast<const unsigned int*>(src_pay) + i);
                }
            }
            first = src[tb];
            last = src[hi - 1];
        }
        // uniform over the CTA
        const bool stable = lo_bits > 0 && ((first >> lo_shift) & lo_mask) != ((last >> lo_shift) & lo_mask);
        if (!stable) {
            // rank = arrival order within the digit, counted in cnt
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const bool v = full || warp * 32 * IPT + j * 32 + lane < count;
                const uint32_t d = static_cast<uint32_t>((e[j] >> shift) & (kRadix - 1));
                rank[j] = v ? atomicAdd(&sm.cnt[d], 1u) : 0u;
            }
        } else {
            // rank = lane order within the warp's row, rows in order, warps in order
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const bool v = full || warp * 32 * IPT + j * 32 + lane < count;
                const uint32_t d = static_cast<uint32_t>((e[j] >> shift) & (kRadix - 1));
                uint32_t peers = __ballot_sync(0xFFFFFFFFu, v);
#pragma unroll
                for (int k = 0; k < kRadixBits; ++k) {
                    const uint32_t bit = (d >> k) & 1u;
                    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
                    peers &= bit ? bal : ~bal;
                }
                const int leader = v ? __ffs(peers) - 1 : static_cast<int>(lane);
                uint32_t base = 0;
                if (v && static_cast<int>(lane) == leader) {
                    base = sm.warp_cnt[warp][d];
                    sm.warp_cnt[warp][d] = static_cast<uint16_t>(base + __popc(peers));
                }
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                rank[j] = base + __popc(peers & lt_mask);
                __syncwarp();
            }
        }
        __syncthreads();  // tile read and ranked: its buffer may take the staged tile
        // thread d: the tile total of digit d (the previous tile's total moves
        // into the running offset), per-warp prefixes when ranked stably, the
        // digit's first staged position and its output base
        {
            uint32_t s = 0;
            if (!stable) {
                s = sm.cnt[tid];
                sm.cnt[tid] = 0;
            } else {
#pragma unroll
                for (int w = 0; w < kRsWarps; ++w) {
                    const uint32_t c = sm.warp_cnt[w][tid];
                    sm.warp_cnt[w][tid] = static_cast<uint16_t>(s);
                    s += c;
                }
            }
            const uint32_t run = sm.running[tid] + sm.tot[tid];
            sm.running[tid] = run;
            sm.tot[tid] = s;
            const uint32_t incl = warp_inclusive_scan(s);
            if (lane == 31) sm.grp_tot[warp] = incl;
            __syncthreads();
            // every warp scans the group totals itself, so thread d can place its
            // digit without another barrier: one lookup per item below, not three
            const uint32_t x = lane < kRadix / 32 ? sm.grp_tot[lane] : 0u;
            const uint32_t grp = __shfl_sync(0xFFFFFFFFu, warp_inclusive_scan(x) - x, warp);
            const uint32_t first_pos = grp + incl - s;
            sm.tile_off[tid] = first_pos;
            sm.out_base[tid] = run - first_pos;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            if (full || warp * 32 * IPT + j * 32 + lane < count) {
                const uint32_t d = static_cast<uint32_t>((e[j] >> shift) & (kRadix - 1));
                uint32_t pos = sm.tile_off[d] + rank[j];
                if (stable) pos += sm.warp_cnt[warp][d];
                sm.in[b][pos] = e[j];
                if constexpr (PAY) sm.in_pay[b][pos] = p[j];
            }
        }
        __syncthreads();
        for (uint32_t q = tid; q < count; q += blockDim.x) {
            const uint64_t x = sm.in[b][q];
            const uint32_t d = static_cast<uint32_t>((x >> shift) & (kRadix - 1));
            const uint32_t g = sm.out_base[d] + q;
            if (narrow)  // the low 32 bits: (bucket within its segment) << bits | tag
                reinterpret_cast<uint32_t*>(dst)[g] = static_cast<uint32_t>(x);
            else
                dst[g] = x;
            if constexpr (PAY) dst_pay[g] = sm.in_pay[b][q];
        }
        if (stable)
            for (int i = tid; i < kRsWarps * kRadix; i += blockDim.x) (&sm.warp_cnt[0][0])[i] = 0;
        __syncthreads();  // the tile is written out and the counters are reset: refill its buffer
        if (tid == 0) issue(t + 2);
    }
    if (__any_sync(0xFFFFFFFFu, failed) && lane == 0) atomicOr(err, ERR_WAIT_LIMIT);
}

// Dynamic shared memory of k_rs_scatter<PAY>.
template <int PAY>
constexpr int rs_scatter_smem() {
    return static_cast<int>(sizeof(RsScatterSmem<PAY>));
}

// start[s] = first index of segment s in the segment-sorted entries, s in [0, nseg];
// start[nseg] = m.
// Each thread owns 8 consecutive positions k (one load per entry plus the
// predecessor of its first); positions run to k == m inclusive.
static __global__ void k_seg_bounds(const uint64_t* ent, uint64_t n, const unsigned long long* n_dev, int seg_shift,
                                    uint64_t nseg, uint32_t* start) {
    constexpr int U = 8;
    const uint64_t m = item_count(n, n_dev);
    for (uint64_t k0 = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) * U; k0 <= m;
         k0 += static_cast<uint64_t>(gridDim.x) * blockDim.x * U) {
        int64_t seg[U + 1];
        seg[0] = k0 == 0 ? -1 : static_cast<int64_t>(ent[k0 - 1] >> seg_shift);
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = k0 + j;
            seg[j + 1] = k < m ? static_cast<int64_t>(ent[k] >> seg_shift) : static_cast<int64_t>(nseg);
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const uint64_t k = k0 + j;
            if (k > m) break;
            for (int64_t s = seg[j] + 1; s <= seg[j + 1]; ++s) start[s] = static_cast<uint32_t>(k);
        }
    }
}

enum SegOp : int { SEG_INSERT = 0, SEG_CONTAINS = 1, SEG_DELETE = 2 };

// Shared-memory segment pass.  round 1: entries carry the primary bucket;
// misses are appended (keyed by the alternate bucket) to `next`.  round 2:
// entries carry the alternate bucket; insert misses are appended to `next`
// for eviction, lookup/delete misses are final.  Hits set bit `payload` of
// `bitmap` when a bitmap is given.  fwd_other: forwarded entries are keyed by
// the key's other bucket (set in round 1).  `cap` is used by k_seg_insert
// only (the two kernels share a launch site).
template <class C, int OP>
__global__ void __launch_bounds__(kSegThreads) k_seg(DevTable t, const uint64_t* ent, const uint32_t* pay,
                                                     const uint32_t* start, uint64_t nseg, int sb_log2, int round,
                                                     uint64_t* next, uint32_t* next_pay,
                                                     unsigned long long* next_count, uint32_t* bitmap, int narrow,
                                                     uint32_t /*cap*/, int fwd_other, uint32_t* /*full*/) {
    extern __shared__ __align__(16) uint64_t seg[];
    __shared__ uint32_t s_warp[32];
    __shared__ unsigned long long s_base;
    constexpr int WPB = C::bucket_bytes / 8;  // 64-bit words per bucket
    const uint64_t sb = 1ull << sb_log2;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    uint32_t n_ok = 0;
    bool err = false;
    for (uint64_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        const uint32_t lo = start[s], hi = start[s + 1];
        if (lo == hi) continue;
        uint64_t* gseg = reinterpret_cast<uint64_t*>(t.buckets + (s << sb_log2) * C::bucket_bytes);
        // the last segment of a table whose bucket count is not a multiple of
        // the segment (AddSub and Offset policies) is partial
        const uint64_t left = t.nb_mask + 1 - (s << sb_log2);
        const uint32_t nbk = left < sb ? static_cast<uint32_t>(left) : static_cast<uint32_t>(sb);
        const uint32_t words = nbk * WPB;
        if (words % 2 == 0) {
            // 16-byte streaming loads, 8 per thread in flight
            const ulonglong2* g2 = reinterpret_cast<const ulonglong2*>(gseg);
            ulonglong2* s2 = reinterpret_cast<ulonglong2*>(seg);
            const uint32_t pairs = words / 2;
            for (uint32_t w0 = tid; w0 < pairs; w0 += blockDim.x * 8) {
                ulonglong2 v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (w0 + j * blockDim.x < pairs) v[j] = __ldcs(g2 + w0 + j * blockDim.x);
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (w0 + j * blockDim.x < pairs) s2[w0 + j * blockDim.x] = v[j];
            }
        } else {  // an odd number of words
            for (uint32_t w = tid; w < words; w += blockDim.x) seg[w] = gseg[w];
        }
        __syncthreads();
        constexpr int U = 8;  // entries per thread in flight
        for (uint32_t base = lo; base < hi; base += blockDim.x * U) {
          uint64_t ev[U];
          uint32_t pv[U];
#pragma unroll
          for (int j = 0; j < U; ++j) {
              const uint32_t k = base + j * blockDim.x + tid;
              ev[j] = 0;
              pv[j] = 0;
              if (k < hi) {
                  ev[j] = narrow ? reinterpret_cast<const uint32_t*>(ent)[k] : ent[k];
                  if (pay) pv[j] = pay[k];
              }
          }
          uint32_t fwd_mask = 0;
#pragma unroll
          for (int j = 0; j < U; ++j) {
            const uint32_t k = base + j * blockDim.x + tid;
            const bool v = k < hi;
            bool ok = false;
            const uint64_t e = ev[j];
            const uint32_t p = pv[j];
            if (v) {
                const uint32_t fp = static_cast<uint32_t>(e) & C::tag_mask;
                const uint64_t lb = (e >> C::bits) & (sb - 1);
                uint64_t* bw = seg + lb * WPB;
                uint64_t c[C::nchunks];
#pragma unroll
                for (int q = 0; q < C::nchunks; ++q) c[q] = bw[q];
                if constexpr (OP == SEG_INSERT)
                    ok = try_insert<C>(bw, c, fp, err);
                else if constexpr (OP == SEG_CONTAINS)
                    ok = has_tag<C>(c, fp);
                else
                    ok = try_remove<C>(bw, c, fp, err);
                if (ok && bitmap) atomicOr(&bitmap[p >> 5], 1u << (p & 31));
            }
            n_ok += ok ? 1u : 0u;
            // misses go to the next round (all of them in round 1; only inserts in round 2)
            if (v && !ok && (round == 1 || OP == SEG_INSERT)) fwd_mask |= 1u << j;
          }
          // one reservation per CTA and step: block-wide prefix sum of the forwards
          const uint32_t cnt = __popc(fwd_mask);
          const uint32_t incl = warp_inclusive_scan(cnt);
          if (lane == 31) s_warp[tid >> 5] = incl;
          __syncthreads();
          if (tid < 32) {
              const uint32_t x = tid < (blockDim.x >> 5) ? s_warp[tid] : 0u;
              const uint32_t xi = warp_inclusive_scan(x);
              if (tid < (blockDim.x >> 5)) s_warp[tid] = xi - x;
              if (tid == 31 && xi) s_base = atomicAdd(next_count, static_cast<unsigned long long>(xi));
          }
          __syncthreads();
          if (fwd_mask) {
              uint64_t o = s_base + s_warp[tid >> 5] + incl - cnt;
#pragma unroll
              for (int j = 0; j < U; ++j) {
                  if ((fwd_mask >> j) & 1u) {
                      const uint64_t e = ev[j];
                      const uint32_t fp = static_cast<uint32_t>(e) & C::tag_mask;
                      // the full bucket index from the segment (entries may be 4-byte)
                      uint64_t b = (s << sb_log2) | ((e >> C::bits) & (sb - 1));
                      uint32_t tg = fp;
                      if (fwd_other) {  // keyed by the other bucket, the tag in that bucket's form
                          b = alt_bucket<C>(b, fp, t.nb_mask);
                          tg = alt_tag<C>(fp);
                      }
                      next[o] = pack_entry<C>(b, tg);
                      if (pay) next_pay[o] = pv[j];
                      ++o;
                  }
              }
          }
          __syncthreads();  // s_warp / s_base reused by the next step
        }
        __syncthreads();
        if constexpr (OP != SEG_CONTAINS) {
            if (words % 2 == 0) {
                ulonglong2* g2 = reinterpret_cast<ulonglong2*>(gseg);
                const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(seg);
                for (uint32_t w = tid; w < words / 2; w += blockDim.x) __stcs(g2 + w, s2[w]);
            } else {
                for (uint32_t w = tid; w < words; w += blockDim.x) gseg[w] = seg[w];
            }
        }
        __syncthreads();
    }
    if constexpr (OP == SEG_INSERT) {
        flush_counter(&t.ctr[round == 2 ? CTR_SECONDARY : CTR_PRIMARY], n_ok);
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

// BFS for a list of keys whose two buckets were full (entries carry (alternate
// bucket, tag)), as a per-lane step machine that keeps one memory operation
// of every lane in flight: each iteration every lane issues exactly one load
// (its next entry, or a bucket) or one compare-and-swap, and only then are the
// results consumed, so a warp waits for one round trip per iteration however
// its lanes' keys diverge.  Per key: fetch the entry, snapshot the start
// bucket (i1 for an even tag, i2 for an odd one), then try the candidates in
// the reference's order (CuckooFilter.cuh:967-1018): candidate slot empty ->
// insert fp into the start bucket; else load the candidate's alternate
// bucket, copy the candidate there if it has room, and swap fp into the
// candidate's slot if the candidate is still there (else undo the copy and
// refresh the snapshot).  A failed compare-and-swap retries from the value it
// returned, as tryInsertAtBucket does.  A lane whose key is done takes the
// next key of its warp's share of the list.  Keys whose candidates all fail go
// to `dfs` for the DFS fallback.
// count_keys: add the keys to the evicting-insert counter (0 when an earlier
// eviction kernel counted them already).
template <class C>
__global__ void __launch_bounds__(256, C::nchunks <= 4 ? 3 : 2) k_evict_bfs_steps(DevTable t, const uint64_t* ent, const uint32_t* pay,
                                                         const unsigned long long* n_dev, uint32_t* bitmap,
                                                         uint64_t* dfs, uint32_t* dfs_pay,
                                                         unsigned long long* dfs_count, uint32_t count_keys) {
    constexpr uint32_t NC = (C::bs / 2) < 8 ? (C::bs / 2) : 8;
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
    // phase = the operation in flight
    enum : uint32_t { P_FETCH, P_SNAP, P_PROBE, P_INS_ALT, P_SWAP, P_INS_START };
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t m = *n_dev;
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
    const uint64_t wid = blockIdx.x * static_cast<uint64_t>(blockDim.x / 32) + threadIdx.x / 32;
    const uint64_t per = (m + nwarps - 1) / nwarps;
    uint64_t next = wid * per;  // warp-uniform cursor into the warp's share
    const uint64_t end = next + per < m ? next + per : m;
    uint32_t n_evk = 0, n_ok = 0, n_ev = 0, n_dup = 0;
    bool err = false;
    bool has = false;
    uint32_t phase = P_FETCH, fp = 0, i = 0, cand = 0, sh = 0, retries = 0;
    int sw = 0, w = 0;
    uint64_t idx = 0, e = 0, start = 0, ab = 0, exp = 0, des = 0;
    const uint64_t* addr = nullptr;  // load or compare-and-swap target
    uint64_t snap[C::nchunks];
#pragma unroll
    for (int q = 0; q < C::nchunks; ++q) snap[q] = 0;

    // Picks candidate i (or the next ones) from the snapshot and sets up its
    // first operation; returns 3 when all candidates are used up.
    auto select = [&]() -> int {
        for (; i < NC; ++i) {
            const uint32_t slot = static_cast<uint32_t>((static_cast<uint64_t>(fp) + 7ull * i) & (C::bs - 1));
            sw = static_cast<int>(slot / C::lanes_per_chunk);
            sh = (slot % C::lanes_per_chunk) * C::bits;
            cand = static_cast<uint32_t>((pick(snap, sw) >> sh) & lane_mask);
            if (cand == 0) {  // reference :980-985: the slot is free, insert fp into the start bucket
                if (plan_insert<C>(snap, fp, w, exp, des)) {
                    phase = P_INS_START;
                    addr = bucket_words<C>(t, start) + w;
                    return 0;
                }
                continue;
            }
            ab = alt_bucket<C>(start, cand, t.nb_mask);
            phase = P_PROBE;
            addr = bucket_words<C>(t, ab);
            return 0;
        }
        return 3;
    };

    for (;;) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !has);
        if (need) {
            if (!has) {
                const uint64_t k = next + __popc(need & lt_mask);
                if (k < end) {
                    has = true;
                    idx = k;
                    phase = P_FETCH;
                    addr = ent + k;
                    i = 0;
                    retries = 0;
                    ++n_evk;
                }
            }
            next += __popc(need);
        }
        if (__ballot_sync(0xFFFFFFFFu, has) == 0) break;
        // issue: one operation per lane, all in flight before any is consumed
        uint64_t ld[C::nchunks];
        uint64_t old = 0;
        const bool do_fetch = has && phase == P_FETCH;
        const bool do_load = has && (phase == P_SNAP || phase == P_PROBE);
        const bool do_cas = has && phase >= P_INS_ALT;
        if (do_fetch) ld[0] = __ldcs(reinterpret_cast<const unsigned long long*>(addr));
        if (do_load) load_rlx<C::bucket_bytes>(const_cast<uint64_t*>(addr), ld);
        if (do_cas) old = cas64(const_cast<uint64_t*>(addr), exp, des);
        // consume
        int outcome = 0;  // 1 stored, 2 stored by a swap, 3 candidates exhausted
        if (has) {
            switch (phase) {
                case P_FETCH: {
                    e = ld[0];
                    if (e & kDfsFlag) {  // BFS already failed for this key: straight to DFS
                        e &= ~kDfsFlag;
                        outcome = 3;
                        break;
                    }
                    fp = static_cast<uint32_t>(e) & C::tag_mask;
                    const uint64_t i2 = e >> C::bits;
                    const uint64_t i1 = alt_bucket<C>(i2, fp, t.nb_mask);
                    start = (fp & 1u) == 0 ? i1 : i2;
                    if ((fp & 1u) == 0) fp = alt_tag<C>(fp);  // the tag in the start bucket's form
                    phase = P_SNAP;
                    addr = bucket_words<C>(t, start);
                    break;
                }
                case P_SNAP:
#pragma unroll
                    for (int q = 0; q < C::nchunks; ++q) snap[q] = ld[q];
                    outcome = select();
                    break;
                case P_PROBE:
                    if (plan_insert<C>(ld, alt_tag<C>(cand), w, exp, des)) {
                        phase = P_INS_ALT;
                        addr = bucket_words<C>(t, ab) + w;
                    } else {
                        ++i;
                        outcome = select();
                    }
                    break;
                case P_INS_ALT:
                    if (old == exp) {  // the candidate is copied: swap fp into its slot
                        exp = pick(snap, sw);
                        des = (exp & ~(lane_mask << sh)) | (static_cast<uint64_t>(fp) << sh);
                        phase = P_SWAP;
                        addr = bucket_words<C>(t, start) + sw;
                    } else {  // the bucket changed: load it again
                        phase = P_PROBE;
                        addr = bucket_words<C>(t, ab);
                        if (++retries >= kCasRetryLimit) err = true;
                    }
                    break;
                case P_SWAP:
                    if (old == exp) {
                        outcome = 2;
                    } else if (((old >> sh) & lane_mask) == cand) {  // other slots of the word changed
                        put(snap, sw, old);
                        exp = old;
                        des = (old & ~(lane_mask << sh)) | (static_cast<uint64_t>(fp) << sh);
                        if (++retries >= kCasRetryLimit) err = true;
                    } else {  // the candidate moved: undo the copy, refresh the snapshot
                        if (!remove_from_pair<C>(t, ab, start, alt_tag<C>(cand), err)) ++n_dup;
                        ++i;
                        if (i == NC) {
                            outcome = 3;
                        } else {
                            phase = P_SNAP;
                            addr = bucket_words<C>(t, start);
                        }
                    }
                    break;
                default:  // P_INS_START
                    if (old == exp) {
                        outcome = 1;
                    } else {
                        put(snap, w, old);
                        if (plan_insert<C>(snap, fp, w, exp, des)) {
                            addr = bucket_words<C>(t, start) + w;
                            if (++retries >= kCasRetryLimit) err = true;
                        } else {
                            ++i;
                            outcome = select();
                        }
                    }
                    break;
            }
        }
        if (outcome == 1 || outcome == 2) {
            ++n_ok;
            if (outcome == 2) ++n_ev;
            record_chain(t, outcome == 2 ? 1u : 0u);
            if (bitmap) atomicOr(&bitmap[pay[idx] >> 5], 1u << (pay[idx] & 31));
        }
        const uint32_t push = __ballot_sync(0xFFFFFFFFu, outcome == 3);
        if (push) {
            unsigned long long base = 0;
            if (lane == static_cast<uint32_t>(__ffs(push) - 1))
                base = atomicAdd(dfs_count, static_cast<unsigned long long>(__popc(push)));
            base = __shfl_sync(0xFFFFFFFFu, base, __ffs(push) - 1);
            if (outcome == 3) {
                const uint64_t o = base + __popc(push & lt_mask);
                dfs[o] = e;
                if (dfs_pay) dfs_pay[o] = pay[idx];
            }
        }
        if (outcome) has = false;
        if (err) has = false;  // a retry bound was hit: stop this key, the host reports the error
    }
    flush_counter(&t.ctr[CTR_OCCUPIED], n_ok + n_dup);
    flush_counter(&t.ctr[CTR_DUP], n_dup);
    flush_counter(&t.ctr[CTR_EVICTED_INSERTS], count_keys ? n_evk : 0u);
    flush_counter(&t.ctr[CTR_EVICTIONS], n_ev);
    if (__any_sync(0xFFFFFFFFu, err) && lane == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// Alternate buckets a key may probe in the fast eviction pass before it is
// left to the step-machine BFS.
constexpr int kBfsFastProbes = 2;
__device__ __forceinline__ bool known_full(const uint32_t* full, uint64_t b) {
    return full && ((full[b >> 5] >> (b & 31)) & 1u);
}

// Empty slots of a bucket image (zero_lanes flags exactly the empty lanes).
template <class C>
__device__ __forceinline__ uint32_t empty_count(const uint64_t (&c)[C::nchunks]) {
    uint32_t n = 0;
#pragma unroll
    for (int j = 0; j < C::nchunks; ++j) n += __popcll(zero_lanes<C::bits>(c[j]));
    return n;
}

// Fast first pass of BFS eviction for a list of keys whose two buckets were
// full (entries carry (alternate bucket, tag)).  Every lane runs the same
// short sequence: load the entry, snapshot the start bucket (i1 for an even
// tag, i2 for an odd one), then take the reference's candidates in order
// (slots (fp + 7i) & (bs-1), CuckooFilter.cuh:967-1018): an empty candidate
// slot -> insert fp into the start bucket; a candidate whose alternate bucket
// is known full (`full`, one bit per bucket, set by the segment rounds and
// kept up to date here; buckets only fill during an insert) is passed over
// without a probe, exactly as the reference's probe of it would find no room;
// otherwise its alternate bucket is loaded, the candidate copied there and fp
// swapped into its slot if the slot still holds it (the copy is undone
// otherwise).  A key whose candidates all fail goes to DFS (flagged for the
// step machine when flag_ok, else through it); a key that used its P probes,
// or whose compare-and-swap found a bucket changed, goes to `rest`, where the
// step-machine BFS starts it over.  One key alone takes the reference's steps.
template <class C, int P>
__global__ void __launch_bounds__(256) k_evict_bfs_fast(DevTable t, const uint64_t* ent, const uint32_t* pay,
                                                        const unsigned long long* n_dev, uint32_t* bitmap,
                                                        uint64_t* rest, uint32_t* rest_pay,
                                                        unsigned long long* rest_count, uint32_t* full,
                                                        uint32_t flag_ok) {
    constexpr uint64_t lane_mask = C::bits == 32 ? 0xFFFFFFFFULL : ((1ULL << C::bits) - 1ULL);
    constexpr int NC = (C::bs / 2) < 8 ? (C::bs / 2) : 8;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t m = *n_dev;
    uint32_t n_evk = 0, n_ok = 0, n_ev = 0, n_dup = 0;
    bool err = false;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    // warp-uniform trip count: every lane reaches the ballot below
    for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * blockDim.x; base < m; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool v = i < m;
        bool done = false, stop = false;
        uint64_t e = 0;
        if (v) {
            ++n_evk;
            e = __ldcs(reinterpret_cast<const unsigned long long*>(ent) + i);
            const uint32_t fp0 = static_cast<uint32_t>(e) & C::tag_mask;
            const uint64_t i2 = e >> C::bits;
            const uint64_t i1 = alt_bucket<C>(i2, fp0, t.nb_mask);
            const uint64_t start = (fp0 & 1u) == 0 ? i1 : i2;
            const uint32_t fp = (fp0 & 1u) == 0 ? alt_tag<C>(fp0) : fp0;  // the tag in the start bucket's form
            uint64_t* sbw = bucket_words<C>(t, start);
            uint64_t snap[C::nchunks];
            load_rlx<C::bucket_bytes>(sbw, snap);
            uint32_t cand[NC];
            uint64_t ab[NC];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const uint32_t slot = static_cast<uint32_t>((static_cast<uint64_t>(fp) + 7ull * q) & (C::bs - 1));
                cand[q] = static_cast<uint32_t>(
                    (pick(snap, static_cast<int>(slot / C::lanes_per_chunk)) >> ((slot % C::lanes_per_chunk) * C::bits)) &
                    lane_mask);
                ab[q] = cand[q] ? alt_bucket<C>(start, cand[q], t.nb_mask) : start;
            }
            // candidates still worth trying: an empty slot, or an alternate
            // bucket not known to be full (bit q, in the reference's order)
            uint32_t avail = 0;
#pragma unroll
            for (int q = 0; q < NC; ++q)
                if (cand[q] == 0 || !known_full(full, ab[q])) avail |= 1u << q;
            // up to P probe rounds; in each, every lane loads its own next
            // candidate's alternate bucket, so a warp waits one round trip per
            // round however its lanes' candidates differ
            for (int r = 0; r < P && !stop && avail; ++r) {
                const int q = __ffs(avail) - 1;
                avail &= avail - 1;
                uint32_t cq = cand[0];
                uint64_t aq = ab[0];
#pragma unroll
                for (int j = 1; j < NC; ++j) {
                    cq = j == q ? cand[j] : cq;
                    aq = j == q ? ab[j] : aq;
                }
                if (cq == 0) {  // reference :980-985: the slot is free, insert fp into the start bucket
                    done = try_insert<C>(sbw, snap, fp, err);
                    if (done) record_chain(t, 0u);
                    stop = true;
                    break;
                }
                uint64_t* abw = bucket_words<C>(t, aq);
                uint64_t img[C::nchunks];
                load_rlx<C::bucket_bytes>(abw, img);
                int w;
                uint64_t exp, des;
                if (!plan_insert<C>(img, alt_tag<C>(cq), w, exp, des)) {  // no room: remember, next candidate
                    if (full) atomicOr(&full[aq >> 5], 1u << (aq & 31));
                    continue;
                }
                stop = true;
                if (cas64(abw + w, exp, des) != exp) break;  // the bucket changed: start over later
                if (full && empty_count<C>(img) == 1) atomicOr(&full[aq >> 5], 1u << (aq & 31));
                const uint32_t slot = static_cast<uint32_t>((static_cast<uint64_t>(fp) + 7ull * q) & (C::bs - 1));
                const int sw = static_cast<int>(slot / C::lanes_per_chunk);
                const int sh = static_cast<int>(slot % C::lanes_per_chunk) * C::bits;
                const uint64_t word = pick(snap, sw);
                const uint64_t swapped = (word & ~(lane_mask << sh)) | (static_cast<uint64_t>(fp) << sh);
                if (cas64(sbw + sw, word, swapped) == word) {
                    done = true;
                    ++n_ev;
                    record_chain(t, 1u);
                } else if (!remove_from_pair<C>(t, aq, start, alt_tag<C>(cq), err)) {
                    ++n_dup;  // the copy could not be taken back: an extra entry
                }
            }
            // probes used up with candidates left: the step machine takes the key
            if (!stop && avail) stop = true;
            if (done) {
                ++n_ok;
                if (bitmap) atomicOr(&bitmap[pay[i] >> 5], 1u << (pay[i] & 31));
            } else if (!stop && flag_ok) {
                e |= kDfsFlag;  // every candidate failed: BFS is over for this key
            }
        }
        const bool to_rest = v && !done;
        const uint32_t push = __ballot_sync(0xFFFFFFFFu, to_rest);
        if (push) {
            unsigned long long o = 0;
            if (lane == static_cast<uint32_t>(__ffs(push) - 1))
                o = atomicAdd(rest_count, static_cast<unsigned long long>(__popc(push)));
            o = __shfl_sync(0xFFFFFFFFu, o, __ffs(push) - 1);
            if (to_rest) {
                const uint64_t at = o + __popc(push & lt_mask);
                rest[at] = e;
                if (rest_pay) rest_pay[at] = pay[i];
            }
        }
    }
    flush_counter(&t.ctr[CTR_OCCUPIED], n_ok + n_dup);
    flush_counter(&t.ctr[CTR_DUP], n_dup);
    flush_counter(&t.ctr[CTR_EVICTED_INSERTS], n_evk);
    flush_counter(&t.ctr[CTR_EVICTIONS], n_ev);
    if (__any_sync(0xFFFFFFFFu, err) && lane == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// Eviction for the keys whose two buckets were full after both segment rounds
// (or, with `continued`, whose BFS candidates all failed); entries carry
// (alternate bucket, tag).  One key per thread, all lanes busy.
template <class C>
__global__ void __launch_bounds__(256) k_evict_list(DevTable t, const uint64_t* ent, const uint32_t* pay,
                                                    const unsigned long long* n_dev, uint32_t policy_bfs,
                                                    uint32_t max_ev, uint32_t* bitmap, uint32_t continued) {
    const uint64_t m = *n_dev;
    uint32_t n_evk = 0, n_fail = 0;
    EvictStats st;
    bool err = false;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t e = ent[i];
        const uint32_t fp = static_cast<uint32_t>(e) & C::tag_mask;
        const uint64_t i2 = e >> C::bits;
        const uint64_t i1 = alt_bucket<C>(i2, fp, t.nb_mask);
        const uint64_t start = (fp & 1u) == 0 ? i1 : i2;
        const uint64_t other = (fp & 1u) == 0 ? i2 : i1;
        const uint32_t sfp = (fp & 1u) == 0 ? alt_tag<C>(fp) : fp;  // the tag in the start bucket's form
        ++n_evk;
        const uint32_t before = st.evictions;
        const bool ok = policy_bfs ? evict_bfs<C>(t, sfp, start, other, max_ev, st, err)
                                   : evict_dfs<C>(t, sfp, start, other, max_ev, st, err);
        if (ok) record_chain(t, st.evictions - before);
        if (ok) {
            if (bitmap) {
                const uint32_t p = pay[i];
                atomicOr(&bitmap[p >> 5], 1u << (p & 31));
            }
        } else {
            ++n_fail;
        }
    }
    flush_counter(&t.ctr[CTR_OCCUPIED], n_evk - n_fail - st.lost + st.dup);
    flush_counter(&t.ctr[CTR_DUP], st.dup);
    flush_counter(&t.ctr[CTR_EVICTED_INSERTS], continued ? 0u : n_evk);
    flush_counter(&t.ctr[CTR_EVICTIONS], st.evictions);
    flush_counter(&t.ctr[CTR_FAILED], n_fail);
    flush_counter(&t.ctr[CTR_LOST], st.lost);
    if (__any_sync(0xFFFFFFFFu, err) && (threadIdx.x & 31) == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// Shared memory of k_seg_insert: the staged segment plus one slot mask per bucket.
template <class C>
constexpr size_t seg_insert_smem(int sb_log2) {
    return (static_cast<size_t>(1) << sb_log2) * (C::bucket_bytes + sizeof(SlotMask<C>));
}

template <class M>
__device__ __forceinline__ uint32_t popc_mask(M m) {
    if constexpr (sizeof(M) == 8)
        return static_cast<uint32_t>(__popcll(static_cast<unsigned long long>(m)));
    else
        return static_cast<uint32_t>(__popc(static_cast<unsigned int>(m)));
}

// Empty-slot mask of a bucket image (bit s set when slot s holds 0).
template <class C>
__device__ __forceinline__ SlotMask<C> empty_mask(const uint64_t* bw) {
    static_assert(C::bs <= 64, "slot masks hold at most 64 slots");
    SlotMask<C> m = 0;
#pragma unroll
    for (int j = 0; j < C::nchunks; ++j) {
        const uint64_t z = zero_lanes<C::bits>(bw[j]);
        if constexpr (C::bits == 16) {
            // the four lane flags (bits 15, 31, 47, 63) gathered into bits 48..51
            // by one multiply: flag l lands at 48 + l, every other product term
            // below bit 48 or above bit 63
            const uint64_t f = (z >> 15) & 0x0001000100010001ULL;
            const uint64_t g = (f * ((1ULL << 48) | (1ULL << 33) | (1ULL << 18) | (1ULL << 3))) >> 48;
            m |= static_cast<SlotMask<C>>(g & 0xFu) << (j * 4);
        } else {
#pragma unroll
            for (int l = 0; l < C::lanes_per_chunk; ++l)
                m |= static_cast<SlotMask<C>>((z >> (l * C::bits + C::bits - 1)) & 1u) << (j * C::lanes_per_chunk + l);
        }
    }
    return m;
}

// The slots a round capped at `cap` tags per bucket may claim in a bucket
// whose empty slots are `m`: the lowest-numbered cap - (tags present) of
// them (all of them when cap >= bs).
template <class C>
__device__ __forceinline__ SlotMask<C> claimable_slots(SlotMask<C> m, uint32_t cap) {
    using M = SlotMask<C>;
    constexpr M kAll = C::bs == 8 * sizeof(M) ? ~static_cast<M>(0) : ((static_cast<M>(1) << (C::bs % (8 * sizeof(M)))) - 1);
    if (cap >= static_cast<uint32_t>(C::bs)) return m;
    if (m == kAll) return (static_cast<M>(1) << cap) - 1;  // an empty bucket: its lowest `cap` slots
    const uint32_t present = C::bs - popc_mask(m);
    uint32_t quota = cap > present ? cap - present : 0u;
    SlotMask<C> r = 0;
    for (; m && quota; --quota) {
        const SlotMask<C> low = m & (~m + 1);
        r |= low;
        m ^= low;
    }
    return r;
}

// Position of the r-th set bit (r counted from 0) of a 16-bit mask that has
// more than r set bits: a binary search over the popcounts of its halves.
__device__ __forceinline__ uint32_t nth_set_bit16(uint32_t m, uint32_t r) {
    uint32_t pos = 0;
#pragma unroll
    for (int w = 8; w >= 1; w >>= 1) {
        const uint32_t c = __popc(m & ((1u << w) - 1u));
        const bool up = r >= c;
        r = up ? r - c : r;
        m = up ? m >> w : m;
        pos += up ? static_cast<uint32_t>(w) : 0u;
    }
    return pos;
}

// Keys per ranked claim batch: the claim words' 16-bit arrival counters are
// rebuilt from the staged segment after at most this many of a segment's keys,
// so no counter can wrap.
constexpr uint32_t kRankBatch = 32768;

// Segment-staged insert.  The staged segment carries one claim word per
// bucket, and a key whose bucket has room stores its tag there with a plain
// shared-memory store into the slot its claim gave it; a key whose bucket has
// no room goes to `next`, keyed by the key's other bucket when fwd_other is
// set, else unchanged (for eviction).
//
// ORDERED claims (RANKED false): the claim word is the mask of claimable
// slots, and a tag takes the first claimable slot circularly from slot
// align_down(fp & (bs-1), tagsPerWord) -- exactly the order in which the
// reference's tryInsertAtBucket scans words and lanes (CuckooFilter.cuh:
// 859-904) -- claimed with one atomic AND (only a claim of the same slot can
// fail and retry).  One key alone so takes the reference's slot.
//
// RANKED claims (batches of at least one key per bucket, whose slot order
// within a bucket is unspecified; buckets of at most 16 slots): the claim word
// holds the 16-bit claimable mask and, above it, a 16-bit arrival counter.
// One atomic add per key returns both: the key with arrival rank r takes the
// r-th claimable slot if there is one.  No claim fails or retries.
//
// cap: at most `cap` tags per bucket after the round (C::bs: no limit): only
// the lowest cap - (tags present) empty slots are claimable.  Capped rounds
// run only for batches of at least one key per bucket.
// PAY: entries carry payloads (key positions; `pay`, `next_pay` and `bitmap`
// are used only then).  NARROW: entries are 4-byte ((bucket within the
// segment) << bits | tag), else 8-byte (bucket << bits | tag).
template <class C, bool PAY, bool NARROW, bool RANKED>
__global__ void __launch_bounds__(kSegInsertThreads, 3) k_seg_insert(DevTable t, const uint64_t* ent, const uint32_t* pay,
                                                            const uint32_t* start, uint64_t nseg, int sb_log2,
                                                            int round, uint64_t* next, uint32_t* next_pay,
                                                            unsigned long long* next_count, uint32_t* bitmap,
                                                            int flags, uint32_t cap, int fwd_other,
                                                            uint32_t* full) {
    using M = SlotMask<C>;
    static_assert(!RANKED || C::bs <= 16, "ranked claims keep a 16-bit counter above a 16-slot mask");
    extern __shared__ __align__(16) uint64_t seg[];
    __shared__ uint32_t s_warp[32];
    __shared__ unsigned long long s_base;
    constexpr int WPB = C::bucket_bytes / 8;
    constexpr int TB = C::bits / 8;  // tag bytes
    constexpr int kMaskBits = 8 * sizeof(M);
    constexpr M kFull = C::bs == kMaskBits ? ~static_cast<M>(0) : ((static_cast<M>(1) << (C::bs % kMaskBits)) - 1);
    const uint32_t sb = 1u << sb_log2;
    const uint32_t seg_words = sb * WPB;
    M* mask = reinterpret_cast<M*>(seg + seg_words);
    uint8_t* seg_bytes = reinterpret_cast<uint8_t*>(seg);
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    const bool fresh = (flags & 2) != 0;  // the table is all zeros: segments are staged as zeros
    // the segment arrives by one bulk copy completing on this barrier
    __shared__ __align__(8) uint64_t seg_bar;
    if (tid == 0) {
        mbar_init(&seg_bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t seg_phase = 0;
    uint32_t n_ok = 0;
    for (uint64_t s = blockIdx.x; s < nseg; s += gridDim.x) {
        const uint32_t lo = start[s], hi = start[s + 1];
        if (lo == hi) continue;
        uint64_t* gseg = reinterpret_cast<uint64_t*>(t.buckets + (s << sb_log2) * C::bucket_bytes);
        // the last segment of a table whose bucket count is not a multiple of
        // the segment (AddSub and Offset policies) is partial
        const uint64_t left = t.nb_mask + 1 - (s << sb_log2);
        const uint32_t nbk = left < sb ? static_cast<uint32_t>(left) : static_cast<uint32_t>(sb);
        const uint32_t words = nbk * WPB;
        bool staged = true;
        if (tid == 0) bulk_wait_read();  // the previous segment's write-back has read the buffer
        if (fresh) {  // the table is all zeros: no load
            __syncthreads();
            for (uint32_t w = tid; w < words; w += blockDim.x) seg[w] = 0;
        } else if (words % 2 == 0) {  // a whole number of 16-byte units: one bulk copy
            if (tid == 0) {
                fence_proxy_async_smem();  // earlier accesses of this shared memory come first
                mbar_arrive_expect_tx(&seg_bar, words * 8u);
                bulk_g2s(seg, gseg, words * 8u, &seg_bar);
            }
            staged = mbar_wait(&seg_bar, seg_phase, kMbarPollLimit);
        } else {
            __syncthreads();
            for (uint32_t w = tid; w < words; w += blockDim.x) seg[w] = gseg[w];
        }
        if (__syncthreads_or(!staged)) {
            // the copy did not land within its poll bound: report it (the
            // host returns CF_ERR_DEVICE), give the copy in flight a second
            // bounded wait, and leave the segment untouched
            if (tid == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_WAIT_LIMIT);
            mbar_wait(&seg_bar, seg_phase, kMbarPollLimit);
            break;
        }
        if (!fresh && words % 2 == 0) seg_phase ^= 1u;
        // claim words from the staged segment (ranked: counters at zero)
        auto build_claims = [&]() {
            for (uint32_t b = tid; b < sb; b += blockDim.x)
                mask[b] = b < nbk ? claimable_slots<C>(empty_mask<C>(seg + static_cast<uint64_t>(b) * WPB), cap)
                                  : static_cast<M>(0);
        };
        if (fresh) {  // every bucket empty: the same claimable slots everywhere
            const M m0 = claimable_slots<C>(kFull, cap);
            for (uint32_t b = tid; b < sb; b += blockDim.x) mask[b] = b < nbk ? m0 : static_cast<M>(0);
        } else {
            build_claims();
        }
        __syncthreads();
        // entries per thread per step: 4-byte entries without payloads stay
        // 32-bit in registers, so twice as many fit (half the block barriers)
        constexpr int U = NARROW && !PAY ? 16 : 8;
        using E = typename std::conditional<NARROW, uint32_t, uint64_t>::type;
        for (uint32_t base = lo; base < hi; base += blockDim.x * U) {
            if constexpr (RANKED) {
                static_assert(kRankBatch % (kSegInsertThreads * U) == 0, "claim batches hold whole steps");
                if (base != lo && (base - lo) % kRankBatch == 0) {
                    // the previous step ended with a barrier: every tag is in the staged segment
                    build_claims();
                    __syncthreads();
                }
            }
            E ev[U];
            uint32_t pv[PAY ? U : 1];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                const uint32_t k = base + j * blockDim.x + tid;
                ev[j] = 0;
                if constexpr (PAY) pv[j] = 0;
                if (k < hi) {
                    if constexpr (NARROW)
                        ev[j] = reinterpret_cast<const uint32_t*>(ent)[k];
                    else
                        ev[j] = ent[k];
                    if constexpr (PAY) pv[j] = pay[k];
                }
            }
            uint32_t fwd_mask = 0;
#pragma unroll
            for (int j = 0; j < U; ++j) {
                const uint32_t k = base + j * blockDim.x + tid;
                if (k >= hi) continue;
                const uint32_t fp = static_cast<uint32_t>(ev[j]) & C::tag_mask;
                const uint32_t lb = static_cast<uint32_t>(static_cast<uint64_t>(ev[j]) >> C::bits) & (sb - 1);
                bool ok = false;
                uint32_t slot = 0;
                if constexpr (RANKED) {
                    const uint32_t old = atomicAdd(reinterpret_cast<uint32_t*>(&mask[lb]), 1u << 16);
                    const uint32_t m = old & 0xFFFFu;
                    const uint32_t r = old >> 16;
                    if (r < static_cast<uint32_t>(__popc(m))) {
                        // claimable slots are usually one run of bits (ranks
                        // fill a bucket in slot order): the r-th is low + r
                        const uint32_t low = static_cast<uint32_t>(__ffs(m)) - 1u;
                        const uint32_t run = m >> low;
                        slot = (run & (run + 1u)) == 0 ? low + r : nth_set_bit16(m, r);
                        ok = true;
                    }
                } else {
                    const uint32_t s0 = ((fp & (C::bs - 1)) / C::tpw) * C::tpw;
                    M m = mask[lb];
                    for (int it = 0; it < 64 && m; ++it) {
                        // first claimable slot circularly from s0
                        const M rot = s0 ? (((m >> s0) | (m << (C::bs - s0))) & kFull) : m;
                        uint32_t off;
                        if constexpr (sizeof(M) == 8)
                            off = __ffsll(static_cast<long long>(rot)) - 1;
                        else
                            off = __ffs(static_cast<int>(rot)) - 1;
                        slot = (s0 + off) & (C::bs - 1);
                        // claim the slot alone: only a claim of the same slot can fail
                        const M bit = static_cast<M>(1) << slot;
                        const M old = atomicAnd(&mask[lb], ~bit);
                        if (old & bit) {
                            ok = true;
                            break;
                        }
                        m = old;
                    }
                }
                if (ok) {
                    uint8_t* dst = seg_bytes + (static_cast<uint64_t>(lb) * C::bucket_bytes + slot * TB);
                    if constexpr (TB == 1)
                        *dst = static_cast<uint8_t>(fp);
                    else if constexpr (TB == 2)
                        *reinterpret_cast<uint16_t*>(dst) = static_cast<uint16_t>(fp);
                    else
                        *reinterpret_cast<uint32_t*>(dst) = fp;
                    ++n_ok;
                    if constexpr (PAY) atomicOr(&bitmap[pv[j] >> 5], 1u << (pv[j] & 31));
                } else {
                    fwd_mask |= 1u << j;
                }
            }
            // one reservation per CTA and step for the tags that found their bucket full
            const uint32_t cnt = __popc(fwd_mask);
            const uint32_t incl = warp_inclusive_scan(cnt);
            if (lane == 31) s_warp[tid >> 5] = incl;
            __syncthreads();
            if (tid < 32) {
                const uint32_t x = tid < (blockDim.x >> 5) ? s_warp[tid] : 0u;
                const uint32_t xi = warp_inclusive_scan(x);
                if (tid < (blockDim.x >> 5)) s_warp[tid] = xi - x;
                if (tid == 31 && xi) s_base = atomicAdd(next_count, static_cast<unsigned long long>(xi));
            }
            __syncthreads();
            if (fwd_mask) {
                uint64_t o = s_base + s_warp[tid >> 5] + incl - cnt;
#pragma unroll
                for (int j = 0; j < U; ++j) {
                    if ((fwd_mask >> j) & 1u) {
                        const uint32_t fp = static_cast<uint32_t>(ev[j]) & C::tag_mask;
                        // the full bucket index from the segment (entries may be 4-byte)
                        uint64_t b = (s << sb_log2) | ((static_cast<uint64_t>(ev[j]) >> C::bits) & (sb - 1));
                        uint32_t tg = fp;
                        if (fwd_other) {  // keyed by the other bucket, the tag in that bucket's form
                            b = alt_bucket<C>(b, fp, t.nb_mask);
                            tg = alt_tag<C>(fp);
                        }
                        next[o] = pack_entry<C>(b, tg);
                        if constexpr (PAY) next_pay[o] = pv[j];
                        ++o;
                    }
                }
            }
            __syncthreads();
        }
        if (full && cap >= static_cast<uint32_t>(C::bs)) {
            // one bit per bucket of the segment, set when an uncapped round
            // left it without an empty slot, read off its claim word: ranked,
            // arrivals reached the claimable slots; ordered, no claimable slot
            // is left.  (A capped round fills no bucket; its bits stay 0,
            // which only means "not known full".)  sb is a multiple of 32
            // whenever the bitmap is kept.
            for (uint32_t b0 = 0; b0 < sb; b0 += blockDim.x) {
                const uint32_t b = b0 + tid;
                bool is_full = false;
                if (b < nbk) {
                    const M cw = mask[b];
                    if constexpr (RANKED)
                        is_full = (static_cast<uint32_t>(cw) >> 16) >= static_cast<uint32_t>(__popc(cw & 0xFFFFu));
                    else
                        is_full = cw == 0;
                }
                const uint32_t word = __ballot_sync(0xFFFFFFFFu, is_full);
                if (lane == 0 && b < sb) full[((s << sb_log2) + b) >> 5] = word;
            }
        }
        if (words % 2 == 0) {
            // the segment leaves by one bulk copy, which reads the buffer
            // while the CTA moves on (the next load waits for that read)
            fence_proxy_async_smem();  // this thread's tag stores, before the copy reads them
            __syncthreads();
            if (tid == 0) {
                bulk_s2g(gseg, seg, words * 8u);
                bulk_commit();
            }
        } else {
            for (uint32_t w = tid; w < words; w += blockDim.x) gseg[w] = seg[w];
        }
        __syncthreads();
    }
    if (tid == 0) bulk_wait_all();
    flush_counter(&t.ctr[round == 2 ? CTR_SECONDARY : CTR_PRIMARY], n_ok);
    flush_counter(&t.ctr[CTR_OCCUPIED], n_ok);
}

// Round 2 by random access (few keys missed their primary bucket): entries
// carry (alternate bucket, tag).  insert: first empty slot of the alternate
// bucket, else eviction; lookup: tag present; delete: remove one copy.
template <class C, int OP>
__global__ void __launch_bounds__(256) k_list_random(DevTable t, const uint64_t* ent, const uint32_t* pay,
                                                     const unsigned long long* n_dev, uint32_t policy_bfs,
                                                     uint32_t max_ev, uint32_t* bitmap) {
    const uint64_t m = *n_dev;
    uint32_t n_sec = 0, n_evk = 0, n_fail = 0;
    EvictStats st;
    bool err = false;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t e = ent[i];
        const uint32_t fp = static_cast<uint32_t>(e) & C::tag_mask;
        const uint64_t i2 = e >> C::bits;
        uint64_t* bw = bucket_words<C>(t, i2);
        uint64_t c[C::nchunks];
        bool ok;
        if constexpr (OP == SEG_CONTAINS) {
            load_nc<C::bucket_bytes>(bw, c);
            ok = has_tag<C>(c, fp);
        } else {
            load_rlx<C::bucket_bytes>(bw, c);
            ok = OP == SEG_INSERT ? try_insert<C>(bw, c, fp, err) : try_remove<C>(bw, c, fp, err);
        }
        if constexpr (OP == SEG_INSERT) {
            if (ok) {
                ++n_sec;
            } else {
                const uint64_t i1 = alt_bucket<C>(i2, fp, t.nb_mask);
                const uint64_t start = (fp & 1u) == 0 ? i1 : i2;
                const uint64_t other = (fp & 1u) == 0 ? i2 : i1;
                const uint32_t sfp = (fp & 1u) == 0 ? alt_tag<C>(fp) : fp;  // the tag in the start bucket's form
                ++n_evk;
                ok = policy_bfs ? evict_bfs<C>(t, sfp, start, other, max_ev, st, err)
                                : evict_dfs<C>(t, sfp, start, other, max_ev, st, err);
                if (!ok) ++n_fail;
            }
        } else if constexpr (OP == SEG_DELETE) {
            n_sec += ok ? 1u : 0u;
        }
        if (ok && bitmap) {
            const uint32_t p = pay[i];
            atomicOr(&bitmap[p >> 5], 1u << (p & 31));
        }
    }
    if constexpr (OP == SEG_INSERT) {
        flush_counter(&t.ctr[CTR_OCCUPIED], n_sec + n_evk - n_fail - st.lost + st.dup);
        flush_counter(&t.ctr[CTR_DUP], st.dup);
        flush_counter(&t.ctr[CTR_SECONDARY], n_sec);
        flush_counter(&t.ctr[CTR_EVICTED_INSERTS], n_evk);
        flush_counter(&t.ctr[CTR_EVICTIONS], st.evictions);
        flush_counter(&t.ctr[CTR_FAILED], n_fail);
        flush_counter(&t.ctr[CTR_LOST], st.lost);
    } else if constexpr (OP == SEG_DELETE) {
        const uint32_t s = __reduce_add_sync(0xFFFFFFFFu, n_sec);
        if ((threadIdx.x & 31) == 0 && s) {
            atomicAdd(&t.ctr[CTR_REMOVED], static_cast<unsigned long long>(s));
            atomicAdd(&t.ctr[CTR_OCCUPIED], ~static_cast<unsigned long long>(s) + 1ull);
        }
    }
    if (__any_sync(0xFFFFFFFFu, err) && (threadIdx.x & 31) == 0) atomicOr(&t.ctr[CTR_ERROR], ERR_CAS_LIMIT);
}

// out[i] = bit i of the bitmap, for i < n.
static __global__ void k_bitmap_expand(const uint32_t* bitmap, uint64_t n, uint8_t* out) {
    for (uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; w * 32 < n;
         w += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t bits = bitmap[w];
        const uint64_t i0 = w * 32;
        if (i0 + 32 <= n && (reinterpret_cast<uintptr_t>(out + i0) & 15) == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint64_t lo = 0, hi = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    lo |= static_cast<uint64_t>((bits >> (16 * h + j)) & 1u) << (8 * j);
                    hi |= static_cast<uint64_t>((bits >> (16 * h + 8 + j)) & 1u) << (8 * j);
                }
                asm volatile("st.global.cs.v2.u64 [%0], {%1,%2};" ::"l"(out + i0 + 16 * h), "l"(lo), "l"(hi)
                             : "memory");
            }
        } else {
            for (uint64_t i = i0; i < n && i < i0 + 32; ++i) out[i] = static_cast<uint8_t>((bits >> (i - i0)) & 1u);
        }
    }
}

}  // namespace cfb
