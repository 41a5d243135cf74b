// cf_registry.cuh -- runtime dispatch from a cf_config to compiled kernels.
//
// The reference fixes every parameter at compile time (CuckooConfig,
// CuckooFilter.cuh:44-74).  Here key width, tag width and bucket size select a
// compiled kernel family; eviction policy, maxEvictions and blockSize are
// runtime arguments of those kernels.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <vector>

#include "cf_kernels.cuh"
#include "cf_region.cuh"
#include "cf_segmented.cuh"

namespace cfb {

// Kernels launched by this library since load (all filters, all devices);
// read through cf_launch_count().
inline std::atomic<unsigned long long>& launch_counter() {
    static std::atomic<unsigned long long> c{0};
    return c;
}
#define CF_COUNT_LAUNCH() (::cfb::launch_counter().fetch_add(1, std::memory_order_relaxed))

// Geometry of the segment-staged path for one filter.
struct SegGeom {
    int sb_log2;     // log2 buckets per segment
    int seg_shift;   // packed entry >> seg_shift = segment id
    int passes;      // radix passes (8-bit digits) over the segment id
    uint64_t nseg;   // segments
};

// Device workspace of the segment-staged path for a chunk of `cap` keys.
struct SegWork {
    uint64_t* ent[2];
    uint32_t* pay[2];
    uint32_t* hist;   // kRadix * max(rs_grid)
    uint32_t* start;  // nseg + 1
    unsigned long long* cnt;   // list lengths (5 used; 8 allocated)
    unsigned long long* h_cnt; // pinned mirror
    uint32_t* bitmap;          // cap / 32 words
    // Known-full buckets of the table, one bit per bucket (full_words words),
    // written by the segment insert rounds and read by eviction; null when
    // not kept (buckets of more than 64 slots, segments of fewer than 32
    // buckets, or the fixed scratch of cf_insert_sorted_noalloc).
    uint32_t* full;
    uint64_t full_words;
    uint64_t cap;
    int rs_grid[3];  // radix CTAs per payload mode (one wave of that scatter kernel)
    int sms;       // streaming multiprocessors
    uint64_t round2_segmented_min;  // list length from which round 2 is segment-staged
    uint32_t round1_cap;            // CF_OPT_ROUND1_CAP (0 = automatic)
    int rg_grid;   // CTAs of the region partition kernels (hist entries: kRgMaxRegions * rg_grid)
    // Insert into a table known to be all zeros: the first segment round
    // stages zeroed segments instead of loading them.
    bool fresh;
};

// Geometry of the region-staged path: region = bucket >> rl, nreg regions.
struct RegionGeom {
    int rl;
    uint32_t nreg;
};

// Dynamic shared memory limit of k_rg_gather (one bit per key of a chunk).
constexpr int kRgGatherMaxSmem = 160 * 1024;

// The eviction kernels run this many waves of CTAs (each warp takes an equal
// share of the list; more, smaller shares were measured faster on B200).
constexpr int kEvictGridWaves = 4;
// Slots of each bucket (in sixteenths) that the first round of a large
// segment-staged insert leaves free for the second round.
constexpr uint32_t kRound1SlackSixteenths = 3;

// Keys per thread of each batch kernel.
constexpr int kContainsKPT = 4;
constexpr int kDeleteKPT = 4;
constexpr int kInsertKPT = 2;

enum KernelId : int { KID_CONTAINS = 0, KID_DELETE = 1, KID_INSERT = 2, KID_COUNT_KERNELS = 3 };

struct LaunchCfg {
    cudaStream_t stream;
    int block;
    int max_grid;        // persistent grid for this kernel and block size
    int kpt = 0;         // keys per thread of the lookup kernel (1, 2, 4; 0 = kContainsKPT)
    int width = 1;       // lanes per key of lookups and deletes (CF_OPT_PROBE_WIDTH; 1 = one lane per key)
    bool full_grid = true;   // one tile per CTA instead of a persistent grid
};

struct OpsTable {
    uint32_t key_bytes, bits, bucket_size, word_bytes, alt_policy;
    uint32_t bucket_bytes;
    int kpt[KID_COUNT_KERNELS];
    uint32_t coop_widths;  // CF_OPT_PROBE_WIDTH values above 1 this geometry supports (bit log2(W))
    cudaError_t (*contains)(const DevTable&, const void*, uint64_t, uint8_t*, const LaunchCfg&);
    cudaError_t (*remove)(const DevTable&, const void*, uint64_t, uint8_t*, const LaunchCfg&);
    cudaError_t (*insert)(const DevTable&, const void*, uint64_t, uint8_t*, const LaunchCfg&, uint32_t policy_bfs,
                          uint32_t max_ev);
    cudaError_t (*count)(const DevTable&, uint64_t nb, unsigned long long* result, const LaunchCfg&);
    cudaError_t (*probe)(const DevTable&, const void*, uint64_t, unsigned long long*, const LaunchCfg&);
    cudaError_t (*occupancy)(int kid, int block, int* blocks_per_sm);
    cudaError_t (*seg_chunk)(const DevTable&, const SegGeom&, const SegWork&, int op, const void* keys, uint64_t m,
                             uint8_t* out, cudaStream_t, uint32_t policy_bfs, uint32_t max_ev);
    cudaError_t (*rg_chunk)(const DevTable&, const RegionGeom&, const SegWork&, int op, const void* keys, uint64_t m,
                            uint8_t* out, cudaStream_t, uint32_t policy_bfs, uint32_t max_ev);
};

inline bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// Per-device launch attributes are remembered for device ordinals below this.
constexpr int kMaxDevices = 64;

// Raises the dynamic shared-memory limit of `Kernel` to `bytes`, once per device.
template <auto Kernel>
cudaError_t ensure_smem_attr(int bytes) {
    static bool set[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!set[dev]) {
        e = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        set[dev] = true;
    }
    return cudaSuccess;
}

// Blocks of `kernel` resident on one SM (at least 1).
template <class K>
int blocks_per_sm(K kernel, int threads, size_t smem) {
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, threads, smem) != cudaSuccess || bps < 1) bps = 1;
    return bps;
}

// CTAs of the radix scatter for payload mode PAY: one wave, at most two CTAs
// per SM (on B200 a 2^31-entry pass took 8.5 ms at two CTAs per SM against
// 9.6 ms at the three that fit).
template <int PAY>
cudaError_t rs_scatter_grid(int sms, int* grid) {
    cudaError_t e = ensure_smem_attr<k_rs_scatter<PAY>>(rs_scatter_smem<PAY>());
    if (e != cudaSuccess) return e;
    static const int bps = blocks_per_sm(k_rs_scatter<PAY>, kRsThreads, rs_scatter_smem<PAY>());
    *grid = sms * (bps < 2 ? bps : 2);
    return cudaSuccess;
}

// One tile of block * kpt keys per CTA (kernels still stride if the batch
// needs more than 2^31 - 1 CTAs).
inline int full_grid_for(uint64_t n, int block, int kpt) {
    const uint64_t tile = static_cast<uint64_t>(block) * kpt;
    const uint64_t tiles = (n + tile - 1) / tile;
    return static_cast<int>(tiles < 0x7FFFFFFFull ? tiles : 0x7FFFFFFFull);
}

inline int grid_for(uint64_t n, int block, int kpt, int max_grid) {
    const uint64_t tile = static_cast<uint64_t>(block) * kpt;
    const uint64_t tiles = (n + tile - 1) / tile;
    return static_cast<int>(tiles < static_cast<uint64_t>(max_grid) ? tiles : max_grid);
}

template <class C, int KPT>
constexpr uintptr_t key_vec_align() {
    return (KPT * C::key_bytes) < 32 ? (KPT * C::key_bytes) : 32;
}

template <class C>
struct Launchers {
    using Key = typename C::Key;
    // keys per thread; buckets wider than 64 bytes keep fewer in flight so
    // their images stay in registers
    static constexpr int CKPT = C::bucket_bytes > 128 ? 1 : C::bucket_bytes > 64 ? 2 : kContainsKPT;
    static constexpr int DKPT = C::bucket_bytes > 64 ? 1 : kDeleteKPT;
    static constexpr int IKPT = C::bucket_bytes > 64 ? 1 : kInsertKPT;

    template <int K>
    static cudaError_t contains_k(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        const int grid = L.full_grid ? full_grid_for(n, L.block, K) : grid_for(n, L.block, K, L.max_grid);
        { k_contains<C, K><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                         aligned(keys, key_vec_align<C, K>()), aligned(out, K)); CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }
    // warp-cooperative lookups and deletes: W lanes per key, kCoopKPT keys per group
    static constexpr int kCoopKPT = 4;
    template <int W>
    static cudaError_t contains_w(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        if constexpr (CoopGeom<C, W>::ok) {
            const int groups = L.block / W;
            const int grid = L.full_grid ? full_grid_for(n, groups, kCoopKPT) : grid_for(n, groups, kCoopKPT, L.max_grid);
            { k_contains_coop<C, kCoopKPT, W><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                                             aligned(out, kCoopKPT)); CF_COUNT_LAUNCH(); }
            return cudaGetLastError();
        } else {
            return cudaErrorInvalidValue;
        }
    }
    template <int W>
    static cudaError_t remove_w(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        if constexpr (CoopGeom<C, W>::ok) {
            const int groups = L.block / W;
            const int grid = L.full_grid ? full_grid_for(n, groups, kCoopKPT) : grid_for(n, groups, kCoopKPT, L.max_grid);
            { k_delete_coop<C, kCoopKPT, W><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                                           aligned(out, kCoopKPT)); CF_COUNT_LAUNCH(); }
            return cudaGetLastError();
        } else {
            return cudaErrorInvalidValue;
        }
    }
    // the probe widths this geometry supports: bit log2(W) set for W lanes per key
    static constexpr uint32_t coop_widths() {
        return (CoopGeom<C, 2>::ok ? 1u << 1 : 0u) | (CoopGeom<C, 4>::ok ? 1u << 2 : 0u) |
               (CoopGeom<C, 8>::ok ? 1u << 3 : 0u) | (CoopGeom<C, 16>::ok ? 1u << 4 : 0u) |
               (CoopGeom<C, 32>::ok ? 1u << 5 : 0u);
    }
    static cudaError_t contains(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        if (n == 0) return cudaSuccess;
        switch (L.width) {
            case 2: return contains_w<2>(t, keys, n, out, L);
            case 4: return contains_w<4>(t, keys, n, out, L);
            case 8: return contains_w<8>(t, keys, n, out, L);
            case 16: return contains_w<16>(t, keys, n, out, L);
            case 32: return contains_w<32>(t, keys, n, out, L);
            default: break;
        }
        switch (L.kpt) {
            case 1: return contains_k<1>(t, keys, n, out, L);
            case 2: return contains_k<2>(t, keys, n, out, L);
            default: return contains_k<CKPT>(t, keys, n, out, L);
        }
    }
    static cudaError_t remove(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        if (n == 0) return cudaSuccess;
        switch (L.width) {
            case 2: return remove_w<2>(t, keys, n, out, L);
            case 4: return remove_w<4>(t, keys, n, out, L);
            case 8: return remove_w<8>(t, keys, n, out, L);
            case 16: return remove_w<16>(t, keys, n, out, L);
            case 32: return remove_w<32>(t, keys, n, out, L);
            default: break;
        }
        constexpr int K = DKPT;
        const int grid = L.full_grid ? full_grid_for(n, L.block, K) : grid_for(n, L.block, K, L.max_grid);
        { k_delete<C, K><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                       aligned(keys, key_vec_align<C, K>()), aligned(out, K)); CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }
    static cudaError_t insert(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L,
                              uint32_t policy_bfs, uint32_t max_ev) {
        if (n == 0) return cudaSuccess;
        constexpr int K = IKPT;
        const int grid = L.full_grid ? full_grid_for(n, L.block, K) : grid_for(n, L.block, K, L.max_grid);
        { k_insert<C, K><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                       aligned(keys, key_vec_align<C, K>()), aligned(out, K),
                                                       policy_bfs, max_ev); CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }
    static cudaError_t count(const DevTable& t, uint64_t nb, unsigned long long* result, const LaunchCfg& L) {
        const int grid = grid_for(nb, L.block, 1, L.max_grid);
        { k_count_occupied<C><<<grid, L.block, 0, L.stream>>>(t, nb, result); CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }
    static cudaError_t probe(const DevTable& t, const void* keys, uint64_t n, unsigned long long* result,
                             const LaunchCfg& L) {
        if (n == 0) return cudaSuccess;
        const int grid = grid_for(n, L.block, 1, L.max_grid);
        { k_probe_count<C><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, result); CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }
    static cudaError_t occupancy(int kid, int block, int* bps) {
        switch (kid) {
            case KID_CONTAINS:
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_contains<C, CKPT>, block, 0);
            case KID_DELETE:
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_delete<C, DKPT>, block, 0);
            default:
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_insert<C, IKPT>, block, 0);
        }
    }

    // One radix pass over n items, scattered by the digit at `shift` into
    // ent[dst].  keys_mode: `src` is the key array; the histogram kernel hashes
    // each key once and writes its packed entry to ent[1], which the scatter
    // then reads (payload = the key's position).  Otherwise `src` is ent[from]
    // with payloads pay[from].  The items are sorted by the `order_bits`
    // segment bits below `shift` (the earlier passes' digits), whose order
    // the scatter keeps.  lo_bits >= 0 (the last pass; lo_bits == order_bits):
    // the histogram kernel also adds every item's segment into w.start.
    static cudaError_t rs_pass(bool keys_mode, bool payload, const DevTable& t, const void* src, int from, uint64_t n,
                               int shift, int order_bits, int dst, const SegWork& w, cudaStream_t s, int lo_bits,
                               int narrow) {
        const int pay = !payload ? 0 : keys_mode ? 1 : 2;
        const int grid = w.rs_grid[pay];
        const int hgrid = grid * kRsHistSub;
        const uint32_t hist_n = static_cast<uint32_t>(kRadix) * static_cast<uint32_t>(hgrid);
        const uint64_t* ent_src = keys_mode ? w.ent[1] : w.ent[from];
        const void* hsrc = keys_mode ? src : static_cast<const void*>(ent_src);
        uint64_t* hout = keys_mode ? w.ent[1] : nullptr;
        if (keys_mode && lo_bits >= 0)
            { k_rs_hist<C, true, true><<<hgrid, kRsHistThreads, 0, s>>>(hsrc, t.nb_mask, n, nullptr, shift, w.hist, hout,
                                                                     lo_bits, w.start); CF_COUNT_LAUNCH(); }
        else if (keys_mode)
            { k_rs_hist<C, true, false><<<hgrid, kRsHistThreads, 0, s>>>(hsrc, t.nb_mask, n, nullptr, shift, w.hist, hout,
                                                                      0, nullptr); CF_COUNT_LAUNCH(); }
        else if (lo_bits >= 0)
            { k_rs_hist<C, false, true><<<hgrid, kRsHistThreads, 0, s>>>(hsrc, t.nb_mask, n, nullptr, shift, w.hist,
                                                                      nullptr, lo_bits, w.start); CF_COUNT_LAUNCH(); }
        else
            { k_rs_hist<C, false, false><<<hgrid, kRsHistThreads, 0, s>>>(hsrc, t.nb_mask, n, nullptr, shift, w.hist,
                                                                       nullptr, 0, nullptr); CF_COUNT_LAUNCH(); }
        { k_scan_u32<<<1, 1024, 0, s>>>(w.hist, hist_n); CF_COUNT_LAUNCH(); }
        unsigned long long* err = t.ctr + CTR_ERROR;
        if (pay == 0)
            { k_rs_scatter<0><<<grid, kRsThreads, rs_scatter_smem<0>(), s>>>(ent_src, nullptr, n, nullptr, shift, order_bits, w.hist,
                                                                          w.ent[dst], nullptr, err, narrow); CF_COUNT_LAUNCH(); }
        else if (pay == 1)
            { k_rs_scatter<1><<<grid, kRsThreads, rs_scatter_smem<1>(), s>>>(ent_src, nullptr, n, nullptr, shift, order_bits, w.hist,
                                                                          w.ent[dst], w.pay[dst], err, narrow); CF_COUNT_LAUNCH(); }
        else
            { k_rs_scatter<2><<<grid, kRsThreads, rs_scatter_smem<2>(), s>>>(ent_src, w.pay[from], n, nullptr, shift,
                                                                          order_bits, w.hist, w.ent[dst], w.pay[dst], err, narrow); CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }

    // Sort n items by segment id; returns the index of the buffer holding the
    // result.  keys_mode: the source is the key array; otherwise ent/pay[from].
    // Up to two passes, the last pass also counts the segments, and
    // *have_start tells that w.start then holds every segment's first index.
    // Entries of the sorted result are 4-byte ((bucket within its segment) <<
    // bits | tag) when the segment starts are counted (at most two passes)
    // and that fits 32 bits; *narrow tells.
    static cudaError_t sort_by_segment(bool keys_mode, bool payload, const DevTable& t, const SegGeom& g,
                                       const SegWork& w, const void* keys, int from, uint64_t n, cudaStream_t s,
                                       int* result, bool* have_start, bool* narrow) {
        int cur = from;
        const bool count_segs = g.passes <= 2;
        *narrow = count_segs && g.sb_log2 + C::bits <= 32;
        if (count_segs) {
            cudaError_t e = cudaMemsetAsync(w.start, 0, (g.nseg + 1) * sizeof(uint32_t), s);
            if (e != cudaSuccess) return e;
        }
        for (int p = 0; p < g.passes; ++p) {
            const bool from_keys = keys_mode && p == 0;
            const int dst = from_keys ? 0 : 1 - cur;
            const int lo_bits = count_segs && p == g.passes - 1 ? kRadixBits * p : -1;
            cudaError_t e = rs_pass(from_keys, payload, t, from_keys ? keys : nullptr, cur, n,
                                    g.seg_shift + kRadixBits * p, kRadixBits * p, dst, w, s, lo_bits,
                                    *narrow && p == g.passes - 1 ? 1 : 0);
            if (e != cudaSuccess) return e;
            cur = dst;
        }
        if (count_segs) { k_scan_u32<<<1, 1024, 0, s>>>(w.start, static_cast<uint32_t>(g.nseg + 1)); CF_COUNT_LAUNCH(); }
        *result = cur;
        *have_start = count_segs;
        return cudaGetLastError();
    }

    // round 1: primary buckets, round 2: alternate buckets, round 3: primary
    // buckets again (inserts whose first round was capped).  The entries
    // left over go to ent/pay[1 - buf] with their count in w.cnt[round - 1]
    // (w.cnt[3] for round 3; w.cnt[2] is the eviction list's).
    static constexpr uint32_t round1_cap() { return C::bs - C::bs * kRound1SlackSixteenths / 16; }

    // Every kernel of a segment round has this signature (k_seg and k_seg_insert).
    using SegKernel = void (*)(DevTable, const uint64_t*, const uint32_t*, const uint32_t*, uint64_t, int, int,
                               uint64_t*, uint32_t*, unsigned long long*, uint32_t*, int, uint32_t, int, uint32_t*);

    // The k_seg_insert instantiation for a round (payloads, 4-byte entries,
    // ranked claims), with its dynamic shared-memory limit raised.
    template <bool RANKED>
    static cudaError_t seg_insert_kernel(bool payload, bool narrow, int smem, SegKernel* k) {
        cudaError_t e = cudaSuccess;
        if (payload && narrow) {
            e = ensure_smem_attr<k_seg_insert<C, true, true, RANKED>>(smem);
            *k = k_seg_insert<C, true, true, RANKED>;
        } else if (payload) {
            e = ensure_smem_attr<k_seg_insert<C, true, false, RANKED>>(smem);
            *k = k_seg_insert<C, true, false, RANKED>;
        } else if (narrow) {
            e = ensure_smem_attr<k_seg_insert<C, false, true, RANKED>>(smem);
            *k = k_seg_insert<C, false, true, RANKED>;
        } else {
            e = ensure_smem_attr<k_seg_insert<C, false, false, RANKED>>(smem);
            *k = k_seg_insert<C, false, false, RANKED>;
        }
        return e;
    }

    // ranked: inserts of a batch of at least one key per bucket claim slots
    // by arrival rank (buckets of at most 16 slots; see k_seg_insert).
    template <int OP>
    static cudaError_t seg_round(const DevTable& t, const SegGeom& g, const SegWork& w, int buf, bool payload,
                                 int round, uint64_t n, bool have_start, bool narrow, cudaStream_t s,
                                 uint32_t cap = C::bs, int fwd_other = -1, bool ranked = false, bool fresh = false) {
        if (fwd_other < 0) fwd_other = round == 1 ? 1 : 0;
        // inserts claim slots on a per-bucket mask of at most 64 bits, staged
        // beside the segment; buckets of more slots insert with
        // compare-and-swap on the staged words
        constexpr bool masked = OP == SEG_INSERT && C::bs <= 64;
        constexpr bool rankable = masked && C::bs <= 16;
        constexpr int kMaxSmem = masked ? kSegBytes + (kSegBytes / C::bucket_bytes) * sizeof(SlotMask<C>) : kSegBytes;
        const int smem = static_cast<int>(masked ? seg_insert_smem<C>(g.sb_log2)
                                                 : (1ull << g.sb_log2) * C::bucket_bytes);
        SegKernel kern = nullptr;
        cudaError_t e = cudaSuccess;
        if constexpr (!masked) {
            e = ensure_smem_attr<k_seg<C, OP>>(kMaxSmem);
            kern = k_seg<C, OP>;
        } else if constexpr (rankable) {
            e = ranked ? seg_insert_kernel<true>(payload, narrow, kMaxSmem, &kern)
                       : seg_insert_kernel<false>(payload, narrow, kMaxSmem, &kern);
        } else {
            e = seg_insert_kernel<false>(payload, narrow, kMaxSmem, &kern);
        }
        if (e != cudaSuccess) return e;
        if (!have_start) {
            const uint64_t bthreads = n / 8 + 1;  // 8 positions per thread
            const int bgrid = static_cast<int>((bthreads + 255) / 256 < 4096 ? (bthreads + 255) / 256 : 4096);
            { k_seg_bounds<<<bgrid, 256, 0, s>>>(w.ent[buf], n, nullptr, g.seg_shift, g.nseg, w.start); CF_COUNT_LAUNCH(); }
        }
        const int other = 1 - buf;
        // one CTA per segment (measured faster on B200 than one wave of CTAs
        // striding over the segments)
        const int grid = static_cast<int>(g.nseg < 0x7FFFFFFFull ? g.nseg : 0x7FFFFFFFull);
        const int threads = masked ? kSegInsertThreads : kSegThreads;
        { kern<<<grid, threads, smem, s>>>(t, w.ent[buf], payload ? w.pay[buf] : nullptr, w.start, g.nseg, g.sb_log2,
                                          round, w.ent[other], payload ? w.pay[other] : nullptr,
                                          &w.cnt[round == 3 ? 3 : round - 1], payload ? w.bitmap : nullptr,
                                          // k_seg: 4-byte entries; k_seg_insert: bit 1, the table is all zeros
                                          masked ? (fresh ? 2 : 0) : (narrow ? 1 : 0), cap, fwd_other,
                                          OP == SEG_INSERT ? w.full : nullptr);
          CF_COUNT_LAUNCH(); }
        return cudaGetLastError();
    }

    template <int OP>
    static cudaError_t seg_chunk_op(const DevTable& t, const SegGeom& g, const SegWork& w, const void* keys,
                                    uint64_t m, uint8_t* out, cudaStream_t s, uint32_t policy_bfs, uint32_t max_ev) {
        const bool payload = out != nullptr;
        // list lengths: round-1, round-2, eviction (DFS), round-3 and fast-eviction leftovers
        cudaError_t e = cudaMemsetAsync(w.cnt, 0, 5 * sizeof(unsigned long long), s);
        if (e == cudaSuccess && payload) e = cudaMemsetAsync(w.bitmap, 0, (m + 31) / 32 * 4, s);
        // known-full buckets: none known at the start of a batch
        if (e == cudaSuccess && OP == SEG_INSERT && w.full)
            e = cudaMemsetAsync(w.full, 0, w.full_words * sizeof(uint32_t), s);
        int a = 0;
        bool have_start = false, narrow = false;
        // Fills of at least one key per bucket: the first round leaves
        // 3/16 of each bucket free (kRound1SlackSixteenths), the second round sends the
        // keys that miss both buckets back to their primary bucket for a
        // third round, and only what misses that goes to eviction.  Far
        // fewer keys need eviction: 4.0 % of a 0.95 fill of 16-slot buckets
        // after two uncapped rounds, 2.0 % after the three capped ones.
        const uint32_t cap1 = OP != SEG_INSERT || C::bs > 64 ? C::bs
                              : w.round1_cap                 ? w.round1_cap
                              : m >= t.nb_mask + 1           ? round1_cap()
                                                             : C::bs;
        const bool round3 = cap1 < C::bs;
        // batches of at least one key per bucket: slot order within a bucket is unspecified
        const bool ranked = OP == SEG_INSERT && m >= t.nb_mask + 1;
        if (e == cudaSuccess) e = sort_by_segment(true, payload, t, g, w, keys, 0, m, s, &a, &have_start, &narrow);
        if (e == cudaSuccess)
            e = seg_round<OP>(t, g, w, a, payload, 1, m, have_start, narrow, s, cap1, 1, ranked,
                              OP == SEG_INSERT && w.fresh);
        // round 2: keys that missed their primary bucket, now in ent/pay[1 - a]
        if (e == cudaSuccess) e = cudaMemcpyAsync(w.h_cnt, w.cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return e;
        const uint64_t m2 = w.h_cnt[0];
        const int b = 1 - a;
        if (m2 > 0) {
            if (m2 >= w.round2_segmented_min) {
                int c = b;
                e = sort_by_segment(false, payload, t, g, w, nullptr, b, m2, s, &c, &have_start, &narrow);
                if (e == cudaSuccess) e = seg_round<OP>(t, g, w, c, payload, 2, m2, have_start, narrow, s, C::bs,
                                                        round3 ? 1 : 0, ranked);
                unsigned long long* left = &w.cnt[1];  // keys for eviction: ent/pay[1 - c], count *left
                bool evict = true;
                if (e == cudaSuccess && OP == SEG_INSERT && round3) {
                    if (e == cudaSuccess)
                        e = cudaMemcpyAsync(w.h_cnt, &w.cnt[1], sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                    const uint64_t m3 = e == cudaSuccess ? w.h_cnt[0] : 0;
                    evict = m3 > 0;
                    if (evict) {
                        int c3 = 1 - c;
                        e = sort_by_segment(false, payload, t, g, w, nullptr, 1 - c, m3, s, &c3, &have_start, &narrow);
                        if (e == cudaSuccess) e = seg_round<OP>(t, g, w, c3, payload, 3, m3, have_start, narrow, s,
                                                                C::bs, 1, ranked);
                        c = c3;
                        left = &w.cnt[3];
                    }
                }
                if (e == cudaSuccess && OP == SEG_INSERT && evict) {
                    uint32_t* bm = payload ? w.bitmap : nullptr;
                    static const int bfs_bps = blocks_per_sm(k_evict_bfs_steps<C>, 256, 0);
                    static const int list_bps = blocks_per_sm(k_evict_list<C>, 256, 0);
                    if (policy_bfs) {
                        // a lockstep pass over the first candidates, then the
                        // step machine for what it could not place, then DFS
                        static const int fast_bps = blocks_per_sm(k_evict_bfs_fast<C, kBfsFastProbes>, 256, 0);
                        uint32_t* p_in = payload ? w.pay[1 - c] : nullptr;
                        uint32_t* p_mid = payload ? w.pay[c] : nullptr;
                        // keys whose candidates all fail are flagged for DFS when
                        // entries leave bit 63 free
                        const int bucket_bits = t.nb_mask ? 64 - __builtin_clzll(t.nb_mask) : 0;
                        const uint32_t flag_ok = bucket_bits + C::bits <= 63 ? 1u : 0u;
                        { k_evict_bfs_fast<C, kBfsFastProbes><<<w.sms * fast_bps * kEvictGridWaves, 256, 0, s>>>(
                              t, w.ent[1 - c], p_in, left, bm, w.ent[c], p_mid, &w.cnt[4], w.full, flag_ok);
                          CF_COUNT_LAUNCH(); }
                        { k_evict_bfs_steps<C><<<w.sms * bfs_bps * kEvictGridWaves, 256, 0, s>>>(
                              t, w.ent[c], p_mid, &w.cnt[4], bm, w.ent[1 - c], p_in, &w.cnt[2], 0u); CF_COUNT_LAUNCH(); }
                        { k_evict_list<C><<<w.sms * list_bps * kEvictGridWaves, 256, 0, s>>>(t, w.ent[1 - c], p_in,
                                                                        &w.cnt[2], 0u, max_ev, bm, 1u); CF_COUNT_LAUNCH(); }
                    } else {
                        { k_evict_list<C><<<w.sms * list_bps * kEvictGridWaves, 256, 0, s>>>(t, w.ent[1 - c],
                                                                        payload ? w.pay[1 - c] : nullptr, left,
                                                                        0u, max_ev, bm, 0u); CF_COUNT_LAUNCH(); }
                    }
                }
            } else {
                const int lgrid = static_cast<int>((m2 + 255) / 256 < 8192 ? (m2 + 255) / 256 : 8192);
                { k_list_random<C, OP><<<lgrid, 256, 0, s>>>(t, w.ent[b], payload ? w.pay[b] : nullptr, &w.cnt[0],
                                                          policy_bfs, max_ev, payload ? w.bitmap : nullptr); CF_COUNT_LAUNCH(); }
            }
            if (e == cudaSuccess) e = cudaGetLastError();
        }
        if (e == cudaSuccess && payload) {
            const int xgrid = static_cast<int>(((m + 31) / 32 + 255) / 256 < 8192 ? ((m + 31) / 32 + 255) / 256 : 8192);
            { k_bitmap_expand<<<xgrid, 256, 0, s>>>(w.bitmap, m, out); CF_COUNT_LAUNCH(); }
            e = cudaGetLastError();
        }
        return e;
    }

    static cudaError_t seg_chunk(const DevTable& t, const SegGeom& g, const SegWork& w, int op, const void* keys,
                                 uint64_t m, uint8_t* out, cudaStream_t s, uint32_t policy_bfs, uint32_t max_ev) {
        switch (op) {
            case SEG_INSERT: return seg_chunk_op<SEG_INSERT>(t, g, w, keys, m, out, s, policy_bfs, max_ev);
            case SEG_CONTAINS: return seg_chunk_op<SEG_CONTAINS>(t, g, w, keys, m, out, s, policy_bfs, max_ev);
            default: return seg_chunk_op<SEG_DELETE>(t, g, w, keys, m, out, s, policy_bfs, max_ev);
        }
    }

    // One region partition pass: histogram, scan, scatter of `m` items
    // (keys, or ent/pay[from] with the count on the device) into ent/pay[dst].
    template <int MODE>
    static void rg_split(const DevTable& t, const RegionGeom& g, const SegWork& w, const void* src,
                         const uint32_t* src_pay, uint64_t m, const unsigned long long* m_dev, bool payload,
                         uint64_t* dst, uint32_t* dst_pay, cudaStream_t s) {
        const int grid = w.rg_grid;
        { k_rg_hist<C, MODE><<<grid, kRgThreads, 0, s>>>(src, t.nb_mask, m, m_dev, g.rl, g.nreg, w.hist); CF_COUNT_LAUNCH(); }
        { k_scan_u32<<<1, 1024, 0, s>>>(w.hist, g.nreg * static_cast<uint32_t>(grid)); CF_COUNT_LAUNCH(); }
        if (payload)
            { k_rg_scatter<C, MODE, true><<<grid, kRgThreads, 0, s>>>(src, src_pay, t.nb_mask, m, m_dev, g.rl, g.nreg,
                                                                    w.hist, dst, dst_pay); CF_COUNT_LAUNCH(); }
        else
            { k_rg_scatter<C, MODE, false><<<grid, kRgThreads, 0, s>>>(src, nullptr, t.nb_mask, m, m_dev, g.rl, g.nreg,
                                                                     w.hist, dst, nullptr); CF_COUNT_LAUNCH(); }
    }

    template <int OP>
    static void rg_probe(const DevTable& t, const SegWork& w, const uint64_t* ent, const uint32_t* pay, uint64_t m,
                         const unsigned long long* m_dev, int round, uint64_t* next, uint32_t* next_pay,
                         unsigned long long* next_count, uint32_t* bitmap, cudaStream_t s) {
        static const int bps = blocks_per_sm(k_rg_probe<C, OP>, kRgThreads, 0);
        { k_rg_probe<C, OP><<<w.sms * bps, kRgThreads, 0, s>>>(t, ent, pay, m, m_dev, round, next, next_pay, next_count,
                                                            bitmap); CF_COUNT_LAUNCH(); }
    }

    // A chunk of m keys through the region-staged path.  Lookups: one pass
    // with both buckets of every key.  Deletes and inserts: primary buckets,
    // then the misses by alternate bucket, then (insert) eviction.
    // ent/pay[0] and ent/pay[1] are adjacent buffers of w.cap entries each, so
    // a lookup's 2m entries fit from ent/pay[0] on.
    template <int OP>
    static cudaError_t rg_chunk_op(const DevTable& t, const RegionGeom& g, const SegWork& w, const void* keys,
                                   uint64_t m, uint8_t* out, cudaStream_t s, uint32_t policy_bfs, uint32_t max_ev) {
        const bool payload = OP == SEG_CONTAINS || out != nullptr;
        uint32_t* bm = payload ? w.bitmap : nullptr;
        cudaError_t e = cudaMemsetAsync(w.cnt, 0, 4 * sizeof(unsigned long long), s);
        if (e == cudaSuccess && payload) e = cudaMemsetAsync(w.bitmap, 0, (m + 31) / 32 * 4, s);
        if (e != cudaSuccess) return e;
        if constexpr (OP == SEG_CONTAINS) {
            // both buckets of every key in one partition pass; hit bits in entry
            // order (w.bitmap, 2m bits); per-chunk gather writes `out`
            rg_split<RG_KEYS_DUAL>(t, g, w, keys, nullptr, m, nullptr, true, w.ent[0], w.pay[0], s);
            static const int lk_bps = blocks_per_sm(k_rg_lookup<C>, kRgThreads, 0);
            { k_rg_lookup<C><<<w.sms * lk_bps, kRgThreads, 0, s>>>(t, w.ent[0], 2 * m, w.bitmap); CF_COUNT_LAUNCH(); }
            e = ensure_smem_attr<k_rg_gather>(kRgGatherMaxSmem);
            if (e != cudaSuccess) return e;
            const uint64_t per = (m + w.rg_grid - 1) / w.rg_grid;
            const uint64_t chunk = (per + kRgTile / 2 - 1) / (kRgTile / 2) * (kRgTile / 2);
            const int smem = static_cast<int>((chunk + 31) / 32 * 4);
            if (smem > kRgGatherMaxSmem) return cudaErrorInvalidValue;
            { k_rg_gather<<<w.rg_grid, kRgThreads, smem, s>>>(w.pay[0], w.bitmap, w.hist, g.nreg, m, 2 * m, out); CF_COUNT_LAUNCH(); }
            return cudaGetLastError();
        } else {
            uint32_t* p0 = payload ? w.pay[0] : nullptr;
            uint32_t* p1 = payload ? w.pay[1] : nullptr;
            rg_split<RG_KEYS>(t, g, w, keys, nullptr, m, nullptr, payload, w.ent[0], p0, s);
            rg_probe<OP>(t, w, w.ent[0], p0, m, nullptr, 1, w.ent[1], p1, &w.cnt[0], bm, s);
            rg_split<RG_ENT>(t, g, w, w.ent[1], p1, 0, &w.cnt[0], payload, w.ent[0], p0, s);
            rg_probe<OP>(t, w, w.ent[0], p0, 0, &w.cnt[0], 2, OP == SEG_INSERT ? w.ent[1] : nullptr,
                         OP == SEG_INSERT ? p1 : nullptr, &w.cnt[1], bm, s);
            if constexpr (OP == SEG_INSERT) {
                // keys whose two buckets are full: ent/pay[1], count cnt[1]
                static const int bfs_bps = blocks_per_sm(k_evict_bfs_steps<C>, 256, 0);
                static const int list_bps = blocks_per_sm(k_evict_list<C>, 256, 0);
                if (policy_bfs) {
                    { k_evict_bfs_steps<C><<<w.sms * bfs_bps * kEvictGridWaves, 256, 0, s>>>(t, w.ent[1], p1, &w.cnt[1], bm, w.ent[0], p0,
                                                                       &w.cnt[2], 1u); CF_COUNT_LAUNCH(); }
                    { k_evict_list<C><<<w.sms * list_bps * kEvictGridWaves, 256, 0, s>>>(t, w.ent[0], p0, &w.cnt[2], 0u, max_ev, bm, 1u); CF_COUNT_LAUNCH(); }
                } else {
                    { k_evict_list<C><<<w.sms * list_bps * kEvictGridWaves, 256, 0, s>>>(t, w.ent[1], p1, &w.cnt[1], 0u, max_ev, bm, 0u); CF_COUNT_LAUNCH(); }
                }
            }
        }
        e = cudaGetLastError();
        if (e == cudaSuccess && payload) {
            const int xgrid = static_cast<int>(((m + 31) / 32 + 255) / 256 < 8192 ? ((m + 31) / 32 + 255) / 256 : 8192);
            { k_bitmap_expand<<<xgrid, 256, 0, s>>>(w.bitmap, m, out); CF_COUNT_LAUNCH(); }
            e = cudaGetLastError();
        }
        return e;
    }

    static cudaError_t rg_chunk(const DevTable& t, const RegionGeom& g, const SegWork& w, int op, const void* keys,
                                uint64_t m, uint8_t* out, cudaStream_t s, uint32_t policy_bfs, uint32_t max_ev) {
        switch (op) {
            case SEG_INSERT: return rg_chunk_op<SEG_INSERT>(t, g, w, keys, m, out, s, policy_bfs, max_ev);
            case SEG_CONTAINS: return rg_chunk_op<SEG_CONTAINS>(t, g, w, keys, m, out, s, policy_bfs, max_ev);
            default: return rg_chunk_op<SEG_DELETE>(t, g, w, keys, m, out, s, policy_bfs, max_ev);
        }
    }

    static OpsTable table() {
        OpsTable o{};
        o.key_bytes = C::key_bytes;
        o.bits = C::bits;
        o.bucket_size = C::bs;
        o.word_bytes = C::word_bytes;
        o.alt_policy = C::alt_policy;
        o.bucket_bytes = C::bucket_bytes;
        o.kpt[KID_CONTAINS] = CKPT;
        o.kpt[KID_DELETE] = DKPT;
        o.kpt[KID_INSERT] = IKPT;
        o.coop_widths = coop_widths();
        o.contains = contains;
        o.remove = remove;
        o.insert = insert;
        o.count = count;
        o.probe = probe;
        o.occupancy = occupancy;
        o.seg_chunk = seg_chunk;
        o.rg_chunk = rg_chunk;
        return o;
    }
};

// Registration hooks, one per translation unit (tag width).
void register_bits8(std::vector<OpsTable>& v);
void register_bits16(std::vector<OpsTable>& v);
void register_bits32(std::vector<OpsTable>& v);

}  // namespace cfb
