// cf_shard.cu -- grouping a device key batch by shard: the exchange step of
// the hash-partitioned multi-GPU form (declared in include/cuckoo_b200.h).
//
// The reference's multi-GPU filter (CuckooFilterMultiGPU.cuh) sends key k to
// GPU hash64(k) % numGPUs (its Partitioner, :44-50), groups each GPU's input
// by destination with a multisplit (:226-234), exchanges the groups all-to-all
// (:247-254) and sends per-key results back the same way (:292-312).  Here
// the batch is cut into contiguous CTA shares of at most kShMaxShare keys and
// the grouping is two HBM passes:
//   1. k_shard_hist: each CTA hashes the keys of its share, counts them per
//      shard (lanes that agree on a shard meet through __match_any_sync and
//      their leader adds) and keeps each key's shard as one byte;
//   2. k_scan_u32 over the (shard, CTA) counts, shard-major, gives every CTA
//      the start of its run inside every shard's group;
//   3. k_shard_scatter: each CTA re-reads its share's keys and shard bytes
//      and writes key and batch position to its runs.  Up to 32 shards, a
//      warp ranks its keys with one ballot per shard (lane d keeps shard d's
//      count, and one atomic per warp and step moves every shard's cursor);
//      beyond 32, lanes that agree on a shard meet through __match_any_sync.
// The workspace holds the (shard, CTA) counts and the shard bytes.
// Per-key results come back in group order.  k_shard_unpartition turns them
// around share by share: run (d, c) holds only positions of share c, so CTA c
// gathers its runs' bytes into shared memory and writes its share of the
// output as one coalesced stretch.  All launches are stream-ordered and
// allocate nothing, so the calls can sit in a CUDA graph.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cuckoo_b200.h"
#include "cf_registry.cuh"

namespace cfb {
int api_fail(int status, const char* msg);
int api_cuda_fail(cudaError_t e, const char* what);
}  // namespace cfb

using namespace cfb;

namespace {

constexpr int kShThreads = 256;
constexpr uint32_t kShMaxShards = 256;
constexpr uint32_t kShBallotShards = 32;  // up to this many shards: ballot ranking
constexpr uint64_t kShMinShare = 8192;    // keys per CTA at least
constexpr uint64_t kShMaxShare = 32768;   // keys per CTA at most (a share's result bytes in shared memory)
constexpr uint32_t kShWideGrid = 1184;    // 148 SMs x 8: grid while shares stay under kShMaxShare
constexpr int kShU = 4;                   // keys per thread in flight

// Keys are read once: streaming loads.
template <int KB>
__device__ __forceinline__ uint64_t sh_load(const void* keys, uint64_t i) {
    if constexpr (KB == 8)
        return ld_once_u64(static_cast<const uint64_t*>(keys) + i);
    else
        return ld_once_u32(static_cast<const uint32_t*>(keys) + i);
}

// splitmix64's output function (Steele, Lea and Flood 2014; Vigna's
// constants): a bijective 64-bit mixer.
__device__ __forceinline__ uint64_t remix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// h % d for d <= 256 with 32-bit divisions only:
// h = hi * 2^32 + lo, so h % d = ((hi % d) * (2^32 % d) + lo % d) % d, and
// every intermediate stays below 2^17.
__device__ __forceinline__ uint32_t mod_small(uint64_t h, uint32_t d) {
    const uint32_t hi = static_cast<uint32_t>(h >> 32), lo = static_cast<uint32_t>(h);
    const uint32_t p32 = static_cast<uint32_t>((0x100000000ull) % d);  // uniform across the grid
    return ((hi % d) * p32 + lo % d) % d;
}

// The shard of a key: the filter's 64-bit hash of the key (remixed for
// CF_SHARD_REMIXED) modulo the shard count.
template <int KB>
__device__ __forceinline__ uint32_t shard_of(uint64_t key, uint32_t ns, uint32_t routing) {
    uint64_t h = hash_key<KB>(key);
    if (routing == CF_SHARD_REMIXED) h = remix64(h);
    return (ns & (ns - 1)) == 0 ? static_cast<uint32_t>(h) & (ns - 1) : mod_small(h, ns);
}

// Ballot ranking of one warp step (ns <= 32; d = ns for lanes without a key):
// *mask = the lanes with this lane's shard; returns, in lane e < ns, how many
// lanes have shard e.
__device__ __forceinline__ uint32_t ballot_rank(uint32_t d, uint32_t ns, uint32_t lane, uint32_t* mask) {
    uint32_t mine = 0, tot = 0;
    for (uint32_t e = 0; e < ns; ++e) {
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, d == e);
        if (d == e) mine = m;
        if (lane == e) tot = static_cast<uint32_t>(__popc(m));
    }
    *mask = mine;
    return tot;
}

template <int KB>
__global__ void __launch_bounds__(kShThreads) k_shard_hist(const void* keys, uint64_t n, uint32_t ns, uint32_t routing,
                                                           uint64_t share, uint32_t* hist, uint8_t* sid) {
    __shared__ uint32_t cnt[kShMaxShards];
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t lo = blockIdx.x * share;
    const uint64_t hi = lo + share < n ? lo + share : n;
    const uint64_t tile = static_cast<uint64_t>(kShU) * blockDim.x;
    for (uint64_t base = lo; base < hi; base += tile) {  // uniform trip count within the CTA
        uint64_t k[kShU];
#pragma unroll
        for (int j = 0; j < kShU; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            k[j] = i < hi ? sh_load<KB>(keys, i) : 0;
        }
#pragma unroll
        for (int j = 0; j < kShU; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            const bool v = i < hi;
            const uint32_t d = v ? shard_of<KB>(k[j], ns, routing) : ns;
            if (v) sid[i] = static_cast<uint8_t>(d);
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
            if (v && lane == static_cast<uint32_t>(__ffs(peers) - 1))
                atomicAdd(&cnt[d], static_cast<uint32_t>(__popc(peers)));
        }
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) hist[static_cast<uint64_t>(d) * gridDim.x + blockIdx.x] = cnt[d];
}

template <int KB>
__global__ void __launch_bounds__(kShThreads) k_shard_scatter(const void* keys, const uint8_t* __restrict__ sid,
                                                              uint64_t n, uint32_t ns, uint64_t share,
                                                              const uint32_t* offs, void* out_keys,
                                                              uint32_t* out_pos) {
    using Key = typename std::conditional<KB == 8, uint64_t, uint32_t>::type;
    __shared__ uint32_t cur[kShMaxShards];
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) cur[d] = offs[static_cast<uint64_t>(d) * gridDim.x + blockIdx.x];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const bool ballot = ns <= kShBallotShards;
    const uint64_t lo = blockIdx.x * share;
    const uint64_t hi = lo + share < n ? lo + share : n;
    const uint64_t tile = static_cast<uint64_t>(kShU) * blockDim.x;
    for (uint64_t base = lo; base < hi; base += tile) {
        uint64_t k[kShU];
        uint32_t ds[kShU];
#pragma unroll
        for (int j = 0; j < kShU; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            k[j] = i < hi ? sh_load<KB>(keys, i) : 0;
            ds[j] = i < hi ? __ldcs(sid + i) : ns;
        }
        // a warp's keys of one step keep their lane order inside each run
#pragma unroll
        for (int j = 0; j < kShU; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
            const bool v = i < hi && ds[j] < ns;  // a shard byte outside 0..ns-1 places nothing
            const uint32_t d = v ? ds[j] : ns;
            uint32_t at;
            if (ballot) {
                uint32_t m;
                const uint32_t tot = ballot_rank(d, ns, lane, &m);
                uint32_t start = 0;
                if (lane < ns && tot) start = atomicAdd(&cur[lane], tot);  // lane e moves shard e's cursor
                at = __shfl_sync(0xFFFFFFFFu, start, v ? d : 0) + static_cast<uint32_t>(__popc(m & lt_mask));
            } else {
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
                const int leader = __ffs(peers) - 1;
                uint32_t start = 0;
                if (v && static_cast<int>(lane) == leader) start = atomicAdd(&cur[d], static_cast<uint32_t>(__popc(peers)));
                at = __shfl_sync(0xFFFFFFFFu, start, leader) + static_cast<uint32_t>(__popc(peers & lt_mask));
            }
            if (v && at < n) {  // (at < n always holds while the shard bytes match the counts)
                static_cast<Key*>(out_keys)[at] = static_cast<Key>(k[j]);
                out_pos[at] = static_cast<uint32_t>(i);
            }
        }
    }
}

// CTA c: the bytes of runs (0, c) .. (ns-1, c) land at their positions inside
// share c, staged in shared memory, then share c of `out` is written in one
// coalesced stretch.  Positions outside share c and runs outside [0, n) (a
// workspace that does not hold this batch's partition) are skipped.
__global__ void __launch_bounds__(kShThreads) k_shard_unpartition(const uint8_t* __restrict__ grouped,
                                                                  const uint32_t* __restrict__ pos, uint64_t n,
                                                                  uint32_t ns, uint64_t share,
                                                                  const uint32_t* __restrict__ offs,
                                                                  uint8_t* __restrict__ out) {
    __shared__ uint8_t buf[kShMaxShare];
    const uint64_t G = gridDim.x, c = blockIdx.x;
    const uint64_t lo = c * share;
    const uint64_t hi = lo + share < n ? lo + share : n;
    const uint64_t cells = static_cast<uint64_t>(ns) * G;
    for (uint32_t d = 0; d < ns; ++d) {
        const uint64_t cell = static_cast<uint64_t>(d) * G + c;
        uint64_t a = offs[cell];
        uint64_t b = cell + 1 < cells ? offs[cell + 1] : n;
        if (b > n) b = n;
        if (a > b) a = b;
        for (uint64_t i0 = a; i0 < b; i0 += static_cast<uint64_t>(kShU) * blockDim.x) {
            uint32_t p[kShU];
            uint8_t g[kShU];
#pragma unroll
            for (int j = 0; j < kShU; ++j) {
                const uint64_t i = i0 + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
                p[j] = i < b ? __ldcs(pos + i) : 0u;
                g[j] = i < b ? __ldcs(grouped + i) : static_cast<uint8_t>(0);
            }
#pragma unroll
            for (int j = 0; j < kShU; ++j) {
                const uint64_t i = i0 + static_cast<uint64_t>(j) * blockDim.x + threadIdx.x;
                const uint64_t o = static_cast<uint64_t>(p[j]) - lo;  // wraps for p < lo
                if (i < b && o < hi - lo) buf[o] = g[j];
            }
        }
    }
    __syncthreads();
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) out[i] = buf[i - lo];
}

// Keys per shard from the scanned starts: shard d's group runs from the start
// of its first CTA's run to the start of shard d + 1's (n for the last shard).
__global__ void k_shard_counts(const uint32_t* starts, uint32_t grid, uint32_t ns, uint64_t n, uint64_t* counts) {
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) {
        const uint64_t a = starts[static_cast<uint64_t>(d) * grid];
        const uint64_t b = d + 1 < ns ? starts[static_cast<uint64_t>(d + 1) * grid] : n;
        counts[d] = b - a;
    }
}

// Keys per CTA: n spread over kShWideGrid CTAs, within [kShMinShare, kShMaxShare].
uint64_t shard_share(uint64_t n) {
    uint64_t s = (n + kShWideGrid - 1) / kShWideGrid;
    if (s < kShMinShare) s = kShMinShare;
    if (s > kShMaxShare) s = kShMaxShare;
    return s;
}

uint32_t shard_grid(uint64_t n) {
    const uint64_t s = shard_share(n);
    const uint64_t g = (n + s - 1) / s;
    return static_cast<uint32_t>(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

// Workspace: the (shard, CTA) counts (uint32, 256-byte aligned), then one
// shard byte per key.
uint64_t shard_counts_bytes(uint64_t n, uint32_t num_shards) {
    return (static_cast<uint64_t>(shard_grid(n)) * num_shards * 4 + 255) & ~255ull;
}

uint64_t cf_shard_workspace_bytes(uint64_t n, uint32_t num_shards) {
    if (num_shards == 0 || num_shards > kShMaxShards) return 0;
    return shard_counts_bytes(n, num_shards) + ((n + 255) & ~255ull);
}

int cf_shard_partition(const void* d_keys, uint64_t n, uint32_t key_bytes, uint32_t num_shards, uint32_t routing,
                       void* d_out_keys, uint32_t* d_out_pos, uint64_t* d_counts, void* d_workspace,
                       uint64_t workspace_bytes, void* stream) {
    if (key_bytes != 4 && key_bytes != 8) return api_fail(CF_ERR_INVALID, "key_bytes must be 4 or 8");
    if (routing != CF_SHARD_REFERENCE && routing != CF_SHARD_REMIXED)
        return api_fail(CF_ERR_INVALID, "routing must be CF_SHARD_REFERENCE or CF_SHARD_REMIXED");
    if (num_shards == 0 || num_shards > kShMaxShards) return api_fail(CF_ERR_INVALID, "num_shards must be 1..256");
    if (n > 0xFFFFFFFFull) return api_fail(CF_ERR_INVALID, "at most 2^32 - 1 keys per call (positions are 32-bit)");
    if (!d_counts || !d_workspace) return api_fail(CF_ERR_INVALID, "counts or workspace is NULL");
    if (n && (!d_keys || !d_out_keys || !d_out_pos))
        return api_fail(CF_ERR_INVALID, "keys, out_keys or out_pos is NULL with n > 0");
    if (workspace_bytes < cf_shard_workspace_bytes(n, num_shards))
        return api_fail(CF_ERR_INVALID, "workspace smaller than cf_shard_workspace_bytes(n, num_shards)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t grid = shard_grid(n);
    const uint64_t share = shard_share(n);
    uint32_t* hist = static_cast<uint32_t*>(d_workspace);
    uint8_t* sid = static_cast<uint8_t*>(d_workspace) + shard_counts_bytes(n, num_shards);
    const uint64_t cells = static_cast<uint64_t>(grid) * num_shards;
    if (key_bytes == 8)
        k_shard_hist<8><<<grid, kShThreads, 0, s>>>(d_keys, n, num_shards, routing, share, hist, sid);
    else
        k_shard_hist<4><<<grid, kShThreads, 0, s>>>(d_keys, n, num_shards, routing, share, hist, sid);
    CF_COUNT_LAUNCH();
    k_scan_u32<<<1, 1024, 0, s>>>(hist, static_cast<uint32_t>(cells));
    CF_COUNT_LAUNCH();
    if (key_bytes == 8)
        k_shard_scatter<8><<<grid, kShThreads, 0, s>>>(d_keys, sid, n, num_shards, share, hist, d_out_keys, d_out_pos);
    else
        k_shard_scatter<4><<<grid, kShThreads, 0, s>>>(d_keys, sid, n, num_shards, share, hist, d_out_keys, d_out_pos);
    CF_COUNT_LAUNCH();
    k_shard_counts<<<1, kShThreads, 0, s>>>(hist, grid, num_shards, n, d_counts);
    CF_COUNT_LAUNCH();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CF_OK : api_cuda_fail(e, "shard partition launch");
}

int cf_shard_unpartition(const uint8_t* d_grouped, const uint32_t* d_pos, uint64_t n, uint32_t num_shards,
                         const void* d_workspace, uint64_t workspace_bytes, uint8_t* d_out, void* stream) {
    if (num_shards == 0 || num_shards > kShMaxShards) return api_fail(CF_ERR_INVALID, "num_shards must be 1..256");
    if (n > 0xFFFFFFFFull) return api_fail(CF_ERR_INVALID, "at most 2^32 - 1 keys per call (positions are 32-bit)");
    if (n == 0) return CF_OK;
    if (!d_grouped || !d_pos || !d_out || !d_workspace)
        return api_fail(CF_ERR_INVALID, "grouped, pos, workspace or out is NULL with n > 0");
    if (workspace_bytes < cf_shard_workspace_bytes(n, num_shards))
        return api_fail(CF_ERR_INVALID, "workspace smaller than cf_shard_workspace_bytes(n, num_shards)");
    k_shard_unpartition<<<shard_grid(n), kShThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_grouped, d_pos, n, num_shards, shard_share(n), static_cast<const uint32_t*>(d_workspace), d_out);
    CF_COUNT_LAUNCH();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CF_OK : api_cuda_fail(e, "shard unpartition launch");
}

}  // extern "C"
