// cf_shard.cu -- grouping a device key batch by shard: the exchange step of
// the hash-partitioned multi-GPU form (declared in include/cuckoo_b200.h).
//
// The reference's multi-GPU filter (CuckooFilterMultiGPU.cuh) sends key k to
// GPU hash64(k) % numGPUs (its Partitioner, :44-50), groups each GPU's input
// by destination with a multisplit (:226-234), exchanges the groups all-to-all
// (:247-254) and sends per-key results back the same way (:292-312).  Here
// the grouping is two HBM passes over the batch:
//   1. k_shard_hist: each CTA counts the keys of its contiguous share per shard
//      (warp-aggregated shared-memory atomics: the lanes of a warp that agree
//      on a shard add once);
//   2. k_scan_u32 over the (shard, CTA) counts, shard-major, gives every CTA
//      the start of its run inside every shard's group;
//   3. k_shard_scatter: each CTA re-reads its share and writes key and batch
//      position to its runs (one shared-memory cursor per shard, advanced
//      once per warp and shard).
// Per-key results come back in group order; k_shard_unpartition writes them
// to their batch positions.  All launches are stream-ordered and allocate
// nothing, so the calls can sit in a CUDA graph.
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
constexpr uint64_t kShMinShare = 8192;  // keys per CTA at least
constexpr uint32_t kShMaxGrid = 1184;   // 148 SMs x 8

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

// The shard of a key: the filter's 64-bit hash of the key (remixed for
// CF_SHARD_REMIXED) modulo the shard count.
template <int KB>
__device__ __forceinline__ uint32_t shard_of(uint64_t key, uint32_t ns, uint32_t routing) {
    const uint64_t h = hash_key<KB>(key);
    return static_cast<uint32_t>((routing == CF_SHARD_REMIXED ? remix64(h) : h) % ns);
}

template <int KB>
__global__ void __launch_bounds__(kShThreads) k_shard_hist(const void* keys, uint64_t n, uint32_t ns, uint32_t routing,
                                                           uint64_t share, uint32_t* hist) {
    __shared__ uint32_t cnt[kShMaxShards];
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t lo = blockIdx.x * share;
    const uint64_t hi = lo + share < n ? lo + share : n;
    for (uint64_t base = lo; base < hi; base += blockDim.x) {  // uniform trip count within the CTA
        const uint64_t i = base + threadIdx.x;
        const bool v = i < hi;
        const uint32_t d = v ? shard_of<KB>(sh_load<KB>(keys, i), ns, routing) : ns;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        if (v && lane == static_cast<uint32_t>(__ffs(peers) - 1)) atomicAdd(&cnt[d], static_cast<uint32_t>(__popc(peers)));
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) hist[static_cast<uint64_t>(d) * gridDim.x + blockIdx.x] = cnt[d];
}

template <int KB>
__global__ void __launch_bounds__(kShThreads) k_shard_scatter(const void* keys, uint64_t n, uint32_t ns,
                                                              uint32_t routing, uint64_t share, const uint32_t* offs,
                                                              void* out_keys, uint32_t* out_pos) {
    using Key = typename std::conditional<KB == 8, uint64_t, uint32_t>::type;
    __shared__ uint32_t cur[kShMaxShards];
    for (uint32_t d = threadIdx.x; d < ns; d += blockDim.x) cur[d] = offs[static_cast<uint64_t>(d) * gridDim.x + blockIdx.x];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t lo = blockIdx.x * share;
    const uint64_t hi = lo + share < n ? lo + share : n;
    for (uint64_t base = lo; base < hi; base += blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const bool v = i < hi;
        const uint64_t key = v ? sh_load<KB>(keys, i) : 0;
        const uint32_t d = v ? shard_of<KB>(key, ns, routing) : ns;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const int leader = __ffs(peers) - 1;
        uint32_t at = 0;
        if (v && static_cast<int>(lane) == leader) at = atomicAdd(&cur[d], static_cast<uint32_t>(__popc(peers)));
        at = __shfl_sync(0xFFFFFFFFu, at, leader) + static_cast<uint32_t>(__popc(peers & lt_mask));
        if (v) {
            static_cast<Key*>(out_keys)[at] = static_cast<Key>(key);
            out_pos[at] = static_cast<uint32_t>(i);
        }
    }
}

__global__ void k_shard_unpartition(const uint8_t* __restrict__ grouped, const uint32_t* __restrict__ pos, uint64_t n,
                                    uint8_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[__ldcs(pos + i)] = __ldcs(grouped + i);
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

uint32_t shard_grid(uint64_t n) {
    const uint64_t g = (n + kShMinShare - 1) / kShMinShare;
    return static_cast<uint32_t>(g < 1 ? 1 : g > kShMaxGrid ? kShMaxGrid : g);
}

}  // namespace

extern "C" {

uint64_t cf_shard_workspace_bytes(uint64_t n, uint32_t num_shards) {
    if (num_shards == 0 || num_shards > kShMaxShards) return 0;
    return (static_cast<uint64_t>(shard_grid(n)) * num_shards * 4 + 255) & ~255ull;
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
    const uint64_t share = (n + grid - 1) / grid;
    uint32_t* hist = static_cast<uint32_t*>(d_workspace);
    const uint32_t cells = grid * num_shards;
    if (key_bytes == 8)
        k_shard_hist<8><<<grid, kShThreads, 0, s>>>(d_keys, n, num_shards, routing, share, hist);
    else
        k_shard_hist<4><<<grid, kShThreads, 0, s>>>(d_keys, n, num_shards, routing, share, hist);
    CF_COUNT_LAUNCH();
    k_scan_u32<<<1, 1024, 0, s>>>(hist, cells);
    CF_COUNT_LAUNCH();
    if (key_bytes == 8)
        k_shard_scatter<8><<<grid, kShThreads, 0, s>>>(d_keys, n, num_shards, routing, share, hist, d_out_keys,
                                                        d_out_pos);
    else
        k_shard_scatter<4><<<grid, kShThreads, 0, s>>>(d_keys, n, num_shards, routing, share, hist, d_out_keys,
                                                        d_out_pos);
    CF_COUNT_LAUNCH();
    k_shard_counts<<<1, kShThreads, 0, s>>>(hist, grid, num_shards, n, d_counts);
    CF_COUNT_LAUNCH();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CF_OK : api_cuda_fail(e, "shard partition launch");
}

int cf_shard_unpartition(const uint8_t* d_grouped, const uint32_t* d_pos, uint64_t n, uint8_t* d_out, void* stream) {
    if (n == 0) return CF_OK;
    if (!d_grouped || !d_pos || !d_out) return api_fail(CF_ERR_INVALID, "grouped, pos or out is NULL with n > 0");
    const uint64_t blocks = (n + 255) / 256;
    k_shard_unpartition<<<static_cast<unsigned>(blocks < 4736 ? blocks : 4736), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_grouped, d_pos, n, d_out);
    CF_COUNT_LAUNCH();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CF_OK : api_cuda_fail(e, "shard unpartition launch");
}

}  // extern "C"
