// cf_registry.cuh -- runtime dispatch from a cf_config to compiled kernels.
//
// The reference fixes every parameter at compile time (CuckooConfig,
// CuckooFilter.cuh:44-74).  Here key width, tag width and bucket size select a
// compiled kernel family; eviction policy, maxEvictions and blockSize are
// runtime arguments of those kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cf_kernels.cuh"

namespace cfb {

// Keys per thread of each batch kernel.
constexpr int kContainsKPT = 4;
constexpr int kDeleteKPT = 4;
constexpr int kInsertKPT = 2;

enum KernelId : int { KID_CONTAINS = 0, KID_DELETE = 1, KID_INSERT = 2, KID_COUNT_KERNELS = 3 };

struct LaunchCfg {
    cudaStream_t stream;
    int block;
    int max_grid;  // persistent grid for this kernel and block size
};

struct OpsTable {
    uint32_t key_bytes, bits, bucket_size, word_bytes;
    uint32_t bucket_bytes;
    int kpt[KID_COUNT_KERNELS];
    cudaError_t (*contains)(const DevTable&, const void*, uint64_t, uint8_t*, const LaunchCfg&);
    cudaError_t (*remove)(const DevTable&, const void*, uint64_t, uint8_t*, const LaunchCfg&);
    cudaError_t (*insert)(const DevTable&, const void*, uint64_t, uint8_t*, const LaunchCfg&, uint32_t policy_bfs,
                          uint32_t max_ev);
    cudaError_t (*count)(const DevTable&, uint64_t nb, unsigned long long* result, const LaunchCfg&);
    cudaError_t (*probe)(const DevTable&, const void*, uint64_t, unsigned long long*, const LaunchCfg&);
    cudaError_t (*occupancy)(int kid, int block, int* blocks_per_sm);
};

inline bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

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

    static cudaError_t contains(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        if (n == 0) return cudaSuccess;
        constexpr int K = kContainsKPT;
        const int grid = grid_for(n, L.block, K, L.max_grid);
        k_contains<C, K><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                         aligned(keys, key_vec_align<C, K>()), aligned(out, K));
        return cudaGetLastError();
    }
    static cudaError_t remove(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L) {
        if (n == 0) return cudaSuccess;
        constexpr int K = kDeleteKPT;
        const int grid = grid_for(n, L.block, K, L.max_grid);
        k_delete<C, K><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                       aligned(keys, key_vec_align<C, K>()), aligned(out, K));
        return cudaGetLastError();
    }
    static cudaError_t insert(const DevTable& t, const void* keys, uint64_t n, uint8_t* out, const LaunchCfg& L,
                              uint32_t policy_bfs, uint32_t max_ev) {
        if (n == 0) return cudaSuccess;
        constexpr int K = kInsertKPT;
        const int grid = grid_for(n, L.block, K, L.max_grid);
        k_insert<C, K><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, out,
                                                       aligned(keys, key_vec_align<C, K>()), aligned(out, K),
                                                       policy_bfs, max_ev);
        return cudaGetLastError();
    }
    static cudaError_t count(const DevTable& t, uint64_t nb, unsigned long long* result, const LaunchCfg& L) {
        const int grid = grid_for(nb, L.block, 1, L.max_grid);
        k_count_occupied<C><<<grid, L.block, 0, L.stream>>>(t, nb, result);
        return cudaGetLastError();
    }
    static cudaError_t probe(const DevTable& t, const void* keys, uint64_t n, unsigned long long* result,
                             const LaunchCfg& L) {
        if (n == 0) return cudaSuccess;
        const int grid = grid_for(n, L.block, 1, L.max_grid);
        k_probe_count<C><<<grid, L.block, 0, L.stream>>>(t, static_cast<const Key*>(keys), n, result);
        return cudaGetLastError();
    }
    static cudaError_t occupancy(int kid, int block, int* bps) {
        switch (kid) {
            case KID_CONTAINS:
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_contains<C, kContainsKPT>, block, 0);
            case KID_DELETE:
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_delete<C, kDeleteKPT>, block, 0);
            default:
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_insert<C, kInsertKPT>, block, 0);
        }
    }

    static OpsTable table() {
        OpsTable o{};
        o.key_bytes = C::key_bytes;
        o.bits = C::bits;
        o.bucket_size = C::bs;
        o.word_bytes = C::word_bytes;
        o.bucket_bytes = C::bucket_bytes;
        o.kpt[KID_CONTAINS] = kContainsKPT;
        o.kpt[KID_DELETE] = kDeleteKPT;
        o.kpt[KID_INSERT] = kInsertKPT;
        o.contains = contains;
        o.remove = remove;
        o.insert = insert;
        o.count = count;
        o.probe = probe;
        o.occupancy = occupancy;
        return o;
    }
};

// Registration hooks, one per translation unit (tag width).
void register_bits8(std::vector<OpsTable>& v);
void register_bits16(std::vector<OpsTable>& v);
void register_bits32(std::vector<OpsTable>& v);

}  // namespace cfb
