// cf_set.cu -- C ABI of filter sets: many independent filters, one launch per
// batched operation (declared in include/cuckoo_b200.h).
//
// The reference runs one filter per object and one kernel launch per batch
// (CuckooFilter.cuh:457-548).  A set owns N filters of one configuration with
// individual capacities, their tables in one device pool, and a device array
// of per-filter descriptors; a batched call takes a device work list (item j =
// keys [offs[j], offs[j+1]) for filter filt[j]) and runs every item in one
// persistent kernel (cf_set.cuh).  The asynchronous calls only launch kernels
// (no allocation, no synchronization), so they can be captured into a CUDA
// graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/cuckoo_b200.h"
#include "cf_registry.cuh"
#include "cf_set.cuh"

namespace cfb {
int api_fail(int status, const char* msg);
int api_cuda_fail(cudaError_t e, const char* what);
int api_validate(const cf_config* cfg);
uint64_t api_num_buckets(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy);
}  // namespace cfb

using namespace cfb;

namespace {

struct LaunchChoice {
    uint32_t block = 256, kpt = 4, width = 1;
};

// Launchers of one configuration, dispatching the runtime (kpt, width) to the
// compiled variants.
struct SetOps {
    uint32_t bits, bucket_size, bucket_bytes, alt_policy;
    cudaError_t (*contains)(const DevTable*, const uint32_t*, const uint64_t*, uint32_t, uint32_t, const void*, uint64_t,
                            uint8_t*, unsigned long long*, const LaunchChoice&, int sms, cudaStream_t);
    cudaError_t (*remove)(const DevTable*, const uint32_t*, const uint64_t*, uint32_t, uint32_t, const void*, uint64_t,
                          uint8_t*, unsigned long long*, const LaunchChoice&, int sms, cudaStream_t);
    cudaError_t (*insert)(const DevTable*, const uint32_t*, const uint64_t*, uint32_t, uint32_t, const void*, uint64_t,
                          uint8_t*, unsigned long long*, const LaunchChoice&, int sms, cudaStream_t, uint32_t, uint32_t);
    bool (*width_ok)(uint32_t width);
};

template <class K>
int grid_of(K kernel, uint32_t block, int sms) {
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, static_cast<int>(block), 0) != cudaSuccess || bps < 1)
        bps = 1;
    return sms * bps;
}

template <class C>
struct SetLaunch {
    using Key = typename C::Key;

    template <int KPT>
    static cudaError_t contains1(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                                 const void* k, uint64_t n, uint8_t* out, unsigned long long* err,
                                 const LaunchChoice& L, int sms, cudaStream_t s) {
        const uint64_t tiles = (n + uint64_t(L.block) * KPT - 1) / (uint64_t(L.block) * KPT);
        const int g = static_cast<int>(std::min<uint64_t>(tiles, grid_of(k_set_contains1<C, KPT>, L.block, sms)));
        k_set_contains1<C, KPT><<<g, L.block, 0, s>>>(d, f, o, ni, nf, static_cast<const Key*>(k), n, out, err);
        CF_COUNT_LAUNCH();
        return cudaGetLastError();
    }
    template <int KPT, int W>
    static cudaError_t containsW(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                                 const void* k, uint64_t n, uint8_t* out, unsigned long long* err,
                                 const LaunchChoice& L, int sms, cudaStream_t s) {
        const uint64_t per = uint64_t(L.block / W) * KPT;
        const uint64_t tiles = (n + per - 1) / per;
        const int g = static_cast<int>(std::min<uint64_t>(tiles, grid_of(k_set_containsW<C, KPT, W>, L.block, sms)));
        k_set_containsW<C, KPT, W><<<g, L.block, 0, s>>>(d, f, o, ni, nf, static_cast<const Key*>(k), n, out, err);
        CF_COUNT_LAUNCH();
        return cudaGetLastError();
    }
    template <int W>
    static cudaError_t containsK(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                                 const void* k, uint64_t n, uint8_t* out, unsigned long long* err,
                                 const LaunchChoice& L, int sms, cudaStream_t s) {
        switch (L.kpt) {
            case 1: return containsW<1, W>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            case 2: return containsW<2, W>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            case 4: return containsW<4, W>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            default: return containsW<8, W>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
        }
    }
    static constexpr bool width_valid(uint32_t w) {
        return w == 1 || ((C::bucket_bytes % w) == 0 && (C::bucket_bytes / w == 4 || C::bucket_bytes / w == 8));
    }
    static bool width_ok(uint32_t w) { return width_valid(w); }
    static cudaError_t contains(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                                const void* k, uint64_t n, uint8_t* out, unsigned long long* err,
                                const LaunchChoice& L, int sms, cudaStream_t s) {
        if (n == 0) return cudaSuccess;
        if (L.width == 1) {
            switch (L.kpt) {
                case 1: return contains1<1>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
                case 2: return contains1<2>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
                case 4: return contains1<4>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
                default: return contains1<8>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            }
        }
        if constexpr (width_valid(2)) if (L.width == 2) return containsK<2>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
        if constexpr (width_valid(4)) if (L.width == 4) return containsK<4>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
        if constexpr (width_valid(8)) if (L.width == 8) return containsK<8>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
        return cudaErrorInvalidValue;
    }
    template <int KPT>
    static cudaError_t remove_k(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                                const void* k, uint64_t n, uint8_t* out, unsigned long long* err,
                                const LaunchChoice& L, int sms, cudaStream_t s) {
        const uint64_t tiles = (n + uint64_t(L.block) * KPT - 1) / (uint64_t(L.block) * KPT);
        const int g = static_cast<int>(std::min<uint64_t>(tiles, grid_of(k_set_delete<C, KPT>, L.block, sms)));
        k_set_delete<C, KPT><<<g, L.block, 0, s>>>(d, f, o, ni, nf, static_cast<const Key*>(k), n, out, err);
        CF_COUNT_LAUNCH();
        return cudaGetLastError();
    }
    static cudaError_t remove(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                              const void* k, uint64_t n, uint8_t* out, unsigned long long* err, const LaunchChoice& L,
                              int sms, cudaStream_t s) {
        if (n == 0) return cudaSuccess;
        switch (L.kpt) {
            case 1: return remove_k<1>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            case 2: return remove_k<2>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            case 4: return remove_k<4>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
            default: return remove_k<8>(d, f, o, ni, nf, k, n, out, err, L, sms, s);
        }
    }
    template <int KPT>
    static cudaError_t insert_k(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                                const void* k, uint64_t n, uint8_t* out, unsigned long long* err,
                                const LaunchChoice& L, int sms, cudaStream_t s, uint32_t bfs, uint32_t max_ev) {
        const uint64_t tiles = (n + uint64_t(L.block) * KPT - 1) / (uint64_t(L.block) * KPT);
        const int g = static_cast<int>(std::min<uint64_t>(tiles, grid_of(k_set_insert<C, KPT>, L.block, sms)));
        k_set_insert<C, KPT><<<g, L.block, 0, s>>>(d, f, o, ni, nf, static_cast<const Key*>(k), n, out, bfs, max_ev, err);
        CF_COUNT_LAUNCH();
        return cudaGetLastError();
    }
    static cudaError_t insert(const DevTable* d, const uint32_t* f, const uint64_t* o, uint32_t ni, uint32_t nf,
                              const void* k, uint64_t n, uint8_t* out, unsigned long long* err, const LaunchChoice& L,
                              int sms, cudaStream_t s, uint32_t bfs, uint32_t max_ev) {
        if (n == 0) return cudaSuccess;
        switch (L.kpt) {
            case 1: return insert_k<1>(d, f, o, ni, nf, k, n, out, err, L, sms, s, bfs, max_ev);
            case 2: return insert_k<2>(d, f, o, ni, nf, k, n, out, err, L, sms, s, bfs, max_ev);
            case 4: return insert_k<4>(d, f, o, ni, nf, k, n, out, err, L, sms, s, bfs, max_ev);
            default: return insert_k<8>(d, f, o, ni, nf, k, n, out, err, L, sms, s, bfs, max_ev);
        }
    }
    static SetOps table() {
        return SetOps{C::bits, C::bs, C::bucket_bytes, C::alt_policy, contains, remove, insert, width_ok};
    }
};

// Set configurations: 64-bit keys with 8-bit tags in 16-slot buckets, 16-bit
// tags in 16-slot buckets, 32-bit tags in 8-slot buckets (one 16- or 32-byte
// bucket per sector), XOR policy; 16/16 also with the AddSub and Offset
// policies.
const std::vector<SetOps>& set_registry() {
    static const std::vector<SetOps> v = {
        SetLaunch<Cfg<8, 8, 16, 8>>::table(), SetLaunch<Cfg<8, 16, 16, 8>>::table(),
        SetLaunch<Cfg<8, 32, 8, 8>>::table(), SetLaunch<Cfg<8, 16, 16, 8, ALT_ADDSUB>>::table(),
        SetLaunch<Cfg<8, 16, 16, 8, ALT_OFFSET>>::table()};
    return v;
}

const SetOps* find_set_ops(const cf_config* c) {
    if (c->key_bytes != 8 || c->word_bytes != 8) return nullptr;
    for (const SetOps& o : set_registry())
        if (o.bits == c->bits_per_tag && o.bucket_size == c->bucket_size && o.alt_policy == c->alt_policy) return &o;
    return nullptr;
}

}  // namespace

struct cf_set {
    cf_config cfg;
    const SetOps* ops;
    int device;
    int sms;
    uint32_t n;
    std::vector<uint64_t> nb;         // buckets per filter
    std::vector<uint64_t> offset;     // byte offset of each table in the pool
    uint8_t* pool;
    uint64_t pool_bytes;
    DevTable* d_descs;
    unsigned long long* d_ctr;        // n * CTR_COUNT
    unsigned long long* d_err;
    LaunchChoice launch[3];           // CF_SET_OP_INSERT, _CONTAINS, _DELETE
};

namespace {

struct Guard {
    int prev = -1;
    explicit Guard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Guard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int check_call(const cf_set* s, const void* keys, uint64_t n, const uint64_t* offs, const uint32_t* filt,
               uint32_t n_items) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    if (n && (!keys || !offs || !filt || n_items == 0))
        return api_fail(CF_ERR_INVALID, "keys, offsets or filters is NULL, or no items, with n > 0");
    return CF_OK;
}

#define SET_CUDA(expr, what)                                  \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return api_cuda_fail(e_, what); \
    } while (0)

}  // namespace

extern "C" {

int cf_set_create(const cf_config* cfg, uint32_t n_filters, const uint64_t* capacities, cf_set** out) {
    if (!out) return api_fail(CF_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (int st = api_validate(cfg)) return st;
    if (n_filters == 0 || !capacities) return api_fail(CF_ERR_INVALID, "n_filters must be > 0 and capacities given");
    const SetOps* ops = find_set_ops(cfg);
    if (!ops)
        return api_fail(CF_ERR_UNSUPPORTED,
                        "filter sets are built for 64-bit keys with 8/16, 16/16 or 32/8 (bits per tag / bucket size) "
                        "and the XOR policy, and 16/16 with the AddSub and Offset policies");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return api_fail(CF_ERR_NOT_LOADED, "no CUDA device");
    cf_set* s = new cf_set{};
    s->cfg = *cfg;
    s->ops = ops;
    s->device = device;
    s->n = n_filters;
    s->nb.resize(n_filters);
    s->offset.resize(n_filters);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n_filters; ++i) {
        if (capacities[i] == 0) {
            delete s;
            return api_fail(CF_ERR_INVALID, "every capacity must be > 0");
        }
        s->nb[i] = api_num_buckets(capacities[i], cfg->bucket_size, cfg->alt_policy);
        s->offset[i] = total;
        total += (s->nb[i] * ops->bucket_bytes + 255) & ~255ull;  // 256-byte aligned tables
    }
    s->pool_bytes = total;
    const uint32_t block = cfg->block_size ? cfg->block_size : 256;
    for (auto& L : s->launch) L.block = block;
    std::vector<DevTable> descs(n_filters);
    cudaError_t e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc(&s->pool, total);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_ctr, sizeof(unsigned long long) * CTR_COUNT * n_filters);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_err, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_descs, sizeof(DevTable) * n_filters);
    if (e == cudaSuccess) {
        for (uint32_t i = 0; i < n_filters; ++i)
            descs[i] = DevTable{s->pool + s->offset[i], s->nb[i] - 1, s->d_ctr + static_cast<uint64_t>(i) * CTR_COUNT};
        e = cudaMemcpy(s->d_descs, descs.data(), sizeof(DevTable) * n_filters, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(s->pool, 0, total);
    if (e == cudaSuccess) e = cudaMemset(s->d_ctr, 0, sizeof(unsigned long long) * CTR_COUNT * n_filters);
    if (e == cudaSuccess) e = cudaMemset(s->d_err, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        const int st = api_cuda_fail(e, "filter set allocation");
        cf_set_destroy(s);
        return st;
    }
    *out = s;
    return CF_OK;
}

int cf_set_destroy(cf_set* s) {
    if (!s) return CF_OK;
    Guard g(s->device);
    if (s->pool) cudaFree(s->pool);
    if (s->d_ctr) cudaFree(s->d_ctr);
    if (s->d_err) cudaFree(s->d_err);
    if (s->d_descs) cudaFree(s->d_descs);
    delete s;
    return CF_OK;
}

int cf_set_size(const cf_set* s, uint32_t* n_filters, uint64_t* pool_bytes) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    if (n_filters) *n_filters = s->n;
    if (pool_bytes) *pool_bytes = s->pool_bytes;
    return CF_OK;
}

int cf_set_get_info(const cf_set* s, uint32_t i, cf_info* out) {
    if (!s || !out) return api_fail(CF_ERR_INVALID, "set or out is NULL");
    if (i >= s->n) return api_fail(CF_ERR_INVALID, "filter index out of range");
    out->num_buckets = s->nb[i];
    out->capacity = s->nb[i] * s->cfg.bucket_size;
    out->size_in_bytes = s->nb[i] * s->ops->bucket_bytes;
    out->bucket_bytes = s->ops->bucket_bytes;
    out->device = s->device;
    return CF_OK;
}

int cf_set_table(cf_set* s, uint32_t i, void** d_table, uint64_t* bytes) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    if (i >= s->n) return api_fail(CF_ERR_INVALID, "filter index out of range");
    if (d_table) *d_table = s->pool + s->offset[i];
    if (bytes) *bytes = s->nb[i] * s->ops->bucket_bytes;
    return CF_OK;
}

int cf_set_contains_async(cf_set* s, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                          const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream) {
    if (int st = check_call(s, d_keys, n, d_offsets, d_filters, n_items)) return st;
    if (n && !d_out) return api_fail(CF_ERR_INVALID, "d_out is NULL with n > 0");
    Guard g(s->device);
    SET_CUDA(s->ops->contains(s->d_descs, d_filters, d_offsets, n_items, s->n, d_keys, n, d_out, s->d_err,
                              s->launch[CF_SET_OP_CONTAINS], s->sms, static_cast<cudaStream_t>(stream)),
             "set contains launch");
    return CF_OK;
}

int cf_set_delete_async(cf_set* s, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                        const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream) {
    if (int st = check_call(s, d_keys, n, d_offsets, d_filters, n_items)) return st;
    Guard g(s->device);
    SET_CUDA(s->ops->remove(s->d_descs, d_filters, d_offsets, n_items, s->n, d_keys, n, d_out, s->d_err,
                            s->launch[CF_SET_OP_DELETE], s->sms, static_cast<cudaStream_t>(stream)),
             "set delete launch");
    return CF_OK;
}

int cf_set_insert_async(cf_set* s, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                        const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream) {
    if (int st = check_call(s, d_keys, n, d_offsets, d_filters, n_items)) return st;
    Guard g(s->device);
    SET_CUDA(s->ops->insert(s->d_descs, d_filters, d_offsets, n_items, s->n, d_keys, n, d_out, s->d_err,
                            s->launch[CF_SET_OP_INSERT], s->sms, static_cast<cudaStream_t>(stream),
                            s->cfg.eviction_policy == CF_EVICT_BFS ? 1u : 0u, s->cfg.max_evictions),
             "set insert launch");
    return CF_OK;
}

int cf_set_sync(cf_set* s, void* stream) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    Guard g(s->device);
    unsigned long long err = 0;
    SET_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "stream synchronize");
    SET_CUDA(cudaMemcpy(&err, s->d_err, sizeof(err), cudaMemcpyDeviceToHost), "error flag read");
    if (err & ERR_BAD_FILTER) {
        cudaMemset(s->d_err, 0, sizeof(err));
        return api_fail(CF_ERR_INVALID, "a work item named a filter outside the set (its keys were skipped)");
    }
    if (err & ERR_CAS_LIMIT) return api_fail(CF_ERR_DEVICE, "a compare-and-swap retry bound was hit on the device");
    return CF_OK;
}

int cf_set_clear(cf_set* s, void* stream) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    Guard g(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SET_CUDA(cudaMemsetAsync(s->pool, 0, s->pool_bytes, st), "pool clear");
    SET_CUDA(cudaMemsetAsync(s->d_ctr, 0, sizeof(unsigned long long) * CTR_COUNT * s->n, st), "counter clear");
    SET_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(unsigned long long), st), "error clear");
    SET_CUDA(cudaStreamSynchronize(st), "stream synchronize");
    return CF_OK;
}

int cf_set_occupied(cf_set* s, uint64_t* out) {
    if (!s || !out) return api_fail(CF_ERR_INVALID, "set or out is NULL");
    Guard g(s->device);
    std::vector<unsigned long long> c(static_cast<size_t>(s->n) * CTR_COUNT);
    SET_CUDA(cudaMemcpy(c.data(), s->d_ctr, c.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
             "counter read");
    for (uint32_t i = 0; i < s->n; ++i) out[i] = c[static_cast<size_t>(i) * CTR_COUNT + CTR_OCCUPIED];
    return CF_OK;
}

int cf_set_get_stats(cf_set* s, uint32_t i, cf_stats* out) {
    if (!s || !out) return api_fail(CF_ERR_INVALID, "set or out is NULL");
    if (i >= s->n) return api_fail(CF_ERR_INVALID, "filter index out of range");
    Guard g(s->device);
    unsigned long long c[CTR_COUNT];
    SET_CUDA(cudaMemcpy(c, s->d_ctr + static_cast<uint64_t>(i) * CTR_COUNT, sizeof(c), cudaMemcpyDeviceToHost),
             "counter read");
    out->occupied = c[CTR_OCCUPIED];
    out->primary = c[CTR_PRIMARY];
    out->secondary = c[CTR_SECONDARY];
    out->evicted_inserts = c[CTR_EVICTED_INSERTS];
    out->evictions = c[CTR_EVICTIONS];
    out->failed = c[CTR_FAILED];
    out->lost = c[CTR_LOST];
    out->removed = c[CTR_REMOVED];
    out->duplicates = c[CTR_DUP];
    return CF_OK;
}

int cf_set_set_launch(cf_set* s, int op, uint32_t block, uint32_t kpt, uint32_t width) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    if (op < 0 || op > 2) return api_fail(CF_ERR_INVALID, "unknown set operation");
    if (block % 32 || block == 0 || block > 512) return api_fail(CF_ERR_INVALID, "block must be 32..512, a multiple of 32");
    if (kpt != 1 && kpt != 2 && kpt != 4 && kpt != 8) return api_fail(CF_ERR_INVALID, "keys per thread must be 1, 2, 4 or 8");
    if (op != CF_SET_OP_CONTAINS && width != 1) return api_fail(CF_ERR_INVALID, "probe width applies to lookups only");
    if (!s->ops->width_ok(width))
        return api_fail(CF_ERR_INVALID, "probe width must be 1 or split a bucket into 4- or 8-byte pieces");
    s->launch[op] = LaunchChoice{block, kpt, width};
    return CF_OK;
}

int cf_set_get_launch(const cf_set* s, int op, uint32_t* block, uint32_t* kpt, uint32_t* width) {
    if (!s) return api_fail(CF_ERR_INVALID, "set is NULL");
    if (op < 0 || op > 2) return api_fail(CF_ERR_INVALID, "unknown set operation");
    if (block) *block = s->launch[op].block;
    if (kpt) *kpt = s->launch[op].kpt;
    if (width) *width = s->launch[op].width;
    return CF_OK;
}

int cf_set_autotune(cf_set* s, int op, const void* d_keys, uint64_t n, const uint64_t* d_offsets,
                    const uint32_t* d_filters, uint32_t n_items, uint8_t* d_out, void* stream, float* best_ms) {
    if (int st = check_call(s, d_keys, n, d_offsets, d_filters, n_items)) return st;
    if (op < 0 || op > 2) return api_fail(CF_ERR_INVALID, "unknown set operation");
    if (op == CF_SET_OP_CONTAINS && n && !d_out) return api_fail(CF_ERR_INVALID, "d_out is NULL with n > 0");
    Guard g(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t a = nullptr, b = nullptr;
    SET_CUDA(cudaEventCreate(&a), "event create");
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return api_fail(CF_ERR_CUDA, "event create failed");
    }
    const LaunchChoice keep = s->launch[op];
    LaunchChoice best = keep;
    float best_t = 1e30f;
    int status = CF_OK;
    const uint32_t blocks[] = {128, 256, 512};
    const uint32_t kpts[] = {1, 2, 4, 8};
    const uint32_t widths[] = {1, 4, 8};
    for (uint32_t blk : blocks) {
        for (uint32_t kp : kpts) {
            for (uint32_t wd : widths) {
                if (op != CF_SET_OP_CONTAINS && wd != 1) continue;
                if (!s->ops->width_ok(wd)) continue;
                s->launch[op] = LaunchChoice{blk, kp, wd};
                float t = 0;
                for (int rep = 0; rep < 2 && status == CF_OK; ++rep) {
                    // inserts and deletes change the set: every trial starts from an
                    // empty set (deletes from the batch inserted with the default launch)
                    if (op != CF_SET_OP_CONTAINS) status = cf_set_clear(s, stream);
                    if (status == CF_OK && op == CF_SET_OP_DELETE) {
                        status = cf_set_insert_async(s, d_keys, n, d_offsets, d_filters, n_items, nullptr, stream);
                    }
                    if (status != CF_OK) break;
                    cudaEventRecord(a, st);
                    if (op == CF_SET_OP_CONTAINS)
                        status = cf_set_contains_async(s, d_keys, n, d_offsets, d_filters, n_items, d_out, stream);
                    else if (op == CF_SET_OP_DELETE)
                        status = cf_set_delete_async(s, d_keys, n, d_offsets, d_filters, n_items, nullptr, stream);
                    else
                        status = cf_set_insert_async(s, d_keys, n, d_offsets, d_filters, n_items, nullptr, stream);
                    cudaEventRecord(b, st);
                    if (status == CF_OK && cudaEventSynchronize(b) != cudaSuccess)
                        status = api_fail(CF_ERR_CUDA, "trial failed");
                    float ms = 0;
                    cudaEventElapsedTime(&ms, a, b);
                    if (rep == 1 || op != CF_SET_OP_CONTAINS) t = ms;  // the lookup's first run warms up
                }
                if (status != CF_OK) break;
                if (t < best_t) {
                    best_t = t;
                    best = s->launch[op];
                }
            }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    s->launch[op] = status == CF_OK ? best : keep;
    if (status == CF_OK && op != CF_SET_OP_CONTAINS) status = cf_set_clear(s, stream);
    if (status == CF_OK) status = cf_set_sync(s, stream);
    if (best_ms) *best_ms = best_t;
    return status;
}

}  // extern "C"
