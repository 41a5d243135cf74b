// cf_api.cu -- C ABI of the B200 cuckoo filter (declared in include/cuckoo_b200.h).
//
// Host side of the reference's CuckooFilter<Config> (CuckooFilter.cuh:140-785):
// the filter owns its table and counters; the synchronous calls mirror the
// reference's (launch, cudaStreamSynchronize, read the occupancy counter).  The
// device-side filter descriptor is passed to kernels by value, never as a host
// `this` pointer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/cuckoo_b200.h"
#include "cf_registry.cuh"

using namespace cfb;

struct cf_filter {
    cf_config cfg;
    const OpsTable* ops;
    uint64_t num_buckets;
    uint64_t table_bytes;
    uint8_t* d_table;
    unsigned long long* d_ctr;  // CTR_COUNT device counters
    unsigned long long* h_ctr;  // pinned mirror
    int device;
    int block;
    int max_grid[KID_COUNT_KERNELS];
    int max_grid_aux;
    int sms;
    // segment-staged path
    bool seg_ok;            // the segment-staged path applies: packed (bucket, tag) entries fit in 64 bits
    bool rg_ok;             // the region-staged path applies
    SegGeom geom;
    void* ws;               // workspace (grown on demand, freed with the filter)
    uint64_t ws_bytes;
    uint64_t ws_limit;      // CF_OPT_WORKSPACE_LIMIT (0 = automatic)
    uint64_t seg_min_keys;  // CF_OPT_SEGMENTED_MIN_KEYS (0 = automatic)
    uint64_t round2_min;    // CF_OPT_ROUND2_SEGMENTED_MIN_KEYS (0 = automatic)
    uint32_t round1_cap;    // CF_OPT_ROUND1_CAP (0 = automatic)
    unsigned long long* h_cnt;
    // region-staged path
    RegionGeom rgeom;
    uint64_t rg_min_keys;   // CF_OPT_REGION_MIN_KEYS (0 = automatic)
    uint32_t staging;       // CF_OPT_STAGING (cf_staging)
    uint64_t rg_bytes;      // CF_OPT_REGION_BYTES (0 = kRgRegionBytes)
    uint32_t lookup_kpt;    // CF_OPT_LOOKUP_KPT (0 = default)
    uint32_t probe_width;   // CF_OPT_PROBE_WIDTH (0 or 1 = one lane per key)
    // The table is all zeros (set by cf_create and cf_clear, which synchronize;
    // cleared by every call that may write the table).  Never set again once
    // cf_table has handed out the table's address (table_exposed).
    bool known_empty;
    bool table_exposed;
    uint32_t persistent;    // CF_OPT_PERSISTENT (0 = one tile per CTA, 1 = persistent grid)
    uint32_t chain_hist;    // CF_OPT_CHAIN_HISTOGRAM
};

namespace {

thread_local char g_err[512] = "";

int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? CF_ERR_NO_MEMORY : CF_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

#define CF_CUDA(expr, what)                          \
    do {                                             \
        cudaError_t e_ = (expr);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

const std::vector<OpsTable>& registry() {
    static std::vector<OpsTable> v = [] {
        std::vector<OpsTable> r;
        register_bits8(r);
        register_bits16(r);
        register_bits32(r);
        return r;
    }();
    return v;
}

const OpsTable* find_ops(const cf_config* c) {
    for (const OpsTable& o : registry())
        if (o.key_bytes == c->key_bytes && o.bits == c->bits_per_tag && o.bucket_size == c->bucket_size &&
            o.word_bytes == c->word_bytes && o.alt_policy == c->alt_policy)
            return &o;
    return nullptr;
}

int validate(const cf_config* c) {
    if (!c) return fail(CF_ERR_INVALID, "config is NULL");
    if (c->key_bytes != 4 && c->key_bytes != 8) return fail(CF_ERR_INVALID, "key_bytes must be 4 or 8");
    if (c->bits_per_tag != 8 && c->bits_per_tag != 16 && c->bits_per_tag != 32)
        return fail(CF_ERR_INVALID, "bits_per_tag must be 8, 16 or 32");
    if (c->bucket_size == 0 || (c->bucket_size & (c->bucket_size - 1)))
        return fail(CF_ERR_INVALID, "bucket_size must be a power of two");
    if (c->word_bytes != 8 && c->word_bytes != 4) return fail(CF_ERR_INVALID, "word_bytes must be 4 or 8");
    if (c->eviction_policy != CF_EVICT_BFS && c->eviction_policy != CF_EVICT_DFS)
        return fail(CF_ERR_INVALID, "eviction_policy must be CF_EVICT_BFS or CF_EVICT_DFS");
    if (c->max_evictions < 1 || c->max_evictions > kMaxEvictionsCap)
        return fail(CF_ERR_INVALID, "max_evictions must be in [1, %u]", kMaxEvictionsCap);
    if (c->block_size != 0 && (c->block_size % 32 != 0 || c->block_size > 512))
        return fail(CF_ERR_INVALID, "block_size must be 0 or a multiple of 32 up to 512");
    if (c->alt_policy != CF_ALT_XOR && c->alt_policy != CF_ALT_ADDSUB && c->alt_policy != CF_ALT_OFFSET)
        return fail(CF_ERR_INVALID, "alt_policy must be CF_ALT_XOR, CF_ALT_ADDSUB or CF_ALT_OFFSET");
    if (!find_ops(c))
        return fail(CF_ERR_UNSUPPORTED,
                    "no kernels for key_bytes=%u bits_per_tag=%u bucket_size=%u word_bytes=%u alt_policy=%u",
                    c->key_bytes, c->bits_per_tag, c->bucket_size, c->word_bytes, c->alt_policy);
    return CF_OK;
}

uint64_t num_buckets_for(uint64_t capacity, uint32_t bucket_size) {
    // std::ceil((double)capacity / bucketSize), then nextPowerOfTwo (helpers.cuh:31-45).
    const double req = std::ceil(static_cast<double>(capacity) / static_cast<double>(bucket_size));
    uint64_t r = static_cast<uint64_t>(req);
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

// calculateNumBuckets of each policy (bucket_policies.cuh:80-83, :166-176, :346-349).
uint64_t num_buckets_policy(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy) {
    if (alt_policy == CF_ALT_XOR) return num_buckets_for(capacity, bucket_size);
    uint64_t r = static_cast<uint64_t>(std::ceil(static_cast<double>(capacity) / static_cast<double>(bucket_size)));
    if (alt_policy == CF_ALT_ADDSUB && (r % 2) != 0) r += 1;
    return r;
}

DevTable dev(const cf_filter* f) {
    return DevTable{f->d_table, f->num_buckets - 1, f->d_ctr, f->chain_hist ? f->d_ctr + CTR_HIST0 : nullptr};
}

LaunchCfg launch(const cf_filter* f, int kid, void* stream) {
    LaunchCfg L{static_cast<cudaStream_t>(stream), f->block, f->max_grid[kid]};
    L.full_grid = f->persistent == 0;
    return L;
}

LaunchCfg launch_aux(const cf_filter* f, void* stream) {
    return LaunchCfg{static_cast<cudaStream_t>(stream), 256, f->max_grid_aux};
}

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int check_filter(const cf_filter* f) {
    if (!f) return fail(CF_ERR_INVALID, "filter is NULL");
    return CF_OK;
}

int check_batch(const cf_filter* f, const void* keys, uint64_t n) {
    if (int s = check_filter(f)) return s;
    if (n && !keys) return fail(CF_ERR_INVALID, "keys is NULL with n > 0");
    return CF_OK;
}

// Synchronize, read the counters, surface device-side errors.
int finish(cf_filter* f, void* stream, uint64_t* occupied_out) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CF_CUDA(cudaMemcpyAsync(f->h_ctr, f->d_ctr, CTR_COUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
            "counter read-back");
    CF_CUDA(cudaStreamSynchronize(s), "stream synchronize");
    if (f->h_ctr[CTR_ERROR] & ERR_CAS_LIMIT)
        return fail(CF_ERR_DEVICE, "a compare-and-swap retry bound was hit on the device");
    if (f->h_ctr[CTR_ERROR] & ERR_WAIT_LIMIT)
        return fail(CF_ERR_DEVICE, "a bulk copy did not complete within its poll bound on the device");
    if (occupied_out) *occupied_out = f->h_ctr[CTR_OCCUPIED];
    return CF_OK;
}

int ilog2(uint64_t v) { return 63 - __builtin_clzll(v); }

// ceil(log2(v)) for v >= 1
int clog2(uint64_t v) { return v <= 1 ? 0 : ilog2(v - 1) + 1; }

void init_geometry(cf_filter* f) {
    const uint64_t bb = f->ops->bucket_bytes;
    uint64_t sb = kSegBytes / bb;
    if (sb > f->num_buckets) sb = f->num_buckets;
    f->geom.sb_log2 = ilog2(sb);  // a power of two at most the bucket count
    sb = 1ull << f->geom.sb_log2;
    // the last segment is partial when the bucket count (AddSub and Offset
    // policies) is not a multiple of the segment
    f->geom.nseg = (f->num_buckets + sb - 1) / sb;
    f->geom.seg_shift = static_cast<int>(f->cfg.bits_per_tag) + f->geom.sb_log2;
    const int seg_bits = clog2(f->geom.nseg);
    f->geom.passes = seg_bits == 0 ? 1 : (seg_bits + kRadixBits - 1) / kRadixBits;
    // (bucket << bits) | tag must fit in 64 bits for every bucket index
    f->seg_ok = clog2(f->num_buckets) + static_cast<int>(f->cfg.bits_per_tag) <= 64 && f->ops->seg_chunk;
    f->rg_ok = f->seg_ok && f->ops->rg_chunk;
    // regions of ~kRgRegionBytes (or CF_OPT_REGION_BYTES), at most kRgMaxRegions
    // of them; the last region is partial when the bucket count is not a power
    // of two (AddSub and Offset policies)
    const int nb_log2 = clog2(f->num_buckets);
    const uint64_t rbytes = f->rg_bytes ? f->rg_bytes : kRgRegionBytes;
    int rl = rbytes > bb ? ilog2(rbytes / bb) : 0;
    if (rl < nb_log2 - 8) rl = nb_log2 - 8;
    if (rl > nb_log2) rl = nb_log2;
    f->rgeom.rl = rl;
    f->rgeom.nreg = static_cast<uint32_t>(((f->num_buckets - 1) >> rl) + 1);
}

// Words of the known-full bucket bitmap (one bit per bucket of the segment
// geometry), kept when the segment insert runs k_seg_insert (at most 64
// slots per bucket) on segments of at least 32 buckets; else 0.
uint64_t full_words(const cf_filter* f) {
    if (f->cfg.bucket_size > 64 || f->geom.sb_log2 < 5) return 0;
    return (f->geom.nseg << f->geom.sb_log2) >> 5;
}

// Bytes of workspace for a chunk of `cap` keys: two entry buffers (8 B per
// key), and with per-key results two payload buffers (4 B) and a result bitmap;
// besides, per table, the radix histogram, the segment starts, the list
// counters and the known-full bucket bitmap.
uint64_t ws_need(const cf_filter* f, uint64_t cap, int grid, bool payload) {
    const uint64_t hist = static_cast<uint64_t>(kRadix) * grid * 4;
    const uint64_t start = (f->geom.nseg + 1) * 4;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    // result bitmap: two bits per key (a region-staged lookup keeps one hit bit per staged entry)
    const uint64_t per_key = payload ? al(cap * 4) * 2 + al((2 * cap + 31) / 32 * 4) : 0;
    return al(cap * 8) * 2 + per_key + al(hist) + al(start) + al(64) + al(full_words(f) * 4);
}

// Automatic workspace limit (CF_OPT_WORKSPACE_LIMIT = 0, the default): the
// device memory free now plus the workspace already held (it is freed before a
// larger one is allocated), less a reserve of 1/16 of the device (at least
// 1 GiB) left to the caller.  The reference allocates what each sorted insert
// needs (CuckooFilter.cuh:475-508); this keeps the whole batch in one chunk
// whenever that fits, and keeps the workspace for the next call.
constexpr uint64_t kMinAutoWorkspace = 256ull << 20;

uint64_t auto_workspace_limit(const cf_filter* f) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 4ull << 30;
    }
    const uint64_t reserve = std::max<uint64_t>(1ull << 30, total_b / 16);
    const uint64_t avail = f->ws_bytes + free_b;
    return avail > reserve + kMinAutoWorkspace ? avail - reserve : kMinAutoWorkspace;
}

int ensure_workspace(cf_filter* f, uint64_t n, bool payload, SegWork* w) {
    // radix passes: one wave of each payload mode's scatter kernel, fixed per-CTA chunks
    int rs_grid[3];
    CF_CUDA(rs_scatter_grid<0>(f->sms, &rs_grid[0]), "radix launch setup");
    CF_CUDA(rs_scatter_grid<1>(f->sms, &rs_grid[1]), "radix launch setup");
    CF_CUDA(rs_scatter_grid<2>(f->sms, &rs_grid[2]), "radix launch setup");
    const int rg_grid = f->sms * 4;
    const int grid = std::max(std::max(rs_grid[0], std::max(rs_grid[1], rs_grid[2])) * kRsHistSub,
                              (rg_grid * static_cast<int>(kRgMaxRegions) + kRadix - 1) / kRadix);
    const uint64_t fixed = ws_need(f, 0, grid, payload) + 4096;
    const uint64_t kMaxChunk = 1ull << 31;  // 32-bit positions and payloads
    uint64_t limit = f->ws_limit;
    bool fits_held = false;  // automatic limit, and the whole batch fits the workspace already held
    if (limit == 0) {  // automatic: the whole batch when device memory allows
        const uint64_t whole = ws_need(f, std::min(n, kMaxChunk), grid, payload);
        fits_held = whole <= f->ws_bytes;
        limit = fits_held ? f->ws_bytes : auto_workspace_limit(f);
    }
    uint64_t cap = 0, need = 0;
    for (;;) {
        cap = n;
        if (fits_held) {
            // one chunk (the fit below is conservative and would split off a
            // sliver of the batch)
        } else if (limit > fixed) {
            const uint64_t fit = (limit - fixed) / (payload ? 25 : 16);
            if (cap > fit) cap = fit;
        } else {
            cap = 0;
        }
        if (cap > kMaxChunk) cap = kMaxChunk;
        if (cap < n) cap = cap / 32 * 32;
        if (cap < 1024 && n > cap) cap = 1024;
        need = ws_need(f, cap, grid, payload);
        if (f->ws_bytes >= need) break;
        if (f->ws) cudaFree(f->ws);
        f->ws = nullptr;
        f->ws_bytes = 0;
        const cudaError_t e = cudaMalloc(&f->ws, need);
        if (e == cudaSuccess) {
            f->ws_bytes = need;
            break;
        }
        // automatic limit: another allocation may have taken the memory since
        // it was measured; retry with half the chunk
        if (e != cudaErrorMemoryAllocation || f->ws_limit != 0 || need <= kMinAutoWorkspace)
            return cuda_fail(e, "workspace allocation");
        cudaGetLastError();
        f->ws = nullptr;
        limit = std::max(kMinAutoWorkspace, need / 2);
    }
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    uint8_t* p = static_cast<uint8_t*>(f->ws);
    w->ent[0] = reinterpret_cast<uint64_t*>(p);
    p += al(cap * 8);
    w->ent[1] = reinterpret_cast<uint64_t*>(p);
    p += al(cap * 8);
    w->hist = reinterpret_cast<uint32_t*>(p);
    p += al(static_cast<uint64_t>(kRadix) * grid * 4);
    w->start = reinterpret_cast<uint32_t*>(p);
    p += al((f->geom.nseg + 1) * 4);
    w->cnt = reinterpret_cast<unsigned long long*>(p);
    p += al(64);
    w->full_words = full_words(f);
    w->full = w->full_words ? reinterpret_cast<uint32_t*>(p) : nullptr;
    p += al(w->full_words * 4);
    w->pay[0] = w->pay[1] = nullptr;
    w->bitmap = nullptr;
    if (payload) {
        w->pay[0] = reinterpret_cast<uint32_t*>(p);
        p += al(cap * 4);
        w->pay[1] = reinterpret_cast<uint32_t*>(p);
        p += al(cap * 4);
        w->bitmap = reinterpret_cast<uint32_t*>(p);
    }
    w->h_cnt = f->h_cnt;
    w->cap = cap;
    for (int i = 0; i < 3; ++i) w->rs_grid[i] = rs_grid[i];
    w->rg_grid = rg_grid;
    w->sms = f->sms;
    return CF_OK;
}

// Keys from which the segment-staged path beats random probes: a random probe
// costs one DRAM transaction, streaming a segment costs its bytes (read, and
// write-back for insert/delete).
// Measured on B200: a random probe costs one DRAM transaction (the device
// completes ~38 G/s); the segment path costs its radix passes, the streamed
// segments and the shared-memory work.  Lookups and deletes beat random
// probing on the segment path only for batches of several keys per bucket;
// the alternate-bucket round of a segment batch pays off from about one key
// per 64 table bytes.
uint64_t auto_threshold(const cf_filter* f, int op) {
    if (op == SEG_INSERT) return f->table_bytes / 64;
    return f->num_buckets * 8;
}

// Batch size from which a batch is segment-staged.  Inserts: one key per
// bucket (on B200 the segment path overtook random inserts between 0.5 and 1
// key per bucket: 0.70 against 0.88 ms at 1, 0.98 against 1.73 ms at 2, on an
// empty 2^28-slot table); lookups and deletes: eight keys per bucket.
uint64_t segmented_threshold(const cf_filter* f, int op) {
    if (f->seg_min_keys) return f->seg_min_keys;
    return op == SEG_INSERT ? f->num_buckets : f->num_buckets * 8;
}

int run_segmented(cf_filter* f, int op, const void* keys, uint64_t n, uint8_t* out, void* stream) {
    if (n == 0) return CF_OK;
    SegWork w{};
    if (int st = ensure_workspace(f, n, out != nullptr, &w)) return st;
    w.round2_segmented_min = f->round2_min ? f->round2_min : auto_threshold(f, op);
    w.round1_cap = f->round1_cap;
    // an insert into a table known to be empty: its first chunk's first
    // round stages zeroed segments instead of loading them
    bool fresh = op == SEG_INSERT && f->known_empty;
    f->known_empty = false;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t kb = f->cfg.key_bytes;
    for (uint64_t c0 = 0; c0 < n; c0 += w.cap) {
        const uint64_t m = n - c0 < w.cap ? n - c0 : w.cap;
        w.fresh = fresh;
        fresh = false;
        CF_CUDA(f->ops->seg_chunk(dev(f), f->geom, w, op, static_cast<const uint8_t*>(keys) + c0 * kb, m,
                                  out ? out + c0 : nullptr, s, f->cfg.eviction_policy == CF_EVICT_BFS ? 1u : 0u,
                                  f->cfg.max_evictions),
                "segment-staged batch");
    }
    return CF_OK;
}

// Region-staged path (cf_region.cuh): keys from which it beats random probes.
// A random probe costs one DRAM transaction (~38 G/s on B200); the region path
// streams ~30 bytes per key plus the table once (lookups) or about twice
// (inserts and deletes), at close to HBM bandwidth.
uint64_t region_threshold(const cf_filter* f, int op) {
    if (f->rg_min_keys) return f->rg_min_keys;
    (void)op;
    return UINT64_MAX;  // automatic choice: not yet (measured slower than the other paths)
}

int run_region(cf_filter* f, int op, const void* keys, uint64_t n, uint8_t* out, void* stream) {
    if (n == 0) return CF_OK;
    if (op != SEG_CONTAINS) f->known_empty = false;
    SegWork w{};
    if (int st = ensure_workspace(f, n, op == SEG_CONTAINS || out != nullptr, &w)) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t kb = f->cfg.key_bytes;
    // lookups stage two entries per key (32-bit entry offsets) and gather each
    // partition chunk's results in shared memory: at most 2^29 keys per chunk
    uint64_t cap = w.cap;
    if (op == SEG_CONTAINS) {
        const uint64_t lim = std::min<uint64_t>(1ull << 29, static_cast<uint64_t>(w.rg_grid) * 1000000ull);
        if (cap > lim) cap = lim;
    }
    for (uint64_t c0 = 0; c0 < n; c0 += cap) {
        const uint64_t m = n - c0 < cap ? n - c0 : cap;
        CF_CUDA(f->ops->rg_chunk(dev(f), f->rgeom, w, op, static_cast<const uint8_t*>(keys) + c0 * kb, m,
                                 out ? out + c0 : nullptr, s, f->cfg.eviction_policy == CF_EVICT_BFS ? 1u : 0u,
                                 f->cfg.max_evictions),
                "region-staged batch");
    }
    return CF_OK;
}

// Execution path of a batch: random probes, segment-staged or region-staged.
enum Path { PATH_RANDOM, PATH_SEGMENT, PATH_REGION };

Path choose_path(const cf_filter* f, int op, uint64_t n, bool sorted_insert) {
    if (!f->seg_ok) return PATH_RANDOM;
    switch (f->staging) {
        case CF_STAGING_RANDOM: return sorted_insert ? PATH_SEGMENT : PATH_RANDOM;
        case CF_STAGING_SEGMENT: return PATH_SEGMENT;
        case CF_STAGING_REGION: return f->rg_ok ? PATH_REGION : PATH_SEGMENT;
        default: break;
    }
    if (f->rg_ok && n >= region_threshold(f, op)) return PATH_REGION;
    if (sorted_insert) return PATH_SEGMENT;
    if (n >= segmented_threshold(f, op)) return PATH_SEGMENT;
    return PATH_RANDOM;
}

int do_insert(cf_filter* f, const void* keys, uint64_t n, uint8_t* out, void* stream) {
    f->known_empty = false;
    CF_CUDA(f->ops->insert(dev(f), keys, n, out, launch(f, KID_INSERT, stream),
                           f->cfg.eviction_policy == CF_EVICT_BFS ? 1u : 0u, f->cfg.max_evictions),
            "insert launch");
    return CF_OK;
}

template <class C>
void host_candidates_t(uint64_t mask, const void* keys, uint64_t n, uint64_t* i1, uint64_t* i2, uint32_t* fp) {
    const auto* k = static_cast<const typename C::Key*>(keys);
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t b;
        uint32_t f;
        candidates<C>(static_cast<uint64_t>(k[i]), mask, b, f);
        if (i1) i1[i] = b;
        if (i2) i2[i] = alt_bucket<C>(b, f, mask);
        if (fp) fp[i] = f;
    }
}

// Bucket size does not enter the hashing; 16 slots stands in for any.
template <int POL>
void host_candidates_p(uint32_t kb, uint32_t bits, uint64_t nbm, const void* keys, uint64_t n, uint64_t* i1,
                       uint64_t* i2, uint32_t* fp) {
    if (kb == 8) {
        if (bits == 8) host_candidates_t<Cfg<8, 8, 16, 8, POL>>(nbm, keys, n, i1, i2, fp);
        else if (bits == 16) host_candidates_t<Cfg<8, 16, 16, 8, POL>>(nbm, keys, n, i1, i2, fp);
        else host_candidates_t<Cfg<8, 32, 8, 8, POL>>(nbm, keys, n, i1, i2, fp);
    } else {
        if (bits == 8) host_candidates_t<Cfg<4, 8, 16, 8, POL>>(nbm, keys, n, i1, i2, fp);
        else if (bits == 16) host_candidates_t<Cfg<4, 16, 16, 8, POL>>(nbm, keys, n, i1, i2, fp);
        else host_candidates_t<Cfg<4, 32, 8, 8, POL>>(nbm, keys, n, i1, i2, fp);
    }
}

void host_candidates(uint32_t pol, uint32_t kb, uint32_t bits, uint64_t nbm, const void* keys, uint64_t n,
                     uint64_t* i1, uint64_t* i2, uint32_t* fp) {
    if (pol == CF_ALT_ADDSUB) host_candidates_p<ALT_ADDSUB>(kb, bits, nbm, keys, n, i1, i2, fp);
    else if (pol == CF_ALT_OFFSET) host_candidates_p<ALT_OFFSET>(kb, bits, nbm, keys, n, i1, i2, fp);
    else host_candidates_p<ALT_XOR>(kb, bits, nbm, keys, n, i1, i2, fp);
}

}  // namespace

namespace cfb {
// Error reporting for the other translation units of the C ABI (filter sets).
int api_fail(int status, const char* msg) { return fail(status, "%s", msg); }
int api_cuda_fail(cudaError_t e, const char* what) { return cuda_fail(e, what); }
int api_validate(const cf_config* cfg) { return validate(cfg); }
uint64_t api_num_buckets(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy) {
    return num_buckets_policy(capacity, bucket_size, alt_policy);
}
}  // namespace cfb

extern "C" {

int cf_abi_version(void) { return CF_ABI_VERSION; }

uint64_t cf_launch_count(void) { return launch_counter().load(std::memory_order_relaxed); }

const char* cf_last_error(void) { return g_err; }

const char* cf_status_string(int status) {
    switch (status) {
        case CF_OK: return "CF_OK";
        case CF_ERR_INVALID: return "CF_ERR_INVALID";
        case CF_ERR_UNSUPPORTED: return "CF_ERR_UNSUPPORTED";
        case CF_ERR_CUDA: return "CF_ERR_CUDA";
        case CF_ERR_NO_MEMORY: return "CF_ERR_NO_MEMORY";
        case CF_ERR_DEVICE: return "CF_ERR_DEVICE";
        case CF_ERR_NOT_LOADED: return "CF_ERR_NOT_LOADED";
        default: return "CF_ERR_UNKNOWN";
    }
}

int cf_config_supported(const cf_config* cfg) { return cfg && find_ops(cfg) != nullptr; }

uint64_t cf_num_buckets_for(uint64_t capacity, uint32_t bucket_size) {
    if (bucket_size == 0) return 0;
    return num_buckets_for(capacity, bucket_size);
}

uint64_t cf_num_buckets_for_policy(uint64_t capacity, uint32_t bucket_size, uint32_t alt_policy) {
    if (bucket_size == 0 || alt_policy > CF_ALT_OFFSET) return 0;
    return num_buckets_policy(capacity, bucket_size, alt_policy);
}

int cf_create(const cf_config* cfg, uint64_t capacity, cf_filter** out) {
    if (!out) return fail(CF_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (int s = validate(cfg)) return s;
    if (capacity == 0) return fail(CF_ERR_INVALID, "capacity must be > 0");
    int device = 0;
    {
        cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess) return fail(CF_ERR_NOT_LOADED, "no CUDA device: %s", cudaGetErrorString(e));
    }
    cf_filter* f = new cf_filter{};
    f->cfg = *cfg;
    f->ops = find_ops(cfg);
    f->device = device;
    f->num_buckets = num_buckets_policy(capacity, cfg->bucket_size, cfg->alt_policy);
    f->table_bytes = f->num_buckets * f->ops->bucket_bytes;
    f->block = cfg->block_size ? static_cast<int>(cfg->block_size) : 256;
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (int k = 0; e == cudaSuccess && k < KID_COUNT_KERNELS; ++k) {
        int bps = 0;
        e = f->ops->occupancy(k, f->block, &bps);
        f->max_grid[k] = sms * (bps > 0 ? bps : 1);
    }
    f->max_grid_aux = sms * 8;
    f->sms = sms;
    init_geometry(f);
    f->ws_limit = 0;  // automatic
    if (e == cudaSuccess) e = cudaHostAlloc(&f->h_cnt, 4 * sizeof(unsigned long long), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&f->d_table, f->table_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&f->d_ctr, CTR_COUNT * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaHostAlloc(&f->h_ctr, CTR_COUNT * sizeof(unsigned long long), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMemset(f->d_table, 0, f->table_bytes);
    if (e == cudaSuccess) e = cudaMemset(f->d_ctr, 0, CTR_COUNT * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        int s = cuda_fail(e, "filter allocation");
        cf_destroy(f);
        return s;
    }
    f->known_empty = true;
    *out = f;
    return CF_OK;
}

int cf_destroy(cf_filter* f) {
    if (!f) return CF_OK;
    DeviceGuard g(f->device);
    if (f->d_table) cudaFree(f->d_table);
    if (f->d_ctr) cudaFree(f->d_ctr);
    if (f->h_ctr) cudaFreeHost(f->h_ctr);
    if (f->h_cnt) cudaFreeHost(f->h_cnt);
    if (f->ws) cudaFree(f->ws);
    delete f;
    return CF_OK;
}

int cf_get_info(const cf_filter* f, cf_info* out) {
    if (int s = check_filter(f)) return s;
    if (!out) return fail(CF_ERR_INVALID, "out is NULL");
    out->num_buckets = f->num_buckets;
    out->capacity = f->num_buckets * f->cfg.bucket_size;
    out->size_in_bytes = f->table_bytes;
    out->bucket_bytes = f->ops->bucket_bytes;
    out->device = f->device;
    return CF_OK;
}

int insert_any(cf_filter* f, const void* keys, uint64_t n, uint8_t* out, void* stream, bool sorted) {
    switch (choose_path(f, SEG_INSERT, n, sorted)) {
        case PATH_REGION: return run_region(f, SEG_INSERT, keys, n, out, stream);
        case PATH_SEGMENT: return run_segmented(f, SEG_INSERT, keys, n, out, stream);
        default: return do_insert(f, keys, n, out, stream);
    }
}

int cf_insert_async(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream) {
    if (int s = check_batch(f, d_keys, n)) return s;
    DeviceGuard g(f->device);
    return insert_any(f, d_keys, n, d_out, stream, false);
}

int cf_insert(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream, uint64_t* occupied_out) {
    if (int s = check_batch(f, d_keys, n)) return s;
    DeviceGuard g(f->device);
    if (int s = insert_any(f, d_keys, n, d_out, stream, false)) return s;
    return finish(f, stream, occupied_out);
}

int cf_insert_sorted(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream,
                     uint64_t* occupied_out) {
    if (int s = check_batch(f, d_keys, n)) return s;
    DeviceGuard g(f->device);
    // (bucket << bits) | tag must fit 64 bits for the staged paths; else the plain path
    if (int s = insert_any(f, d_keys, n, d_out, stream, true)) return s;
    return finish(f, stream, occupied_out);
}

int cf_contains_async(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream) {
    if (int s = check_batch(f, d_keys, n)) return s;
    if (n && !d_out) return fail(CF_ERR_INVALID, "d_out is NULL with n > 0");
    DeviceGuard g(f->device);
    switch (choose_path(f, SEG_CONTAINS, n, false)) {
        case PATH_REGION: return run_region(f, SEG_CONTAINS, d_keys, n, d_out, stream);
        case PATH_SEGMENT: return run_segmented(f, SEG_CONTAINS, d_keys, n, d_out, stream);
        default: break;
    }
    LaunchCfg L = launch(f, KID_CONTAINS, stream);
    L.kpt = static_cast<int>(f->lookup_kpt);
    L.width = static_cast<int>(f->probe_width);
    CF_CUDA(f->ops->contains(dev(f), d_keys, n, d_out, L), "contains launch");
    return CF_OK;
}

int cf_contains(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream) {
    if (int s = cf_contains_async(f, d_keys, n, d_out, stream)) return s;
    DeviceGuard g(f->device);
    CF_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "stream synchronize");
    return CF_OK;
}

int cf_delete_async(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream) {
    if (int s = check_batch(f, d_keys, n)) return s;
    f->known_empty = false;
    DeviceGuard g(f->device);
    switch (choose_path(f, SEG_DELETE, n, false)) {
        case PATH_REGION: return run_region(f, SEG_DELETE, d_keys, n, d_out, stream);
        case PATH_SEGMENT: return run_segmented(f, SEG_DELETE, d_keys, n, d_out, stream);
        default: break;
    }
    LaunchCfg L = launch(f, KID_DELETE, stream);
    L.width = static_cast<int>(f->probe_width);
    CF_CUDA(f->ops->remove(dev(f), d_keys, n, d_out, L), "delete launch");
    return CF_OK;
}

int cf_delete(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream, uint64_t* occupied_out) {
    if (int s = cf_delete_async(f, d_keys, n, d_out, stream)) return s;
    DeviceGuard g(f->device);
    return finish(f, stream, occupied_out);
}

int cf_clear(cf_filter* f, void* stream) {
    if (int s = check_filter(f)) return s;
    DeviceGuard g(f->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CF_CUDA(cudaMemsetAsync(f->d_table, 0, f->table_bytes, s), "table clear");
    CF_CUDA(cudaMemsetAsync(f->d_ctr, 0, CTR_COUNT * sizeof(unsigned long long), s), "counter clear");
    CF_CUDA(cudaStreamSynchronize(s), "stream synchronize");
    f->known_empty = !f->table_exposed;
    return CF_OK;
}

int cf_occupied(cf_filter* f, uint64_t* out) {
    if (int s = check_filter(f)) return s;
    if (!out) return fail(CF_ERR_INVALID, "out is NULL");
    DeviceGuard g(f->device);
    unsigned long long v = 0;
    CF_CUDA(cudaMemcpy(&v, f->d_ctr + CTR_OCCUPIED, sizeof(v), cudaMemcpyDeviceToHost), "occupancy read");
    *out = v;
    return CF_OK;
}

int cf_count_occupied_slots(cf_filter* f, uint64_t* out) {
    if (int s = check_filter(f)) return s;
    if (!out) return fail(CF_ERR_INVALID, "out is NULL");
    DeviceGuard g(f->device);
    unsigned long long* d_res = nullptr;
    CF_CUDA(cudaMalloc(&d_res, sizeof(unsigned long long)), "scratch allocation");
    unsigned long long v = 0;
    cudaError_t e = cudaMemset(d_res, 0, sizeof(v));
    if (e == cudaSuccess) e = f->ops->count(dev(f), f->num_buckets, d_res, launch_aux(f, nullptr));
    if (e == cudaSuccess) e = cudaMemcpy(&v, d_res, sizeof(v), cudaMemcpyDeviceToHost);
    cudaFree(d_res);
    CF_CUDA(e, "occupied-slot count");
    *out = v;
    return CF_OK;
}

int cf_get_stats(cf_filter* f, cf_stats* out) {
    if (int s = check_filter(f)) return s;
    if (!out) return fail(CF_ERR_INVALID, "out is NULL");
    DeviceGuard g(f->device);
    unsigned long long c[CTR_COUNT];
    CF_CUDA(cudaMemcpy(c, f->d_ctr, sizeof(c), cudaMemcpyDeviceToHost), "counter read");
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

int cf_get_chain_histogram(cf_filter* f, uint64_t* bins) {
    if (int s = check_filter(f)) return s;
    if (!bins) return fail(CF_ERR_INVALID, "bins is NULL");
    DeviceGuard g(f->device);
    unsigned long long h[kChainBins];
    CF_CUDA(cudaMemcpy(h, f->d_ctr + CTR_HIST0, sizeof(h), cudaMemcpyDeviceToHost), "histogram read");
    for (int i = 0; i < kChainBins; ++i) bins[i] = h[i];
    return CF_OK;
}

int cf_reset_stats(cf_filter* f) {
    if (int s = check_filter(f)) return s;
    DeviceGuard g(f->device);
    CF_CUDA(cudaMemset(f->d_ctr + 1, 0, (CTR_COUNT - 1) * sizeof(unsigned long long)), "counter reset");
    return CF_OK;
}

int cf_table(cf_filter* f, void** d_table, uint64_t* bytes) {
    if (int s = check_filter(f)) return s;
    if (d_table) {  // the caller may write the table at any time
        f->known_empty = false;
        f->table_exposed = true;
    }
    if (d_table) *d_table = f->d_table;
    if (bytes) *bytes = f->table_bytes;
    return CF_OK;
}

int cf_load_table(cf_filter* f, const void* src, uint64_t bytes, void* stream) {
    if (int s = check_filter(f)) return s;
    if (!src) return fail(CF_ERR_INVALID, "src is NULL");
    if (bytes != f->table_bytes)
        return fail(CF_ERR_INVALID, "image is %llu bytes, table is %llu", static_cast<unsigned long long>(bytes),
                    static_cast<unsigned long long>(f->table_bytes));
    DeviceGuard g(f->device);
    f->known_empty = false;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CF_CUDA(cudaMemcpyAsync(f->d_table, src, bytes, cudaMemcpyDefault, s), "table load");
    CF_CUDA(cudaMemsetAsync(f->d_ctr + CTR_OCCUPIED, 0, sizeof(unsigned long long), s), "counter reset");
    CF_CUDA(f->ops->count(dev(f), f->num_buckets, f->d_ctr + CTR_OCCUPIED, launch_aux(f, stream)), "recount");
    CF_CUDA(cudaStreamSynchronize(s), "stream synchronize");
    return CF_OK;
}

int cf_set_option(cf_filter* f, int option, uint64_t value) {
    if (int s = check_filter(f)) return s;
    switch (option) {
        case CF_OPT_WORKSPACE_LIMIT:
            f->ws_limit = value;
            return CF_OK;
        case CF_OPT_SEGMENTED_MIN_KEYS:
            f->seg_min_keys = value;
            return CF_OK;
        case CF_OPT_ROUND2_SEGMENTED_MIN_KEYS:
            f->round2_min = value;
            return CF_OK;
        case CF_OPT_REGION_MIN_KEYS:
            f->rg_min_keys = value;
            return CF_OK;
        case CF_OPT_STAGING:
            if (value > CF_STAGING_REGION) return fail(CF_ERR_INVALID, "unknown staging mode %llu",
                                                       static_cast<unsigned long long>(value));
            f->staging = static_cast<uint32_t>(value);
            return CF_OK;
        case CF_OPT_LOOKUP_KPT:
            if (value != 0 && value != 1 && value != 2 && value != 4)
                return fail(CF_ERR_INVALID, "lookup keys per thread must be 0, 1, 2 or 4");
            f->lookup_kpt = static_cast<uint32_t>(value);
            return CF_OK;
        case CF_OPT_PROBE_WIDTH:
            if (value > 1 && ((value & (value - 1)) != 0 || value > 32 ||
                              !((f->ops->coop_widths >> __builtin_ctzll(value)) & 1u)))
                return fail(CF_ERR_INVALID,
                            "probe width %llu not supported for %u-byte buckets (lanes of 4 or 8 bytes, at most 64 slots)",
                            static_cast<unsigned long long>(value), f->ops->bucket_bytes);
            f->probe_width = static_cast<uint32_t>(value);
            return CF_OK;
        case CF_OPT_PERSISTENT:
            if (value > 1) return fail(CF_ERR_INVALID, "persistent must be 0 or 1");
            f->persistent = static_cast<uint32_t>(value);
            return CF_OK;
        case CF_OPT_CHAIN_HISTOGRAM:
            if (value > 1) return fail(CF_ERR_INVALID, "chain histogram must be 0 or 1");
            f->chain_hist = static_cast<uint32_t>(value);
            return CF_OK;
        case CF_OPT_ROUND1_CAP:
            if (value > f->cfg.bucket_size)
                return fail(CF_ERR_INVALID, "round-1 cap must be 0 (automatic) or 1..bucket_size");
            f->round1_cap = static_cast<uint32_t>(value);
            return CF_OK;
        case CF_OPT_REGION_BYTES:
            if (value & (value - 1)) return fail(CF_ERR_INVALID, "region bytes must be 0 or a power of two");
            f->rg_bytes = value;
            init_geometry(f);
            return CF_OK;
        default:
            return fail(CF_ERR_INVALID, "unknown option %d", option);
    }
}

int cf_get_option(cf_filter* f, int option, uint64_t* value) {
    if (int s = check_filter(f)) return s;
    if (!value) return fail(CF_ERR_INVALID, "value is NULL");
    switch (option) {
        case CF_OPT_WORKSPACE_LIMIT: *value = f->ws_limit; return CF_OK;
        case CF_OPT_SEGMENTED_MIN_KEYS: *value = f->seg_min_keys; return CF_OK;
        case CF_OPT_WORKSPACE_BYTES: *value = f->ws_bytes; return CF_OK;
        case CF_OPT_ROUND2_SEGMENTED_MIN_KEYS: *value = f->round2_min; return CF_OK;
        case CF_OPT_REGION_MIN_KEYS: *value = f->rg_min_keys; return CF_OK;
        case CF_OPT_STAGING: *value = f->staging; return CF_OK;
        case CF_OPT_REGION_BYTES: *value = f->rg_bytes ? f->rg_bytes : kRgRegionBytes; return CF_OK;
        case CF_OPT_REGION_COUNT: *value = f->rgeom.nreg; return CF_OK;
        case CF_OPT_LOOKUP_KPT: *value = f->lookup_kpt; return CF_OK;
        case CF_OPT_PROBE_WIDTH: *value = f->probe_width; return CF_OK;
        case CF_OPT_PERSISTENT: *value = f->persistent; return CF_OK;
        case CF_OPT_ROUND1_CAP: *value = f->round1_cap; return CF_OK;
        case CF_OPT_CHAIN_HISTOGRAM: *value = f->chain_hist; return CF_OK;
        default: return fail(CF_ERR_INVALID, "unknown option %d", option);
    }
}

int cf_store_table(cf_filter* f, void* dst, uint64_t bytes, void* stream) {
    if (int s = check_filter(f)) return s;
    if (!dst) return fail(CF_ERR_INVALID, "dst is NULL");
    if (bytes != f->table_bytes)
        return fail(CF_ERR_INVALID, "buffer is %llu bytes, table is %llu", static_cast<unsigned long long>(bytes),
                    static_cast<unsigned long long>(f->table_bytes));
    DeviceGuard g(f->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CF_CUDA(cudaMemcpyAsync(dst, f->d_table, bytes, cudaMemcpyDefault, s), "table store");
    CF_CUDA(cudaStreamSynchronize(s), "stream synchronize");
    return CF_OK;
}

int cf_hash_candidates(const cf_config* cfg, uint64_t num_buckets, const void* h_keys, uint64_t n, uint64_t* i1,
                       uint64_t* i2, uint32_t* fp) {
    if (!cfg) return fail(CF_ERR_INVALID, "config is NULL");
    const uint32_t pol = cfg->alt_policy;
    if (pol > CF_ALT_OFFSET) return fail(CF_ERR_INVALID, "alt_policy must be CF_ALT_XOR, CF_ALT_ADDSUB or CF_ALT_OFFSET");
    if (num_buckets == 0 || (pol == CF_ALT_XOR && (num_buckets & (num_buckets - 1))))
        return fail(CF_ERR_INVALID, "num_buckets must be a power of two for the XOR policy, > 0 otherwise");
    if (pol == CF_ALT_ADDSUB && num_buckets % 2 != 0)
        return fail(CF_ERR_INVALID, "num_buckets must be even for the AddSub policy");
    if (n && !h_keys) return fail(CF_ERR_INVALID, "keys is NULL with n > 0");
    const uint32_t kb = cfg->key_bytes, bits = cfg->bits_per_tag;
    if ((kb != 4 && kb != 8) || (bits != 8 && bits != 16 && bits != 32))
        return fail(CF_ERR_INVALID, "key_bytes must be 4/8 and bits_per_tag 8/16/32");
    host_candidates(pol, kb, bits, num_buckets - 1, h_keys, n, i1, i2, fp);
    return CF_OK;
}

int cf_hash64(uint32_t value_bytes, const void* h_values, uint64_t n, uint64_t* out) {
    if (value_bytes != 1 && value_bytes != 2 && value_bytes != 4 && value_bytes != 8)
        return fail(CF_ERR_INVALID, "value_bytes must be 1, 2, 4 or 8");
    if (n && (!h_values || !out)) return fail(CF_ERR_INVALID, "values or out is NULL with n > 0");
    const uint8_t* p = static_cast<const uint8_t*>(h_values);
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t v = 0;
        std::memcpy(&v, p + i * value_bytes, value_bytes);
        out[i] = value_bytes == 8   ? xxh64_u64(v)
                 : value_bytes == 4 ? xxh64_u32(static_cast<uint32_t>(v))
                 : value_bytes == 2 ? xxh64_u16(static_cast<uint32_t>(v))
                                    : xxh64_u8(static_cast<uint32_t>(v));
    }
    return CF_OK;
}

int cf_alt_buckets(const cf_config* cfg, uint64_t num_buckets, const uint64_t* buckets, const uint32_t* tags,
                   uint64_t n, uint64_t* out) {
    if (!cfg) return fail(CF_ERR_INVALID, "config is NULL");
    const uint32_t pol = cfg->alt_policy;
    if (pol > CF_ALT_OFFSET) return fail(CF_ERR_INVALID, "alt_policy must be CF_ALT_XOR, CF_ALT_ADDSUB or CF_ALT_OFFSET");
    if (num_buckets == 0 || (pol == CF_ALT_XOR && (num_buckets & (num_buckets - 1))))
        return fail(CF_ERR_INVALID, "num_buckets must be a power of two for the XOR policy, > 0 otherwise");
    if (pol == CF_ALT_ADDSUB && num_buckets % 2 != 0)
        return fail(CF_ERR_INVALID, "num_buckets must be even for the AddSub policy");
    if (n && (!buckets || !tags || !out)) return fail(CF_ERR_INVALID, "buckets, tags or out is NULL with n > 0");
    const uint32_t bits = cfg->bits_per_tag;
    if (bits != 8 && bits != 16 && bits != 32) return fail(CF_ERR_INVALID, "bits_per_tag must be 8, 16 or 32");
    const uint64_t nbm = num_buckets - 1;
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t t = bits == 32 ? tags[i] : (tags[i] & ((1u << bits) - 1u));
        uint64_t a;
#define CF_ALT_CASE(B)                                                                   \
    if (pol == CF_ALT_ADDSUB) a = alt_bucket<Cfg<8, B, 16, 8, ALT_ADDSUB>>(buckets[i], t, nbm); \
    else if (pol == CF_ALT_OFFSET) a = alt_bucket<Cfg<8, B, 16, 8, ALT_OFFSET>>(buckets[i], t, nbm); \
    else a = alt_bucket<Cfg<8, B, 16, 8>>(buckets[i], t, nbm);
        if (bits == 8) {
            CF_ALT_CASE(8)
        } else if (bits == 16) {
            CF_ALT_CASE(16)
        } else {
            CF_ALT_CASE(32)
        }
#undef CF_ALT_CASE
        out[i] = a;
    }
    return CF_OK;
}

int cf_probe_count(cf_filter* f, const void* d_keys, uint64_t n, uint64_t* primary_hits, void* stream) {
    if (int s = check_batch(f, d_keys, n)) return s;
    if (!primary_hits) return fail(CF_ERR_INVALID, "primary_hits is NULL");
    DeviceGuard g(f->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long* d_res = nullptr;
    CF_CUDA(cudaMalloc(&d_res, sizeof(unsigned long long)), "scratch allocation");
    unsigned long long v = 0;
    cudaError_t e = cudaMemsetAsync(d_res, 0, sizeof(v), s);
    if (e == cudaSuccess) e = f->ops->probe(dev(f), d_keys, n, d_res, launch_aux(f, stream));
    if (e == cudaSuccess) e = cudaMemcpyAsync(&v, d_res, sizeof(v), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_res);
    CF_CUDA(e, "probe count");
    *primary_hits = v;
    return CF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Sorted insert without allocation (cf_insert_sorted_noalloc).
//
// cf_insert_sorted grows a cudaMalloc'd workspace on demand and may free and
// re-allocate it.  Some callers cannot allow that: a cudaMalloc or cudaFree
// can synchronize the whole device (stalling the other streams of a serving
// process), and some hosts hand the library a device whose memory is already
// fully reserved by another allocator.  For them the segment-staged insert
// runs here on a fixed scratch area that is part of the library's own device
// image: a file-scope __device__ array, present on every GPU on which this
// library's code is loaded, until the process exits.  Nothing is allocated per
// call.  Like cf_insert_sorted, the call synchronizes its stream before it
// returns (it reads the per-round key counts back to the host).

namespace {

constexpr uint64_t kNoAllocMaxKeys = CF_NOALLOC_MAX_KEYS;
constexpr uint64_t kNoAllocMaxSegments = 1ull << 18;  // tables up to 16 GiB (64 KiB segments)
constexpr int kNoAllocMaxGrid = 2048;                  // radix-pass CTAs

constexpr uint64_t na_al(uint64_t x) { return (x + 255) & ~255ull; }
// Layout: two entry buffers, two payload buffers, the result bitmap (two bits
// per key, as the workspace allocator sizes it), the radix histogram, the
// segment starts and the list counters.
constexpr uint64_t kNaEnt = na_al(kNoAllocMaxKeys * 8);
constexpr uint64_t kNaPay = na_al(kNoAllocMaxKeys * 4);
constexpr uint64_t kNaBitmap = na_al((2 * kNoAllocMaxKeys + 31) / 32 * 4);
constexpr uint64_t kNaHist = na_al(static_cast<uint64_t>(kRadix) * kNoAllocMaxGrid * kRsHistSub * 4);
constexpr uint64_t kNaStart = na_al((kNoAllocMaxSegments + 1) * 4);
constexpr uint64_t kNaCnt = 256;
constexpr uint64_t kNoAllocScratchBytes = 2 * kNaEnt + 2 * kNaPay + kNaBitmap + kNaHist + kNaStart + kNaCnt;

// The scratch.  In host code this name is only a handle: the device address
// comes from cudaGetSymbolAddress (noalloc_scratch).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch on the current device.  Looked up on every
// call (the lookup allocates nothing), so an address never outlives the
// context it came from, e.g. across a cudaDeviceReset.
int noalloc_scratch(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "scratch address lookup");
    *out = p;
    return CF_OK;
}

}  // namespace

extern "C" {

uint64_t cf_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int cf_insert_sorted_noalloc(cf_filter* f, const void* d_keys, uint64_t n, uint8_t* d_out, void* stream,
                             uint64_t* occupied_out) {
    if (int s = check_batch(f, d_keys, n)) return s;
    if (n > kNoAllocMaxKeys)
        return fail(CF_ERR_INVALID, "%llu keys exceed the %llu-key limit of cf_insert_sorted_noalloc; split the batch",
                    static_cast<unsigned long long>(n), static_cast<unsigned long long>(kNoAllocMaxKeys));
    if (!f->seg_ok)
        return fail(CF_ERR_UNSUPPORTED, "bucket index and tag do not fit one 64-bit entry for this table");
    if (f->geom.nseg > kNoAllocMaxSegments)
        return fail(CF_ERR_UNSUPPORTED, "table of %llu segments exceeds the %llu-segment limit of the fixed scratch",
                    static_cast<unsigned long long>(f->geom.nseg), static_cast<unsigned long long>(kNoAllocMaxSegments));
    DeviceGuard g(f->device);
    f->known_empty = false;
    void* base = nullptr;
    if (int s = noalloc_scratch(&base)) return s;
    SegWork w{};
    CF_CUDA(rs_scatter_grid<0>(f->sms, &w.rs_grid[0]), "radix launch setup");
    CF_CUDA(rs_scatter_grid<1>(f->sms, &w.rs_grid[1]), "radix launch setup");
    CF_CUDA(rs_scatter_grid<2>(f->sms, &w.rs_grid[2]), "radix launch setup");
    for (int i = 0; i < 3; ++i)
        if (w.rs_grid[i] > kNoAllocMaxGrid) return fail(CF_ERR_UNSUPPORTED, "radix grid %d too large", w.rs_grid[i]);
    uint8_t* p = static_cast<uint8_t*>(base);
    w.ent[0] = reinterpret_cast<uint64_t*>(p);
    w.ent[1] = reinterpret_cast<uint64_t*>(p + kNaEnt);
    p += 2 * kNaEnt;
    w.pay[0] = reinterpret_cast<uint32_t*>(p);
    w.pay[1] = reinterpret_cast<uint32_t*>(p + kNaPay);
    p += 2 * kNaPay;
    w.bitmap = reinterpret_cast<uint32_t*>(p);
    p += kNaBitmap;
    w.hist = reinterpret_cast<uint32_t*>(p);
    p += kNaHist;
    w.start = reinterpret_cast<uint32_t*>(p);
    p += kNaStart;
    w.cnt = reinterpret_cast<unsigned long long*>(p);
    w.full = nullptr;  // no known-full bitmap in the fixed scratch: eviction probes every candidate
    w.full_words = 0;
    w.h_cnt = f->h_cnt;
    w.cap = kNoAllocMaxKeys;
    w.sms = f->sms;
    w.rg_grid = f->sms * 4;
    w.round2_segmented_min = f->round2_min ? f->round2_min : auto_threshold(f, SEG_INSERT);
    w.round1_cap = f->round1_cap;
    if (n) {
        // the segment pass clears the list counters, the result bitmap and the
        // segment starts itself; the other buffers are written before read
        CF_CUDA(f->ops->seg_chunk(dev(f), f->geom, w, SEG_INSERT, d_keys, n, d_out, static_cast<cudaStream_t>(stream),
                                  f->cfg.eviction_policy == CF_EVICT_BFS ? 1u : 0u, f->cfg.max_evictions),
                "segment-staged batch");
    }
    return finish(f, stream, occupied_out);
}

}  // extern "C"
