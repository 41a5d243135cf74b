// ref_gpu.cu -- C-ABI shim that runs the reference's own CUDA kernels.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against
// the reference's include/CuckooFilter.cuh where it lies, for sm_100a, into
// oracle/_ref/libref_gpu.so.  Nothing of the reference is copied: this file only
// instantiates the reference's CuckooFilter<Config> and forwards to its public
// member functions (CuckooFilter.cuh:457 insertMany, :475 insertManySorted,
// :518 containsMany, :536 deleteMany, :675 clear, :699 occupiedSlots).
//
// The reference kernels dereference the filter object's `this` pointer on the
// device (CuckooFilter.cuh:459,501,520,543), so the object is placed in managed
// memory, as the reference's own multi-GPU wrapper does
// (CuckooFilterMultiGPU.cuh:356-357).  Built with the sm_100a gencode, the
// reference's 256-bit load path (CuckooFilter.cuh:302-319) is live.
#include <cstdint>
#include <new>

#include <CuckooFilter.cuh>

namespace {

using XorU64_16_BFS = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
using XorU64_16_DFS = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::DFS>;
using XorU64_8_BFS = CuckooConfig<uint64_t, 8, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
using XorU64_8_DFS = CuckooConfig<uint64_t, 8, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::DFS>;
using XorU64_32_BFS = CuckooConfig<uint64_t, 32, 500, 256, 8, XorAltBucketPolicy, EvictionPolicy::BFS>;
using XorU64_32_DFS = CuckooConfig<uint64_t, 32, 500, 256, 8, XorAltBucketPolicy, EvictionPolicy::DFS>;
using XorU32_16_DFS = CuckooConfig<uint32_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::DFS>;
using XorU64_16_DFS_E16 = CuckooConfig<uint64_t, 16, 16, 256, 16, XorAltBucketPolicy, EvictionPolicy::DFS>;
using XorU64_16_BFS_E16 = CuckooConfig<uint64_t, 16, 16, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
using XorU64_32_DFS_E16 = CuckooConfig<uint64_t, 32, 16, 256, 8, XorAltBucketPolicy, EvictionPolicy::DFS>;
using XorU64_32_BFS_E16 = CuckooConfig<uint64_t, 32, 16, 256, 8, XorAltBucketPolicy, EvictionPolicy::BFS>;
// 32-bit WordType (the reference's word-width comparison, benchmark/cuckoo_atomics_comparison.cu)
using XorU64_8_DFS_W32 = CuckooConfig<uint64_t, 8, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::DFS, uint32_t>;
using XorU64_8_BFS_W32 = CuckooConfig<uint64_t, 8, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS, uint32_t>;
using XorU64_16_DFS_W32 = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::DFS, uint32_t>;
using XorU64_16_BFS_E16_W32 =
    CuckooConfig<uint64_t, 16, 16, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS, uint32_t>;
// AddSub and Offset alternate-bucket policies (benchmark/bucket_policy_benchmark.cu:16-17)
using AddSubU64_16_BFS = CuckooConfig<uint64_t, 16, 500, 256, 16, AddSubAltBucketPolicy, EvictionPolicy::BFS>;
using AddSubU64_16_DFS = CuckooConfig<uint64_t, 16, 500, 256, 16, AddSubAltBucketPolicy, EvictionPolicy::DFS>;
using OffsetU64_16_BFS = CuckooConfig<uint64_t, 16, 500, 256, 16, OffsetAltBucketPolicy, EvictionPolicy::BFS>;
using OffsetU64_16_DFS = CuckooConfig<uint64_t, 16, 500, 256, 16, OffsetAltBucketPolicy, EvictionPolicy::DFS>;
using OffsetU64_16_DFS_E16 = CuckooConfig<uint64_t, 16, 16, 256, 16, OffsetAltBucketPolicy, EvictionPolicy::DFS>;
using AddSubU64_16_DFS_E16 = CuckooConfig<uint64_t, 16, 16, 256, 16, AddSubAltBucketPolicy, EvictionPolicy::DFS>;

template <typename Cfg>
struct Shim {
    using F = CuckooFilter<Cfg>;
    using K = typename Cfg::KeyType;

    static void* create(size_t capacity) {
        void* mem = nullptr;
        if (cudaMallocManaged(&mem, sizeof(F)) != cudaSuccess) return nullptr;
        new (mem) F(capacity);
        return mem;
    }
    static void destroy(void* h) {
        static_cast<F*>(h)->~F();
        cudaFree(h);
    }
    static size_t insert(void* h, const void* keys, size_t n, cudaStream_t s, int sorted) {
        F* f = static_cast<F*>(h);
        return sorted ? f->insertManySorted(static_cast<const K*>(keys), n, s)
                      : f->insertMany(static_cast<const K*>(keys), n, s);
    }
    static void contains(void* h, const void* keys, size_t n, uint8_t* out, cudaStream_t s) {
        static_cast<F*>(h)->containsMany(static_cast<const K*>(keys), n, reinterpret_cast<bool*>(out), s);
    }
    static size_t remove(void* h, const void* keys, size_t n, uint8_t* out, cudaStream_t s) {
        return static_cast<F*>(h)->deleteMany(static_cast<const K*>(keys), n, reinterpret_cast<bool*>(out), s);
    }
    static void clear(void* h) { static_cast<F*>(h)->clear(); }
    static size_t occupied(void* h) { return static_cast<F*>(h)->occupiedSlots(); }
    static void* table(void* h) { return static_cast<F*>(h)->d_buckets; }
    static size_t table_bytes(void* h) { return static_cast<F*>(h)->sizeInBytes(); }
    static size_t num_buckets(void* h) { return static_cast<F*>(h)->getNumBuckets(); }
};

struct Ops {
    void* (*create)(size_t);
    void (*destroy)(void*);
    size_t (*insert)(void*, const void*, size_t, cudaStream_t, int);
    void (*contains)(void*, const void*, size_t, uint8_t*, cudaStream_t);
    size_t (*remove)(void*, const void*, size_t, uint8_t*, cudaStream_t);
    void (*clear)(void*);
    size_t (*occupied)(void*);
    void* (*table)(void*);
    size_t (*table_bytes)(void*);
    size_t (*num_buckets)(void*);
};

template <typename Cfg>
constexpr Ops ops_of() {
    using S = Shim<Cfg>;
    return Ops{S::create, S::destroy, S::insert, S::contains, S::remove,
               S::clear,  S::occupied, S::table, S::table_bytes, S::num_buckets};
}

// Index = configuration id used by the Python side (oracle/refgpu.py).
const Ops kOps[] = {
    ops_of<XorU64_16_BFS>(),     ops_of<XorU64_16_DFS>(),     ops_of<XorU64_8_BFS>(),
    ops_of<XorU64_8_DFS>(),      ops_of<XorU64_32_BFS>(),     ops_of<XorU64_32_DFS>(),
    ops_of<XorU32_16_DFS>(),     ops_of<XorU64_16_DFS_E16>(), ops_of<XorU64_16_BFS_E16>(),
    ops_of<XorU64_32_DFS_E16>(), ops_of<XorU64_32_BFS_E16>(), ops_of<XorU64_8_DFS_W32>(),
    ops_of<XorU64_8_BFS_W32>(),  ops_of<XorU64_16_DFS_W32>(), ops_of<XorU64_16_BFS_E16_W32>(),
    ops_of<AddSubU64_16_BFS>(),  ops_of<AddSubU64_16_DFS>(),  ops_of<OffsetU64_16_BFS>(),
    ops_of<OffsetU64_16_DFS>(),  ops_of<OffsetU64_16_DFS_E16>(), ops_of<AddSubU64_16_DFS_E16>(),
};
constexpr int kNumOps = sizeof(kOps) / sizeof(kOps[0]);

const Ops* get(int id) { return (id >= 0 && id < kNumOps) ? &kOps[id] : nullptr; }

}  // namespace

extern "C" {

int refg_num_configs() { return kNumOps; }

void* refg_create(int id, size_t capacity) {
    const Ops* o = get(id);
    return o ? o->create(capacity) : nullptr;
}
void refg_destroy(int id, void* h) { if (const Ops* o = get(id)) o->destroy(h); }
size_t refg_insert(int id, void* h, const void* keys, size_t n, void* stream, int sorted) {
    return get(id)->insert(h, keys, n, static_cast<cudaStream_t>(stream), sorted);
}
void refg_contains(int id, void* h, const void* keys, size_t n, uint8_t* out, void* stream) {
    get(id)->contains(h, keys, n, out, static_cast<cudaStream_t>(stream));
}
size_t refg_delete(int id, void* h, const void* keys, size_t n, uint8_t* out, void* stream) {
    return get(id)->remove(h, keys, n, out, static_cast<cudaStream_t>(stream));
}
void refg_clear(int id, void* h) { get(id)->clear(h); }
size_t refg_occupied(int id, void* h) { return get(id)->occupied(h); }
void* refg_table(int id, void* h) { return get(id)->table(h); }
size_t refg_table_bytes(int id, void* h) { return get(id)->table_bytes(h); }
size_t refg_num_buckets(int id, void* h) { return get(id)->num_buckets(h); }

}  // extern "C"
