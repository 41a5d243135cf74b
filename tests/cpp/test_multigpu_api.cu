// test_multigpu_api.cu -- the C++ drop-in include/CuckooFilterMultiGPU.cuh,
// written the way the reference's multi-GPU example uses its class
// (src/multi_gpu_main.cu: insert a host vector, look it up, look up keys never
// inserted, delete some, look up the rest).  The shards share one GPU here
// (the machine that runs the tests has one), which exercises the same
// grouping, copies and per-shard calls without kernels that wait on each
// other.  Checked: counts, per-key results aligned with the keys, that every
// key sits in shard hash64(key) % numShards (or its remixed form), multi-round
// batches, clear, both host container types and the transfer-plan form.
//
// Build (tests/test_cpp_multigpu.py does this):
//   nvcc -std=c++17 -Iinclude tests/cpp/test_multigpu_api.cu \
//        -Lcuckoo-filter_b200/lib -lcuckoo_b200 -o test_multigpu_api
#include <CuckooFilterMultiGPU.cuh>
#include <thrust/host_vector.h>

#include <cstdio>
#include <random>
#include <vector>

namespace {

int g_failures = 0;

#define EXPECT(cond, msg)                                                                         \
    do {                                                                                          \
        if (!(cond)) {                                                                            \
            ++g_failures;                                                                         \
            std::fprintf(stderr, "  FAILED %s:%d: %s (%s)\n", __FILE__, __LINE__, #cond, msg); \
        }                                                                                         \
    } while (0)

using Config = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
using Multi = CuckooFilterMultiGPU<Config>;

std::vector<uint64_t> keys_of(uint64_t seed, size_t n) {
    std::mt19937_64 rng(seed);
    std::vector<uint64_t> v(n);
    for (auto& k : v) k = rng();
    return v;
}

uint64_t remix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

std::vector<uint32_t> shards_of(const std::vector<uint64_t>& keys, size_t n, cf_shard_routing routing) {
    std::vector<uint64_t> h(keys.size());
    cuckoo_b200::check(cf_hash64(8, keys.data(), keys.size(), h.data()), "cf_hash64");
    std::vector<uint32_t> s(keys.size());
    for (size_t i = 0; i < keys.size(); ++i) s[i] = (routing == CF_SHARD_REMIXED ? remix64(h[i]) : h[i]) % n;
    return s;
}

// Every key found in the shard it routes to, and the shard holds no more
// tags than keys were routed to it.
void check_placement(const Multi& f, const std::vector<uint64_t>& keys, cf_shard_routing routing) {
    const size_t n = f.numShards();
    const auto sh = shards_of(keys, n, routing);
    for (size_t s = 0; s < n; ++s) {
        std::vector<uint64_t> mine;
        for (size_t i = 0; i < keys.size(); ++i)
            if (sh[i] == s) mine.push_back(keys[i]);
        cudaSetDevice(f.shardDevice(s));
        uint64_t* d = nullptr;
        uint8_t* o = nullptr;
        cudaMalloc(&d, mine.size() * 8 + 8);
        cudaMalloc(&o, mine.size() + 1);
        cudaMemcpy(d, mine.data(), mine.size() * 8, cudaMemcpyHostToDevice);
        cuckoo_b200::check(cf_contains(f.shard(s), d, mine.size(), o, nullptr), "cf_contains");
        std::vector<uint8_t> h(mine.size());
        cudaMemcpy(h.data(), o, mine.size(), cudaMemcpyDeviceToHost);
        size_t found = 0;
        for (uint8_t b : h) found += b;
        EXPECT(found == mine.size(), "every key is in the shard it routes to");
        uint64_t occ = 0;
        cuckoo_b200::check(cf_occupied(f.shard(s), &occ), "cf_occupied");
        EXPECT(occ == mine.size(), "a shard holds exactly the keys routed to it");
        cudaFree(d);
        cudaFree(o);
    }
}

void Scenario(const char* name, size_t shards, cf_shard_routing routing, size_t slice) {
    Multi f(shards, 1 << 20, std::vector<int>{0}, routing);
    if (slice) f.setSliceKeys(slice);
    // SDIV(capacity, numGPUs) * 1.02 (the reference's per-GPU capacity)
    EXPECT(f.numShards() == shards && f.capacityPerGPU() == size_t(double(((1 << 20) + shards - 1) / shards) * 1.02),
           "geometry");
    const auto keys = keys_of(11 + shards, 300000);
    EXPECT(f.insertMany(keys) == keys.size(), "insertMany returns totalOccupiedSlots()");
    thrust::host_vector<bool> out;
    f.containsMany(keys, out);
    size_t found = 0;
    for (bool b : out) found += b;
    EXPECT(out.size() == keys.size() && found == keys.size(), "every inserted key found");
    const auto neg = keys_of(999, 100000);
    std::vector<bool> nout;
    f.containsMany(neg, nout);
    size_t fp = 0;
    for (bool b : nout) fp += b;
    EXPECT(fp < neg.size() / 100, "few false positives");
    check_placement(f, keys, routing);
    // results aligned with the keys: interleave stored and never-stored keys
    std::vector<uint64_t> mix;
    for (size_t i = 0; i < 20000; ++i) {
        mix.push_back(keys[i]);
        mix.push_back(neg[i]);
    }
    std::vector<bool> mout;
    f.containsMany(mix, mout);
    size_t pos_ok = 0, neg_hits = 0;
    for (size_t i = 0; i < mix.size(); i += 2) {
        pos_ok += mout[i];
        neg_hits += mout[i + 1];
    }
    EXPECT(pos_ok == 20000 && neg_hits < 400, "per-key results follow the caller's order");
    std::vector<uint64_t> half(keys.begin(), keys.begin() + keys.size() / 2);
    std::vector<uint64_t> rest(keys.begin() + keys.size() / 2, keys.end());
    thrust::host_vector<bool> dout;
    EXPECT(f.deleteMany(half, dout) == rest.size(), "deleteMany returns totalOccupiedSlots()");
    size_t removed = 0;
    for (bool b : dout) removed += b;
    EXPECT(removed == half.size(), "every stored key deleted");
    std::vector<bool> rout;
    f.containsMany(rest, rout);
    found = 0;
    for (bool b : rout) found += b;
    EXPECT(found == rest.size(), "the other keys stay");
    EXPECT(f.deleteMany(rest) == 0, "deleteMany without results");
    EXPECT(f.totalOccupiedSlots() == 0 && f.loadFactor() == 0.0f, "empty after deleting everything");
    f.insertMany(rest);
    f.clear();
    EXPECT(f.totalOccupiedSlots() == 0, "clear");
    EXPECT(f.totalCapacity() > 0 && f.sizeInBytes() == f.totalCapacity() * 2, "totals (16-bit tags)");
    f.synchronizeAllGPUs();
    std::printf("[  OK  ] %s\n", name);
}

void ReferenceConstructors() {
    int ndev = 0;
    cudaGetDeviceCount(&ndev);
    Multi a(1, 100000);
    const auto keys = keys_of(5, 50000);
    EXPECT(a.insertMany(keys) == keys.size(), "one GPU, default constructor");
    Multi b(1, 100000, "no_such_plan.txt");
    EXPECT(b.insertMany(keys) == keys.size(), "transfer-plan constructor");
    EXPECT(ndev >= 1, "a device");
    std::printf("[  OK  ] ReferenceConstructors\n");
}

}  // namespace

int main() {
    try {
        Scenario("FourShardsReferenceRouting", 4, CF_SHARD_REFERENCE, 0);
        Scenario("ThreeShardsRemixedRouting", 3, CF_SHARD_REMIXED, 0);
        Scenario("EightShardsManyRounds", 8, CF_SHARD_REFERENCE, 7001);
        Scenario("OneShard", 1, CF_SHARD_REFERENCE, 0);
        ReferenceConstructors();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "exception: %s\n", e.what());
        return 2;
    }
    std::printf("%d failures\n", g_failures);
    return g_failures ? 1 : 0;
}
