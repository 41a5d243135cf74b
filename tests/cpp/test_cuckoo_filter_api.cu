// test_cuckoo_filter_api.cu -- the reference's behavioural test suite
// (tests/test_cuckoo_filter.cu of the reference: 12 cases on
// CuckooConfig<uint32_t, 16, 500, 256, 16>) run against this repository's
// C++ drop-in header include/CuckooFilter.cuh, i.e. through the C ABI of
// libcuckoo_b200.so.  The cases are restated, not copied: same scenarios, same
// expectations, a minimal assertion harness instead of gtest (not installed).
//
// Build (tests/test_cpp_api.py does this):
//   nvcc -std=c++17 -Iinclude tests/cpp/test_cuckoo_filter_api.cu \
//        -Lcuckoo-filter_b200/lib -lcuckoo_b200 -o test_cuckoo_filter_api
#include <CuckooFilter.cuh>

#include <algorithm>
#include <cstdio>
#include <limits>
#include <random>
#include <vector>

namespace {

int g_failures = 0;
int g_checks = 0;

#define EXPECT(cond, msg)                                                                \
    do {                                                                                 \
        ++g_checks;                                                                      \
        if (!(cond)) {                                                                   \
            ++g_failures;                                                                \
            std::fprintf(stderr, "  FAILED %s:%d: %s (%s)\n", __FILE__, __LINE__, #cond, msg); \
        }                                                                                \
    } while (0)

using Config = CuckooConfig<uint32_t, 16, 500, 256, 16>;
using Filter = CuckooFilter<Config>;
constexpr double kTargetLoad = 0.95;

std::vector<uint32_t> random_keys(std::mt19937& rng, size_t n) {
    std::uniform_int_distribution<uint32_t> dist(1, std::numeric_limits<uint32_t>::max());
    std::vector<uint32_t> v(n);
    for (auto& k : v) k = dist(rng);
    return v;
}

std::vector<uint8_t> host(const thrust::device_vector<uint8_t>& d) {
    std::vector<uint8_t> h(d.size());
    thrust::copy(d.begin(), d.end(), h.begin());
    return h;
}

size_t count_true(const std::vector<uint8_t>& v) { return std::count(v.begin(), v.end(), uint8_t{1}); }

void BasicInsertAndQuery(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 2, 3, 4, 5, 100, 200, 300};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> out(keys.size());
    EXPECT(f.insertMany(d) == keys.size(), "all keys inserted");
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == keys.size(), "every key found");
}

void EmptyFilter(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 2, 3, 4, 5};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> out(keys.size());
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == 0, "an empty filter finds nothing");
}

void ClearOperation(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 2, 3, 4, 5};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> out(keys.size());
    f.insertMany(d);
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == keys.size(), "found before clear");
    f.clear();
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == 0, "nothing found after clear");
    EXPECT(f.loadFactor() == 0.0f, "load factor 0 after clear");
}

void LoadFactor(std::mt19937& rng) {
    Filter f(10000);
    EXPECT(f.loadFactor() == 0.0f, "empty load factor");
    auto keys = random_keys(rng, 5000);
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    const size_t inserted = f.insertMany(d);
    const float lf = f.loadFactor();
    EXPECT(lf > 0.0f && lf <= 1.0f, "load factor in (0, 1]");
    EXPECT(lf == static_cast<float>(inserted) / static_cast<float>(f.capacity()), "load factor = inserted / capacity");
    EXPECT(inserted > 0, "some keys inserted");
}

void NearCapacityInsertion(std::mt19937& rng) {
    const size_t n = static_cast<size_t>((1 << 20) * kTargetLoad);
    Filter f(n);
    auto keys = random_keys(rng, n);
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> out(n);
    const size_t inserted = f.insertMany(d);
    EXPECT(inserted > n * 0.99, "at least 99% inserted");
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) > inserted * 0.99, "at least 99% of inserted found");
}

void DuplicateInsertions(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 1, 2, 2, 3, 3, 4, 4, 5, 5};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    EXPECT(f.insertMany(d) == keys.size(), "duplicates are stored as separate copies");
    std::vector<uint32_t> uniq = {1, 2, 3, 4, 5};
    thrust::device_vector<uint32_t> du(uniq.begin(), uniq.end());
    thrust::device_vector<uint8_t> out(uniq.size());
    f.containsMany(du, out);
    EXPECT(count_true(host(out)) == uniq.size(), "every unique key found");
}

void BasicDeletion(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 2, 3, 4, 5, 100, 200, 300};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> out(keys.size());
    EXPECT(f.insertMany(d) == keys.size(), "all inserted");
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == keys.size(), "found before deletion");
    thrust::device_vector<uint8_t> del(keys.size());
    const size_t remaining = f.deleteMany(d, del);
    EXPECT(count_true(host(del)) == keys.size(), "every key deleted");
    EXPECT(remaining == 0, "nothing remains");
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == 0, "nothing found after deletion");
}

void DeleteNonExistentKeys(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 2, 3, 4, 5};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> del(keys.size());
    f.deleteMany(d, del);
    EXPECT(count_true(host(del)) == 0, "no absent key deleted");
}

void PartialDeletion(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> ins = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
    thrust::device_vector<uint32_t> di(ins.begin(), ins.end());
    EXPECT(f.insertMany(di) == ins.size(), "all inserted");
    std::vector<uint32_t> dk = {2, 4, 6, 8, 10};
    thrust::device_vector<uint32_t> dd(dk.begin(), dk.end());
    thrust::device_vector<uint8_t> del(dk.size());
    const size_t remaining = f.deleteMany(dd, del);
    EXPECT(count_true(host(del)) == dk.size(), "every even key deleted");
    EXPECT(remaining == 5, "five keys remain");
    thrust::device_vector<uint8_t> out(dk.size());
    f.containsMany(dd, out);
    EXPECT(count_true(host(out)) == 0, "deleted keys not found");
    std::vector<uint32_t> rest = {1, 3, 5, 7, 9};
    thrust::device_vector<uint32_t> dr(rest.begin(), rest.end());
    thrust::device_vector<uint8_t> ro(rest.size());
    f.containsMany(dr, ro);
    EXPECT(count_true(host(ro)) == rest.size(), "remaining keys still found");
}

void DeleteAndReinsert(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 2, 3, 4, 5};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    thrust::device_vector<uint8_t> out(keys.size());
    f.insertMany(d);
    f.deleteMany(d);
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == 0, "not found after deletion");
    EXPECT(f.insertMany(d) == keys.size(), "reinserted");
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == keys.size(), "found after reinsertion");
}

void LoadFactorAfterDeletion(std::mt19937& rng) {
    Filter f(10000);
    auto keys = random_keys(rng, 1000);
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    f.insertMany(d);
    const float before = f.loadFactor();
    EXPECT(before > 0.0f, "positive load factor");
    const size_t remaining = f.deleteMany(d);
    const float after = f.loadFactor();
    EXPECT(after < before, "load factor decreases");
    EXPECT(after == static_cast<float>(remaining) / static_cast<float>(f.capacity()), "load factor = remaining / capacity");
}

void DeleteDuplicates(std::mt19937&) {
    Filter f(10000);
    std::vector<uint32_t> keys = {1, 1, 1, 2, 2, 3};
    thrust::device_vector<uint32_t> d(keys.begin(), keys.end());
    f.insertMany(d);
    std::vector<uint32_t> dk = {1, 1, 1};
    thrust::device_vector<uint32_t> dd(dk.begin(), dk.end());
    thrust::device_vector<uint8_t> del(dk.size());
    f.deleteMany(dd, del);
    EXPECT(count_true(host(del)) >= 1, "at least one deletion succeeds");
}

// Beyond the reference's suite: the sorted insert, the static helpers and the
// error path of the drop-in.
void SortedInsertAndHelpers(std::mt19937& rng) {
    using Cfg64 = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
    CuckooFilter<Cfg64> f(1 << 16);
    EXPECT(f.getNumBuckets() == (1u << 12) && f.numBuckets == (1u << 12), "numBuckets");
    EXPECT(f.sizeInBytes() == (1u << 12) * 32, "sizeInBytes");
    std::vector<uint64_t> keys(50000);
    std::uniform_int_distribution<uint64_t> dist;
    for (auto& k : keys) k = dist(rng);
    thrust::device_vector<uint64_t> d(keys.begin(), keys.end());
    const size_t occ = f.insertManySorted(d);
    EXPECT(occ == keys.size(), "sorted insert stores all keys at 76% load");
    EXPECT(f.countOccupiedSlots() == occ, "image count equals the counter");
    thrust::device_vector<uint8_t> out(keys.size());
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == keys.size(), "no false negatives");
    // static helpers: key 1 at 2^16 buckets (known answer of the reference's hashing)
    EXPECT(CuckooFilter<Cfg64>::hash64(1) == 0x9F29CB17A2A49995ull, "hash64 known answer");
    auto [i1, i2, fp] = CuckooFilter<Cfg64>::getCandidateBuckets(1, 1 << 16);
    EXPECT(i1 == 39317 && i2 == 24287 && fp == 51991, "getCandidateBuckets known answer");
    EXPECT(CuckooFilter<Cfg64>::getAlternateBucket(i2, fp, 1 << 16) == i1, "alternate bucket is an involution");
    EXPECT(CuckooFilter<Cfg64>::calculateNumBuckets(1 << 20) == (1 << 16), "calculateNumBuckets");
    bool threw = false;
    try {
        f.containsMany(nullptr, 5, nullptr);
    } catch (const cuckoo_b200::Error& e) {
        threw = e.status() == CF_ERR_INVALID;
    }
    EXPECT(threw, "a NULL batch raises cuckoo_b200::Error(CF_ERR_INVALID)");
}

// The AddSub and Offset alternate-bucket policies through the drop-in
// (the reference's bucket_policy_benchmark.cu:16-17 configurations).
template <template <typename, typename, std::size_t, std::size_t> class Policy>
void PolicyFilter(std::mt19937& rng) {
    using Cfg = CuckooConfig<uint64_t, 16, 500, 128, 16, Policy>;
    using F = CuckooFilter<Cfg>;
    const size_t cap = 100003;  // not a power of two: these policies keep ceil(cap / 16) buckets
    F f(cap);
    EXPECT(f.getNumBuckets() == F::calculateNumBuckets(cap) && f.getNumBuckets() >= cap / 16, "bucket count");
    std::vector<uint64_t> keys(static_cast<size_t>(0.9 * f.capacity()));
    std::uniform_int_distribution<uint64_t> dist;
    for (auto& k : keys) k = dist(rng);
    thrust::device_vector<uint64_t> d(keys.begin(), keys.end());
    EXPECT(f.insertMany(d) == keys.size(), "all keys stored at 90% load");
    thrust::device_vector<uint8_t> out(keys.size());
    f.containsMany(d, out);
    EXPECT(count_true(host(out)) == keys.size(), "no false negatives");
    auto [i1, i2, fp] = F::getCandidateBuckets(keys[0], f.getNumBuckets());
    auto [alt, afp] = F::getAlternateBucketWithNewFp(i1, fp, f.getNumBuckets());
    EXPECT(alt == i2, "alternate of the primary bucket is i2");
    auto [back, bfp] = F::getAlternateBucketWithNewFp(alt, afp, f.getNumBuckets());
    EXPECT(back == i1 && bfp == fp, "moving twice returns the tag home");
    thrust::device_vector<uint8_t> del(keys.size());
    EXPECT(f.deleteMany(d, del) == 0, "every key deleted");
}

void AddSubPolicy(std::mt19937& rng) { PolicyFilter<AddSubAltBucketPolicy>(rng); }
void OffsetPolicy(std::mt19937& rng) { PolicyFilter<OffsetAltBucketPolicy>(rng); }

}  // namespace

int main() {
    struct Case {
        const char* name;
        void (*fn)(std::mt19937&);
    } cases[] = {{"BasicInsertAndQuery", BasicInsertAndQuery},
                 {"EmptyFilter", EmptyFilter},
                 {"ClearOperation", ClearOperation},
                 {"LoadFactor", LoadFactor},
                 {"NearCapacityInsertion", NearCapacityInsertion},
                 {"DuplicateInsertions", DuplicateInsertions},
                 {"BasicDeletion", BasicDeletion},
                 {"DeleteNonExistentKeys", DeleteNonExistentKeys},
                 {"PartialDeletion", PartialDeletion},
                 {"DeleteAndReinsert", DeleteAndReinsert},
                 {"LoadFactorAfterDeletion", LoadFactorAfterDeletion},
                 {"DeleteDuplicates", DeleteDuplicates},
                 {"SortedInsertAndHelpers", SortedInsertAndHelpers},
                 {"AddSubPolicy", AddSubPolicy},
                 {"OffsetPolicy", OffsetPolicy}};
    for (const Case& c : cases) {
        std::mt19937 rng(42);  // the reference's fixture seeds every case with 42
        const int before = g_failures;
        try {
            c.fn(rng);
        } catch (const std::exception& e) {
            ++g_failures;
            std::fprintf(stderr, "  EXCEPTION in %s: %s\n", c.name, e.what());
        }
        std::printf("[%s] %s\n", g_failures == before ? "  OK  " : "FAILED", c.name);
    }
    std::printf("%d checks, %d failures\n", g_checks, g_failures);
    return g_failures == 0 ? 0 : 1;
}
