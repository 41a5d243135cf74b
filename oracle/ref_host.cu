// ref_host.cu -- C-ABI shim over the reference's own host-callable hashing.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the reference
// headers where they lie (include/hashutil.cuh, include/bucket_policies.cuh,
// include/helpers.cuh); output goes to oracle/_ref/libref_host.so.  It pins the
// oracle's hashing to the reference's: XorAltBucketPolicy::getCandidateBuckets
// (bucket_policies.cuh:46-61), calculateNumBuckets (:80-83) and
// xxhash::xxhash64 (hashutil.cuh:71-161) are called exactly as compiled from
// the reference sources.
#include <cstdint>
#include <cstring>

#include <bucket_policies.cuh>

namespace {

template <typename Key, typename Tag, size_t bits, size_t bs>
void candidates(const void* keys, size_t n, uint64_t nb, uint64_t* i1, uint64_t* i2, uint32_t* fp) {
    using P = XorAltBucketPolicy<Key, Tag, bits, bs>;
    const Key* k = static_cast<const Key*>(keys);
    for (size_t i = 0; i < n; ++i) {
        auto [a, b, f] = P::getCandidateBuckets(k[i], nb);
        i1[i] = a;
        i2[i] = b;
        fp[i] = f;
    }
}

template <typename Key>
int dispatch(uint32_t bits, uint32_t bs, const void* keys, size_t n, uint64_t nb, uint64_t* i1,
             uint64_t* i2, uint32_t* fp) {
    // bucketSize only enters calculateNumBuckets, never getCandidateBuckets;
    // instantiate with 16 and pass the bucket count explicitly.
    (void)bs;
    switch (bits) {
        case 8: candidates<Key, uint8_t, 8, 16>(keys, n, nb, i1, i2, fp); return 0;
        case 16: candidates<Key, uint16_t, 16, 16>(keys, n, nb, i1, i2, fp); return 0;
        case 32: candidates<Key, uint32_t, 32, 16>(keys, n, nb, i1, i2, fp); return 0;
        default: return -1;
    }
}

}  // namespace

extern "C" {

int ref_candidates(uint32_t key_bytes, uint32_t bits, uint32_t bucket_size, uint64_t num_buckets,
                   const void* keys, size_t n, uint64_t* i1, uint64_t* i2, uint32_t* fp) {
    if (key_bytes == 8) return dispatch<uint64_t>(bits, bucket_size, keys, n, num_buckets, i1, i2, fp);
    if (key_bytes == 4) return dispatch<uint32_t>(bits, bucket_size, keys, n, num_buckets, i1, i2, fp);
    return -1;
}

uint64_t ref_xxhash64(const void* data, size_t len) {
    switch (len) {
        case 1: { uint8_t v; std::memcpy(&v, data, 1); return xxhash::xxhash64(v); }
        case 2: { uint16_t v; std::memcpy(&v, data, 2); return xxhash::xxhash64(v); }
        case 4: { uint32_t v; std::memcpy(&v, data, 4); return xxhash::xxhash64(v); }
        case 8: { uint64_t v; std::memcpy(&v, data, 8); return xxhash::xxhash64(v); }
        default: return 0;
    }
}

uint64_t ref_num_buckets(uint64_t capacity, uint32_t bucket_size) {
    switch (bucket_size) {
        case 2: return XorAltBucketPolicy<uint64_t, uint32_t, 32, 2>::calculateNumBuckets(capacity);
        case 4: return XorAltBucketPolicy<uint64_t, uint16_t, 16, 4>::calculateNumBuckets(capacity);
        case 8: return XorAltBucketPolicy<uint64_t, uint16_t, 16, 8>::calculateNumBuckets(capacity);
        case 16: return XorAltBucketPolicy<uint64_t, uint16_t, 16, 16>::calculateNumBuckets(capacity);
        case 32: return XorAltBucketPolicy<uint64_t, uint16_t, 16, 32>::calculateNumBuckets(capacity);
        case 64: return XorAltBucketPolicy<uint64_t, uint8_t, 8, 64>::calculateNumBuckets(capacity);
        default: return 0;
    }
}

}  // extern "C"
