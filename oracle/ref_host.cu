// ref_host.cu -- C-ABI shim over the reference's own host-callable hashing.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the reference
// headers where they lie (include/hashutil.cuh, include/bucket_policies.cuh,
// include/helpers.cuh); output goes to oracle/_ref/libref_host.so.  It pins the
// oracle's hashing to the reference's: XorAltBucketPolicy::getCandidateBuckets
// (bucket_policies.cuh:46-61), calculateNumBuckets (:80-83) and
// xxhash::xxhash64 (hashutil.cuh:71-161) are called exactly as compiled from
// the reference sources.  The same holds for AddSubAltBucketPolicy and
// OffsetAltBucketPolicy (bucket_policies.cuh:95-350): candidates, the
// alternate bucket with the tag it is stored under there
// (getAlternateBucketWithNewFp, CuckooFilter.cuh:394-401) and the bucket count.
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

template <template <typename, typename, size_t, size_t> class Pol, typename Key, typename Tag, size_t bits>
void pol_candidates(const void* keys, size_t n, uint64_t nb, uint64_t* i1, uint64_t* i2, uint32_t* fp) {
    using P = Pol<Key, Tag, bits, 16>;
    const Key* k = static_cast<const Key*>(keys);
    for (size_t i = 0; i < n; ++i) {
        auto [a, b, f] = P::getCandidateBuckets(k[i], nb);
        i1[i] = a;
        i2[i] = b;
        fp[i] = f;
    }
}

template <template <typename, typename, size_t, size_t> class Pol, typename Key>
int pol_dispatch(uint32_t bits, const void* keys, size_t n, uint64_t nb, uint64_t* i1, uint64_t* i2,
                 uint32_t* fp) {
    switch (bits) {
        case 8: pol_candidates<Pol, Key, uint8_t, 8>(keys, n, nb, i1, i2, fp); return 0;
        case 16: pol_candidates<Pol, Key, uint16_t, 16>(keys, n, nb, i1, i2, fp); return 0;
        case 32: pol_candidates<Pol, Key, uint32_t, 32>(keys, n, nb, i1, i2, fp); return 0;
        default: return -1;
    }
}

template <template <typename, typename, size_t, size_t> class Pol>
int pol_keys(uint32_t key_bytes, uint32_t bits, const void* keys, size_t n, uint64_t nb, uint64_t* i1,
             uint64_t* i2, uint32_t* fp) {
    if (key_bytes == 8) return pol_dispatch<Pol, uint64_t>(bits, keys, n, nb, i1, i2, fp);
    if (key_bytes == 4) return pol_dispatch<Pol, uint32_t>(bits, keys, n, nb, i1, i2, fp);
    return -1;
}

// Alternate bucket of (bucket, tag) and the tag as stored there.
template <typename Tag, size_t bits>
uint64_t pol_alt(uint32_t policy, uint64_t nb, uint64_t bucket, uint32_t tag, uint32_t* new_tag) {
    const Tag t = static_cast<Tag>(tag);
    if (policy == 1) {
        *new_tag = tag;
        return AddSubAltBucketPolicy<uint64_t, Tag, bits, 16>::getAlternateBucket(bucket, t, nb);
    }
    if (policy == 2) {
        auto [alt, nt] = OffsetAltBucketPolicy<uint64_t, Tag, bits, 16>::getAlternateBucketWithNewFp(bucket, t, nb);
        *new_tag = nt;
        return alt;
    }
    *new_tag = tag;
    return XorAltBucketPolicy<uint64_t, Tag, bits, 16>::getAlternateBucket(bucket, t, nb);
}

}  // namespace

extern "C" {

// policy: 0 XorAltBucketPolicy, 1 AddSubAltBucketPolicy, 2 OffsetAltBucketPolicy.
int ref_candidates_policy(uint32_t policy, uint32_t key_bytes, uint32_t bits, uint64_t num_buckets,
                          const void* keys, size_t n, uint64_t* i1, uint64_t* i2, uint32_t* fp) {
    switch (policy) {
        case 0: return pol_keys<XorAltBucketPolicy>(key_bytes, bits, keys, n, num_buckets, i1, i2, fp);
        case 1: return pol_keys<AddSubAltBucketPolicy>(key_bytes, bits, keys, n, num_buckets, i1, i2, fp);
        case 2: return pol_keys<OffsetAltBucketPolicy>(key_bytes, bits, keys, n, num_buckets, i1, i2, fp);
        default: return -1;
    }
}

int ref_alt_policy(uint32_t policy, uint32_t bits, uint64_t num_buckets, const uint64_t* buckets,
                   const uint32_t* tags, size_t n, uint64_t* alt, uint32_t* new_tags) {
    for (size_t i = 0; i < n; ++i) {
        switch (bits) {
            case 8: alt[i] = pol_alt<uint8_t, 8>(policy, num_buckets, buckets[i], tags[i], &new_tags[i]); break;
            case 16: alt[i] = pol_alt<uint16_t, 16>(policy, num_buckets, buckets[i], tags[i], &new_tags[i]); break;
            case 32: alt[i] = pol_alt<uint32_t, 32>(policy, num_buckets, buckets[i], tags[i], &new_tags[i]); break;
            default: return -1;
        }
    }
    return 0;
}

uint64_t ref_num_buckets_policy(uint32_t policy, uint64_t capacity) {
    switch (policy) {
        case 1: return AddSubAltBucketPolicy<uint64_t, uint16_t, 16, 16>::calculateNumBuckets(capacity);
        case 2: return OffsetAltBucketPolicy<uint64_t, uint16_t, 16, 16>::calculateNumBuckets(capacity);
        default: return XorAltBucketPolicy<uint64_t, uint16_t, 16, 16>::calculateNumBuckets(capacity);
    }
}

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
