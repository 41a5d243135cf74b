/*
 * CuckooFilter.cuh -- C++ drop-in for the batch API of the reference's
 * header-only GPU cuckoo filter (reference include/CuckooFilter.cuh).
 *
 * Code written against the reference's
 *
 *     CuckooConfig<T, bitsPerTag, maxEvictions, blockSize, bucketSize,
 *                  AltBucketPolicy, evictionPolicy, WordType>     (CuckooFilter.cuh:44-74)
 *     CuckooFilter<Config> filter(capacity);                     (:420)
 *     filter.insertMany / insertManySorted / containsMany / deleteMany
 *
 * compiles unchanged against this header (put this repository's include/
 * directory first on the include path and link libcuckoo_b200.so).  Every call
 * forwards to the C ABI declared in cuckoo_b200.h, which runs the library's own
 * sm_100a kernels; nothing here launches a kernel itself, so the header also
 * compiles with a plain C++17 host compiler (g++ -I<cuda>/include).
 *
 * Semantics kept from the reference: keys and outputs are device pointers,
 * bool outputs are one byte each (0/1), every batch call is synchronous on
 * its stream, and insertMany/insertManySorted/deleteMany return
 * occupiedSlots() after the batch.  Differences: a failed insert never drops a
 * previously stored tag, and errors are reported by throwing
 * cuckoo_b200::Error (define CUCKOO_B200_EXIT_ON_ERROR to print the message
 * and exit the process instead, as the reference's CUDA_CALL does,
 * helpers.cuh:202-210).
 */
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

#include "cuckoo_b200.h"

#if defined(__CUDACC__) && __has_include(<thrust/device_vector.h>)
#include <thrust/device_vector.h>
#define CUCKOO_FILTER_HAS_THRUST 1
#endif

/* Eviction policy (reference CuckooFilter.cuh:19-22). */
enum class EvictionPolicy { BFS, DFS };

namespace cuckoo_b200 {

/* A non-zero cf_status from the library, with its message. */
class Error : public std::runtime_error {
   public:
    Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
    int status() const noexcept { return status_; }

   private:
    int status_;
};

inline void check(int status, const char* call) {
    if (status == CF_OK) return;
    std::string msg = std::string(call) + ": " + cf_status_string(status) + ": " + cf_last_error();
#ifdef CUCKOO_B200_EXIT_ON_ERROR
    std::fprintf(stderr, "%s\n", msg.c_str());
    std::exit(1);
#else
    throw Error(status, msg);
#endif
}

/* Candidate buckets and tag of host keys, evaluated by the library (the
 * kernels' own hashing). */
inline void candidates(const cf_config& cfg, std::uint64_t num_buckets, const void* key, std::uint64_t* i1,
                       std::uint64_t* i2, std::uint32_t* fp) {
    check(cf_hash_candidates(&cfg, num_buckets, key, 1, i1, i2, fp), "cf_hash_candidates");
}

}  // namespace cuckoo_b200

namespace cuckoo_b200 {

/* Host-side functions shared by the alternate-bucket policies: evaluated by
 * the library with the same code the kernels use. */
template <typename KeyType, typename TagType, std::size_t bitsPerTag, std::size_t bucketSize, cf_alt_policy ALT>
struct AltPolicyBase {
    static constexpr cf_alt_policy alt_policy = ALT;

    static cf_config config() {
        cf_config c{};
        c.key_bytes = sizeof(KeyType);
        c.bits_per_tag = static_cast<std::uint32_t>(bitsPerTag);
        c.bucket_size = static_cast<std::uint32_t>(bucketSize);
        c.word_bytes = 8;
        c.eviction_policy = CF_EVICT_DFS;
        c.max_evictions = 500;
        c.block_size = 0;
        c.alt_policy = ALT;
        return c;
    }

    /* (i1, i2, fp): fp as stored in the primary bucket i1. */
    static std::tuple<std::size_t, std::size_t, TagType> getCandidateBuckets(const KeyType& key,
                                                                            std::size_t numBuckets) {
        std::uint64_t i1 = 0, i2 = 0;
        std::uint32_t fp = 0;
        const cf_config c = config();
        candidates(c, numBuckets, &key, &i1, &i2, &fp);
        return {static_cast<std::size_t>(i1), static_cast<std::size_t>(i2), static_cast<TagType>(fp)};
    }

    static std::size_t getAlternateBucket(std::size_t bucket, TagType fp, std::size_t numBuckets) {
        const cf_config c = config();
        const std::uint64_t b = bucket;
        const std::uint32_t t = fp;
        std::uint64_t out = 0;
        check(cf_alt_buckets(&c, numBuckets, &b, &t, 1, &out), "cf_alt_buckets");
        return static_cast<std::size_t>(out);
    }

    static std::size_t calculateNumBuckets(std::size_t capacity) {
        return static_cast<std::size_t>(
            cf_num_buckets_for_policy(capacity, static_cast<std::uint32_t>(bucketSize), ALT));
    }
};

}  // namespace cuckoo_b200

/*
 * XOR alternate-bucket policy (reference bucket_policies.cuh:15-84): tag from
 * the upper 32 bits of xxHash64(key) (0 maps to 1), primary bucket from the
 * lower 32 bits, alternate bucket = bucket ^ (xxHash64(tag) & (numBuckets - 1)),
 * numBuckets = nextPowerOfTwo(ceil(capacity / bucketSize)).
 */
template <typename KeyType, typename TagType, std::size_t bitsPerTag, std::size_t bucketSize>
struct XorAltBucketPolicy
    : cuckoo_b200::AltPolicyBase<KeyType, TagType, bitsPerTag, bucketSize, CF_ALT_XOR> {
    static constexpr bool usesChoiceBit = false;
    static constexpr char name[] = "XorAltBucketPolicy";
};

/*
 * Additive/subtractive policy (reference bucket_policies.cuh:95-177): the
 * table is two halves; a key's primary bucket is in the first half (lower 32
 * hash bits mod numBuckets/2), its alternate in the second:
 * (bucket + h(tag) mod half) mod half + half, and back by subtracting.
 * numBuckets = ceil(capacity / bucketSize) rounded up to even.
 */
template <typename KeyType, typename TagType, std::size_t bitsPerTag, std::size_t bucketSize>
struct AddSubAltBucketPolicy
    : cuckoo_b200::AltPolicyBase<KeyType, TagType, bitsPerTag, bucketSize, CF_ALT_ADDSUB> {
    static constexpr bool usesChoiceBit = false;
    static constexpr char name[] = "AddSubAltBucketPolicy";
};

/*
 * Offset policy with a choice bit (reference bucket_policies.cuh:179-350): the
 * tag's top bit is 0 in the primary bucket and 1 in the alternate; the
 * alternate is (bucket + off) mod numBuckets from the primary and
 * (bucket - off) mod numBuckets back, off = h(tag without the bit) mod
 * numBuckets (0 maps to 1).  Any numBuckets = ceil(capacity / bucketSize).
 */
template <typename KeyType, typename TagType, std::size_t bitsPerTag, std::size_t bucketSize>
struct OffsetAltBucketPolicy
    : cuckoo_b200::AltPolicyBase<KeyType, TagType, bitsPerTag, bucketSize, CF_ALT_OFFSET> {
    static_assert(bitsPerTag >= 2, "bitsPerTag must be at least 2 for choice bit");
    static constexpr bool usesChoiceBit = true;
    static constexpr char name[] = "OffsetAltBucketPolicy";
    static constexpr std::size_t choiceBitPos = bitsPerTag - 1;
    static constexpr TagType choiceBitMask = TagType(TagType(1) << choiceBitPos);
    static constexpr TagType pureFpMask = TagType(choiceBitMask - 1);

    static TagType getPureFingerprint(TagType fp) { return fp & pureFpMask; }
    static TagType getChoiceBit(TagType fp) { return (fp >> choiceBitPos) & 1; }
    static TagType setChoiceBit(TagType fp, TagType choice) {
        return TagType((fp & pureFpMask) | TagType(choice << choiceBitPos));
    }
    /* The alternate bucket and the tag as stored there (choice bit flipped). */
    static std::tuple<std::size_t, TagType> getAlternateBucketWithNewFp(std::size_t bucket, TagType fp,
                                                                        std::size_t numBuckets) {
        const std::size_t alt =
            cuckoo_b200::AltPolicyBase<KeyType, TagType, bitsPerTag, bucketSize,
                                       CF_ALT_OFFSET>::getAlternateBucket(bucket, fp, numBuckets);
        return {alt, TagType(fp ^ choiceBitMask)};
    }
};

/*
 * Compile-time configuration (reference CuckooFilter.cuh:44-74).  Same
 * parameters and defaults; blockSize is the kernels' threads per block (0 lets
 * the library choose) and maxEvictions is capped at 512 by the library.
 */
template <typename T, std::size_t bitsPerTag_, std::size_t maxEvictions_ = 500, std::size_t blockSize_ = 256,
          std::size_t bucketSize_ = 16,
          template <typename, typename, std::size_t, std::size_t> class AltBucketPolicy_ = XorAltBucketPolicy,
          EvictionPolicy evictionPolicy_ = EvictionPolicy::DFS, typename WordType_ = std::uint64_t>
struct CuckooConfig {
    using KeyType = T;
    static constexpr std::size_t bitsPerTag = bitsPerTag_;
    static constexpr std::size_t maxEvictions = maxEvictions_;
    static constexpr std::size_t blockSize = blockSize_;
    static constexpr std::size_t bucketSize = bucketSize_;
    static constexpr EvictionPolicy evictionPolicy = evictionPolicy_;
    using TagType = std::conditional_t<bitsPerTag <= 8, std::uint8_t,
                                       std::conditional_t<bitsPerTag <= 16, std::uint16_t, std::uint32_t>>;
    using WordType = WordType_;
    static_assert(std::is_same_v<WordType, std::uint32_t> || std::is_same_v<WordType, std::uint64_t>,
                  "WordType must be uint32_t or uint64_t");
    static_assert(sizeof(TagType) <= sizeof(WordType), "TagType must fit within WordType");
    using AltBucketPolicy = AltBucketPolicy_<KeyType, TagType, bitsPerTag, bucketSize_>;
};

/*
 * The filter (reference CuckooFilter.cuh:140-785).  Owns its device table;
 * not copyable.  The table lives on the device that was current at
 * construction.
 */
template <typename Config>
class CuckooFilter {
   public:
    using T = typename Config::KeyType;
    using TagType = typename Config::TagType;
    static constexpr std::size_t bitsPerTag = Config::bitsPerTag;
    static constexpr std::size_t bucketSize = Config::bucketSize;
    static constexpr std::size_t maxEvictions = Config::maxEvictions;
    static constexpr std::size_t blockSize = Config::blockSize;
    static_assert(std::is_same_v<T, std::uint32_t> || std::is_same_v<T, std::uint64_t> ||
                      std::is_same_v<T, std::int32_t> || std::is_same_v<T, std::int64_t>,
                  "keys must be 4- or 8-byte integers");
    static_assert(bitsPerTag == 8 || bitsPerTag == 16 || bitsPerTag == 32, "bitsPerTag must be 8, 16 or 32");
    static_assert((bucketSize & (bucketSize - 1)) == 0, "Bucket size must be a power of 2");

    std::size_t numBuckets;  // public, as in the reference (:349)

    explicit CuckooFilter(std::size_t capacity) : numBuckets(calculateNumBuckets(capacity)) {
        const cf_config c = config();
        cuckoo_b200::check(cf_create(&c, capacity, &f_), "cf_create");
    }

    CuckooFilter(const CuckooFilter&) = delete;
    CuckooFilter& operator=(const CuckooFilter&) = delete;

    ~CuckooFilter() { cf_destroy(f_); }

    /* The library's configuration record for Config. */
    static cf_config config() {
        cf_config c{};
        c.key_bytes = sizeof(T);
        c.bits_per_tag = static_cast<std::uint32_t>(bitsPerTag);
        c.bucket_size = static_cast<std::uint32_t>(bucketSize);
        c.word_bytes = sizeof(typename Config::WordType);
        c.eviction_policy = Config::evictionPolicy == EvictionPolicy::BFS ? CF_EVICT_BFS : CF_EVICT_DFS;
        c.max_evictions = static_cast<std::uint32_t>(maxEvictions);
        c.block_size = static_cast<std::uint32_t>(blockSize);
        c.alt_policy = Config::AltBucketPolicy::alt_policy;
        return c;
    }

    /* insertMany (:457-464): returns occupiedSlots() after the batch. */
    std::size_t insertMany(const T* d_keys, const std::size_t n, cudaStream_t stream = {}) {
        std::uint64_t occ = 0;
        cuckoo_b200::check(cf_insert(f_, d_keys, n, nullptr, stream, &occ), "insertMany");
        return static_cast<std::size_t>(occ);
    }

    /* insertManySorted (:475-508): keys are grouped by primary bucket first. */
    std::size_t insertManySorted(const T* d_keys, const std::size_t n, cudaStream_t stream = {}) {
        std::uint64_t occ = 0;
        cuckoo_b200::check(cf_insert_sorted(f_, d_keys, n, nullptr, stream, &occ), "insertManySorted");
        return static_cast<std::size_t>(occ);
    }

    /* containsMany (:518-523): d_output[i] = key i may be present. */
    void containsMany(const T* d_keys, const std::size_t n, bool* d_output, cudaStream_t stream = {}) {
        cuckoo_b200::check(cf_contains(f_, d_keys, n, reinterpret_cast<std::uint8_t*>(d_output), stream),
                           "containsMany");
    }

    /* deleteMany (:536-548): removes one copy per key; d_output (optional)
     * receives true for each key removed.  Returns occupiedSlots(). */
    std::size_t deleteMany(const T* d_keys, const std::size_t n, bool* d_output = nullptr, cudaStream_t stream = {}) {
        std::uint64_t occ = 0;
        cuckoo_b200::check(cf_delete(f_, d_keys, n, reinterpret_cast<std::uint8_t*>(d_output), stream, &occ),
                           "deleteMany");
        return static_cast<std::size_t>(occ);
    }

#ifdef CUCKOO_FILTER_HAS_THRUST
    /* Thrust overloads (:550-670). Outputs are resized to the key count. */
    std::size_t insertMany(const thrust::device_vector<T>& d_keys, cudaStream_t stream = {}) {
        return insertMany(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(), stream);
    }
    std::size_t insertManySorted(const thrust::device_vector<T>& d_keys, cudaStream_t stream = {}) {
        return insertManySorted(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(), stream);
    }
    void containsMany(const thrust::device_vector<T>& d_keys, thrust::device_vector<bool>& d_output,
                      cudaStream_t stream = {}) {
        d_output.resize(d_keys.size());
        containsMany(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(),
                     thrust::raw_pointer_cast(d_output.data()), stream);
    }
    void containsMany(const thrust::device_vector<T>& d_keys, thrust::device_vector<std::uint8_t>& d_output,
                      cudaStream_t stream = {}) {
        d_output.resize(d_keys.size());
        containsMany(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(),
                     reinterpret_cast<bool*>(thrust::raw_pointer_cast(d_output.data())), stream);
    }
    std::size_t deleteMany(const thrust::device_vector<T>& d_keys, thrust::device_vector<bool>& d_output,
                           cudaStream_t stream = {}) {
        d_output.resize(d_keys.size());
        return deleteMany(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(),
                          thrust::raw_pointer_cast(d_output.data()), stream);
    }
    std::size_t deleteMany(const thrust::device_vector<T>& d_keys, thrust::device_vector<std::uint8_t>& d_output,
                           cudaStream_t stream = {}) {
        d_output.resize(d_keys.size());
        return deleteMany(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(),
                          reinterpret_cast<bool*>(thrust::raw_pointer_cast(d_output.data())), stream);
    }
    std::size_t deleteMany(const thrust::device_vector<T>& d_keys, cudaStream_t stream = {}) {
        return deleteMany(thrust::raw_pointer_cast(d_keys.data()), d_keys.size(), nullptr, stream);
    }
#endif

    /* clear (:675-682): empty table, counters zeroed. */
    void clear() { cuckoo_b200::check(cf_clear(f_, nullptr), "clear"); }

    /* loadFactor (:688): occupied / capacity, in float as the reference computes it. */
    [[nodiscard]] float loadFactor() {
        return static_cast<float>(occupiedSlots()) / static_cast<float>(numBuckets * bucketSize);
    }

    /* occupiedSlots (:699-704): the device counter. */
    std::size_t occupiedSlots() {
        std::uint64_t v = 0;
        cuckoo_b200::check(cf_occupied(f_, &v), "occupiedSlots");
        return static_cast<std::size_t>(v);
    }

    /* evictionCount / resetEvictionCount (:714-726).  Always counted here
     * (the reference counts only under CUCKOO_FILTER_COUNT_EVICTIONS). */
    std::size_t evictionCount() {
        cf_stats s{};
        cuckoo_b200::check(cf_get_stats(f_, &s), "evictionCount");
        return static_cast<std::size_t>(s.evictions);
    }
    void resetEvictionCount() { cuckoo_b200::check(cf_reset_stats(f_), "resetEvictionCount"); }

    std::size_t capacity() { return numBuckets * bucketSize; }                       // :732
    [[nodiscard]] std::size_t getNumBuckets() const { return numBuckets; }           // :740
    [[nodiscard]] std::size_t sizeInBytes() const { return numBuckets * bucketSize * bitsPerTag / 8; }  // :748

    /* countOccupiedSlots (:759-785): non-empty slots of the table image. */
    std::size_t countOccupiedSlots() {
        std::uint64_t v = 0;
        cuckoo_b200::check(cf_count_occupied_slots(f_, &v), "countOccupiedSlots");
        return static_cast<std::size_t>(v);
    }

    /* Static hashing helpers (:362-414). */
    static std::uint64_t hash64(const T& key) {
        std::uint64_t h = 0;
        cuckoo_b200::check(cf_hash64(sizeof(T), &key, 1, &h), "cf_hash64");
        return h;
    }
    static std::tuple<std::size_t, std::size_t, TagType> getCandidateBuckets(const T& key, std::size_t numBuckets) {
        return Config::AltBucketPolicy::getCandidateBuckets(key, numBuckets);
    }
    static std::size_t getAlternateBucket(std::size_t bucket, TagType fp, std::size_t numBuckets) {
        return Config::AltBucketPolicy::getAlternateBucket(bucket, fp, numBuckets);
    }
    /* The alternate bucket and the tag as stored there (CuckooFilter.cuh:394-401). */
    static std::tuple<std::size_t, TagType> getAlternateBucketWithNewFp(std::size_t bucket, TagType fp,
                                                                        std::size_t numBuckets) {
        if constexpr (Config::AltBucketPolicy::usesChoiceBit)
            return Config::AltBucketPolicy::getAlternateBucketWithNewFp(bucket, fp, numBuckets);
        else
            return {Config::AltBucketPolicy::getAlternateBucket(bucket, fp, numBuckets), fp};
    }
    static std::size_t calculateNumBuckets(std::size_t capacity) {
        return Config::AltBucketPolicy::calculateNumBuckets(capacity);
    }

    /* The underlying C handle (for the library's extensions: statistics,
     * table import/export, options). */
    cf_filter* handle() const { return f_; }

   private:
    cf_filter* f_ = nullptr;
};
