// cf_device.cuh -- device primitives of the B200 cuckoo filter.
//
// Hashing and bucket derivation are bit-exact with the reference:
//   xxHash64, seed 0, over the little-endian bytes of the value
//     (reference include/hashutil.cuh:71-161; only the < 32-byte branch is
//     reachable for 1/2/4/8-byte inputs, and each size is written out here as
//     straight-line code);
//   fingerprint = (uint32)(h >> 32) & tagMask, 0 -> 1; primary = (uint32)h & (nb-1);
//   alternate  = bucket ^ (xxHash64(tag as TagType) & (nb-1))
//     (include/bucket_policies.cuh:46-61, :72-74).
// Table layout is the reference's (include/CuckooFilter.cuh:224-237): bucket b is
// bucketBytes contiguous bytes at b*bucketBytes; slot s holds its tag at byte
// offset s*(bits/8), packed little-endian into 64-bit words, 0 = empty.
#pragma once

#include <cstdint>

namespace cfb {

// ----------------------------------------------------------------- xxHash64

constexpr uint64_t XP1 = 11400714785074694791ULL;
constexpr uint64_t XP2 = 14029467366897019727ULL;
constexpr uint64_t XP3 = 1609587929392839161ULL;
constexpr uint64_t XP4 = 9650029242287828579ULL;
constexpr uint64_t XP5 = 2870177450012600261ULL;

__host__ __device__ __forceinline__ uint64_t rotl64(uint64_t x, int r) {
    return (x << r) | (x >> (64 - r));
}

__host__ __device__ __forceinline__ uint64_t xxh_avalanche(uint64_t h) {
    h ^= h >> 33;
    h *= XP2;
    h ^= h >> 29;
    h *= XP3;
    h ^= h >> 32;
    return h;
}

// XXH64 of an 8-byte value: one 8-byte lane step, then the avalanche.
__host__ __device__ __forceinline__ uint64_t xxh64_u64(uint64_t v) {
    uint64_t h = XP5 + 8;
    uint64_t k = rotl64(v * XP2, 31) * XP1;
    h ^= k;
    h = rotl64(h, 27) * XP1 + XP4;
    return xxh_avalanche(h);
}

// XXH64 of a 4-byte value: the 4-byte step, then the avalanche.
__host__ __device__ __forceinline__ uint64_t xxh64_u32(uint32_t v) {
    uint64_t h = XP5 + 4;
    h ^= static_cast<uint64_t>(v) * XP1;
    h = rotl64(h, 23) * XP2 + XP3;
    return xxh_avalanche(h);
}

// XXH64 of a 2-byte value: two single-byte steps (low byte first).
__host__ __device__ __forceinline__ uint64_t xxh64_u16(uint32_t v) {
    uint64_t h = XP5 + 2;
    h ^= static_cast<uint64_t>(v & 0xFF) * XP5;
    h = rotl64(h, 11) * XP1;
    h ^= static_cast<uint64_t>((v >> 8) & 0xFF) * XP5;
    h = rotl64(h, 11) * XP1;
    return xxh_avalanche(h);
}

// XXH64 of a 1-byte value.
__host__ __device__ __forceinline__ uint64_t xxh64_u8(uint32_t v) {
    uint64_t h = XP5 + 1;
    h ^= static_cast<uint64_t>(v & 0xFF) * XP5;
    h = rotl64(h, 11) * XP1;
    return xxh_avalanche(h);
}

template <int KEY_BYTES>
__host__ __device__ __forceinline__ uint64_t hash_key(uint64_t key) {
    if constexpr (KEY_BYTES == 8) {
        return xxh64_u64(key);
    } else {
        return xxh64_u32(static_cast<uint32_t>(key));
    }
}

template <int BITS>
__host__ __device__ __forceinline__ uint64_t hash_tag(uint32_t tag) {
    if constexpr (BITS == 8) {
        return xxh64_u8(tag);
    } else if constexpr (BITS == 16) {
        return xxh64_u16(tag);
    } else {
        return xxh64_u32(tag);
    }
}

// ------------------------------------------------------------ configuration

// KB = key bytes (4/8), BITS = tag bits (8/16/32), BS = slots per bucket,
// WB = CAS word bytes (8; the reference's WordType).
// Alternate-bucket policy (reference include/bucket_policies.cuh): XOR (:15-84),
// AddSub (:95-177), Offset (:179-350).
constexpr int ALT_XOR = 0;
constexpr int ALT_ADDSUB = 1;
constexpr int ALT_OFFSET = 2;

template <int KB, int BITS, int BS, int WB, int POL = ALT_XOR>
struct Cfg {
    static constexpr int alt_policy = POL;
    // The Offset policy keeps a choice bit in the tag's top bit: 0 while the tag
    // is in its primary bucket, 1 in its alternate.
    static constexpr uint32_t choice_bit = POL == ALT_OFFSET ? (1u << (BITS - 1)) : 0u;
    static constexpr int key_bytes = KB;
    static constexpr int bits = BITS;
    static constexpr int bs = BS;
    static constexpr int word_bytes = WB;
    static constexpr int bucket_bytes = BS * BITS / 8;
    static constexpr int nchunks = bucket_bytes / 8;     // 64-bit chunks per bucket
    static constexpr int lanes_per_chunk = 64 / BITS;    // tags per 64-bit chunk (the unit of every atomic here)
    static constexpr int tpw = WB * 8 / BITS;            // tags per WordType word (the reference's scan unit)
    static constexpr int wc = BS / tpw;                  // WordType words per bucket
    // Slot scans start at align_down(tag & (bs-1), tpw).  With 64-bit words a
    // scan can go chunk by chunk; with 32-bit words it goes slot by slot.
    static constexpr bool chunk_scan = tpw == lanes_per_chunk;
    static constexpr uint32_t tag_mask = BITS == 32 ? 0xFFFFFFFFu : ((1u << BITS) - 1u);
    static_assert(KB == 4 || KB == 8, "key must be 4 or 8 bytes");
    static_assert(BITS == 8 || BITS == 16 || BITS == 32, "tag must be 8, 16 or 32 bits");
    static_assert((BS & (BS - 1)) == 0, "bucket size must be a power of two");
    static_assert(bucket_bytes >= 8 && bucket_bytes % 8 == 0, "bucket must be a whole number of 8-byte chunks");
    static_assert(WB == 4 || WB == 8, "WordType is uint32_t or uint64_t");
    static_assert(BITS <= WB * 8, "a tag must fit in one word");
    static_assert(BS % tpw == 0, "bucket size must be a multiple of tags per word");
    static_assert(BS <= 128, "at most 128 slots per bucket");
    static_assert(nchunks <= 32, "at most 32 chunks (256 bytes) per bucket");
    static_assert(POL == ALT_XOR || POL == ALT_ADDSUB || POL == ALT_OFFSET, "alternate-bucket policy");
    using Key = typename std::conditional<KB == 8, uint64_t, uint32_t>::type;
};

// Bucket derivation (getCandidateBuckets of the configured policy).
// `nbm` is the bucket count minus one: the index mask of the XOR policy, whose
// bucket count is a power of two; AddSub and Offset take any (even, for
// AddSub) bucket count and reduce modulo it.
template <class C>
__host__ __device__ __forceinline__ void candidates(uint64_t key, uint64_t nbm, uint64_t& i1, uint32_t& fp) {
    const uint64_t h = hash_key<C::key_bytes>(key);
    const uint32_t hb = static_cast<uint32_t>(h);
    if constexpr (C::alt_policy == ALT_OFFSET) {
        // (bitsPerTag - 1) fingerprint bits, choice bit 0 (:232-247)
        const uint32_t f = static_cast<uint32_t>(h >> 32) & (C::choice_bit - 1u);
        fp = f == 0 ? 1u : f;
        i1 = static_cast<uint64_t>(hb) % (nbm + 1);
    } else {
        const uint32_t f = static_cast<uint32_t>(h >> 32) & C::tag_mask;
        fp = f == 0 ? 1u : f;
        if constexpr (C::alt_policy == ALT_ADDSUB)
            i1 = static_cast<uint64_t>(hb) % ((nbm + 1) / 2);  // first half (:128-137)
        else
            i1 = static_cast<uint64_t>(hb) & nbm;
    }
}

// The other bucket of a tag stored in bucket b (getAlternateBucket).
template <class C>
__host__ __device__ __forceinline__ uint64_t alt_bucket(uint64_t b, uint32_t tag, uint64_t nbm) {
    if constexpr (C::alt_policy == ALT_ADDSUB) {
        // first half -> second by adding, second -> first by subtracting (:150-160)
        const uint64_t half = (nbm + 1) / 2;
        const uint64_t fh = hash_tag<C::bits>(tag) % half;
        return b < half ? ((b + fh) % half) + half : (b - fh) % half;
    } else if constexpr (C::alt_policy == ALT_OFFSET) {
        // +offset from the primary, -offset from the alternate (:300-323)
        const uint64_t nb = nbm + 1;
        uint64_t off = hash_tag<C::bits>(tag & (C::choice_bit - 1u)) % nb;
        off = off == 0 ? 1 : off;
        return (tag & C::choice_bit) == 0 ? (b + off) % nb : (b + nb - off) % nb;
    } else {
        return b ^ (hash_tag<C::bits>(tag) & nbm);
    }
}

// The tag as stored once it moves to its other bucket
// (getAlternateBucketWithNewFp, CuckooFilter.cuh:394-401): the Offset policy
// flips the choice bit; XOR and AddSub keep the tag.
template <class C>
__host__ __device__ __forceinline__ uint32_t alt_tag(uint32_t tag) {
    return tag ^ C::choice_bit;
}

// ------------------------------------------------------------------- SWAR

// Exact per-lane "lane == 0" test: the top bit of each lane of the result is set
// iff that lane is zero.  Unlike the borrow-based test, no lane above a zero
// lane is flagged, so the flags can be used directly.
template <int BITS>
__device__ __forceinline__ uint64_t zero_lanes(uint64_t v) {
    constexpr uint64_t lo7 = BITS == 8 ? 0x7F7F7F7F7F7F7F7FULL
                           : BITS == 16 ? 0x7FFF7FFF7FFF7FFFULL
                                        : 0x7FFFFFFF7FFFFFFFULL;
    return ~(((v & lo7) + lo7) | v | lo7);
}

template <int BITS>
__device__ __forceinline__ uint64_t replicate(uint32_t tag) {
    if constexpr (BITS == 8) {
        return static_cast<uint64_t>(tag) * 0x0101010101010101ULL;
    } else if constexpr (BITS == 16) {
        return static_cast<uint64_t>(tag) * 0x0001000100010001ULL;
    } else {
        return static_cast<uint64_t>(tag) * 0x0000000100000001ULL;
    }
}

// Index of the lowest flagged lane of a zero_lanes() result (mask != 0).
template <int BITS>
__device__ __forceinline__ int lowest_lane(uint64_t mask) {
    return (__ffsll(static_cast<long long>(mask)) - 1) / BITS;
}

// ------------------------------------------------------------------- loads

// Read-only bucket load through the non-coherent path, no L1 allocation (the
// table is not written while a lookup batch runs).  The non-coherent loads
// here are not `volatile`: their data does not change during a kernel, so the
// compiler may batch and hoist them.
template <int BYTES>
__device__ __forceinline__ void load_nc(const void* p, uint64_t* c) {
    if constexpr (BYTES == 8) {
        asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(c[0]) : "l"(p));
    } else if constexpr (BYTES == 16) {
        asm("ld.global.nc.L1::no_allocate.v2.u64 {%0,%1}, [%2];" : "=l"(c[0]), "=l"(c[1]) : "l"(p));
    } else {
#pragma unroll
        for (int i = 0; i < BYTES / 32; ++i) {
            asm("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                         : "=l"(c[4 * i]), "=l"(c[4 * i + 1]), "=l"(c[4 * i + 2]), "=l"(c[4 * i + 3])
                         : "l"(static_cast<const char*>(p) + 32 * i));
        }
    }
}

// As load_nc, but the loads stay in program order relative to each other, so a
// run of them is issued back to back before any result is used (the compiler
// may otherwise sink each load next to its use and serialize them).
template <int BYTES>
__device__ __forceinline__ void load_nc_issue(const void* p, uint64_t* c) {
    if constexpr (BYTES == 8) {
        asm volatile("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(c[0]) : "l"(p));
    } else if constexpr (BYTES == 16) {
        asm volatile("ld.global.nc.L1::no_allocate.v2.u64 {%0,%1}, [%2];" : "=l"(c[0]), "=l"(c[1]) : "l"(p));
    } else {
#pragma unroll
        for (int i = 0; i < BYTES / 32; ++i) {
            asm volatile("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                         : "=l"(c[4 * i]), "=l"(c[4 * i + 1]), "=l"(c[4 * i + 2]), "=l"(c[4 * i + 3])
                         : "l"(static_cast<const char*>(p) + 32 * i));
        }
    }
}

// Bucket load for read-modify-write paths: relaxed at GPU scope so the values
// are at least as new as L2; they only seed compare-and-swap expectations.
template <int BYTES>
__device__ __forceinline__ void load_rlx(const void* p, uint64_t* c) {
    if constexpr (BYTES == 8) {
        asm volatile("ld.relaxed.gpu.global.L1::no_allocate.u64 %0, [%1];" : "=l"(c[0]) : "l"(p) : "memory");
    } else if constexpr (BYTES == 16) {
        asm volatile("ld.relaxed.gpu.global.L1::no_allocate.v2.u64 {%0,%1}, [%2];"
                     : "=l"(c[0]), "=l"(c[1])
                     : "l"(p)
                     : "memory");
    } else {
#pragma unroll
        for (int i = 0; i < BYTES / 32; ++i) {
            asm volatile("ld.relaxed.gpu.global.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                         : "=l"(c[4 * i]), "=l"(c[4 * i + 1]), "=l"(c[4 * i + 2]), "=l"(c[4 * i + 3])
                         : "l"(static_cast<const char*>(p) + 32 * i)
                         : "memory");
        }
    }
}

__device__ __forceinline__ uint64_t load_word_rlx(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t cas64(uint64_t* p, uint64_t expected, uint64_t desired) {
    return atomicCAS(reinterpret_cast<unsigned long long*>(p), expected, desired);
}

// Streaming key loads (read once).
__device__ __forceinline__ uint64_t ld_stream_u64(const uint64_t* p) {
    uint64_t v;
    asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t* p) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void ld_stream_v4u64(const uint64_t* p, uint64_t& a, uint64_t& b, uint64_t& c,
                                                uint64_t& d) {
    asm("ld.global.nc.L1::no_allocate.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
                 : "l"(p));
}
__device__ __forceinline__ void ld_stream_v4u32(const uint32_t* p, uint32_t& a, uint32_t& b, uint32_t& c,
                                                uint32_t& d) {
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
                 : "l"(p));
}

// Streaming loads that L2 may evict first (data read once).
__device__ __forceinline__ uint64_t ld_once_u64(const uint64_t* p) {
    return static_cast<uint64_t>(__ldcs(reinterpret_cast<const unsigned long long*>(p)));
}
__device__ __forceinline__ uint32_t ld_once_u32(const uint32_t* p) { return __ldcs(p); }

// L2 policy that keeps lines resident ahead of normal and streaming data.
__device__ __forceinline__ uint64_t l2_policy_keep() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// Fire-and-forget bitwise OR into global memory under an L2 cache policy.
__device__ __forceinline__ void red_or_policy(uint32_t* p, uint32_t v, uint64_t pol) {
    asm volatile("red.relaxed.gpu.global.or.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol) : "memory");
}

// ------------------------------------------- bulk copies (TMA) and mbarriers
//
// One-dimensional cp.async.bulk global -> shared copies completing on an
// mbarrier's transaction count, and shared -> global copies completing as
// bulk async-groups.  Source and destination must be 16-byte aligned and the
// size a multiple of 16 bytes.  No multicast form is used.

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// Makes initialised mbarriers visible to the async proxy (before __syncthreads).
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Orders this thread's earlier generic shared-memory accesses before later
// async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// One-dimensional cp.async.bulk shared -> global copy (bulk async-group
// completion).  Both addresses 16-byte aligned, size a multiple of 16 bytes.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until this thread's committed bulk stores have read their shared-memory source.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Waits until this thread's committed bulk stores have completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Waits until the phase with parity `parity` of `bar` completes.  Returns
// false after `limit` unsuccessful polls (each poll may suspend the thread for
// a hardware-defined interval), so a copy that never lands cannot hang the CTA.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
constexpr uint32_t kMbarPollLimit = 1u << 22;

}  // namespace cfb
