/*
 * CuckooFilterMultiGPU.cuh -- C++ drop-in for the reference's hash-partitioned
 * multi-GPU filter (reference include/CuckooFilterMultiGPU.cuh).
 *
 * Code written against the reference's
 *
 *     CuckooFilterMultiGPU<Config> filter(numGPUs, capacity);          (:335)
 *     filter.insertMany(h_keys);                                        (:452)
 *     filter.containsMany(h_keys, h_output);                            (:469)
 *     filter.deleteMany(h_keys, h_output);  filter.deleteMany(h_keys);  (:487, :504)
 *     filter.loadFactor(), totalOccupiedSlots(), totalCapacity(),
 *            sizeInBytes(), clear(), synchronizeAllGPUs()               (:520-592)
 *
 * compiles unchanged against this header and libcuckoo_b200.so.  One host
 * thread drives every shard, as in the reference, and shard i owns an
 * independent filter of SDIV(capacity, numGPUs) * 1.02 slots (:337) on its
 * device.  A batch of host keys is cut into one slice per shard; each slice is
 * copied to its shard's device and grouped by destination shard there
 * (cf_shard_partition, on the device).  The groups then cross to their
 * destination devices with one peer copy per (source, destination) pair
 * (NVLink through NVSwitch).  Each shard runs the batch operation on what it
 * received (the library's single-GPU path), and per-key results travel back
 * the same way and are put in batch order (cf_shard_unpartition).
 *
 * Differences from the reference:
 *  - results are aligned with the caller's keys (the reference leaves them in
 *    its multisplit order);
 *  - the transfer-plan constructor (:376) accepts a plan path and ignores it:
 *    NVSwitch gives every GPU pair the same bandwidth;
 *  - an extra constructor places shards on chosen devices (shards may share a
 *    device) and selects the routing.  CF_SHARD_REFERENCE (the default) is the
 *    reference's hash64(key) % numGPUs; CF_SHARD_REMIXED keeps a shard's keys
 *    spread over all its buckets (see cuckoo_b200.h).
 * Host key and result containers are any type with data()/size() (keys) and
 * resize()/operator[] (results), thrust::host_vector included.  Errors throw
 * cuckoo_b200::Error.
 */
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <string>
#include <vector>

#include "CuckooFilter.cuh"

namespace cuckoo_b200 {

inline void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    check(CF_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

template <typename Config>
class CuckooFilterMultiGPU {
   public:
    using T = typename Config::KeyType;
    static constexpr float defaultMemoryFactor = 0.8f;

    CuckooFilterMultiGPU(std::size_t numGPUs, std::size_t capacity, float memFactor = defaultMemoryFactor)
        : CuckooFilterMultiGPU(numGPUs, capacity, first_devices(numGPUs), CF_SHARD_REFERENCE, memFactor) {}

    /* The reference's transfer-plan form; the plan is not needed here. */
    CuckooFilterMultiGPU(std::size_t numGPUs, std::size_t capacity, const char* /*transferPlanPath*/,
                         float memFactor = defaultMemoryFactor)
        : CuckooFilterMultiGPU(numGPUs, capacity, first_devices(numGPUs), CF_SHARD_REFERENCE, memFactor) {}

    /* Shard i on devices[i % devices.size()], with the given routing. */
    CuckooFilterMultiGPU(std::size_t numGPUs, std::size_t capacity, std::vector<int> devices,
                         cf_shard_routing routing, float memFactor = defaultMemoryFactor)
        : n_(numGPUs), capacityPerGPU_(static_cast<std::size_t>(double((capacity + numGPUs - 1) / numGPUs) * 1.02)),
          routing_(routing) {
        if (n_ == 0 || n_ > 256) check(CF_ERR_INVALID, "numGPUs must be 1..256");
        if (devices.empty()) check(CF_ERR_INVALID, "no devices");
        const cf_config cfg = ::CuckooFilter<Config>::config();
        s_.resize(n_);
        for (std::size_t i = 0; i < n_; ++i) {
            Shard& sh = s_[i];
            sh.dev = devices[i % devices.size()];
            cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
            cuda_check(cudaStreamCreateWithFlags(&sh.stream, cudaStreamNonBlocking), "cudaStreamCreate");
            check(cf_create(&cfg, capacityPerGPU_, &sh.f), "cf_create");
        }
        enable_peers();
        // keys per shard slice: a share of the free memory of the shard's
        // device (memFactor of it, split between the shards it holds)
        slice_ = std::size_t(1) << 26;
        for (std::size_t i = 0; i < n_; ++i) {
            cuda_check(cudaSetDevice(s_[i].dev), "cudaSetDevice");
            std::size_t free_b = 0, total_b = 0;
            cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            std::size_t on_dev = 0;
            for (const Shard& o : s_) on_dev += o.dev == s_[i].dev;
            const std::size_t per_key = 3 * sizeof(T) + 12;
            const std::size_t fit = static_cast<std::size_t>(double(free_b) * memFactor) / (per_key * on_dev);
            slice_ = std::max<std::size_t>(1024, std::min(slice_, fit));
        }
    }

    CuckooFilterMultiGPU(const CuckooFilterMultiGPU&) = delete;
    CuckooFilterMultiGPU& operator=(const CuckooFilterMultiGPU&) = delete;

    ~CuckooFilterMultiGPU() {
        for (Shard& sh : s_) {
            cudaSetDevice(sh.dev);
            if (sh.stream) cudaStreamSynchronize(sh.stream);
            const std::initializer_list<void*> bufs = {sh.in,   sh.grouped,  sh.pos,         sh.counts, sh.ws,
                                                       sh.recv, sh.res_recv, sh.res_grouped, sh.out};
            for (void* p : bufs)
                if (p) cudaFree(p);
            if (sh.h_counts) cudaFreeHost(sh.h_counts);
            if (sh.h_out) cudaFreeHost(sh.h_out);
            cf_destroy(sh.f);
            if (sh.stream) cudaStreamDestroy(sh.stream);
        }
    }

    /* insertMany (:452): returns totalOccupiedSlots() afterwards. */
    template <class HostKeys>
    std::size_t insertMany(const HostKeys& h_keys) {
        run(OP_INSERT, h_keys.data(), h_keys.size(), nullptr);
        return totalOccupiedSlots();
    }

    /* containsMany (:469): h_output[i] = key i may be present. */
    template <class HostKeys, class HostOut>
    void containsMany(const HostKeys& h_keys, HostOut& h_output) {
        h_output.resize(h_keys.size());
        std::vector<std::uint8_t> res(h_keys.size());
        run(OP_CONTAINS, h_keys.data(), h_keys.size(), res.data());
        for (std::size_t i = 0; i < res.size(); ++i) h_output[i] = res[i] != 0;
    }

    /* deleteMany (:487): h_output[i] = key i was removed; returns totalOccupiedSlots(). */
    template <class HostKeys, class HostOut>
    std::size_t deleteMany(const HostKeys& h_keys, HostOut& h_output) {
        h_output.resize(h_keys.size());
        std::vector<std::uint8_t> res(h_keys.size());
        run(OP_DELETE, h_keys.data(), h_keys.size(), res.data());
        for (std::size_t i = 0; i < res.size(); ++i) h_output[i] = res[i] != 0;
        return totalOccupiedSlots();
    }

    /* deleteMany (:504) without per-key results. */
    template <class HostKeys>
    std::size_t deleteMany(const HostKeys& h_keys) {
        run(OP_DELETE, h_keys.data(), h_keys.size(), nullptr);
        return totalOccupiedSlots();
    }

    [[nodiscard]] float loadFactor() const {
        return static_cast<float>(totalOccupiedSlots()) / static_cast<float>(totalCapacity());
    }

    void synchronizeAllGPUs() {
        for (Shard& sh : s_) {
            cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
            cuda_check(cudaStreamSynchronize(sh.stream), "cudaStreamSynchronize");
        }
    }

    [[nodiscard]] std::size_t totalOccupiedSlots() const {
        std::size_t t = 0;
        for (const Shard& sh : s_) {
            std::uint64_t occ = 0;
            check(cf_occupied(sh.f, &occ), "cf_occupied");
            t += occ;
        }
        return t;
    }

    void clear() {
        for (Shard& sh : s_) {
            cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
            check(cf_clear(sh.f, sh.stream), "cf_clear");
        }
        synchronizeAllGPUs();
    }

    [[nodiscard]] std::size_t totalCapacity() const { return sum_info(&cf_info::capacity); }
    [[nodiscard]] std::size_t sizeInBytes() const { return sum_info(&cf_info::size_in_bytes); }

    /* Extensions: the shard count, per-shard capacity, and shard i's filter and device. */
    [[nodiscard]] std::size_t numShards() const { return n_; }
    [[nodiscard]] std::size_t capacityPerGPU() const { return capacityPerGPU_; }
    [[nodiscard]] cf_filter* shard(std::size_t i) const { return s_.at(i).f; }
    [[nodiscard]] int shardDevice(std::size_t i) const { return s_.at(i).dev; }
    /* Keys of a batch per shard and round (batches above numShards() times
     * this run in rounds); set from the free memory at construction. */
    [[nodiscard]] std::size_t sliceKeys() const { return slice_; }
    void setSliceKeys(std::size_t keys) { slice_ = std::max<std::size_t>(1, keys); }

   private:
    enum Op { OP_INSERT, OP_CONTAINS, OP_DELETE };

    struct Shard {
        int dev = 0;
        cudaStream_t stream = nullptr;
        cf_filter* f = nullptr;
        T* in = nullptr;                   // this shard's slice of the batch
        T* grouped = nullptr;              // the slice grouped by destination shard
        std::uint32_t* pos = nullptr;      // batch position of each grouped key
        std::uint64_t* counts = nullptr;   // keys per destination shard (device)
        std::uint64_t* h_counts = nullptr; // the same, pinned host copy
        void* ws = nullptr;                // grouping workspace
        std::uint64_t ws_bytes = 0;
        std::size_t cap = 0;               // capacity of in/grouped/pos/res_grouped/out
        T* recv = nullptr;                 // keys received from every shard
        std::uint8_t* res_recv = nullptr;  // results of the received keys
        std::size_t recv_cap = 0;
        std::uint8_t* res_grouped = nullptr;  // results back, in group order
        std::uint8_t* out = nullptr;          // results in batch order
        std::uint8_t* h_out = nullptr;        // pinned host copy of out
    };

    static std::vector<int> first_devices(std::size_t n) {
        std::vector<int> d(n);
        for (std::size_t i = 0; i < n; ++i) d[i] = static_cast<int>(i);
        return d;
    }

    std::size_t sum_info(std::uint64_t cf_info::*field) const {
        std::size_t t = 0;
        for (const Shard& sh : s_) {
            cf_info info{};
            check(cf_get_info(sh.f, &info), "cf_get_info");
            t += info.*field;
        }
        return t;
    }

    void enable_peers() {
        for (const Shard& a : s_)
            for (const Shard& b : s_) {
                if (a.dev == b.dev) continue;
                int ok = 0;
                if (cudaDeviceCanAccessPeer(&ok, a.dev, b.dev) != cudaSuccess || !ok) continue;
                cuda_check(cudaSetDevice(a.dev), "cudaSetDevice");
                const cudaError_t e = cudaDeviceEnablePeerAccess(b.dev, 0);
                if (e != cudaSuccess) cudaGetLastError();  // already enabled, or copies go through the host
            }
    }

    template <class P>
    static void grow(P*& p, std::size_t count) {
        if (p) cuda_check(cudaFree(p), "cudaFree");
        p = nullptr;
        cuda_check(cudaMalloc(reinterpret_cast<void**>(&p), std::max<std::size_t>(count, 1) * sizeof(P)), "cudaMalloc");
    }

    void reserve(Shard& sh, std::size_t m) {
        if (m <= sh.cap) return;
        cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
        grow(sh.in, m);
        grow(sh.grouped, m);
        grow(sh.pos, m);
        grow(sh.res_grouped, m);
        grow(sh.out, m);
        if (sh.h_out) cuda_check(cudaFreeHost(sh.h_out), "cudaFreeHost");
        cuda_check(cudaMallocHost(reinterpret_cast<void**>(&sh.h_out), m), "cudaMallocHost");
        if (!sh.counts) {
            grow(sh.counts, n_);
            cuda_check(cudaMallocHost(reinterpret_cast<void**>(&sh.h_counts), n_ * sizeof(std::uint64_t)),
                       "cudaMallocHost");
        }
        const std::uint64_t wsb = cf_shard_workspace_bytes(m, static_cast<std::uint32_t>(n_));
        if (sh.ws) cuda_check(cudaFree(sh.ws), "cudaFree");
        cuda_check(cudaMalloc(&sh.ws, wsb), "cudaMalloc");
        sh.ws_bytes = wsb;
        sh.cap = m;
    }

    void reserve_recv(Shard& sh, std::size_t m) {
        if (m <= sh.recv_cap) return;
        cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
        grow(sh.recv, m);
        grow(sh.res_recv, m);
        sh.recv_cap = m;
    }

    void sync_all() { synchronizeAllGPUs(); }

    /* One batch of host keys through partition, exchange, shard operation and,
     * with `res`, the results back in batch order. */
    void run(Op op, const T* keys, std::size_t n, std::uint8_t* res) {
        const std::size_t N = n_;
        const std::size_t chunk = slice_ * N;
        std::vector<std::size_t> len(N), off(N);
        std::vector<std::uint64_t> cnt(N * N), sdisp(N * N), rdisp(N * N), recv(N);
        for (std::size_t done = 0; done < n; done += chunk) {
            const std::size_t m = std::min(chunk, n - done);
            for (std::size_t s = 0, o = 0; s < N; ++s) {  // slices: m / N keys, the first m % N one more
                len[s] = m / N + (s < m % N ? 1 : 0);
                off[s] = o;
                o += len[s];
            }
            // 1. slice to its device, grouped by destination shard there
            for (std::size_t s = 0; s < N; ++s) {
                Shard& sh = s_[s];
                reserve(sh, len[s]);
                cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
                if (len[s])
                    cuda_check(cudaMemcpyAsync(sh.in, keys + done + off[s], len[s] * sizeof(T), cudaMemcpyHostToDevice,
                                               sh.stream),
                               "copy keys to the device");
                check(cf_shard_partition(sh.in, len[s], sizeof(T), static_cast<std::uint32_t>(N), routing_, sh.grouped,
                                         sh.pos, sh.counts, sh.ws, sh.ws_bytes, sh.stream),
                      "cf_shard_partition");
                cuda_check(cudaMemcpyAsync(sh.h_counts, sh.counts, N * sizeof(std::uint64_t), cudaMemcpyDeviceToHost,
                                           sh.stream),
                           "copy counts");
            }
            sync_all();
            for (std::size_t d = 0; d < N; ++d) recv[d] = 0;
            for (std::size_t s = 0; s < N; ++s)
                for (std::size_t d = 0, o = 0; d < N; ++d) {
                    cnt[s * N + d] = s_[s].h_counts[d];
                    sdisp[s * N + d] = o;
                    o += cnt[s * N + d];
                    rdisp[d * N + s] = recv[d];
                    recv[d] += cnt[s * N + d];
                }
            // 2. groups to their destination shards, one peer copy per pair
            for (std::size_t d = 0; d < N; ++d) reserve_recv(s_[d], recv[d]);
            for (std::size_t s = 0; s < N; ++s) {
                Shard& src = s_[s];
                cuda_check(cudaSetDevice(src.dev), "cudaSetDevice");
                for (std::size_t d = 0; d < N; ++d) {
                    const std::uint64_t c = cnt[s * N + d];
                    if (!c) continue;
                    Shard& dst = s_[d];
                    cuda_check(cudaMemcpyPeerAsync(dst.recv + rdisp[d * N + s], dst.dev, src.grouped + sdisp[s * N + d],
                                                   src.dev, c * sizeof(T), src.stream),
                               "peer copy of keys");
                }
            }
            sync_all();
            // 3. each shard's operation on the keys it received
            for (std::size_t d = 0; d < N; ++d) {
                Shard& sh = s_[d];
                if (!recv[d]) continue;
                cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
                if (op == OP_INSERT)
                    check(cf_insert(sh.f, sh.recv, recv[d], nullptr, sh.stream, nullptr), "insertMany");
                else if (op == OP_CONTAINS)
                    check(cf_contains(sh.f, sh.recv, recv[d], sh.res_recv, sh.stream), "containsMany");
                else
                    check(cf_delete(sh.f, sh.recv, recv[d], res ? sh.res_recv : nullptr, sh.stream, nullptr),
                          "deleteMany");
            }
            if (!res) continue;
            // 4. results back to their source shards, then into batch order
            for (std::size_t d = 0; d < N; ++d) {
                Shard& dst = s_[d];
                cuda_check(cudaSetDevice(dst.dev), "cudaSetDevice");
                for (std::size_t s = 0; s < N; ++s) {
                    const std::uint64_t c = cnt[s * N + d];
                    if (!c) continue;
                    Shard& src = s_[s];
                    cuda_check(cudaMemcpyPeerAsync(src.res_grouped + sdisp[s * N + d], src.dev,
                                                   dst.res_recv + rdisp[d * N + s], dst.dev, c, dst.stream),
                               "peer copy of results");
                }
            }
            sync_all();
            for (std::size_t s = 0; s < N; ++s) {
                Shard& sh = s_[s];
                if (!len[s]) continue;
                cuda_check(cudaSetDevice(sh.dev), "cudaSetDevice");
                check(cf_shard_unpartition(sh.res_grouped, sh.pos, len[s], static_cast<std::uint32_t>(N), sh.ws,
                                           sh.ws_bytes, sh.out, sh.stream),
                      "cf_shard_unpartition");
                cuda_check(cudaMemcpyAsync(sh.h_out, sh.out, len[s], cudaMemcpyDeviceToHost, sh.stream),
                           "copy results to the host");
            }
            sync_all();
            for (std::size_t s = 0; s < N; ++s)
                std::copy(s_[s].h_out, s_[s].h_out + len[s], res + done + off[s]);
        }
    }

    std::size_t n_;
    std::size_t capacityPerGPU_;
    cf_shard_routing routing_;
    std::size_t slice_ = 0;
    std::vector<Shard> s_;
};

}  // namespace cuckoo_b200

using cuckoo_b200::CuckooFilterMultiGPU;
