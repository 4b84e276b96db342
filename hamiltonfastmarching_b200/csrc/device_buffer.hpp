// Owning device allocation (RAII) used by the host orchestration.
//
// Allocations are stream-ordered (cudaMallocAsync / cudaFreeAsync on the device's default memory
// pool, whose release threshold is raised once so that freed blocks stay cached): repeated solves
// reuse memory without device-wide synchronisation.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace hfm {

// Stream on which the calling thread's solve runs (set by the orchestration).
cudaStream_t &current_stream();
// The calling thread's persistent solver kernels use 1/share of the device's resident CTAs (a
// serving lane leaves the rest of the SMs to the lanes that run beside it).
int &solver_share();
void keep_pool_cached();
// Held from the launch of a cooperative (grid-synchronising) kernel until it completes: two such
// kernels in flight from different threads could each hold part of the SMs while waiting at a grid
// barrier for blocks that the other keeps from becoming resident.
std::mutex &cooperative_mutex();
// Kernel launches issued by this library (all threads), for launch accounting.
void count_launch(unsigned n = 1);

// Sets the calling thread's current stream for a scope (device allocations of the scope are
// stream-ordered on it).
struct StreamScope {
    cudaStream_t saved;
    explicit StreamScope(cudaStream_t s) : saved(current_stream()) { current_stream() = s; }
    ~StreamScope() { current_stream() = saved; }
    StreamScope(const StreamScope &) = delete;
    StreamScope &operator=(const StreamScope &) = delete;
};

// Large host<->device copies of pageable memory: through two page-locked staging buffers of the
// calling thread, the host-side copies split over a pool of worker threads and overlapped with the
// DMA of the previous chunk. Copies below kStagedMin bytes go straight through cudaMemcpyAsync.
// staged_upload returns once the host source has been read (the DMA may still be in flight on `s`);
// staged_download returns once the destination is written.
constexpr size_t kStagedMin = size_t(8) << 20;
void staged_upload(void *dst_dev, const void *src_host, size_t bytes, cudaStream_t s);
// Sets up the calling thread's staging buffers and the copy workers ahead of the first transfer.
void staging_warm_up();
// Small page-locked host words for asynchronous device-to-host reads (bump-allocated from a pool
// set up once per process and kept: page-locking memory synchronises the device, which must not
// happen while a persistent solver runs). 16-byte aligned; throws when the pool is spent.
void *pinned_words(size_t bytes);
void staged_download(void *dst_host, const void *src_dev, size_t bytes, cudaStream_t s);

// Counted kernel launch: launch(kernel, grid, block, shared_bytes, stream, args...).
template <typename... KArgs, typename... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                   Args &&...args) {
    count_launch();
    kernel<<<grid, block, smem, stream>>>(std::forward<Args>(args)...);
}

template <typename T>
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { alloc(n); }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }

    void alloc(size_t n) {
        release();
        if (n == 0) return;
        keep_pool_cached();
        HFM_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&p_), n * sizeof(T), current_stream()));
        n_ = n;
    }
    void release() {
        if (p_) cudaFreeAsync(p_, current_stream());
        p_ = nullptr;
        n_ = 0;
    }
    void zero(cudaStream_t s = current_stream()) {
        if (n_) HFM_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    void upload(const T *h, size_t n, cudaStream_t s = current_stream()) {
        if (n > n_) alloc(n);
        if (!n) return;
        staged_upload(p_, h, n * sizeof(T), s);
    }
    void upload(const std::vector<T> &v, cudaStream_t s = current_stream()) { upload(v.data(), v.size(), s); }
    void download(T *h, size_t n, cudaStream_t s = current_stream()) const {
        if (n) HFM_CUDA(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }

private:
    T *p_ = nullptr;
    size_t n_ = 0;
};

}  // namespace hfm
