// Owning device allocation (RAII) used by the host orchestration.
//
// Allocations are stream-ordered (cudaMallocAsync / cudaFreeAsync on the device's default memory
// pool, whose release threshold is raised once so that freed blocks stay cached): repeated solves
// reuse memory without device-wide synchronisation.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
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
// Kernel launches issued by this library (all threads), for launch accounting.
void count_launch(unsigned n = 1);

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
    static constexpr size_t kPinThreshold = size_t(64) << 20;
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
        // Large pageable sources are page-locked for the transfer (DMA at full link speed instead
        // of staged copies); if locking is refused the copy proceeds from pageable memory.
        const size_t bytes = n * sizeof(T);
        if (bytes >= kPinThreshold &&
            cudaHostRegister(const_cast<T *>(h), bytes, cudaHostRegisterReadOnly) == cudaSuccess) {
            const cudaError_t e = cudaMemcpyAsync(p_, h, bytes, cudaMemcpyHostToDevice, s);
            const cudaError_t e2 = cudaStreamSynchronize(s);
            cudaHostUnregister(const_cast<T *>(h));
            HFM_CUDA(e);
            HFM_CUDA(e2);
            return;
        }
        cudaGetLastError();
        HFM_CUDA(cudaMemcpyAsync(p_, h, bytes, cudaMemcpyHostToDevice, s));
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
