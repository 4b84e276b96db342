// Owning device allocation (RAII) used by the host orchestration.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>
#include <vector>

#include "common.cuh"

namespace hfm {

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
        HFM_CUDA(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)));
        n_ = n;
    }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    void zero(cudaStream_t s = 0) {
        if (n_) HFM_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    void upload(const T *h, size_t n, cudaStream_t s = 0) {
        if (n > n_) alloc(n);
        if (n) HFM_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T> &v, cudaStream_t s = 0) { upload(v.data(), v.size(), s); }
    void download(T *h, size_t n, cudaStream_t s = 0) const {
        if (n) HFM_CUDA(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }

private:
    T *p_ = nullptr;
    size_t n_ = 0;
};

}  // namespace hfm
