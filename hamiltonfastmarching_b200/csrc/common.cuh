// Shared device utilities of the solve path: error handling, round-to-nearest arithmetic that the
// compiler may not fuse, grid geometry of the tiled layout, and a bounded grid-wide barrier.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <limits>
#include <string>

#include "../../include/hfm_b200.h"
#include "io.hpp"

#define HFM_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw ::hfm::Error(e_ == cudaErrorMemoryAllocation ? HFM_ERR_NOMEM : HFM_ERR_CUDA,      \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

namespace hfm {

// Device-side error bits, written to a status word the host reads after each phase.
enum : unsigned {
    kErrBarrierTimeout = 1u,   // a grid barrier wait exceeded its iteration limit
    kErrRoundCap = 2u,         // the solver exceeded its round cap
    kErrTableOverflow = 4u,    // a tile's dependency table overflowed
    kErrSelling = 8u,          // Selling did not terminate / non positive definite metric
    kErrIndexRange = 16u,      // a flow or queue index left its array (the access was skipped)
};

// ------------------------------------------------------------------------------------------
// Arithmetic with explicit rounding. The reference is compiled for x86-64 without fused
// multiply-add, so every product and sum is rounded on its own; these wrappers keep nvcc from
// contracting a*b+c into an FMA on the parity-critical paths.
template <typename R> struct Arith;
#ifdef __CUDA_ARCH__
#define HFM_RN(dev, host) return dev
#else
#define HFM_RN(dev, host) return host
#endif
// On the host these compile to plain IEEE operations: the host compiler targets x86-64 without
// FMA, like the reference build.
template <> struct Arith<double> {
    static __host__ __device__ __forceinline__ double add(double a, double b) { HFM_RN(__dadd_rn(a, b), a + b); }
    static __host__ __device__ __forceinline__ double sub(double a, double b) { HFM_RN(__dsub_rn(a, b), a - b); }
    static __host__ __device__ __forceinline__ double mul(double a, double b) { HFM_RN(__dmul_rn(a, b), a * b); }
    static __host__ __device__ __forceinline__ double div(double a, double b) { HFM_RN(__ddiv_rn(a, b), a / b); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
    static __host__ __device__ __forceinline__ double inf() { HFM_RN(__longlong_as_double(0x7ff0000000000000LL), std::numeric_limits<double>::infinity()); }
};
template <> struct Arith<float> {
    static __host__ __device__ __forceinline__ float add(float a, float b) { HFM_RN(__fadd_rn(a, b), a + b); }
    static __host__ __device__ __forceinline__ float sub(float a, float b) { HFM_RN(__fsub_rn(a, b), a - b); }
    static __host__ __device__ __forceinline__ float mul(float a, float b) { HFM_RN(__fmul_rn(a, b), a * b); }
    static __host__ __device__ __forceinline__ float div(float a, float b) { HFM_RN(__fdiv_rn(a, b), a / b); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
    static __host__ __device__ __forceinline__ float inf() { HFM_RN(__int_as_float(0x7f800000), std::numeric_limits<float>::infinity()); }
};
#undef HFM_RN

// ------------------------------------------------------------------------------------------
// Tiled grid geometry. Axes are (a0, a1, a2) = (x, y, z|theta); a2 is the fastest axis of the
// row-major value array. 2D grids use a2 of extent 1. A tile holds 64 cells: 8x8x1 in 2D and
// 4x4x4 in 3D; a warp owns a tile and each lane two of its cells (local l and l+32).
struct GridGeom {
    int dims[3];
    int periodic[3];
    int tshift[3];     // log2 of tile extents
    int ntiles[3];     // tiles per axis
    long long ncells;  // dims product
    long long ntile;   // ntiles product

    __host__ __device__ int text(int a) const { return 1 << tshift[a]; }
    __host__ __device__ long long lin(int x0, int x1, int x2) const {
        return ((long long)x0 * dims[1] + x1) * dims[2] + x2;
    }
    __host__ __device__ void tile_coords(long long t, int &t0, int &t1, int &t2) const {
        t2 = (int)(t % ntiles[2]);
        long long r = t / ntiles[2];
        t1 = (int)(r % ntiles[1]);
        t0 = (int)(r / ntiles[1]);
    }
    __host__ __device__ long long tile_of(int x0, int x1, int x2) const {
        return ((long long)(x0 >> tshift[0]) * ntiles[1] + (x1 >> tshift[1])) * ntiles[2] + (x2 >> tshift[2]);
    }
    __host__ __device__ int local_of(int x0, int x1, int x2) const {
        const int m0 = (1 << tshift[0]) - 1, m1 = (1 << tshift[1]) - 1, m2 = (1 << tshift[2]) - 1;
        return (((x0 & m0) << tshift[1] | (x1 & m1)) << tshift[2]) | (x2 & m2);
    }
    __host__ __device__ void local_coords(int l, int &l0, int &l1, int &l2) const {
        l2 = l & ((1 << tshift[2]) - 1);
        l1 = (l >> tshift[2]) & ((1 << tshift[1]) - 1);
        l0 = l >> (tshift[1] + tshift[2]);
    }
    // Wraps periodic axes; returns false if the point leaves a closed axis.
    __host__ __device__ bool wrap(int &x0, int &x1, int &x2) const {
        int *x[3] = {&x0, &x1, &x2};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (periodic[a]) {
                int r = *x[a] % dims[a];
                *x[a] = r < 0 ? r + dims[a] : r;
            } else if (*x[a] < 0 || *x[a] >= dims[a]) {
                return false;
            }
        }
        return true;
    }
};

// Tiles of 64 cells: log2 extents `shift` (summing to 6, unused axes 0), or 8x8 / 4x4x4 if null.
GridGeom make_geom(int ndim, const int *dims, const int *periodic, const int *shift = nullptr);

// Bounded sense-reversing barrier across all CTAs of a cooperative launch. Every wait gives up
// after `limit` polls, sets kErrBarrierTimeout in *status and lets the caller return.
__device__ __forceinline__ bool grid_barrier(unsigned *count, volatile unsigned *gen, unsigned nblocks,
                                             unsigned *status, unsigned long long limit) {
    __syncthreads();
    __shared__ int s_fail;
    if (threadIdx.x == 0) {
        s_fail = 0;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(count, 1u) == nblocks - 1) {
            *count = 0;
            __threadfence();
            atomicAdd((unsigned *)gen, 1u);
        } else {
            unsigned long long spins = 0;
            while (*gen == g) {
                if (++spins > limit) {
                    atomicOr(status, kErrBarrierTimeout);
                    s_fail = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile unsigned *)status & kErrBarrierTimeout) s_fail = 1;
    }
    __syncthreads();
    return s_fail == 0;
}

}  // namespace hfm
