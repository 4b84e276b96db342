// Selling / Voronoi reduction of symmetric positive definite matrices in FP64, device side.
//
// Every product and sum goes through Arith<double> (explicit round-to-nearest, never fused), in
// the operation order of the reference so that integer offsets and weights are bit-identical:
//   packed index, scalar product      JMM_CPPLibs/.../LinearAlgebra/Implementation/SymmetricMatrixType.hxx:11-30
//   trace, determinant, comatrix      SymmetricMatrixType.hxx:189-243
//   obtuse superbase (Selling)        JMM_CPPLibs/.../LinearAlgebra/Implementation/BasisReduction.hpp:65-99
//   tensor decomposition              BasisReduction.hpp:102-157, Perp/Cross VectorType.h:98-113
//   small-weight tolerance            Headers/Specializations/CommonTraits.h:82-105
#pragma once

#include <float.h>

#include "common.cuh"

namespace hfm {

using A64 = Arith<double>;

__host__ __device__ __forceinline__ int sym_idx(int i, int j) {
    return i < j ? (j * (j + 1)) / 2 + i : (i * (i + 1)) / 2 + j;
}

// sum_i u_i (sum_j m_ij v_j), accumulated from zero in index order.
template <int D>
__host__ __device__ __forceinline__ double sym_scal(const double *m, const int *u, const int *v) {
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double si = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j) si = A64::add(si, A64::mul(m[sym_idx(i, j)], (double)v[j]));
        sum = A64::add(sum, A64::mul((double)u[i], si));
    }
    return sum;
}

template <int D>
__host__ __device__ __forceinline__ double sym_trace(const double *m) {
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) r = A64::add(r, m[sym_idx(i, i)]);
    return r;
}

template <int D>
__host__ __device__ __forceinline__ double sym_det(const double *m) {
#define C_(i, j) m[sym_idx(i, j)]
    if (D == 2) return A64::sub(A64::mul(C_(0, 0), C_(1, 1)), A64::mul(C_(1, 0), C_(0, 1)));
    const double a = A64::mul(C_(0, 0), A64::sub(A64::mul(C_(1, 1), C_(2, 2)), A64::mul(C_(1, 2), C_(2, 1))));
    const double b = A64::mul(C_(0, 1), A64::sub(A64::mul(A64::mul(2.0, C_(1, 2)), C_(2, 0)), A64::mul(C_(1, 0), C_(2, 2))));
    const double c = A64::mul(C_(0, 2), A64::mul(C_(1, 1), C_(2, 0)));
    return A64::sub(A64::add(a, b), c);
#undef C_
}

// Comatrix()/Determinant(): the division is a product with the rounded reciprocal.
template <int D>
__host__ __device__ __forceinline__ void sym_inverse(const double *m, double *out) {
#define C_(i, j) m[sym_idx(i, j)]
    double co[6];
    if (D == 2) {
        co[0] = C_(1, 1);
        co[1] = -C_(1, 0);
        co[2] = C_(0, 0);
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j) {
                const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                co[sym_idx(i, j)] = A64::sub(A64::mul(C_(i1, j1), C_(i2, j2)), A64::mul(C_(i1, j2), C_(i2, j1)));
            }
    }
#undef C_
    const double b = A64::div(1.0, sym_det<D>(m));
#pragma unroll
    for (int k = 0; k < D * (D + 1) / 2; ++k) out[k] = A64::mul(co[k], b);
}

// Offsets (3 components, unused ones zero) and raw weights of the tensor decomposition.
// Returns false if the matrix is rejected or Selling does not terminate within 200 sweeps.
template <int D>
__host__ __device__ bool tensor_decomposition(const double *d, int off[6][3], double w[6]) {
    if (!(sym_det<D>(d) > 0.0) || !(sym_trace<D>(d) > 0.0)) return false;  // NaN too
    int sb[4][3];
#pragma unroll
    for (int i = 0; i <= D; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) sb[i][j] = (j < D) ? ((i < D) ? (i == j) : -1) : 0;
    bool reduced = true;
    for (int it = 0; reduced && it < 200; ++it) {
        reduced = false;
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
            for (int j = i + 1; j <= D; ++j) {
                if (sym_scal<D>(d, sb[i], sb[j]) > 0.0) {
                    reduced = true;
                    if (D == 2) {
                        const int k = 3 - i - j;
#pragma unroll
                        for (int c = 0; c < 2; ++c) sb[k][c] = sb[i][c] - sb[j][c];
                    } else {
                        const int k = (i != 0 && j != 0) ? 0 : ((i != 1 && j != 1) ? 1 : 2);
                        const int l = 6 - i - j - k;
#pragma unroll
                        for (int c = 0; c < 3; ++c) { sb[k][c] += sb[i][c]; sb[l][c] += sb[i][c]; }
                    }
#pragma unroll
                    for (int c = 0; c < D; ++c) sb[i][c] = -sb[i][c];
                }
            }
    }
    if (reduced) return false;
    if (D == 2) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int j = (i + 1) % 3, k = (i + 2) % 3;
            off[i][0] = -sb[i][1];
            off[i][1] = sb[i][0];
            off[i][2] = 0;
            w[i] = -sym_scal<2>(d, sb[j], sb[k]);
        }
    } else {
        int r = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = i + 1; j < 4; ++j) {
                const int k = (i != 0 && j != 0) ? 0 : ((i != 1 && j != 1) ? 1 : 2);
                const int l = 6 - i - j - k;
                const int *u = sb[k], *v = sb[l];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
                    off[r][c] = u[c1] * v[c2] - u[c2] * v[c1];
                }
                w[r] = -sym_scal<3>(d, sb[i], sb[j]);
                ++r;
            }
    }
    return true;
}

// Riemann stencil at one point: D = (dual ? M : M^-1) o (1/(h_i h_j)), then Selling and the
// 1000*eps*Tr(D) cut-off (Headers/Specializations/Riemannian.h:41-71, CommonTraits.h:82-105).
template <int D>
__host__ __device__ bool riemann_stencil(const double *metric, bool dual, const double *h, int off[6][3], double w[6]) {
    double m[6], d[6];
    if (dual) {
#pragma unroll
        for (int k = 0; k < D * (D + 1) / 2; ++k) m[k] = metric[k];
    } else {
        sym_inverse<D>(metric, m);
    }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            const double g = A64::mul(h[i], h[j]);
            d[sym_idx(i, j)] = A64::mul(m[sym_idx(i, j)], A64::div(1.0, g));
        }
    if (!tensor_decomposition<D>(d, off, w)) return false;
    const double atol = A64::mul(1000.0 * DBL_EPSILON, sym_trace<D>(d));
#pragma unroll
    for (int k = 0; k < (D == 2 ? 3 : 6); ++k) w[k] = w[k] < atol ? 0.0 : w[k];
    return true;
}

}  // namespace hfm
