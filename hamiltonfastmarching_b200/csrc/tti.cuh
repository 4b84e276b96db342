// TTI3 local solver: tilted transversely isotropic norms as an extremum over t in [tmin, tmax] of
// Riemannian norms, discretised with the Selling decompositions met along the segment
// D(t) = (1 - t) D0 + t D1 (semi-Lagrangian scheme of the reference, FP64).
//
// Norm (JMM_CPPLibs/JMM_CPPLibs/LinearAlgebra/TTINorm.h:19-28, Implementation/TTINorm.hxx):
// the dual unit ball is <l, q> + 1/2 <q, Q q> = 1 with q = (p0^2 + p1^2, p2^2), p = A^-T p0,
// A the transform (columns scaled by the grid scales, Headers/Experimental/Implementation/
// TTI.hpp:24-34). The local solve (TTI.hpp:142-276) walks the Selling path interval by interval
// (BasisReduction.hpp:207-287); on each interval the neighbour set is fixed and the update value,
// a sorted-prefix quadratic solve with weights linear in t and right-hand side Multiplier(t)
// (TTINorm.hxx:99-226), is extremised with endpoint derivative tests and a safeguarded Newton
// search (derivatives carried by a second-order forward-mode number).
#pragma once

#include <cstdint>
#include <limits>

#include "selling.cuh"

namespace hfm {

struct TTICell {
    double D0[6], D1[6];            // extremal matrices of the Selling path, packed (xx,xy,yy,xz,yz,zz)
    double l0, l1, q00, q01, q11;   // linear and quadratic coefficients
    double tmin, tmax;
    int dir;                        // -1: infimum over t, +1: supremum
    int8_t sb[12];                  // obtuse superbase of D(tmin)
};

// x + dx t + ddx t^2 / 2 around the point of evaluation
struct Dual2 {
    double v, d, dd;
};
__host__ __device__ __forceinline__ Dual2 dconst(double v) { return {v, 0.0, 0.0}; }
__host__ __device__ __forceinline__ Dual2 operator+(Dual2 a, Dual2 b) { return {a.v + b.v, a.d + b.d, a.dd + b.dd}; }
__host__ __device__ __forceinline__ Dual2 operator-(Dual2 a, Dual2 b) { return {a.v - b.v, a.d - b.d, a.dd - b.dd}; }
__host__ __device__ __forceinline__ Dual2 operator*(Dual2 a, double s) { return {a.v * s, a.d * s, a.dd * s}; }
__host__ __device__ __forceinline__ Dual2 operator*(Dual2 a, Dual2 b) {
    return {a.v * b.v, a.d * b.v + a.v * b.d, a.dd * b.v + 2.0 * (a.d * b.d) + a.v * b.dd};
}
__host__ __device__ __forceinline__ Dual2 operator/(Dual2 a, Dual2 b) {
    const double q = a.v / b.v, qd = (a.d - q * b.d) / b.v;
    return {q, qd, (a.dd - 2.0 * qd * b.d - q * b.dd) / b.v};
}
__host__ __device__ __forceinline__ Dual2 dsqrt(Dual2 a) {
    const double s = sqrt(a.v), sd = a.d / (2.0 * s);
    return {s, sd, (a.dd - 2.0 * sd * sd) / (2.0 * s)};
}

__host__ __device__ __forceinline__ double tti_inf() { return std::numeric_limits<double>::infinity(); }

// Smallest positive s with q s^2 / 2 + l s - 1 = 0 (TTINorm.hxx:46-60).
__host__ __device__ __forceinline__ double tti_spr(double l, double q) {
    if (q == 0.0) return 1.0 / l;
    const double sd = sqrt(l * l + 2.0 * q);
    const double rm = (-l - sd) / q, rp = (-l + sd) / q;
    const double lo = rm < rp ? rm : rp, hi = rm < rp ? rp : rm;
    return lo > 0 ? lo : hi;
}

// Pairs (i < j) of superbase indices in lexicographic order and their complements (k < l).
__host__ __device__ __forceinline__ void tti_pair(int r, int &i, int &j) {
    const int I[6] = {0, 0, 0, 1, 1, 2}, J[6] = {1, 2, 3, 2, 3, 3};
    i = I[r];
    j = J[r];
}
__host__ __device__ __forceinline__ int tti_lin(int i, int j) {
    if (i > j) { const int s = i; i = j; j = s; }
    return i == 0 ? j - 1 : (i == 1 ? j + 1 : 5);
}
__host__ __device__ __forceinline__ void tti_compl(int i, int j, int &k, int &l) {
    k = (i != 0 && j != 0) ? 0 : ((i != 1 && j != 1) ? 1 : 2);
    l = 6 - i - j - k;
}
__host__ __device__ __forceinline__ void tti_cross(const int *u, const int *v, int *o) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
}

// Norm set-up from the 14 metric values (linear 2, quadratic xx,xy,yy, then the transform, which
// the reference reads row by row: element 5 + 3 i + j is its transform(i, j)), the grid scales and
// the obtuse superbase at tmin. T below holds that transform transposed, T(i, j) = element
// 5 + i + 3 j; MakeNorm scales column j of the transform by h_j (TTI.hpp:24-34), i.e. row i of T by
// h_i. False if the element is not a valid TTI norm.
__host__ __device__ inline bool tti_setup(const double *m, const double *h, TTICell &n) {
    n.l0 = m[0]; n.l1 = m[1];
    n.q00 = m[2]; n.q01 = m[3]; n.q11 = m[4];
    double T[3][3], B[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[i][j] = m[5 + i + 3 * j] * h[i];
    double det = 0.0;
    for (int i = 0; i < 3; ++i)
        det += T[i][0] * T[(i + 1) % 3][1] * T[(i + 2) % 3][2] - T[i][2] * T[(i + 1) % 3][1] * T[(i + 2) % 3][0];
    if (!(det != 0.0)) return false;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            B[j][i] = (T[(i + 1) % 3][(j + 1) % 3] * T[(i + 2) % 3][(j + 2) % 3] -
                       T[(i + 1) % 3][(j + 2) % 3] * T[(i + 2) % 3][(j + 1) % 3]) / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) {
            n.D0[sym_idx(i, j)] = B[0][i] * B[0][j] + B[1][i] * B[1][j];
            n.D1[sym_idx(i, j)] = B[2][i] * B[2][j];
        }
    if (!(n.l0 >= 0 && n.l1 >= 0 && n.l0 + n.l1 > 0)) return false;
    const double r0 = tti_spr(n.l0, n.q00), r1 = tti_spr(n.l1, n.q11);
    const double a0 = n.l0 + n.q00 * r0, a1 = n.l1 + n.q01 * r0;
    const double b0 = n.l0 + n.q01 * r1, b1 = n.l1 + n.q11 * r1;
    double tmin = a1 / (a0 + a1), tmax = b1 / (b0 + b1);
    if (tmin < tmax) {
        n.dir = -1;
    } else {
        const double s = tmin;
        tmin = tmax;
        tmax = s;
        n.dir = 1;
    }
    n.tmin = tmin;
    n.tmax = tmax;
    if (!(tmin == tmin && tmax == tmax)) return false;
    // obtuse superbase of D(tmin), from the canonical one
    double D[6];
    for (int k = 0; k < 6; ++k) D[k] = (1. - tmin) * n.D0[k] + tmin * n.D1[k];
    if (!(sym_det<3>(D) > 0.0) || !(sym_trace<3>(D) > 0.0)) return false;  // NaN too
    int sb[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    bool reduced = true;
    for (int it = 0; reduced && it < 200; ++it) {
        reduced = false;
        for (int i = 0; i < 3; ++i)
            for (int j = i + 1; j <= 3; ++j)
                if (sym_scal<3>(D, sb[i], sb[j]) > 0.0) {
                    reduced = true;
                    int k, l;
                    tti_compl(i, j, k, l);
                    for (int c = 0; c < 3; ++c) {
                        sb[k][c] += sb[i][c];
                        sb[l][c] += sb[i][c];
                        sb[i][c] = -sb[i][c];
                    }
                }
    }
    if (reduced) return false;
    for (int i = 0; i < 4; ++i)
        for (int c = 0; c < 3; ++c) {
            if (sb[i][c] < -127 || sb[i][c] > 127) return false;
            n.sb[3 * i + c] = (int8_t)sb[i][c];
        }
    return true;
}

// Multiplier(t): beta such that diag(1 - t, t) / beta is tangent to the dual unit ball.
__host__ __device__ inline Dual2 tti_multiplier(const TTICell &n, Dual2 t) {
    if (n.q00 == 0.0 && n.q01 == 0.0 && n.q11 == 0.0) return dconst(1. / (n.l0 + n.l1));
    const double Q00 = n.q11, Q01 = -n.q01, Q11 = n.q00;  // comatrix of the quadratic part
    const double Ql0 = Q00 * n.l0 + Q01 * n.l1, Ql1 = Q01 * n.l0 + Q11 * n.l1;
    const double detQ = Q00 * Q11 - Q01 * Q01, lQl = n.l0 * Ql0 + n.l1 * Ql1;
    const Dual2 v0 = dconst(1.0) - t, v1 = t;
    const Dual2 Qv0 = v0 * Q00 + v1 * Q01, Qv1 = v0 * Q01 + v1 * Q11;
    const Dual2 detVL = v0 * n.l1 - v1 * n.l0;
    const Dual2 lQv = Qv0 * n.l0 + Qv1 * n.l1;
    const Dual2 vQv = v0 * Qv0 + v1 * Qv1;
    const Dual2 num = detVL * detVL + vQv * 2.0;
    const double sgn = num.v > 0 ? 1.0 : -1.0;
    const Dual2 delta = vQv * (2 * detQ + lQl);
    if (delta.v < 1e-10) return dconst(tti_spr(n.l0, n.q00) * v0.v);  // degenerate conic
    return num / (dsqrt(delta) * sgn + lQv);
}

struct TTIPath {
    int sb[4][3];
    int off[6][3];
    double w0[6], w1[6];
};

__host__ __device__ __forceinline__ void tti_weights(const TTICell &n, TTIPath &P) {
    for (int r = 0; r < 6; ++r) {
        int i, j;
        tti_pair(r, i, j);
        P.w0[r] = -sym_scal<3>(n.D0, P.sb[i], P.sb[j]);
        P.w1[r] = -sym_scal<3>(n.D1, P.sb[i], P.sb[j]);
    }
}

__host__ __device__ __forceinline__ void tti_path_start(const TTICell &n, TTIPath &P) {
    for (int i = 0; i < 4; ++i)
        for (int c = 0; c < 3; ++c) P.sb[i][c] = n.sb[3 * i + c];
    tti_weights(n, P);
    for (int r = 0; r < 6; ++r) {
        int i, j, k, l;
        tti_pair(r, i, j);
        tti_compl(i, j, k, l);
        tti_cross(P.sb[k], P.sb[l], P.off[r]);
    }
}

// Next breakpoint of the path (t = +inf if none) and the pair whose weight vanishes there.
__host__ __device__ __forceinline__ void tti_next(const TTIPath &P, double &t, int &in, int &jn) {
    t = tti_inf();
    in = jn = -1;
    for (int r = 0; r < 6; ++r) {
        const double s0 = P.w0[r], s1 = P.w1[r];
        if (s1 >= s0 || 0 >= s0) continue;
        const double tr = s0 / (s0 - s1);
        if (tr >= t) continue;
        t = tr;
        tti_pair(r, in, jn);
    }
}

// Selling step across the breakpoint of pair (i, j); offsets are kept up to sign.
__host__ __device__ __forceinline__ void tti_step(const TTICell &n, TTIPath &P, int i, int j) {
    int k, l;
    tti_compl(i, j, k, l);
    for (int c = 0; c < 3; ++c) {
        P.sb[k][c] += P.sb[i][c];
        P.sb[l][c] += P.sb[i][c];
        P.sb[i][c] = -P.sb[i][c];
    }
    tti_cross(P.sb[k], P.sb[l], P.off[tti_lin(i, j)]);
    const int a = tti_lin(i, k), b = tti_lin(i, l);
    for (int c = 0; c < 3; ++c) {
        const int s = P.off[a][c];
        P.off[a][c] = P.off[b][c];
        P.off[b][c] = s;
    }
    tti_weights(n, P);
}

// Update value at t: sorted-prefix solve with weights w0 + t (w1 - w0) (clamped at 0) and right-hand
// side Multiplier(t); with `ad`, the value and its t-derivatives recomputed on the same prefix.
__host__ __device__ inline Dual2 tti_update(const TTICell &n, Dual2 t, const double *val, const TTIPath &P, bool ad) {
    const double INF = tti_inf();
    int idx[6] = {0, 1, 2, 3, 4, 5};
    for (int i = 1; i < 6; ++i) {
        const int x = idx[i];
        int k = i - 1;
        while (k >= 0 && val[idx[k]] > val[x]) {
            idx[k + 1] = idx[k];
            --k;
        }
        idx[k + 1] = x;
    }
    const double vmin = val[idx[0]];
    if (vmin == INF) return dconst(INF);
    const Dual2 mult = tti_multiplier(n, t);
    double a = 0, b = 0, c = -mult.v, sol = INF;
    int r = 0;
    for (; r < 6; ++r) {
        const int i = idx[r];
        const double v = val[i] - vmin;
        if (v >= sol) break;
        const double w_ = P.w0[i] + t.v * (P.w1[i] - P.w0[i]);
        const double w = w_ > 0 ? w_ : 0.0, wv = w * v;
        a += w;
        b += wv;
        c += wv * v;
        if (a <= mult.v * 1e-10) continue;
        const double delta = b * b - a * c;
        sol = (b + sqrt(delta > 0 ? delta : 0.0)) / a;
    }
    if (!ad) return dconst(vmin + sol);
    if (sol == INF) return dconst(INF);
    Dual2 A = dconst(0), B = dconst(0), C = mult * -1.0;
    for (int q = 0; q < r; ++q) {
        const int i = idx[q];
        const double v = val[i] - vmin;
        const Dual2 w = dconst(P.w0[i]) + t * (P.w1[i] - P.w0[i]);
        A = A + w;
        B = B + w * v;
        C = C + (w * v) * v;
    }
    return dconst(vmin) + (B + dsqrt(B * B - A * C)) / A;
}

// Local solve from the neighbour values get(o0, o1, o2) (+inf when unavailable). Returns +inf if
// no neighbour is available; *t_act, *interior describe the extremum. Every loop is bounded.
template <typename Get>
__host__ __device__ inline double tti_solve(const TTICell &n, Get get, double *t_act, bool *interior) {
    const double INF = tti_inf();
    TTIPath P;
    tti_path_start(n, P);
    double vals[6];
    bool need[6] = {true, true, true, true, true, true};
    double t0 = n.tmin;
    const double sgn = -(double)n.dir;
    double best = INF, tb = INF;
    bool inner = false;
    for (int guard = 0; guard < 64; ++guard) {
        double t1;
        int ni, nj;
        tti_next(P, t1, ni, nj);
        if (t1 > n.tmax) t1 = n.tmax;
        for (int r = 0; r < 6; ++r)
            if (need[r]) {
                const double vp = get(P.off[r][0], P.off[r][1], P.off[r][2]);
                const double vm = get(-P.off[r][0], -P.off[r][1], -P.off[r][2]);
                vals[r] = vp < vm ? vp : vm;
                need[r] = false;
            }
        do {
            const Dual2 v0 = tti_update(n, Dual2{t0, 1.0, 0.0}, vals, P, true) * sgn;
            if (v0.d >= 0 && v0.v < INF) {
                if (v0.v < best) { best = v0.v; tb = t0; inner = false; }
                break;
            }
            const Dual2 v1 = tti_update(n, Dual2{t1, 1.0, 0.0}, vals, P, true) * sgn;
            if (v1.d <= 0 && v1.v < INF) {
                if (v1.v < best) { best = v1.v; tb = t1; inner = false; }
                break;
            }
            if (v0.v == INF && v1.v == INF) break;
            double x0 = t0, x1 = t1, x = (v1.d * t0 - v0.d * t1) / (v1.d - v0.d), xo = INF;
            for (int it = 0; fabs(xo - x) > 100 * 2.220446049250313e-16 && it < 100; ++it) {
                xo = x;
                const Dual2 v = tti_update(n, Dual2{x, 1.0, 0.0}, vals, P, true) * sgn;
                if (v.d <= 0) x0 = x;
                else x1 = x;
                if (v.dd > 0) {
                    x -= v.d / v.dd;
                    if (x0 < x && x < x1) continue;
                }
                x = (x0 + x1) / 2.;
            }
            const double v = sgn * tti_update(n, dconst(x), vals, P, false).v;
            if (v < best) { best = v; tb = x; inner = true; }
        } while (false);
        if (t1 == n.tmax || ni < 0) break;
        t0 = t1;
        tti_step(n, P, ni, nj);
        int k, l;
        tti_compl(ni, nj, k, l);
        need[tti_lin(ni, nj)] = true;
        const int a = tti_lin(ni, k), b = tti_lin(ni, l);
        const double s = vals[a];
        vals[a] = vals[b];
        vals[b] = s;
        const bool sn = need[a];
        need[a] = need[b];
        need[b] = sn;
    }
    if (t_act) *t_act = tb;
    if (interior) *interior = inner;
    return sgn * best;
}

// Distinct offsets (up to sign) met along the path from tmin to tmax (SetNeighbors,
// TTI.hpp:67-92). Returns their number, or -1 if more than `cap`.
__host__ __device__ inline int tti_neighbors(const TTICell &n, int (*out)[3], int cap) {
    TTIPath P;
    tti_path_start(n, P);
    int cnt = 0;
    auto push = [&](const int *o) -> bool {
        for (int q = 0; q < cnt; ++q)
            if ((out[q][0] == o[0] && out[q][1] == o[1] && out[q][2] == o[2]) ||
                (out[q][0] == -o[0] && out[q][1] == -o[1] && out[q][2] == -o[2]))
                return true;
        if (cnt >= cap) return false;
        out[cnt][0] = o[0];
        out[cnt][1] = o[1];
        out[cnt][2] = o[2];
        ++cnt;
        return true;
    };
    for (int r = 0; r < 6; ++r)
        if (!push(P.off[r])) return -1;
    if (n.tmax == n.tmin) return cnt;
    for (int guard = 0; guard < 64; ++guard) {
        double t;
        int i, j;
        tti_next(P, t, i, j);
        if (t >= n.tmax || i < 0) break;
        tti_step(n, P, i, j);
        if (!push(P.off[tti_lin(i, j)])) return -1;
    }
    return cnt;
}

// Selling decomposition at t (from scratch), for the recomputation of the adjoint.
__host__ __device__ inline bool tti_path_at(const TTICell &n, double t, TTIPath &P) {
    double D[6];
    for (int k = 0; k < 6; ++k) D[k] = (1. - t) * n.D0[k] + t * n.D1[k];
    if (!(sym_det<3>(D) > 0.0) || !(sym_trace<3>(D) > 0.0)) return false;  // NaN too
    int sb[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    bool reduced = true;
    for (int it = 0; reduced && it < 200; ++it) {
        reduced = false;
        for (int i = 0; i < 3; ++i)
            for (int j = i + 1; j <= 3; ++j)
                if (sym_scal<3>(D, sb[i], sb[j]) > 0.0) {
                    reduced = true;
                    int k, l;
                    tti_compl(i, j, k, l);
                    for (int c = 0; c < 3; ++c) {
                        sb[k][c] += sb[i][c];
                        sb[l][c] += sb[i][c];
                        sb[i][c] = -sb[i][c];
                    }
                }
    }
    if (reduced) return false;
    for (int i = 0; i < 4; ++i)
        for (int c = 0; c < 3; ++c) P.sb[i][c] = sb[i][c];
    tti_weights(n, P);
    for (int r = 0; r < 6; ++r) {
        int i, j, k, l;
        tti_pair(r, i, j);
        tti_compl(i, j, k, l);
        tti_cross(P.sb[k], P.sb[l], P.off[r]);
    }
    return true;
}

}  // namespace hfm
