// GPU solve path for Eulerian schemes: per-cell Selling stencils (Riemann) or per-angle shared
// stencils (ReedsShepp2, Elastica2), wall visibility, and a tiled fast-iterative solver.
//
// The fixed point solved here is the one the reference's fast marching reaches
// (Headers/Base/Implementation/HamiltonFastMarching.hxx:86-169 with the Hopf-Lax update of
// Headers/Base/Implementation/EulerianStencil.hxx:104-153): at every cell x the value is the root of
//     sum_i w_i (t - v_i)^2 = 1
// over the neighbour values v_i sorted increasingly, a neighbour being used only while it is
// strictly below the root obtained from the smaller ones; the accumulation starts from the
// smallest value (minVal), adds (w, w v, w v^2) in increasing order, and takes
// (b + sqrt(max(0, b^2 - a c)))/a. Fast marching adds neighbours exactly in that order (they are
// accepted by increasing value), so with unfused FP64 arithmetic the converged tiles reproduce
// its arrival times.
//
// Layout in HBM: values RowMajor (the output array itself); per-cell stencil data tile-major
// (64 consecutive entries per tile and slot) so that a warp streams its tile's stencils with
// coalesced loads. Scheduling: a persistent cooperative kernel processes an active-tile list
// round by round (one warp per tile, local Jacobi sweeps voted with __any_sync), and appends to
// the next list, through atomics, the tiles whose stencils read a cell that changed.
#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <iterator>
#include <chrono>
#include <cmath>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "device_buffer.hpp"
#include "selling.cuh"
#include "tti.cuh"
#include "solver.hpp"

namespace hfm {

GridGeom make_geom(int ndim, const int *dims, const int *periodic, const int *shift) {
    GridGeom g{};
    for (int a = 0; a < 3; ++a) {
        g.dims[a] = a < ndim ? dims[a] : 1;
        g.periodic[a] = a < ndim ? periodic[a] : 0;
    }
    if (shift) { for (int a = 0; a < 3; ++a) g.tshift[a] = a < ndim ? shift[a] : 0; }
    else if (ndim == 2) { g.tshift[0] = 3; g.tshift[1] = 3; g.tshift[2] = 0; }
    else { g.tshift[0] = 2; g.tshift[1] = 2; g.tshift[2] = 2; }
    g.ncells = 1;
    g.ntile = 1;
    for (int a = 0; a < 3; ++a) {
        g.ntiles[a] = (g.dims[a] + (1 << g.tshift[a]) - 1) >> g.tshift[a];
        g.ncells *= g.dims[a];
        g.ntile *= g.ntiles[a];
    }
    return g;
}

// Kernels live in a named namespace: nvcc's host launch wrappers for __global__ templates do not
// bind to their generated stubs inside an anonymous namespace.
namespace detail {

constexpr unsigned kVisPlus = 1u << 24, kVisMinus = 1u << 25, kFixed = 1u << 28, kDead = 1u << 29;
constexpr unsigned kShFixed = 1u << 30, kShDead = 1u << 31;
constexpr int kWarpsPerCta = 4;
// Stencil families of the solver kernels (the KIND template parameter): per-cell Riemann
// stencils, shared per-angle stencils (curvature models), per-cell TTI Selling paths.
// kKindShare2: shared stencils of two groups of forward differences whose value is the smaller of
// the two groups' solutions (Dubins2, nmax = 2). kKindShareS2: shared stencils over R^3 x S^2
// (ReedsShepp3), one class per (theta, phi) pair (see s2_step).
constexpr int kKindRiemann = 0, kKindShare = 1, kKindTTI = 2, kKindShare2 = 3, kKindShareS2 = 4;
constexpr bool is_share(int kind) { return kind == kKindShare || kind == kKindShare2 || kind == kKindShareS2; }
// Value increases a tile may take before it accepts decreases only (termination guard).
constexpr unsigned kUpBudget = 128;
// Tile dependency tables: a small hash table per warp first (fast, high occupancy), the large one
// only for grids whose tiles read more distinct tiles (detected by the overflow status).
constexpr int kDepCapSmall = 128, kDepWarpsSmall = 4;
constexpr int kDepCapLarge = 1024, kDepWarpsLarge = 2;
constexpr unsigned long long kBarrierPolls = 1ull << 25;

__host__ __device__ __forceinline__ unsigned pack_off(int o0, int o1, int o2) {
    return (unsigned)(uint8_t)(int8_t)o0 | ((unsigned)(uint8_t)(int8_t)o1 << 8) | ((unsigned)(uint8_t)(int8_t)o2 << 16);
}
__device__ __forceinline__ int off_c(unsigned code, int c) { return (int)(int8_t)((code >> (8 * c)) & 0xffu); }

// One instance of a batch: its grid and where its tiles, cells and tables start in the batch's
// global arrays. A single solve is a batch of one.
struct Inst {
    GridGeom g;
    long long tile0;     // first global tile
    long long cell0;     // first global cell (RowMajor values of the instance start here)
    long long cls0;      // first class of its shared-stencil table
    long long metric0;   // first metric row
    long long mult0;     // first entry of its compact speed-multiplier field
    double h[3];
    int dual, metric_const, has_walls;
    int mult_depth, mult_inverse, pad;
    int nth, nph;        // ReedsShepp3: theta and phi extents (0 elsewhere)
};

// Instance holding global cell x (binary search over the increasing cell0 offsets).
__device__ __forceinline__ int inst_of_cell(const Inst *inst, int n, long long x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (inst[mid].cell0 <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Pending work of a tile: the cells whose inputs changed since their last solve and the smallest
// new value among the changes behind them, updated and taken together by 16-byte atomics (a push
// and the claim that consumes its cells always agree on the wake-up value).
struct alignas(16) DirtyWake {
    unsigned long long mask;   // cells of the tile
    unsigned long long wake;   // bit pattern of a non-negative double (+inf: none)
};
constexpr unsigned long long kInfWake = 0x7ff0000000000000ull;

__device__ __forceinline__ void dirty_add(DirtyWake *dw, unsigned long long bits, unsigned long long wake) {
    DirtyWake old;  // a torn read only costs a failed compare
    old.mask = ((volatile unsigned long long *)dw)[0];
    old.wake = ((volatile unsigned long long *)dw)[1];
    while (true) {
        DirtyWake nw;
        nw.mask = old.mask | bits;
        nw.wake = wake < old.wake ? wake : old.wake;  // non-negative doubles order as their bits
        if (nw.mask == old.mask && nw.wake == old.wake) return;
        const DirtyWake seen = atomicCAS(dw, old, nw);
        if (seen.mask == old.mask && seen.wake == old.wake) return;
        old = seen;
    }
}

template <typename Real>
struct Dev {
    const Inst *inst;         // [ninst]
    int ninst;
    const int *tile_inst;     // [ntile] instance of each global tile
    long long ncells;         // total cells
    long long ntile;          // total tiles
    long long ntc;            // tile-major cell count = ntile * 64
    long long sstride;        // distance between the stencil slots of a cell in code / weight (ntc,
                              // or the arena's size when this is a view of one arena instance)
    Real *values;             // RowMajor
    unsigned *code;           // [ND][ntc] per-cell offsets + visibility/flags (per-cell stencils)
    Real *weight;             // [ND][ntc]
    Real *mult;               // [ntc] speed multiplier (shared stencils)
    unsigned *vis;            // [ntc] slot visibility + flags (shared stencils)
    const int8_t *cls_off;    // [nclass][ND][3]
    const Real *cls_w;        // [nclass][ND]
    const int8_t *cls_ang;    // [nclass][ND][2] theta and phi steps of the differences (kKindShareS2)
    const int *cls_d2;        // [nclass][NB] third-coordinate step of each slot, periodized (kKindShareS2)
    // reverse tile dependencies: tile T -> tiles whose stencils read T, with the cells they read;
    // entries [dep_ptr[T], dep_end[T]) (dep_end null: dep_ptr[T + 1], a CSR over the tile space)
    const long long *dep_ptr;
    const long long *dep_end;
    const int *dep_tile;
    const unsigned long long *dep_mask;    // cells of T read by the dependent tile
    const unsigned long long *dep_dmask;   // cells of the dependent tile that read T
    DirtyWake *dirty;                      // [ntile] cells whose inputs changed since their last solve
    // value-ordered scheduling: key = smallest changed value among the tiles that woke the tile
    unsigned long long *key;               // [ntile] bit patterns of non-negative doubles
    // with the dirty bits, the smallest changed value (unscaled) behind them: a dirty cell whose
    // value is at or below it cannot change (see process_tile); false: every dirty cell is solved
    bool skip_settled;
    // largest value among a tile's solvable cells (+inf while any is unreached); values only
    // decrease, so a stale entry is an upper bound
    unsigned long long *maxval;            // [ntile]
    unsigned long long *rstat;             // [8][nslots][4] per round slot (and instance slot of a
                                           // resident solver): min key, max key, tiles solved, -
    int nslots;                            // 0 or 1: one statistics row per round (batch solver)
    unsigned *live;                        // [3][nslots] tiles of each instance slot in each list, or null
    // per instance: key = value * kscale, so that the keys of a batch measure the progress of each
    // instance's front on a common scale (nullptr: keys are the values)
    const double *kscale;
    const TTICell *tti;                    // [ntc] TTI norms (TTI kind)
    // static factoring of a single TTI instance (null: none): factor values, adimensional
    // gradients and mask over the box [fac_lo, fac_lo + fac_dims) of cells
    const double *fac_val;
    const double *fac_grad;
    const uint8_t *fac_mask;
    int fac_lo[3], fac_dims[3];
    int fac_sub;                           // the box is a subdomain (corrections vanish outside it)
    unsigned *tile_up;                     // [ntile] value increases taken by each tile
    unsigned up_budget;                    // increases a tile may take before it takes only
                                           // decreases (0: kUpBudget)
    // Diagonal models (a single instance): the speed (or cost) vector per cell, for the first
    // variations, which have one component per axis (var_dim = ndim; 1 elsewhere)
    const double *diag_src;
    int diag_inverse;
    int var_dim;
    unsigned order_lo, order_hi;           // tiles solved per round kept in [lo, hi]; lo = 0: plain FIM
    // active-tile lists (triple buffered) and their dedupe flags
    int *list[3];
    unsigned *count[3];
    unsigned *claim[3];
    unsigned *flag[3];
    unsigned *bar_count;
    unsigned *bar_gen;
    unsigned *status;
    unsigned long long *stats;  // rounds, tile activations, local solves
    int max_rounds;
    int sweeps;
};

// Shared stencils over R^3 x S^2 (ReedsShepp3 and ReedsSheppForward3, Curvature3.h:11-107). The
// grid (x, y, z, theta, phi) is held RowMajor as the 3-D grid (x, y, w),
// w = (z * ntheta + theta) * nphi + phi: values, tiles and scheduling are those of a 3-D grid, and
// the class of a cell is its (theta, phi) pair. Angular indices are periodized as
// PeriodicGrid.hxx:120-160 does: theta reflects at the poles (index 2 ntheta - 1 - t) while phi
// turns by nphi / 2, phi wraps.
__host__ __device__ __forceinline__ void s2_wrap(int nth, int nph, int &th, int &ph) {
    th %= 2 * nth;
    if (th < 0) th += 2 * nth;
    if (th >= nth) {
        th = 2 * nth - th - 1;
        ph += nph / 2;
    }
    ph %= nph;
    if (ph < 0) ph += nph;
}

// Step (dz, dtheta, dphi) from third coordinate x2 (z closed): false where it leaves the domain.
__host__ __device__ __forceinline__ bool s2_step(const Inst &I, int x2, int dz, int dth, int dph, int &y2) {
    const int nth = I.nth, nph = I.nph, nang = nth * nph;
    int z = x2 / nang;
    const int r = x2 - z * nang;
    int th = r / nph + dth, ph = r % nph + dph;
    z += dz;
    if (z < 0 || z >= I.g.dims[2] / nang) return false;
    s2_wrap(nth, nph, th, ph);
    y2 = (z * nth + th) * nph + ph;
    return true;
}

// Global class of the cell at third coordinate x2 of a shared-stencil instance.
template <int KIND>
__host__ __device__ __forceinline__ long long share_class(const Inst &I, int x2) {
    if constexpr (KIND == kKindShareS2) return I.cls0 + x2 % (I.nth * I.nph);
    else return I.cls0 + x2;
}

// Neighbour through slot `slot` of class cls (kKindShareS2) of a cell whose visibility bit for
// that slot is set (so the step stays in the domain): the x, y steps of the difference and the
// periodized third-coordinate step of the slot's table.
template <typename Real, int ND, int NB>
__device__ __forceinline__ void s2_visible_neighbor(const Dev<Real> &P, long long cls, int k, int slot, int s, int x0,
                                                    int x1, int x2, int &y0, int &y1, int &y2) {
    const int8_t *o = P.cls_off + (cls * ND + k) * 3;
    y0 = x0 + s * __ldg(o);
    y1 = x1 + s * __ldg(o + 1);
    y2 = x2 + __ldg(P.cls_d2 + cls * NB + slot);
}

// Neighbour y = x + s e of difference k of class cls (kKindShareS2): false outside the domain.
template <typename Real, int ND>
__device__ __forceinline__ bool s2_neighbor(const Dev<Real> &P, const Inst &I, long long cls, int k, int s, int x0,
                                            int x1, int x2, int &y0, int &y1, int &y2) {
    const int8_t *o = P.cls_off + (cls * ND + k) * 3;
    const int8_t *a = P.cls_ang + (cls * ND + k) * 2;
    y0 = x0 + s * __ldg(o);
    y1 = x1 + s * __ldg(o + 1);
    if (y0 < 0 || y0 >= I.g.dims[0] || y1 < 0 || y1 >= I.g.dims[1]) return false;
    return s2_step(I, x2, s * __ldg(o + 2), s * __ldg(a), s * __ldg(a + 1), y2);
}

// --------------------------------------------------------------------------------------------
// Hopf-Lax update over neighbour candidates v[k] (+inf if unusable) with weights w[k], taken in
// increasing order (ties by k); see the file header. `used` receives the bitmask of taken k.
//
// Fast marching adds the next neighbour iff its value is below the current root r (computed with
// rounding). For t above the vertex of q(t) = a t^2 - 2 b t + c (t measured from minVal), t < r
// iff q(t) < 0, so the decision is taken from the sign of q, which needs no square root or
// division; only when |q| is within 1e-12 of the magnitude of its terms (far wider than the
// rounding of q and of the root) is the root computed and compared exactly as fast marching does.
// The root itself is computed once, after the last addition.
template <typename Real>
__device__ __forceinline__ Real quad_root(Real minVal, Real a, Real b, Real c) {
    using A = Arith<Real>;
    if (a == Real(0)) return A::inf();
    const Real d2 = A::sub(A::mul(b, b), A::mul(a, c));
    const Real d = A::sqrt(Real(0) < d2 ? d2 : Real(0));
    return A::add(minVal, A::div(A::add(b, d), a));
}

// Compare-exchange of (value, index) pairs by value, then index: a total order, so a sorting
// network gives the selection order of the loop below (smallest value, ties by index).
template <typename Real>
__device__ __forceinline__ void cex(Real &va, Real &wa, int &ka, Real &vb, Real &wb, int &kb) {
    const bool sw = vb < va || (vb == va && kb < ka);
    const Real tv = sw ? vb : va, tw = sw ? wb : wa;
    const int tk = sw ? kb : ka;
    vb = sw ? va : vb;
    wb = sw ? wa : wb;
    kb = sw ? ka : kb;
    va = tv;
    wa = tw;
    ka = tk;
}

// Sorting networks for the small stencils (2, 3, 4, 6 and 8 differences; optimal sizes).
template <typename Real, int ND>
__device__ __forceinline__ void sort_candidates(Real (&v)[ND], Real (&w)[ND], int (&k)[ND]) {
#define HFM_CX(a, b) cex<Real>(v[a], w[a], k[a], v[b], w[b], k[b])
    if constexpr (ND == 2) {
        HFM_CX(0, 1);
    } else if constexpr (ND == 3) {
        HFM_CX(1, 2); HFM_CX(0, 2); HFM_CX(0, 1);
    } else if constexpr (ND == 4) {
        HFM_CX(0, 1); HFM_CX(2, 3); HFM_CX(0, 2); HFM_CX(1, 3); HFM_CX(1, 2);
    } else if constexpr (ND == 6) {
        HFM_CX(1, 2); HFM_CX(0, 2); HFM_CX(0, 1); HFM_CX(4, 5); HFM_CX(3, 5); HFM_CX(3, 4);
        HFM_CX(0, 3); HFM_CX(1, 4); HFM_CX(2, 5); HFM_CX(2, 4); HFM_CX(1, 3); HFM_CX(2, 3);
    } else if constexpr (ND == 8) {
        HFM_CX(0, 2); HFM_CX(1, 3); HFM_CX(4, 6); HFM_CX(5, 7); HFM_CX(0, 4); HFM_CX(1, 5); HFM_CX(2, 6);
        HFM_CX(3, 7); HFM_CX(0, 1); HFM_CX(2, 3); HFM_CX(4, 5); HFM_CX(6, 7); HFM_CX(2, 4); HFM_CX(3, 5);
        HFM_CX(1, 4); HFM_CX(3, 6); HFM_CX(1, 2); HFM_CX(3, 4); HFM_CX(5, 6);
    }
#undef HFM_CX
}

template <typename Real, int ND>
__device__ __forceinline__ Real hopf_lax_sorted(const Real (&v_in)[ND], const Real (&w_in)[ND], unsigned *used) {
    using A = Arith<Real>;
    const Real INF = A::inf();
    const Real band = sizeof(Real) == 8 ? Real(1e-12) : Real(1e-5);
    if constexpr (ND == 2 || ND == 3 || ND == 4 || ND == 6 || ND == 8) {
        // the same additions in the same order as the selection loop below, on sorted candidates
        Real v[ND], w[ND];
        int k[ND];
#pragma unroll
        for (int i = 0; i < ND; ++i) { v[i] = v_in[i]; w[i] = w_in[i]; k[i] = i; }
        sort_candidates<Real, ND>(v, w, k);
        unsigned taken = 0;
        Real minVal = v[0], a = 0, b = 0, c = -1;
#pragma unroll
        for (int it = 0; it < ND; ++it) {
            const Real bv = v[it], bw = w[it];
            if (!(bv < INF)) break;
            if (it > 0) {
                const Real t = A::sub(bv, minVal);
                const Real at2 = A::mul(A::mul(a, t), t), bt2 = A::mul(Real(2), A::mul(b, t));
                const Real q = A::add(A::sub(at2, bt2), c);
                const Real mag = A::add(A::add(fabs(at2), fabs(bt2)), fabs(c));
                if (q > band * mag) break;
                if (!(q < -band * mag) && !(bv < quad_root<Real>(minVal, a, b, c))) break;
            }
            const Real dv = A::sub(bv, minVal);
            const Real wv = A::mul(bw, dv);
            a = A::add(a, bw);
            b = A::add(b, wv);
            c = A::add(c, A::mul(wv, dv));
            taken |= 1u << k[it];
        }
        if (used) *used = taken;
        return taken ? quad_root<Real>(minVal, a, b, c) : INF;
    }
    const Real (&v)[ND] = v_in;
    const Real (&w)[ND] = w_in;
    unsigned taken = 0;
    Real minVal = 0, a = 0, b = 0, c = -1;
    for (int it = 0; it < ND; ++it) {
        Real bv = INF, bw = 0;
        int bk = -1;
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            if (!((taken >> k) & 1u) && v[k] < bv) { bv = v[k]; bw = w[k]; bk = k; }
        }
        if (bk < 0) break;
        if (it == 0) {
            minVal = bv;
        } else {
            // stop unless bv < root(a, b, c)
            const Real t = A::sub(bv, minVal);
            const Real at2 = A::mul(A::mul(a, t), t), bt2 = A::mul(Real(2), A::mul(b, t));
            const Real q = A::add(A::sub(at2, bt2), c);
            const Real mag = A::add(A::add(fabs(at2), fabs(bt2)), fabs(c));
            if (q > band * mag) break;
            if (!(q < -band * mag) && !(bv < quad_root<Real>(minVal, a, b, c))) break;
        }
        const Real dv = A::sub(bv, minVal);
        const Real wv = A::mul(bw, dv);
        a = A::add(a, bw);
        b = A::add(b, wv);
        c = A::add(c, A::mul(wv, dv));
        taken |= 1u << bk;
    }
    if (used) *used = taken;
    return taken ? quad_root<Real>(minVal, a, b, c) : INF;
}

// Hopf-Lax update of two groups of forward differences (EulerianStencil<.,0,6,2>, Dubins2):
// neighbours are taken in increasing order of value, each one only while below the current value,
// and added to every difference whose offset reaches it (EulerianStencil.hxx:104-153); the
// differences k < ND/2 accumulate in group 0, the others in group 1, from one shared minVal; the
// value is minVal plus the smaller group root, group 0 on ties (QuadraticMax<.,2>::Solve,
// EulerianStencil.hxx:30-50). `used` receives the added differences and, in bit ND, the group.
template <typename Real, int ND>
__device__ __forceinline__ Real hopf_lax_two_groups(const Real (&v)[ND], const Real (&w)[ND], const unsigned (&oc)[ND],
                                                    unsigned *used) {
    using A = Arith<Real>;
    const Real INF = A::inf();
    Real minVal = 0, a0 = 0, b0 = 0, c0 = -1, a1 = 0, b1 = 0, c1 = -1;
    Real value = INF;
    int imin = 0;
    unsigned taken = 0;
    for (int it = 0; it < ND; ++it) {
        Real bv = INF;
        int bk = -1;
#pragma unroll
        for (int k = 0; k < ND; ++k)
            if (!((taken >> k) & 1u) && v[k] < bv) { bv = v[k]; bk = k; }
        if (bk < 0) break;
        if (it == 0) minVal = bv;
        else if (!(bv < value)) break;  // ConditionalUpdate: values[x] <= acceptedValue
        const unsigned ob = oc[bk];
        const Real dv = A::sub(bv, minVal);
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            if (((taken >> k) & 1u) || oc[k] != ob || !(v[k] < INF)) continue;
            taken |= 1u << k;
            const Real wv = A::mul(w[k], dv);
            const Real wv2 = A::mul(wv, dv);
            if (k < ND / 2) { a0 = A::add(a0, w[k]); b0 = A::add(b0, wv); c0 = A::add(c0, wv2); }
            else { a1 = A::add(a1, w[k]); b1 = A::add(b1, wv); c1 = A::add(c1, wv2); }
        }
        Real res = INF;
        imin = 0;
        if (a0 != Real(0)) {
            const Real d2 = A::sub(A::mul(b0, b0), A::mul(a0, c0));
            res = A::div(A::add(b0, A::sqrt(Real(0) < d2 ? d2 : Real(0))), a0);
        }
        if (a1 != Real(0)) {
            const Real d2 = A::sub(A::mul(b1, b1), A::mul(a1, c1));
            const Real r1 = A::div(A::add(b1, A::sqrt(Real(0) < d2 ? d2 : Real(0))), a1);
            if (r1 < res) { res = r1; imin = 1; }
        }
        value = A::add(minVal, res);
    }
    if (used) *used = taken | ((unsigned)imin << ND);
    return taken ? value : INF;
}

// Local solve at one cell. `sv` holds the current values of the warp's tile (nullptr: read all
// neighbours from global memory). `side` receives, per symmetric difference, 1 if the -e
// neighbour provided the candidate.
template <typename Real, int NFWD, int NSYM, int KIND>
__device__ __forceinline__ Real solve_cell_stencil(const Dev<Real> &P, const Inst &I, long long c, int x0, int x1,
                                                   int x2, int tx0, int tx1, int tx2, const Real *sv, unsigned *used,
                                                   unsigned *side) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    using A = Arith<Real>;
    const Real INF = A::inf();
    const GridGeom &g = I.g;
    const Real *values = P.values + I.cell0;
    const long long cls = share_class<KIND>(I, x2);
    Real v[ND], w[ND];
    [[maybe_unused]] unsigned oc[ND];  // packed offsets (two-group stencils: shared neighbours)
    Real m2 = 1;
    unsigned visw = 0;
    if (SHARE) {
        const Real m = P.mult[c];
        m2 = A::mul(m, m);
        visw = P.vis[c];
    }
    unsigned sides = 0;
    auto fetch_at = [&](int n0, int n1, int n2) -> Real {
        if (sv) {
            const unsigned l0 = n0 - tx0, l1 = n1 - tx1, l2 = n2 - tx2;
            if (l0 < (1u << g.tshift[0]) && l1 < (1u << g.tshift[1]) && l2 < (1u << g.tshift[2]))
                return sv[((l0 << g.tshift[1] | l1) << g.tshift[2]) | l2];
        }
        return __ldcg(values + g.lin(n0, n1, n2));
    };
    auto fetch = [&](int o0, int o1, int o2) -> Real {
        int n2 = x2 + o2;
        if (SHARE && g.periodic[2]) {
            n2 %= g.dims[2];
            if (n2 < 0) n2 += g.dims[2];
        }
        return fetch_at(x0 + o0, x1 + o1, n2);
    };
#pragma unroll
    for (int k = 0; k < ND; ++k) {
        int o0, o1, o2;
        bool vp, vm = false;
        if (SHARE) {
            const int8_t *o = P.cls_off + (cls * ND + k) * 3;
            o0 = __ldg(o); o1 = __ldg(o + 1); o2 = __ldg(o + 2);
            if constexpr (KIND == kKindShare2) oc[k] = pack_off(o0, o1, o2);
            w[k] = A::mul(__ldg(P.cls_w + cls * ND + k), m2);
            if (k < NFWD) {
                vp = (visw >> k) & 1u;
            } else {
                const int s = NFWD + 2 * (k - NFWD);
                vp = (visw >> s) & 1u;
                vm = (visw >> (s + 1)) & 1u;
            }
        } else {
            const unsigned cd = P.code[k * P.sstride + c];
            o0 = off_c(cd, 0); o1 = off_c(cd, 1); o2 = off_c(cd, 2);
            w[k] = P.weight[k * P.sstride + c];
            vp = cd & kVisPlus;
            vm = (k >= NFWD) && (cd & kVisMinus);
        }
        Real val = INF;
        if constexpr (KIND == kKindShareS2) {
            // the visibility bits hold only steps that stay in the domain
            constexpr int NB = NFWD + 2 * NSYM;
            const int slot = k < NFWD ? k : NFWD + 2 * (k - NFWD);
            int y0, y1, y2;
            if (vp) {
                s2_visible_neighbor<Real, ND, NB>(P, cls, k, slot, 1, x0, x1, x2, y0, y1, y2);
                val = fetch_at(y0, y1, y2);
            }
            if (vm) {
                s2_visible_neighbor<Real, ND, NB>(P, cls, k, slot + 1, -1, x0, x1, x2, y0, y1, y2);
                const Real vv = fetch_at(y0, y1, y2);
                if (vv < val) { val = vv; if (k >= NFWD) sides |= 1u << (k - NFWD); }
            }
        } else {
            if (vp) val = fetch(o0, o1, o2);
            if (vm) {
                const Real vv = fetch(-o0, -o1, -o2);
                if (vv < val) { val = vv; if (k >= NFWD) sides |= 1u << (k - NFWD); }
            }
        }
        v[k] = val;
    }
    if (side) *side = sides;
    if constexpr (KIND == kKindShare2) return hopf_lax_two_groups<Real, ND>(v, w, oc, used);
    else return hopf_lax_sorted<Real, ND>(v, w, used);
}

// TTI local solve of a cell of the factoring box (StaticFactoring.hxx:33-64 with TTI.hpp:160-276).
// A neighbour y = x + e enters with u(y) + <grad(x), e> + value(x) - value(y) (order-1 Correction;
// the last two terms 0 when y leaves a subdomain box). Fast marching re-solves x from its accepted
// neighbours each time one of them is accepted below x's current value, and keeps the smallest
// result; with the corrections the neighbours above that value can change a solve, so that order
// is reproduced: the neighbours the update can read, in increasing value, each one triggering a
// solve over the neighbours at or below its value while it is below the smallest result so far.
template <typename Real, typename Get>
__device__ double solve_cell_tti_factored(const Dev<Real> &P, long long c, const int (&b)[3], long long bi, Get raw,
                                          double *t_act, bool *interior) {
    using A = Arith<double>;
    const double INF = A::inf();
    const double fx = P.fac_val[bi];
    const double *gx = P.fac_grad + 3 * bi;
    auto corr = [&](int o0, int o1, int o2) -> double {
        const int e0 = b[0] + o0, e1 = b[1] + o1, e2 = b[2] + o2;
        if ((unsigned)e0 >= (unsigned)P.fac_dims[0] || (unsigned)e1 >= (unsigned)P.fac_dims[1] ||
            (unsigned)e2 >= (unsigned)P.fac_dims[2])
            return 0.0;  // out of a subdomain box; a whole-domain box holds every neighbour read
        const long long ei = ((long long)e0 * P.fac_dims[1] + e1) * P.fac_dims[2] + e2;
        double deriv = 0.0;
        deriv = A::add(deriv, A::mul(gx[0], (double)o0));
        deriv = A::add(deriv, A::mul(gx[1], (double)o1));
        deriv = A::add(deriv, A::mul(gx[2], (double)o2));
        return A::add(deriv, A::sub(fx, P.fac_val[ei]));
    };
    // the values of the neighbours the update can read (the cell's Selling-path offsets, both signs)
    constexpr int kMax = 2 * kTTISlots;
    double th[kMax];
    int nth = 0;
    for (int k = 0; k < kTTISlots; ++k) {
        if (P.weight[k * P.sstride + c] == Real(0)) continue;
        const unsigned cd = P.code[k * P.sstride + c];
        const int o0 = off_c(cd, 0), o1 = off_c(cd, 1), o2 = off_c(cd, 2);
        for (int sg = 1; sg >= -1; sg -= 2) {
            const double v = raw(sg * o0, sg * o1, sg * o2);
            if (!(v < INF)) continue;
            int q = nth++;
            while (q > 0 && th[q - 1] > v) { th[q] = th[q - 1]; --q; }
            th[q] = v;
        }
    }
    double best = INF, tb = INF;
    bool ib = false;
    for (int q = 0; q < nth; ++q) {
        const double theta = th[q];
        if (q > 0 && theta == th[q - 1]) continue;
        if (!(theta < best)) break;  // ConditionalUpdate: values[x] <= acceptedValue
        auto get = [&](int o0, int o1, int o2) -> double {
            const double v = raw(o0, o1, o2);
            if (!(v <= theta)) return INF;
            return A::add(v, corr(o0, o1, o2));
        };
        double ta = INF;
        bool in = false;
        const double sv = tti_solve(P.tti[c], get, &ta, &in);
        if (sv < best) { best = sv; tb = ta; ib = in; }
    }
    if (t_act) *t_act = tb;
    if (interior) *interior = ib;
    return best;
}

// TTI local solve at one cell (FP64): neighbour values from the tile in shared memory or global
// memory, +inf outside the domain.
template <typename Real>
__device__ __forceinline__ Real solve_cell_tti(const Dev<Real> &P, const Inst &I, long long c, int x0, int x1, int x2,
                                               int tx0, int tx1, int tx2, const Real *sv, double *t_act,
                                               bool *interior) {
    const GridGeom &g = I.g;
    const Real *values = P.values + I.cell0;
    auto get = [&](int o0, int o1, int o2) -> double {
        const int n0 = x0 + o0, n1 = x1 + o1, n2 = x2 + o2;
        if ((unsigned)n0 >= (unsigned)g.dims[0] || (unsigned)n1 >= (unsigned)g.dims[1] ||
            (unsigned)n2 >= (unsigned)g.dims[2])
            return Arith<double>::inf();
        if (sv) {
            const unsigned l0 = n0 - tx0, l1 = n1 - tx1, l2 = n2 - tx2;
            if (l0 < (1u << g.tshift[0]) && l1 < (1u << g.tshift[1]) && l2 < (1u << g.tshift[2]))
                return (double)sv[((l0 << g.tshift[1] | l1) << g.tshift[2]) | l2];
        }
        return (double)__ldcg(values + g.lin(n0, n1, n2));
    };
    if (P.fac_val) {
        const int b[3] = {x0 - P.fac_lo[0], x1 - P.fac_lo[1], x2 - P.fac_lo[2]};
        if ((unsigned)b[0] < (unsigned)P.fac_dims[0] && (unsigned)b[1] < (unsigned)P.fac_dims[1] &&
            (unsigned)b[2] < (unsigned)P.fac_dims[2]) {
            const long long bi = ((long long)b[0] * P.fac_dims[1] + b[1]) * P.fac_dims[2] + b[2];
            if (P.fac_mask[bi]) return (Real)solve_cell_tti_factored<Real>(P, c, b, bi, get, t_act, interior);
        }
    }
    return (Real)tti_solve(P.tti[c], get, t_act, interior);
}

template <typename Real, int NFWD, int NSYM, int KIND>
__device__ __forceinline__ Real solve_cell(const Dev<Real> &P, const Inst &I, long long c, int x0, int x1, int x2,
                                           int tx0, int tx1, int tx2, const Real *sv, unsigned *used, unsigned *side) {
    if constexpr (KIND == kKindTTI) {
        if (used) *used = 0;
        if (side) *side = 0;
        return solve_cell_tti<Real>(P, I, c, x0, x1, x2, tx0, tx1, tx2, sv, nullptr, nullptr);
    } else {
        return solve_cell_stencil<Real, NFWD, NSYM, KIND>(P, I, c, x0, x1, x2, tx0, tx1, tx2, sv, used, side);
    }
}

template <typename Real, int KIND>
__device__ __forceinline__ void cell_flags(const Dev<Real> &P, long long c, bool &fixed, bool &dead) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    if (SHARE) {
        const unsigned f = P.vis[c];
        fixed = f & kShFixed;
        dead = f & kShDead;
    } else {
        const unsigned f = P.code[c];
        fixed = f & kFixed;
        dead = f & kDead;
    }
}

// Appends tile D (of instance slot `inst`) to list `li` unless it is already there (flag dedupe).
// Called by all lanes with their own `want`; one atomicAdd per warp reserves the slots. A resident
// solver also counts the tiles of each instance per list (all lanes of a call push tiles of one
// instance).
template <typename Real>
__device__ __forceinline__ void push_tiles(const Dev<Real> &P, int li, int D, bool want, int lane, int inst) {
    if (want) want = atomicExch(&P.flag[li][D], 1u) == 0u;
    const unsigned ballot = __ballot_sync(0xffffffffu, want);
    if (!ballot) return;
    unsigned base = 0;
    if (lane == __ffs(ballot) - 1) {
        base = atomicAdd(P.count[li], (unsigned)__popc(ballot));
        if (P.live) atomicAdd(P.live + li * P.nslots + inst, (unsigned)__popc(ballot));
    }
    base = __shfl_sync(0xffffffffu, base, __ffs(ballot) - 1);
    if (want) P.list[li][base + __popc(ballot & ((1u << lane) - 1u))] = D;
}

// Statistics row of round slot `slot` for instance slot `inst` (one row per round slot when the
// solver keeps no per-instance statistics).
template <typename Real>
__device__ __forceinline__ unsigned long long *stat_row(const Dev<Real> &P, int slot, int inst) {
    const int ns = P.nslots > 1 ? P.nslots : 1;
    return P.rstat + ((long long)slot * ns + (ns > 1 ? inst : 0)) * 4;
}

// Warp-local smallest and largest wake-up keys pushed for one instance in one round, merged into
// its statistics row with two atomics when the instance or round changes and before the round's
// barrier (instead of two atomics on the same row per pushed tile). Warp-uniform.
struct StatAcc {
    int inst = -1, slot = 0;
    unsigned long long mn = ~0ull, mx = 0ull;
};

template <typename Real>
__device__ __forceinline__ void stat_flush(const Dev<Real> &P, StatAcc &a, int lane) {
    if (a.inst >= 0 && lane == 0) {
        unsigned long long *row = stat_row(P, a.slot, a.inst);
        if (a.mn != ~0ull) atomicMin(row + 0, a.mn);
        if (a.mx) atomicMax(row + 1, a.mx);
    }
    a.inst = -1;
    a.mn = ~0ull;
    a.mx = 0ull;
}

template <typename Real>
__device__ __forceinline__ void stat_add(const Dev<Real> &P, StatAcc &a, int slot, int inst, unsigned long long kmin,
                                         unsigned long long kmax, int lane) {
    if (a.inst != inst || a.slot != slot) {
        stat_flush(P, a, lane);
        a.inst = inst;
        a.slot = slot;
    }
    a.mn = kmin < a.mn ? kmin : a.mn;
    a.mx = kmax > a.mx ? kmax : a.mx;
}

// Pushes the dependents of tile T that read a cell of `mask`, marking as dirty the cells of each
// dependent that read T; if `self_pending` is non-zero T itself is pushed with those cells dirty.
// Dirty bits are set before the dedupe flag so that a dependent already queued, or one that has
// just claimed itself, sees them on its next activation. The wake-up value `mu` (smallest changed
// value of T) goes with the dirty bits in one atomic update.
template <typename Real>
__device__ __forceinline__ void push_dependents(const Dev<Real> &P, int li, int slot, int T, unsigned long long mask,
                                                unsigned long long self_pending, unsigned long long mu,
                                                unsigned long long kb, int lane, StatAcc &acc) {
    bool any = false;
    const int inst = P.tile_inst[T];
    if (mask) {
        const long long b = P.dep_ptr[T], e = P.dep_end ? P.dep_end[T] : P.dep_ptr[T + 1];
        for (long long base = b; base < e; base += 32) {
            const long long i = base + lane;
            bool want = false;
            int D = 0;
            if (i < e) {
                D = P.dep_tile[i];
                want = (P.dep_mask[i] & mask) != 0ull;
                // a neighbour value v improves x only if v < u(x) (ConditionalUpdate,
                // HamiltonFastMarching.hxx:151): no cell of D can gain from values >= max u(D).
                // Not with static factoring: D's values can rise during an activation that has not
                // yet published its larger maximum, so a stale maximum would drop a needed wake-up
                if (want && !P.fac_val) {
                    const double mx = __longlong_as_double(__ldcg(P.maxval + D));
                    want = __longlong_as_double(mu) < mx * (1.0 + 16.0 * DBL_EPSILON);
                }
                if (want) {
                    dirty_add(P.dirty + D, P.dep_dmask[i], mu);
                    atomicMin(P.key + D, kb);
                }
            }
            any |= __any_sync(0xffffffffu, want);
            push_tiles(P, li, D, want, lane, inst);
        }
    }
    if (self_pending && lane == 0) {
        dirty_add(P.dirty + T, self_pending, mu);
        atomicMin(P.key + T, kb);
    }
    push_tiles(P, li, T, self_pending != 0ull && lane == 0, lane, inst);
    if (any || self_pending) stat_add(P, acc, slot, inst, kb, kb, lane);
}

// Class of a list entry at the start of a round. Stale: no key and no pending cell (its cells were
// solved after it was queued; a later push queues the tile again, so it is dropped). In the band:
// key at most theta, or pending cells without a key (a push that raced with the tile's own
// activation). Carried: a key above theta.
constexpr int kEntryStale = 0, kEntryBand = 1, kEntryCarried = 2;

template <typename Real>
__device__ __forceinline__ int entry_class(const Dev<Real> &P, int T, unsigned long long kt, double theta) {
    if (kt == 0x7ff0000000000000ull) {
        const unsigned long long m = ((volatile const unsigned long long *)(P.dirty + T))[0];
        return m ? kEntryBand : kEntryStale;
    }
    return __longlong_as_double(kt) <= theta ? kEntryBand : kEntryCarried;
}

// Cells of the warp's tile that the cell at (x0,x1,x2) reads through its visible stencil entries.
template <typename Real, int NFWD, int NSYM, int KIND>
__device__ __forceinline__ unsigned long long intile_reads(const Dev<Real> &P, const Inst &I, long long c, int x0,
                                                           int x1, int x2, int tx0, int tx1, int tx2) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    const GridGeom &g = I.g;
    unsigned long long m = 0;
    const unsigned visw = SHARE ? P.vis[c] : 0u;
    [[maybe_unused]] const long long cls = share_class<KIND>(I, x2);
#pragma unroll
    for (int k = 0; k < ND; ++k) {
        int o0, o1, o2;
        unsigned bits;
        if (SHARE) {
            const int8_t *o = P.cls_off + (cls * ND + k) * 3;
            o0 = __ldg(o); o1 = __ldg(o + 1); o2 = __ldg(o + 2);
            bits = k < NFWD ? ((visw >> k) & 1u) : ((visw >> (NFWD + 2 * (k - NFWD))) & 3u);
        } else {
            const unsigned cd = P.code[k * P.sstride + c];
            o0 = off_c(cd, 0); o1 = off_c(cd, 1); o2 = off_c(cd, 2);
            bits = ((cd & kVisPlus) ? 1u : 0u) | ((cd & kVisMinus) ? 2u : 0u);
        }
#pragma unroll
        for (int si = 0; si < 2; ++si) {
            if (!((bits >> si) & 1u)) continue;
            const int s = si ? -1 : 1;
            int n0 = x0 + s * o0, n1 = x1 + s * o1, n2 = x2 + s * o2;
            if constexpr (KIND == kKindShareS2) {
                s2_visible_neighbor<Real, ND, NFWD + 2 * NSYM>(P, cls, k, k < NFWD ? k : NFWD + 2 * (k - NFWD) + si, s,
                                                              x0, x1, x2, n0, n1, n2);
            } else if (SHARE && g.periodic[2]) {
                n2 %= g.dims[2];
                if (n2 < 0) n2 += g.dims[2];
            }
            const unsigned l0 = n0 - tx0, l1 = n1 - tx1, l2 = n2 - tx2;
            if (l0 < (1u << g.tshift[0]) && l1 < (1u << g.tshift[1]) && l2 < (1u << g.tshift[2]))
                m |= 1ull << (((l0 << g.tshift[1] | l1) << g.tshift[2]) | l2);
        }
    }
    return m;
}

// One activation of tile T: solve the dirty cells, then, sweep after sweep, the cells reading an
// in-tile cell that changed in the previous sweep, until nothing changes (warp vote) or the sweep
// budget is spent (T re-queues itself with the cells still pending).
//
// A cell is solved only if its value is above the smallest new value among the neighbours that
// changed since its last solve (the tile's wake-up value for the dirty cells, the smallest value
// changed in the previous sweep for the others). The Hopf-Lax update uses only the candidates
// below the cell's current value, which such changes leave in place, so the skipped solve would
// return the same value bit for bit (fast marching's own rule: a neighbour accepted at or above a
// cell's tentative value does not update it, HamiltonFastMarching.hxx:151). Not applied to TTI3,
// whose update is an extremum over a family of such solves.
template <typename Real, int NFWD, int NSYM, int KIND>
__device__ __forceinline__ void process_tile(const Dev<Real> &P, int T, Real *sv, int lane, int li_next, int slot,
                                             unsigned long long &n_solves, StatAcc &acc) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    const Inst &I = P.inst[P.tile_inst[T]];
    const GridGeom &g = I.g;
    int t0, t1, t2;
    g.tile_coords(T - I.tile0, t0, t1, t2);
    const int tx0 = t0 << g.tshift[0], tx1 = t1 << g.tshift[1], tx2 = t2 << g.tshift[2];
    unsigned long long dirty = 0, wk = 0ull;
    if (lane == 0) {
        const DirtyWake taken = atomicExch(P.dirty + T, DirtyWake{0ull, kInfWake});
        dirty = taken.mask;
        wk = taken.wake;
    }
    dirty = __shfl_sync(0xffffffffu, dirty, 0);
    double lim = -1.0;  // solve a cell only if its value is above lim
    if (KIND != kKindTTI && P.skip_settled) lim = __longlong_as_double(__shfl_sync(0xffffffffu, wk, 0));
    __threadfence();
    Real cur[2];
    [[maybe_unused]] Real first[2];  // TTI3: the values before the activation (see the wake-up key)
    bool upd[2], todo[2], chg[2] = {false, false};
    unsigned long long reads[2] = {0ull, 0ull};
    int xs[2][3];
    long long gi[2];
    const Real INF = Arith<Real>::inf();
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int l = lane + 32 * j;
        int l0, l1, l2;
        g.local_coords(l, l0, l1, l2);
        xs[j][0] = tx0 + l0; xs[j][1] = tx1 + l1; xs[j][2] = tx2 + l2;
        const bool valid = xs[j][0] < g.dims[0] && xs[j][1] < g.dims[1] && xs[j][2] < g.dims[2];
        bool fixed = true, dead = true;
        const long long c = (long long)T * 64 + l;
        if (valid) cell_flags<Real, KIND>(P, c, fixed, dead);
        gi[j] = valid ? I.cell0 + g.lin(xs[j][0], xs[j][1], xs[j][2]) : 0;
        cur[j] = (valid && !dead) ? __ldcg(P.values + gi[j]) : INF;
        upd[j] = valid && !dead && !fixed;
        todo[j] = upd[j] && ((dirty >> l) & 1ull) && (double)cur[j] > lim;
        sv[l] = cur[j];
        if constexpr (KIND == kKindTTI) first[j] = cur[j];
    }
    // nothing to solve (every dirty cell settled): the values and the tile's largest value stand
    if (!__any_sync(0xffffffffu, todo[0] || todo[1])) return;
    bool have_reads = false;  // in-tile read masks, built once a sweep has changed a cell
    __syncwarp();
    bool converged = false;
    unsigned ups = 0;  // increases taken by this lane in this activation
    unsigned tile_ups = 0;
    if (lane == 0) tile_ups = __ldcg(P.tile_up + T);
    const bool strict = __shfl_sync(0xffffffffu, tile_ups, 0) >= (P.up_budget ? P.up_budget : kUpBudget);
    for (int sweep = 0; sweep < P.sweeps; ++sweep) {
        Real nv[2] = {cur[0], cur[1]};
        // one copy of the (large) local solve for both cells; the per-cell operands are selected,
        // not indexed, so that they stay in registers
#pragma unroll 1
        for (int j = 0; j < 2; ++j) {
            if (j ? todo[1] : todo[0]) {
                const Real r = solve_cell<Real, NFWD, NSYM, KIND>(
                    P, I, (long long)T * 64 + lane + 32 * j, j ? xs[1][0] : xs[0][0], j ? xs[1][1] : xs[0][1],
                    j ? xs[1][2] : xs[0][2], tx0, tx1, tx2, sv, nullptr, nullptr);
                if (j) nv[1] = r;
                else nv[0] = r;
                ++n_solves;
            }
        }
        __syncwarp();
        bool now[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            // Any change is taken, so that the field converges to the exact fixed point of the
            // local solves (what fast marching computes from the final neighbour values, whatever
            // the schedule). Rounding can make a recomputation land an ulp above the current value
            // and such increases can cycle (observed on TTI3, whose extremum over t is found
            // iteratively): a tile that has taken kUpBudget increases takes only decreases from
            // then on, so the iteration terminates (values then decrease in a finite set); its
            // cells keep the smallest value they were computed at (fast marching's own rule,
            // HamiltonFastMarching.hxx:151-176), equal to the fixed point up to rounding.
            now[j] = strict ? nv[j] < cur[j] : nv[j] != cur[j];
            ups += (now[j] && nv[j] > cur[j]) ? 1u : 0u;
            if (now[j]) {
                cur[j] = nv[j];
                sv[lane + 32 * j] = nv[j];
                chg[j] = true;
            }
        }
        __syncwarp();
        const unsigned long long C = (unsigned long long)__ballot_sync(0xffffffffu, now[0]) |
                                     ((unsigned long long)__ballot_sync(0xffffffffu, now[1]) << 32);
        if (!C) { converged = true; break; }
        if (!have_reads) {
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (upd[j])
                    reads[j] = intile_reads<Real, NFWD, NSYM, KIND>(P, I, (long long)T * 64 + lane + 32 * j, xs[j][0],
                                                                    xs[j][1], xs[j][2], tx0, tx1, tx2);
            have_reads = true;
        }
        if (KIND != kKindTTI && P.skip_settled) {  // smallest value changed in this sweep
            double m = Arith<double>::inf();
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (now[j] && (double)cur[j] < m) m = (double)cur[j];
#pragma unroll
            for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
            lim = m;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) todo[j] = upd[j] && (reads[j] & C) != 0ull && (double)cur[j] > lim;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) ups += __shfl_xor_sync(0xffffffffu, ups, o);
    if (lane == 0 && ups) __stcg(P.tile_up + T, tile_ups + ups);
    unsigned long long pending = 0;
    if (!converged)
        pending = (unsigned long long)__ballot_sync(0xffffffffu, todo[0]) |
                  ((unsigned long long)__ballot_sync(0xffffffffu, todo[1]) << 32);
#pragma unroll
    for (int j = 0; j < 2; ++j)
        if (chg[j]) __stcg(P.values + gi[j], cur[j]);
    const unsigned lo = __ballot_sync(0xffffffffu, chg[0]);
    const unsigned hi = __ballot_sync(0xffffffffu, chg[1]);
    const unsigned long long mask = (unsigned long long)lo | ((unsigned long long)hi << 32);
    // largest solvable value of the tile, for the wake-up pruning of its sources
    double mx = 0.0;
#pragma unroll
    for (int j = 0; j < 2; ++j)
        if (upd[j] && !((double)cur[j] <= mx)) mx = (double)cur[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) __stcg(P.maxval + T, (unsigned long long)__double_as_longlong(mx));
    // smallest changed value: the wake-up key of the dependents. A TTI3 update can rise (static
    // factoring makes it non-monotone), and a neighbour that rose may have been below a dependent's
    // value before: the smaller of the old and new values wakes the dependents then.
    double mu = Arith<double>::inf();
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        if (!chg[j]) continue;
        double m = (double)cur[j];
        if constexpr (KIND == kKindTTI) m = (double)first[j] < m ? (double)first[j] : m;
        mu = m < mu ? m : mu;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) mu = fmin(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    __threadfence();
    const double kv = P.kscale ? mu * P.kscale[P.tile_inst[T]] : mu;
    push_dependents(P, li_next, slot, T, mask, pending, (unsigned long long)__double_as_longlong(mu),
                    (unsigned long long)__double_as_longlong(kv), lane, acc);
}

// Persistent cooperative solver: rounds over the triple-buffered active-tile lists. Round r solves
// the active tiles whose key is at most theta_r = (smallest key) + delta_r and carries the others to
// the next list; delta_r doubles when a round solved fewer than order_lo tiles and halves above
// order_hi, so the band follows the arrival front with enough tiles in flight. Every block derives
// the same theta_r from the same round statistics read after the barrier.
// Resident CTAs per SM requested from the register allocator (measured on B200: the solve is
// latency-bound, and more resident warps beat the spills this costs, except for the 27-offset
// Elastica stencil whose local solve needs the registers).
template <typename Real, int NFWD, int NSYM, int KIND>
constexpr int fim_min_blocks() {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    // ReedsShepp3: 4 blocks per SM (up to 128 registers), which keeps its 8-difference update and
    // the sphere periodization out of local memory
    return KIND == kKindTTI ? 1 : KIND == kKindShareS2 ? 4 : SHARE ? (NFWD + NSYM > 8 ? (sizeof(Real) == 8 ? 1 : 4) : 8) : 8;
}

template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void __launch_bounds__(kWarpsPerCta * 32, (fim_min_blocks<Real, NFWD, NSYM, KIND>())) fim_kernel(Dev<Real> P) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    __shared__ Real s_vals[kWarpsPerCta][64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long kInfBits = 0x7ff0000000000000ull;
    unsigned long long n_act = 0, n_solves = 0, n_carry = 0;
    StatAcc acc;
    double delta = Arith<double>::inf();
    int r = 0;
    bool ok = true;
    for (; r < P.max_rounds; ++r) {
        const int cur = r % 3, nxt = (r + 1) % 3, old = (r + 2) % 3;
        const int slot = r & 7, nslot = (r + 1) & 7, rslot = (r + 4) & 7;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            *P.count[old] = 0;
            *P.claim[old] = 0;
            P.rstat[rslot * 4 + 0] = kInfBits;
            P.rstat[rslot * 4 + 1] = 0ull;
            P.rstat[rslot * 4 + 2] = 0ull;
        }
        const unsigned n = *(volatile unsigned *)P.count[cur];
        const double mk = __longlong_as_double(*(volatile unsigned long long *)(P.rstat + slot * 4 + 0));
        const double theta = (P.order_lo == 0u) ? Arith<double>::inf() : mk + delta;
        unsigned long long solved = 0;
        while (true) {
            unsigned i = 0;
            if (lane == 0) i = atomicAdd(P.claim[cur], 1u);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= n) break;
            const int T = P.list[cur][i];
            unsigned long long kt = 0;
            int cls = 0;
            if (lane == 0) {
                P.flag[cur][T] = 0u;
                kt = *(volatile unsigned long long *)(P.key + T);
                cls = entry_class(P, T, kt, theta);
            }
            kt = __shfl_sync(0xffffffffu, kt, 0);
            cls = __shfl_sync(0xffffffffu, cls, 0);
            if (cls == kEntryStale) continue;
            if (cls == kEntryCarried) {
                // not yet in the band: carry to the next round with its key
                push_tiles(P, nxt, T, lane == 0, lane, 0);
                stat_add(P, acc, nslot, 0, kt, 0ull, lane);
                ++n_carry;
                continue;
            }
            if (lane == 0) atomicExch(P.key + T, kInfBits);
            __threadfence();  // the key is cleared before the tile's pending cells are taken
            process_tile<Real, NFWD, NSYM, KIND>(P, T, s_vals[warp], lane, nxt, nslot, n_solves, acc);
            ++n_act;
            ++solved;
        }
        stat_flush(P, acc, lane);
        if (lane == 0 && solved) atomicAdd(P.rstat + slot * 4 + 2, solved);
        ok = grid_barrier(P.bar_count, P.bar_gen, gridDim.x, P.status, kBarrierPolls);
        if (!ok) break;
        if (*(volatile unsigned *)P.count[nxt] == 0u) { ++r; break; }
        if (P.order_lo) {
            const unsigned long long np = *(volatile unsigned long long *)(P.rstat + slot * 4 + 2);
            if (r == 0) {
                const double lo_k = __longlong_as_double(*(volatile unsigned long long *)(P.rstat + nslot * 4 + 0));
                const double hi_k = __longlong_as_double(*(volatile unsigned long long *)(P.rstat + nslot * 4 + 1));
                delta = hi_k > lo_k ? 2.0 * (hi_k - lo_k) : Arith<double>::inf();
            } else if (np < P.order_lo) {
                delta *= 2.0;
            } else if (np > P.order_hi) {
                delta *= 0.5;
            }
        }
    }
    if (ok && r >= P.max_rounds && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(P.status, (unsigned)kErrRoundCap);
    if (lane == 0) {
        atomicAdd(P.stats + 1, n_act);
        atomicAdd(P.stats + 3, n_carry);
    }
    n_solves += __shfl_xor_sync(0xffffffffu, n_solves, 16);
    n_solves += __shfl_xor_sync(0xffffffffu, n_solves, 8);
    n_solves += __shfl_xor_sync(0xffffffffu, n_solves, 4);
    n_solves += __shfl_xor_sync(0xffffffffu, n_solves, 2);
    n_solves += __shfl_xor_sync(0xffffffffu, n_solves, 1);
    if (lane == 0) atomicAdd(P.stats + 2, n_solves);
    if (blockIdx.x == 0 && threadIdx.x == 0) P.stats[0] = (unsigned long long)r;
}

// Seeds the first list: every tile holding a seed, and the dependents reading a seed cell.
template <typename Real>
__global__ void init_lists_kernel(Dev<Real> P, const int *seed_tiles, const unsigned long long *seed_masks, int n) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= n) return;
    StatAcc acc;
    push_dependents(P, 0, 0, seed_tiles[wid], seed_masks[wid], ~0ull, 0ull, 0ull, lane, acc);
    stat_flush(P, acc, lane);
}

// --------------------------------------------------------------------------------------------
// Stencil construction and layout.

template <typename Real>
__global__ void from_double_kernel(const double *in, Real *out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (Real)in[i];
}

template <typename Real>
__global__ void fill_kernel(Real *p, long long n, Real v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

// One thread per cell: Riemann Selling stencil, written tile-major for the solver and optionally
// RowMajor for export. Non positive definite metrics set kErrSelling.
// Global cell x of a batch -> its instance, coordinates and global tile-major index.
struct CellRef {
    int i;
    int x0, x1, x2;
    long long xl;   // cell index within the instance
    long long c;    // global tile-major index
};
__device__ __forceinline__ CellRef cell_ref(const Inst *inst, int ninst, long long x) {
    CellRef r;
    r.i = inst_of_cell(inst, ninst, x);
    const Inst &I = inst[r.i];
    r.xl = x - I.cell0;
    r.x2 = (int)(r.xl % I.g.dims[2]);
    const long long q = r.xl / I.g.dims[2];
    r.x1 = (int)(q % I.g.dims[1]);
    r.x0 = (int)(q / I.g.dims[1]);
    r.c = (I.tile0 + I.g.tile_of(r.x0, r.x1, r.x2)) * 64 + I.g.local_of(r.x0, r.x1, r.x2);
    return r;
}

template <int D, typename Real>
__global__ void riemann_stencil_kernel(Dev<Real> P, const double *metric, int8_t *plain_off, double *plain_w) {
    constexpr int NS = D * (D + 1) / 2, NK = D == 2 ? 3 : 6;
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    double m[6];
    const double *src = metric + (I.metric0 + (I.metric_const ? 0 : R.xl)) * NS;
#pragma unroll
    for (int k = 0; k < NS; ++k) m[k] = src[k];
    int off[6][3];
    double w[6];
    if (!riemann_stencil<D>(m, I.dual != 0, I.h, off, w)) {
        atomicOr(P.status, (unsigned)kErrSelling);
#pragma unroll
        for (int k = 0; k < NK; ++k) { w[k] = 0.0; off[k][0] = off[k][1] = off[k][2] = 0; }
    }
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        P.code[k * P.sstride + R.c] = pack_off(off[k][0], off[k][1], off[k][2]);
        P.weight[k * P.sstride + R.c] = (Real)w[k];
        if (plain_off) {
#pragma unroll
            for (int a = 0; a < 3; ++a) plain_off[(x * NK + k) * 3 + a] = (int8_t)off[k][a];
            plain_w[x * NK + k] = w[k];
        }
    }
}

// Diagonal2 / Diagonal3 (Headers/Specializations/Isotropic.h:61-115): one symmetric difference
// per axis, weight baseWeight * speed_i^2 with baseWeight = 1 / h_i^2 (EulerianStencil.h:79-81), the
// speed vector per cell (or the inverse of the cost vector, component-wise).
template <typename Real>
__global__ void diagonal_stencil_kernel(Dev<Real> P, int D, const double *speed, int8_t *plain_off, double *plain_w) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    const double *src = speed + (I.metric0 + (I.metric_const ? 0 : R.xl)) * D;
    for (int k = 0; k < D; ++k) {
        double sp = src[k];
        if (I.mult_inverse) sp = 1.0 / sp;
        const double base = 1. / (I.h[k] * I.h[k]);
        const double w = base * (sp * sp);
        int o[3] = {0, 0, 0};
        o[k] = 1;
        P.code[k * P.sstride + R.c] = pack_off(o[0], o[1], o[2]);
        P.weight[k * P.sstride + R.c] = (Real)w;
        if (plain_off) {
            for (int a = 0; a < 3; ++a) plain_off[(x * D + k) * 3 + a] = (int8_t)o[a];
            plain_w[x * D + k] = w;
        }
        if (!(w >= 0.0) || !(w < Arith<double>::inf())) atomicOr(P.status, (unsigned)kErrSelling);
    }
}

// One thread per cell: the TTI norm (tile-major) and the distinct offsets of its Selling path as
// the cell's stencil slots (weight 1; unused slots weight 0), for the visibility and dependency
// passes. Invalid norms set kErrSelling; paths with more than NSYM offsets kErrTableOverflow.
template <int NSYM, typename Real>
__global__ void tti_setup_kernel(Dev<Real> P, const double *metric) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    double m[14];
    const double *src = metric + (I.metric0 + (I.metric_const ? 0 : R.xl)) * 14;
#pragma unroll
    for (int k = 0; k < 14; ++k) m[k] = src[k];
    TTICell cell;
    int off[NSYM][3];
    int n = -1;
    if (tti_setup(m, I.h, cell)) n = tti_neighbors(cell, off, NSYM);
    else atomicOr(P.status, (unsigned)kErrSelling);
    if (n < 0 && (P.status[0] & kErrSelling) == 0) atomicOr(P.status, (unsigned)kErrTableOverflow);
    ((TTICell *)P.tti)[R.c] = cell;
#pragma unroll
    for (int k = 0; k < NSYM; ++k) {
        const bool on = k < n && abs(off[k][0]) < 128 && abs(off[k][1]) < 128 && abs(off[k][2]) < 128;
        P.code[k * P.sstride + R.c] = on ? pack_off(off[k][0], off[k][1], off[k][2]) : 0u;
        P.weight[k * P.sstride + R.c] = on ? Real(1) : Real(0);
    }
}

// Per instance, the sum over cells of 1 / sqrt((l0 + l1) / 2) of the TTI norms (a slowness scale:
// the key scale of batched ordering).
template <typename Real>
__global__ void tti_scale_kernel(Dev<Real> P, const double *metric, double *out) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool in = x < P.ncells;
    int i = -1;
    double v = 0.0;
    if (in) {
        i = inst_of_cell(P.inst, P.ninst, x);
        const Inst &I = P.inst[i];
        const double *m = metric + (I.metric0 + (I.metric_const ? 0 : x - I.cell0)) * 14;
        const double s = 0.5 * (m[0] + m[1]);
        v = s > 0 ? 1.0 / sqrt(s) : 0.0;
    }
    const unsigned same = __match_any_sync(0xffffffffu, i);
    const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
    for (int o = 0; o < 32; ++o) {
        const double w = __shfl_sync(0xffffffffu, v, o);
        if (lane == leader && o != lane && ((same >> o) & 1u)) v += w;
    }
    if (in && lane == leader) atomicAdd(out + i, v);
}

// Largest L1 norm of a non-zero-weight offset whose target lies in the domain (MaxStencilWidth,
// HamiltonFastMarching.hxx:36-45 over the reversed offsets of HFM_StencilRecompute.hxx:91-116),
// per instance.
template <typename Real, int NSYM>
__global__ void width_kernel(Dev<Real> P, unsigned *maxw) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool in = x < P.ncells;
    int i = -1;
    unsigned best = 0;
    if (in) {
        const CellRef R = cell_ref(P.inst, P.ninst, x);
        i = R.i;
        const GridGeom &g = P.inst[R.i].g;
#pragma unroll
        for (int k = 0; k < NSYM; ++k) {
            if (P.weight[k * P.sstride + R.c] == Real(0)) continue;
            const unsigned cd = P.code[k * P.sstride + R.c];
            const int o0 = off_c(cd, 0), o1 = off_c(cd, 1), o2 = off_c(cd, 2);
            const unsigned l1 = abs(o0) + abs(o1) + abs(o2);
            for (int s = 1; s >= -1; s -= 2) {
                int n0 = R.x0 + s * o0, n1 = R.x1 + s * o1, n2 = R.x2 + s * o2;
                if (g.wrap(n0, n1, n2) && l1 > best) best = l1;
            }
        }
    }
    // one atomic per (warp, instance) instead of one per cell on a single word
    const unsigned same = __match_any_sync(0xffffffffu, i);
    const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
    for (int o = 0; o < 32; ++o) {
        const unsigned w = __shfl_sync(0xffffffffu, best, o);
        if (lane == leader && ((same >> o) & 1u) && w > best) best = w;
    }
    if (in && lane == leader && best) atomicMax(maxw + i, best);
}

// Speed multiplier to the tile-major layout (shared stencils).
// The compact field (depth 0: one value, 1: per angle, 2: per (x,y), 3: per cell) is broadcast
// here; a cost is inverted in double precision (IEEE division, as the reference's 1./cost).
template <typename Real>
__global__ void mult_layout_kernel(Dev<Real> P, const double *src) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    long long k = 0;
    if (I.mult_depth == 3) {
        k = R.xl;
    } else if (I.nth > 0) {  // ReedsShepp3: (x, y, z) or (theta, phi)
        const int nang = I.nth * I.nph;
        if (I.mult_depth == 2) k = ((long long)R.x0 * I.g.dims[1] + R.x1) * (I.g.dims[2] / nang) + R.x2 / nang;
        else if (I.mult_depth == 1) k = R.x2 % nang;
    } else if (I.mult_depth == 2) {
        k = (long long)R.x0 * I.g.dims[1] + R.x1;
    } else if (I.mult_depth == 1) {
        k = R.x2;
    }
    double m = src[I.mult0 + k];
    if (I.mult_inverse) m = 1.0 / m;
    P.mult[R.c] = (Real)m;
}

// --------------------------------------------------------------------------------------------
// Walls: distance to the nearest wall cell (breadth-first search distance of
// Headers/ExtraAlgorithms/WallObstructionTest.h:48-88, which on a box grid is the L1 distance,
// computed here by separable forward/backward scans per axis), capped at the stencil width.

__global__ void walls_from_f64_kernel(long long n, const double *src, uint8_t *dst) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < n) dst[x] = src[x] != 0.0 ? 1 : 0;
}

__global__ void wall_init_kernel(long long n, const uint8_t *walls, int *d) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < n) d[x] = walls[x] ? 0 : (1 << 29);
}

__global__ void wall_scan_kernel(GridGeom g, int axis, int *d) {
    // d points at the instance's first cell
    const long long nl = g.ncells / g.dims[axis];
    const long long line = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (line >= nl) return;
    long long stride = 1;
    for (int a = 2; a > axis; --a) stride *= g.dims[a];
    const long long inner = stride;
    const long long base = (line / inner) * inner * g.dims[axis] + (line % inner);
    const int n = g.dims[axis];
    const int laps = g.periodic[axis] ? 2 : 1;
    int prev = 1 << 29;
    for (int lap = 0; lap < laps; ++lap)
        for (int i = 0; i < n; ++i) {
            int v = d[base + i * stride];
            if (prev + 1 < v) { v = prev + 1; d[base + i * stride] = v; }
            prev = v;
        }
    prev = 1 << 29;
    for (int lap = 0; lap < laps; ++lap)
        for (int i = n - 1; i >= 0; --i) {
            int v = d[base + i * stride];
            if (prev + 1 < v) { v = prev + 1; d[base + i * stride] = v; }
            prev = v;
        }
}

template <typename Real>
__global__ void wall_cap_kernel(Dev<Real> P, const int *d, const unsigned *cap, int8_t *wd) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const int i = inst_of_cell(P.inst, P.ninst, x);
    wd[x] = d[x] <= (int)cap[i] ? (int8_t)d[x] : (int8_t)127;
}

// Visible(base, v, sum) of WallObstructionTest.h:95-150: a discrete walk from `base` toward `sum`.
__device__ bool wall_visible(const GridGeom &g, const int8_t *wd, int b0, int b1, int b2, int v0, int v1, int v2,
                             int s0, int s1, int s2) {
    int w = wd[g.lin(s0, s1, s2)];
    if (w == 127) return true;
    if (w == 0) return false;
    const int v[3] = {v0, v1, v2};
    int vSign[3] = {0, 0, 0};
    int vSum = 0, vProd = 1, vMax = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (v[i] != 0) {
            vSign[i] = v[i] > 0 ? 1 : -1;
            const int av = abs(v[i]);
            vSum += av;
            vProd *= av;
            vMax = max(vMax, av);
        }
    }
    if (vSum <= w) return true;
    int pos[3] = {b0, b1, b2};
    long long vNext[3], vInc[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        vNext[i] = v[i] == 0 ? 2147483647LL : (long long)(vProd / abs(v[i]));
        vInc[i] = 2 * vNext[i];
    }
    for (int i = 1; i < vMax; ++i) {
        const long long thr = (2LL * i * vProd) / vMax;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (v[j] != 0 && vNext[j] <= thr) {
                vNext[j] += vInc[j];
                --vSum;
                pos[j] += vSign[j];
            }
        }
        int p0 = pos[0], p1 = pos[1], p2 = pos[2];
        g.wrap(p0, p1, p2);
        w = wd[g.lin(p0, p1, p2)];
        if (vSum <= w) return true;
        if (w == 0) return false;
    }
    return true;
}

// Visibility bits of every (cell, neighbour slot): the neighbour y = x + s e may update x iff the
// difference has non-zero weight, y lies in the domain, and Visible(y, -s e, x) holds
// (ConditionalUpdate, HamiltonFastMarching.hxx:136-154). Also marks padding cells dead.
template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void visibility_kernel(Dev<Real> P, const int8_t *wd_all, const uint8_t *cls_enabled) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= P.ntc) return;
    const int T = (int)(c >> 6), l = (int)(c & 63);
    const Inst &I = P.inst[P.tile_inst[T]];
    const GridGeom &g = I.g;
    const int8_t *wd = (wd_all && I.has_walls) ? wd_all + I.cell0 : nullptr;
    int t0, t1, t2, l0, l1, l2;
    g.tile_coords(T - I.tile0, t0, t1, t2);
    g.local_coords(l, l0, l1, l2);
    const int x0 = (t0 << g.tshift[0]) + l0, x1 = (t1 << g.tshift[1]) + l1, x2 = (t2 << g.tshift[2]) + l2;
    if (x0 >= g.dims[0] || x1 >= g.dims[1] || x2 >= g.dims[2]) {
        if (SHARE) P.vis[c] = kShDead;
        else P.code[c] = kDead;
        return;
    }
    unsigned visw = 0;
    const long long cls = share_class<KIND>(I, x2);
#pragma unroll 1
    for (int k = 0; k < ND; ++k) {
        int o[3];
        bool nonzero;
        if (SHARE) {
            const int8_t *oo = P.cls_off + (cls * ND + k) * 3;
            o[0] = oo[0]; o[1] = oo[1]; o[2] = oo[2];
            nonzero = P.cls_w[cls * ND + k] != Real(0);
        } else {
            const unsigned cd = P.code[k * P.sstride + c];
            o[0] = off_c(cd, 0); o[1] = off_c(cd, 1); o[2] = off_c(cd, 2);
            nonzero = P.weight[k * P.sstride + c] != Real(0);
        }
        unsigned bits = 0;
        for (int si = 0; si < (k < NFWD ? 1 : 2); ++si) {
            const int s = si == 0 ? 1 : -1;
            const int slot = k < NFWD ? k : NFWD + 2 * (k - NFWD) + si;
            if (!nonzero) continue;
            if (SHARE && !cls_enabled[cls * (NFWD + 2 * NSYM) + slot]) continue;
            int y0 = x0 + s * o[0], y1 = x1 + s * o[1], y2 = x2 + s * o[2];
            if constexpr (KIND == kKindShareS2) {
                if (!s2_neighbor<Real, ND>(P, I, cls, k, s, x0, x1, x2, y0, y1, y2)) continue;
            } else if (!g.wrap(y0, y1, y2)) {
                continue;
            }
            if (wd && !wall_visible(g, wd, y0, y1, y2, -s * o[0], -s * o[1], -s * o[2], x0, x1, x2)) continue;
            if (SHARE) visw |= 1u << slot;
            else bits |= si == 0 ? kVisPlus : kVisMinus;
        }
        if (!SHARE) P.code[k * P.sstride + c] |= bits;
    }
    if (SHARE) P.vis[c] = visw;
}

template <typename Real, int KIND>
__global__ void seeds_kernel(Dev<Real> P, const long long *idx, const double *val, int n) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    // idx: global cell indices
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long x = idx[i];
    const long long c = cell_ref(P.inst, P.ninst, x).c;
    P.values[x] = (Real)val[i];
    if (SHARE) P.vis[c] |= kShFixed;
    else P.code[c] |= kFixed;
}

// --------------------------------------------------------------------------------------------
// Tile dependency graph. Pass 0 counts, pass 1 writes, for every tile D, the distinct source
// tiles T != D its visible stencil entries read, with the 64-bit mask of the cells read in T.

template <typename Real, int NFWD, int NSYM, int KIND, int kDepCap, int kDepWarps>
__global__ void __launch_bounds__(kDepWarps * 32)
    deps_kernel(Dev<Real> P, int pass, unsigned *cnt, const long long *offs, int *src, int *dst,
                unsigned long long *msk, unsigned long long *dmsk) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    __shared__ int keys[kDepWarps][kDepCap];
    __shared__ unsigned long long masks[kDepWarps][kDepCap];
    __shared__ unsigned long long dmasks[kDepWarps][kDepCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long D = (long long)blockIdx.x * kDepWarps + warp;
    if (D >= P.ntile) return;
    int *K = keys[warp];
    unsigned long long *M = masks[warp];
    unsigned long long *DM = dmasks[warp];
    for (int i = lane; i < kDepCap; i += 32) { K[i] = -1; M[i] = 0ull; DM[i] = 0ull; }
    __syncwarp();
    const Inst &I = P.inst[P.tile_inst[D]];
    const GridGeom &g = I.g;
    int t0, t1, t2;
    g.tile_coords(D - I.tile0, t0, t1, t2);
    bool overflow = false;
    for (int j = 0; j < 2; ++j) {
        const int l = lane + 32 * j;
        int l0, l1, l2;
        g.local_coords(l, l0, l1, l2);
        const int x0 = (t0 << g.tshift[0]) + l0, x1 = (t1 << g.tshift[1]) + l1, x2 = (t2 << g.tshift[2]) + l2;
        const long long c = D * 64 + l;
        if (x0 >= g.dims[0] || x1 >= g.dims[1] || x2 >= g.dims[2]) continue;
        unsigned visw = SHARE ? P.vis[c] : 0u;
        [[maybe_unused]] const long long cls = share_class<KIND>(I, x2);
        for (int k = 0; k < ND; ++k) {
            int o[3];
            unsigned bits;
            if (SHARE) {
                const int8_t *oo = P.cls_off + (cls * ND + k) * 3;
                o[0] = oo[0]; o[1] = oo[1]; o[2] = oo[2];
                bits = k < NFWD ? ((visw >> k) & 1u) : ((visw >> (NFWD + 2 * (k - NFWD))) & 3u);
            } else {
                const unsigned cd = P.code[k * P.sstride + c];
                o[0] = off_c(cd, 0); o[1] = off_c(cd, 1); o[2] = off_c(cd, 2);
                bits = ((cd & kVisPlus) ? 1u : 0u) | ((cd & kVisMinus) ? 2u : 0u);
            }
            for (int si = 0; si < 2; ++si) {
                if (!((bits >> si) & 1u)) continue;
                const int s = si == 0 ? 1 : -1;
                int y0 = x0 + s * o[0], y1 = x1 + s * o[1], y2 = x2 + s * o[2];
                if constexpr (KIND == kKindShareS2) {
                    if (!s2_neighbor<Real, ND>(P, I, cls, k, s, x0, x1, x2, y0, y1, y2)) continue;
                } else {
                    g.wrap(y0, y1, y2);
                }
                const int T = (int)(I.tile0 + g.tile_of(y0, y1, y2));
                if (T == D) continue;
                const int b = g.local_of(y0, y1, y2);
                unsigned h = ((unsigned)T * 2654435761u) & (kDepCap - 1);
                int probes = 0;
                while (true) {
                    const int prev = atomicCAS(&K[h], -1, T);
                    if (prev == -1 || prev == T) {
                        atomicOr(&M[h], 1ull << b);
                        atomicOr(&DM[h], 1ull << l);
                        break;
                    }
                    h = (h + 1) & (kDepCap - 1);
                    if (++probes >= kDepCap) { overflow = true; break; }
                }
            }
        }
    }
    if (overflow) atomicOr(P.status, (unsigned)kErrTableOverflow);
    __syncwarp();
    unsigned total = 0;
    for (int base = 0; base < kDepCap; base += 32) {
        const bool has = K[base + lane] != -1;
        const unsigned bal = __ballot_sync(0xffffffffu, has);
        if (pass == 1 && has) {
            const long long pos = offs[D] + total + __popc(bal & ((1u << lane) - 1u));
            src[pos] = K[base + lane];
            dst[pos] = (int)D;
            msk[pos] = M[base + lane];
            dmsk[pos] = DM[base + lane];
        }
        total += __popc(bal);
    }
    if (pass == 0 && lane == 0) cnt[D] = total;
}

__global__ void dep_count_kernel(long long n, const int *src, unsigned *rcnt) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(rcnt + src[i], 1u);
}

__global__ void dep_scatter_kernel(long long n, const int *src, const int *dst, const unsigned long long *msk,
                                   const unsigned long long *dmsk, const long long *rptr, unsigned *cursor, int *rtile,
                                   unsigned long long *rmask, unsigned long long *rdmask) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int T = src[i];
    const long long pos = rptr[T] + atomicAdd(cursor + T, 1u);
    rtile[pos] = dst[i];
    rmask[pos] = msk[i];
    rdmask[pos] = dmsk[i];
}

// --------------------------------------------------------------------------------------------
// Post-processing.

// Per instance, the sum over cells of the norm scale of the Riemann metric: sqrt(tr(M)/d) for a
// primal metric, sqrt(d/tr(D)) for a dual one (the key scale of batched ordering).
template <int D, typename Real>
__global__ void metric_scale_kernel(Dev<Real> P, const double *metric, double *out) {
    constexpr int NS = D * (D + 1) / 2;
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool in = x < P.ncells;
    int i = -1;
    double v = 0.0;
    if (in) {
        i = inst_of_cell(P.inst, P.ninst, x);
        const Inst &I = P.inst[i];
        const double *m = metric + (I.metric0 + (I.metric_const ? 0 : x - I.cell0)) * NS;
        const double tr = D == 2 ? m[0] + m[2] : m[0] + m[2] + m[5];
        v = I.dual ? sqrt(D / tr) : sqrt(tr / D);
        if (!(v < 1e300)) v = 0.0;
    }
    // segmented warp sum: the first lane of each instance adds the others' terms
    const unsigned same = __match_any_sync(0xffffffffu, i);
    const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
    for (int o = 0; o < 32; ++o) {
        const double w = __shfl_sync(0xffffffffu, v, o);
        if (lane == leader && o != lane && ((same >> o) & 1u)) v += w;
    }
    if (in && lane == leader) atomicAdd(out + i, v);
}

template <typename Real>
// Reached cells per instance (the reference's nAccepted).
__global__ void count_finite_kernel(Dev<Real> P, unsigned long long *out) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool in = x < P.ncells;
    const int i = in ? inst_of_cell(P.inst, P.ninst, x) : -1;
    const bool fin = in && P.values[x] < Arith<Real>::inf();
    const unsigned same = __match_any_sync(0xffffffffu, i);
    const unsigned cnt = __popc(__ballot_sync(0xffffffffu, fin) & same);
    if (in && cnt && (threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(out + i, (unsigned long long)cnt);
}

// activeNeighs bitsets in the reference layout (EulerianStencil.h:35-49): forward difference k
// at bit k, symmetric difference j at bits nfwd+2j (+e) and nfwd+2j+1 (-e). A used forward
// difference also marks the other forward differences with the same offset, as the reference's
// update adds every difference matching the accepted offset (EulerianStencil.hxx:114-123).
template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void active_kernel(Dev<Real> P, unsigned long long *active) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    if constexpr (KIND == kKindTTI) {
        // the semi-Lagrangian scheme records the extremum t instead of a bitset (TTI.h:45-60):
        // t at an interior extremum, -t at an interval endpoint, +inf where no update was made;
        // the bits of that double are stored
        const CellRef R = cell_ref(P.inst, P.ninst, x);
        const Inst &I = P.inst[R.i];
        bool fixed, dead;
        cell_flags<Real, KIND>(P, R.c, fixed, dead);
        double code = Arith<double>::inf();
        if (!fixed && !dead && (double)P.values[x] < Arith<double>::inf()) {
            double ta = Arith<double>::inf();
            bool inner = false;
            solve_cell_tti<Real>(P, I, R.c, R.x0, R.x1, R.x2, 0, 0, 0, nullptr, &ta, &inner);
            code = inner ? ta : -ta;
        }
        active[x] = (unsigned long long)__double_as_longlong(code);
        return;
    }
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    const int x0 = R.x0, x1 = R.x1, x2 = R.x2;
    const long long c = R.c;
    const long long cls = share_class<KIND>(I, x2);
    bool fixed, dead;
    cell_flags<Real, KIND>(P, c, fixed, dead);
    unsigned long long bits = 0;
    if (!fixed && !dead) {
        unsigned used = 0, side = 0;
        solve_cell<Real, NFWD, NSYM, KIND>(P, I, c, x0, x1, x2, 0, 0, 0, nullptr, &used, &side);
        for (int k = 0; k < ND; ++k) {
            if (!((used >> k) & 1u)) continue;
            if (k < NFWD) {
                bits |= 1ull << k;
                if (SHARE) {
                    const int8_t *ok = P.cls_off + (cls * ND + k) * 3;
                    for (int k2 = 0; k2 < NFWD; ++k2) {
                        const int8_t *o2 = P.cls_off + (cls * ND + k2) * 3;
                        if (o2[0] == ok[0] && o2[1] == ok[1] && o2[2] == ok[2]) bits |= 1ull << k2;
                    }
                }
            } else {
                bits |= 1ull << (NFWD + 2 * (k - NFWD) + ((side >> (k - NFWD)) & 1u));
            }
        }
        // the group of a two-group stencil, in the bit after the differences (SetIMax)
        if constexpr (KIND == kKindShare2) bits |= (unsigned long long)((used >> ND) & 1u) << ND;
    }
    active[x] = bits;
}

template <typename Real>
__global__ void to_double_kernel(const Real *in, double *out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

struct EventTimer {
    cudaEvent_t a, b;
    EventTimer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~EventTimer() { cudaEventDestroy(a); cudaEventDestroy(b); }
    void start(cudaStream_t s) { cudaEventRecord(a, s); }
    float stop(cudaStream_t s) {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

void check_status(const DeviceBuffer<unsigned> &status, const char *phase) {
    unsigned st = 0;
    status.download(&st, 1);
    HFM_CUDA(cudaDeviceSynchronize());
    if (st & kErrSelling)
        throw Error(HFM_ERR_VALUE, "ObtuseSuperbase error : input must be positive definite (metric rejected by Selling)");
    if (st & kErrTableOverflow) throw Error(HFM_ERR_UNSUPPORTED, "stencil too wide for the tile dependency table");
    if (st & kErrBarrierTimeout)
        throw Error(HFM_ERR_NOT_CONVERGED, std::string(phase) + ": a grid barrier wait exceeded its limit");
    if (st & kErrRoundCap) throw Error(HFM_ERR_NOT_CONVERGED, std::string(phase) + ": round cap reached before convergence");
    if (st & kErrIndexRange) throw Error(HFM_ERR_CUDA, std::string(phase) + ": a flow index left its array");
}

// --------------------------------------------------------------------------------------------
// Reverse first variation (Headers/ExtraAlgorithms/FirstVariation.h:198-251, 341-385).
//
// flow_kernel stores, for every reached cell x, the upwind differences of its final update in
// stencil order with w_i = Weight_i * max(0, u(x) - u(y_i)), normalised by their sum, and
// var(x) = (sum_i w_i (u - u_i)) / sum_i w_i (times the speed multiplier for shared stencils):
// the same products and sums, in the same order, as ValueVariation. adjoint_kernel then sweeps
// the upwind graph in reverse topological order: a cell is ready once every downwind cell that
// reads it has been processed (in-degree counters), which is the order of the reference's
// decreasing-value traversal restricted to the actual dependencies. A ready cell gathers
// lambda = (its inspection weight) + sum of w * lambda(downwind) over a reverse adjacency sorted
// by decreasing downwind value, the order in which the reference's traversal adds them
// (FirstVariation.h:341-385): the result does not depend on the schedule.

template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void flow_kernel(Dev<Real> P, int *fidx, double *fw, double *var, uint8_t *nflow, int *indeg) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    // the adjoint runs on a batch of one instance
    constexpr int ND = NFWD + NSYM;
    using A = Arith<double>;
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const Inst &I = P.inst[0];
    const GridGeom &g = I.g;
    const long long N = g.ncells;
    if (x >= N) return;
    if constexpr (KIND == kKindShareS2) {
        // ReedsShepp3 first variations are refused by the host before any launch
        if (x == 0) atomicOr(P.status, (unsigned)kErrIndexRange);
        return;
    }
    const int x2 = (int)(x % g.dims[2]);
    const long long r = x / g.dims[2];
    const int x1 = (int)(r % g.dims[1]);
    const int x0 = (int)(r / g.dims[1]);
    const long long c = (I.tile0 + g.tile_of(x0, x1, x2)) * 64 + g.local_of(x0, x1, x2);
    bool fixed, dead;
    cell_flags<Real, KIND>(P, c, fixed, dead);
    const double u = (double)P.values[x];
    nflow[x] = 0;
    var[x * (P.var_dim > 1 ? P.var_dim : 1)] = 0.0;
    if constexpr (KIND == kKindTTI) {
        // semi-Lagrangian ValueVariation (FirstVariation.h:169-196): the update recomputed at the
        // extremum t (TTI.hpp:278-389), flow weights (sol - v) w(t), and the local derivative
        // value - sum of the normalised weights times the neighbour values. A seed has no flow
        // and the derivative is its value (HamiltonFastMarching.hxx:194-195).
        if (fixed) var[x] = u;
        if (fixed || dead || !(u < Arith<double>::inf())) return;
        double ta = 0.0;
        bool inner = false;
        solve_cell_tti<Real>(P, I, c, x0, x1, x2, 0, 0, 0, nullptr, &ta, &inner);
        if (!(ta < Arith<double>::inf())) return;
        const TTICell &tc = P.tti[c];
        TTIPath path;
        if (!tti_path_at(tc, ta, path)) return;
        // candidates (value, weights at both ends, cell), sorted by value: the sort moves whole
        // records, so no array is read through an index array
        struct Cand {
            double v, wa, wb;
            int cell;
        } cand[6];
        for (int r = 0; r < 6; ++r) {
            double vs[2] = {Arith<double>::inf(), Arith<double>::inf()};
            int cs[2] = {-1, -1};
            for (int si = 0; si < 2; ++si) {
                const int s = si ? -1 : 1;
                const int y0 = x0 + s * path.off[r][0], y1 = x1 + s * path.off[r][1], y2 = x2 + s * path.off[r][2];
                if ((unsigned)y0 >= (unsigned)g.dims[0] || (unsigned)y1 >= (unsigned)g.dims[1] ||
                    (unsigned)y2 >= (unsigned)g.dims[2])
                    continue;
                cs[si] = (int)g.lin(y0, y1, y2);
                vs[si] = (double)P.values[cs[si]];
            }
            const bool plus = vs[0] < vs[1];  // the +e neighbour only when strictly smaller
            Cand cd{plus ? vs[0] : vs[1], path.w0[r], path.w1[r], plus ? cs[0] : cs[1]};
            int k = r - 1;
            while (k >= 0 && cand[k].v > cd.v) {
                cand[k + 1] = cand[k];
                --k;
            }
            cand[k + 1] = cd;
        }
        const double vmin = cand[0].v;
        if (!(vmin < Arith<double>::inf())) return;
        double a = 0, b = 0, cc = -tti_multiplier(tc, dconst(ta)).v, sol = Arith<double>::inf();
        int r = 0;
        for (; r < 6; ++r) {
            const double v = cand[r].v - vmin;
            if (v >= sol) break;
            const double w = (1 - ta) * cand[r].wa + ta * cand[r].wb;
            a += w;
            b += w * v;
            cc += (w * v) * v;
            if (a <= 100 * fabs(cc) * 2.220446049250313e-16) continue;
            sol = (b + sqrt(b * b - a * cc)) / a;
        }
        double wd[6], ws = 0.0;
        const int n = r;
        for (int q = 0; q < n; ++q) {
            const double v = cand[q].v - vmin;
            const double w0 = (1 - ta) * cand[q].wa + ta * cand[q].wb;
            const double d = (sol - v) * w0;
            wd[q] = d > 0 ? d : 0.0;
            ws += wd[q];
        }
        double vd = sol + vmin;
        for (int j = 0; j < n; ++j) {
            wd[j] = wd[j] / ws;
            vd -= wd[j] * (double)P.values[cand[j].cell];
        }
        var[x] = vd;
        nflow[x] = (uint8_t)n;
        for (int j = 0; j < n; ++j) {
            fidx[j * N + x] = cand[j].cell;
            fw[j * N + x] = wd[j];
            atomicAdd(indeg + cand[j].cell, 1);
        }
        return;
    }
    const int vdim = P.var_dim > 1 ? P.var_dim : 1;
    for (int i = 1; i < vdim; ++i) var[x * vdim + i] = 0.0;
    if (fixed || dead || !(u < Arith<double>::inf())) return;
    unsigned used = 0, side = 0;
    solve_cell<Real, NFWD, NSYM, KIND>(P, I, c, x0, x1, x2, 0, 0, 0, nullptr, &used, &side);
    double m = 1.0;
    if (SHARE) m = (double)P.mult[c];
    double ws = 0.0, v = 0.0;
    double vv[3] = {0.0, 0.0, 0.0};  // per axis (Diagonal models: difference k is along axis k)
    int n = 0;
    int ys[2 * ND > 32 ? 32 : 2 * ND];
    double ww[2 * ND > 32 ? 32 : 2 * ND];
    for (int k = 0; k < ND; ++k) {
        int o0, o1, o2;
        double wb;
        if (SHARE) {
            const int8_t *o = P.cls_off + ((I.cls0 + x2) * ND + k) * 3;
            o0 = o[0]; o1 = o[1]; o2 = o[2];
            wb = A::mul((double)P.cls_w[(I.cls0 + x2) * ND + k], A::mul(m, m));
        } else {
            const unsigned cd = P.code[k * P.sstride + c];
            o0 = off_c(cd, 0); o1 = off_c(cd, 1); o2 = off_c(cd, 2);
            wb = (double)P.weight[k * P.sstride + c];
        }
        // active bits of this difference (see active_kernel)
        unsigned act = 0;  // bit0: +e, bit1: -e
        if (k < NFWD) {
            if ((used >> k) & 1u) act = 1;
            else if (SHARE) {
                for (int k2 = 0; k2 < NFWD; ++k2) {
                    if (!((used >> k2) & 1u)) continue;
                    const int8_t *o2p = P.cls_off + ((I.cls0 + x2) * ND + k2) * 3;
                    if (o2p[0] == o0 && o2p[1] == o1 && o2p[2] == o2) { act = 1; break; }
                }
            }
        } else if ((used >> k) & 1u) {
            act = ((side >> (k - NFWD)) & 1u) ? 2u : 1u;
        }
        // a two-group stencil recomputes with the named group only (HopfLaxRecompute,
        // EulerianStencil.hxx:157-200)
        if (KIND == kKindShare2 && (k < ND / 2 ? 0u : 1u) != ((used >> ND) & 1u)) act = 0;
        for (int si = 0; si < 2; ++si) {
            if (!((act >> si) & 1u)) continue;
            const int s = si ? -1 : 1;
            int y0 = x0 + s * o0, y1 = x1 + s * o1, y2 = x2 + s * o2;
            if (!g.wrap(y0, y1, y2)) {  // an active neighbour is inside the grid
                atomicOr(P.status, (unsigned)kErrIndexRange);
                continue;
            }
            const long long y = g.lin(y0, y1, y2);
            const double d = A::sub(u, (double)P.values[y]);
            const double vd = 0.0 < d ? d : 0.0;
            const double w = A::mul(wb, vd);
            ws = A::add(ws, w);
            v = A::add(v, A::mul(w, vd));
            if (vdim > 1 && k < 3) vv[k] = A::add(vv[k], A::mul(w, vd));
            if (n < 32) { ys[n] = (int)y; ww[n] = w; ++n; }
        }
    }
    if (ws != 0.0) {
        const double inv = A::div(1.0, ws);
        for (int j = 0; j < n; ++j) ww[j] = A::mul(ww[j], inv);
        v = SHARE ? A::mul(inv, A::mul(m, v)) : A::mul(inv, v);
        if (vdim > 1) {  // inv * (speed_i * var_i) (FirstVariation.h:243-247 with the vector multiplier)
            const double *sp = P.diag_src + (I.metric0 + (I.metric_const ? 0 : x)) * vdim;
            for (int i = 0; i < vdim && i < 3; ++i) {
                const double si = P.diag_inverse ? A::div(1.0, sp[i]) : sp[i];
                vv[i] = A::mul(inv, A::mul(si, vv[i]));
            }
        }
    }
    if (vdim > 1) {
        for (int i = 0; i < vdim && i < 3; ++i) var[x * vdim + i] = vv[i];
    } else {
        var[x] = v;
    }
    nflow[x] = (uint8_t)n;
    for (int j = 0; j < n; ++j) {
        fidx[j * N + x] = ys[j];
        fw[j * N + x] = ww[j];
        atomicAdd(indeg + ys[j], 1);
    }
}

#include "geodesic.cuh"
#include "stopping.cuh"

struct AdjDev {
    long long N;
    const int *fidx;
    const double *fw;
    const double *var;
    const uint8_t *nflow;
    const long long *rptr;   // reverse adjacency: downwind cells reading y, sorted
    const int *rx;
    const double *rw;
    double *lam;             // lambda of the processed cells
    int *indeg;
    double *acc;             // inspection weights
    double *sens;
    int var_dim;             // components of var / sens per cell
    int *list[3];            // list[0]: the ready queue (the three point at it)
    unsigned *count[3];      // [0] cells queued, [1] slots claimed
    long long *seed_idx;
    double *seed_w;
    unsigned *seed_count;
    unsigned seed_cap;
    unsigned *bar_count;
    unsigned *bar_gen;
    unsigned *status;
    unsigned long long *processed;  // cells processed (diagnostics)
};

__global__ void adjoint_roots_kernel(AdjDev A) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool want = x < A.N && A.indeg[x] == 0;
    const unsigned bal = __ballot_sync(0xffffffffu, want);
    if (!bal) return;
    unsigned base = 0;
    if (lane == __ffs(bal) - 1) base = atomicAdd(A.count[0], (unsigned)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, __ffs(bal) - 1);
    if (want) A.list[0][base + __popc(bal & ((1u << lane) - 1u))] = (int)x;
}

// The sweeps run over a ready queue instead of rounds: list[0] holds every cell once, in the order
// the cells become ready (count[0] of them so far, the slots beyond still -1); warps claim 32 slots
// at a time (count[1]) and each lane processes its cell as soon as its slot is filled, so a cell is
// processed one queue hop after its last dependency and no grid barrier separates fronts. Every
// cell is pushed exactly once and the graph is acyclic, so a claimed slot is always filled by a
// cell whose own dependencies other warps are processing (all blocks are resident: cooperative
// launch). A warp that sees no progress for kQueuePolls polls sets kErrBarrierTimeout and leaves.
constexpr unsigned long long kQueuePolls = 1ull << 24;

__device__ __forceinline__ void queue_push(int *q, unsigned *tail, bool want, int v, int lane) {
    const unsigned bal = __ballot_sync(0xffffffffu, want);
    if (!bal) return;
    unsigned base = 0;
    if (lane == __ffs(bal) - 1) base = atomicAdd(tail, (unsigned)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, __ffs(bal) - 1);
    if (want) ((volatile int *)q)[base + __popc(bal & ((1u << lane) - 1u))] = v;
}

__global__ void adjoint_kernel(AdjDev A) {
    const int lane = threadIdx.x & 31;
    int *q = A.list[0];
    unsigned long long processed = 0;
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(A.count[1], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((long long)base >= A.N) break;
        const long long i = (long long)base + lane;
        bool pending = i < A.N;
        unsigned long long idle = 0;
        while (__any_sync(0xffffffffu, pending)) {
            int x = -1;
            if (pending) x = ((volatile int *)q)[i];
            if (x >= A.N) {  // a queued cell is a cell of the grid
                atomicOr(A.status, (unsigned)kErrIndexRange);
                x = -1;
                pending = false;
            }
            const bool ready = pending && x >= 0;
            if (!__any_sync(0xffffffffu, ready)) {
                if (!__any_sync(0xffffffffu, pending)) break;
                if (++idle > kQueuePolls) {
                    if (lane == 0) atomicOr(A.status, (unsigned)kErrBarrierTimeout);
                    return;
                }
                __nanosleep(32);
                continue;
            }
            idle = 0;
            __threadfence();  // the downstream values written before this cell was queued
            int nf = 0;
            if (ready) {
                double lam = __ldcg(A.acc + x);
                for (long long k = A.rptr[x], e = A.rptr[x + 1]; k < e; ++k)
                    lam = __dadd_rn(lam, __dmul_rn(A.rw[k], __ldcg(A.lam + A.rx[k])));
                __stcg(A.lam + x, lam);
                nf = A.nflow[x];
                if (lam != 0.0) {
                    for (int v = 0; v < A.var_dim; ++v)
                        A.sens[(long long)x * A.var_dim + v] = lam * A.var[(long long)x * A.var_dim + v];
                    if (nf == 0) {
                        const unsigned si = atomicAdd(A.seed_count, 1u);
                        if (si < A.seed_cap) { A.seed_idx[si] = x; A.seed_w[si] = lam; }
                    }
                }
                __threadfence();
                ++processed;
            }
            for (int j = 0; __any_sync(0xffffffffu, j < nf); ++j) {
                bool want = false;
                int y = 0;
                if (j < nf) {
                    y = A.fidx[j * A.N + x];
                    if ((unsigned)y < (unsigned)A.N) want = atomicSub(A.indeg + y, 1) == 1;
                    else atomicOr(A.status, (unsigned)kErrIndexRange);
                }
                queue_push(q, A.count[0], want, y, lane);
            }
            if (ready) pending = false;
        }
    }
    if (processed) atomicAdd(A.processed, processed);
}

// Reverse adjacency of the upwind graph: for every cell y, the (downwind cell, weight) pairs of
// the cells whose final update read y.
__global__ void flow_scatter_kernel(long long N, const int *fidx, const double *fw, const uint8_t *nflow,
                                    const long long *rptr, unsigned *cursor, int *rx, double *rw) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= N) return;
    const int nf = nflow[x];
    for (int j = 0; j < nf; ++j) {
        const int y = fidx[j * N + x];
        const long long pos = rptr[y] + atomicAdd(cursor + y, 1u);
        rx[pos] = (int)x;
        rw[pos] = fw[j * N + x];
    }
}

// Sorts each cell's reverse adjacency by decreasing downwind value, then decreasing index, then
// weight bits (a fixed order whatever the scatter order was).
template <typename Real>
__global__ void flow_sort_kernel(long long N, const long long *rptr, int *rx, double *rw, const Real *values) {
    const long long y = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (y >= N) return;
    const long long b = rptr[y], e = rptr[y + 1];
    auto before = [&](int xa, double wa, int xb, double wb) {
        const Real va = values[xa], vb = values[xb];
        if (va != vb) return va > vb;
        if (xa != xb) return xa > xb;
        return __double_as_longlong(wa) > __double_as_longlong(wb);
    };
    for (long long i = b + 1; i < e; ++i) {
        const int xi = rx[i];
        const double wi = rw[i];
        long long k = i - 1;
        while (k >= b && before(xi, wi, rx[k], rw[k])) {
            rx[k + 1] = rx[k];
            rw[k + 1] = rw[k];
            --k;
        }
        rx[k + 1] = xi;
        rw[k + 1] = wi;
    }
}

// Upwind flow graph of a solved single instance: per cell its normalised flow (fidx, fw, nflow)
// and local derivative (var), and the reverse adjacency (rptr, rx, rw: the downwind cells that
// read each cell, sorted) with the reverse degrees (indeg0).
struct FlowGraph {
    long long N = 0, ne = 0;
    DeviceBuffer<int> fidx, indeg0, rx;
    DeviceBuffer<double> fw, var, rw;
    DeviceBuffer<uint8_t> nflow;
    DeviceBuffer<long long> rptr;
};

template <typename Real, int NFWD, int NSYM, int KIND>
void build_flow_graph(const Dev<Real> &P, long long N, FlowGraph &G, cudaStream_t s) {
    constexpr int ND = NFWD + NSYM;
    constexpr int NF = 2 * ND > 32 ? 32 : 2 * ND;
    if (N >= (1ll << 31)) throw Error(HFM_ERR_UNSUPPORTED, "grid too large for the first variation");
    G.N = N;
    G.fidx.alloc((size_t)NF * N);
    G.indeg0.alloc(N);
    G.fw.alloc((size_t)NF * N);
    G.var.alloc((size_t)N * (P.var_dim > 1 ? P.var_dim : 1));
    G.nflow.alloc(N);
    G.indeg0.zero(s);
    launch(flow_kernel<Real, NFWD, NSYM, KIND>, nblocks(N, 128), 128, 0, s, P, G.fidx.get(), G.fw.get(), G.var.get(),
           G.nflow.get(), G.indeg0.get());
    HFM_CUDA(cudaGetLastError());
    // reverse adjacency (CSR over y, offsets scanned on the host)
    G.rptr.alloc(N + 1);
    std::vector<int> hdeg(N);
    G.indeg0.download(hdeg.data(), N, s);
    HFM_CUDA(cudaStreamSynchronize(s));
    std::vector<long long> hrptr(N + 1);
    long long ne = 0;
    for (long long y = 0; y < N; ++y) { hrptr[y] = ne; ne += hdeg[y]; }
    hrptr[N] = ne;
    G.ne = ne;
    G.rptr.upload(hrptr, s);
    G.rx.alloc(std::max(1ll, ne));
    G.rw.alloc(std::max(1ll, ne));
    DeviceBuffer<unsigned> cursor(N);
    cursor.zero(s);
    launch(flow_scatter_kernel, nblocks(N, 256), 256, 0, s, N, G.fidx.get(), G.fw.get(), G.nflow.get(), G.rptr.get(),
           cursor.get(), G.rx.get(), G.rw.get());
    launch(flow_sort_kernel<Real>, nblocks(N, 256), 256, 0, s, N, G.rptr.get(), G.rx.get(), G.rw.get(), P.values);
    HFM_CUDA(cudaGetLastError());
    HFM_CUDA(cudaStreamSynchronize(s));
}

template <typename Real, int NFWD, int NSYM, int KIND>
void run_adjoint(const Dev<Real> &P, long long N, const EulerProblem &p, EulerResult &res,
                 DeviceBuffer<unsigned> &status, cudaStream_t s, FlowGraph *graph = nullptr) {
    FlowGraph own;
    if (!graph) {
        build_flow_graph<Real, NFWD, NSYM, KIND>(P, N, own, s);
        graph = &own;
    }
    FlowGraph &G = *graph;
    DeviceBuffer<int> indeg(N);
    const int vdim = P.var_dim > 1 ? P.var_dim : 1;
    DeviceBuffer<double> acc(N), sens((size_t)N * vdim), lam(N);
    DeviceBuffer<int> &fidx = G.fidx, &indeg0 = G.indeg0, &rx = G.rx;
    DeviceBuffer<double> &fw = G.fw, &var = G.var, &rw = G.rw;
    DeviceBuffer<uint8_t> &nflow = G.nflow;
    DeviceBuffer<long long> &rptr = G.rptr;
    DeviceBuffer<int> queue(N);
    DeviceBuffer<unsigned> counters(8);
    const unsigned seed_cap = 1u << 20;
    DeviceBuffer<long long> seed_idx(seed_cap);
    DeviceBuffer<double> seed_w(seed_cap);
    DeviceBuffer<unsigned long long> rounds(1);
    AdjDev A{};
    A.N = N;
    A.fidx = fidx.get();
    A.fw = fw.get();
    A.var = var.get();
    A.nflow = nflow.get();
    A.rptr = rptr.get();
    A.rx = rx.get();
    A.rw = rw.get();
    A.lam = lam.get();
    A.indeg = indeg.get();
    A.acc = acc.get();
    A.sens = sens.get();
    A.var_dim = vdim;
    for (int i = 0; i < 3; ++i) { A.list[i] = queue.get(); A.count[i] = counters.get() + i; }
    A.seed_count = counters.get() + 3;
    A.bar_count = counters.get() + 4;
    A.bar_gen = counters.get() + 5;
    A.seed_idx = seed_idx.get();
    A.seed_w = seed_w.get();
    A.seed_cap = seed_cap;
    A.status = status.get();
    A.processed = rounds.get();
    int dev = 0, nsm = 0, per_sm = 0;
    HFM_CUDA(cudaGetDevice(&dev));
    HFM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    HFM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel, 256, 0));
    if (per_sm < 1) throw Error(HFM_ERR_CUDA, "adjoint kernel cannot be resident");
    const double *hvals = p.h_values_out ? p.h_values_out : res.values.data();
    for (size_t gi = 0; gi < p.adjoint_index.size(); ++gi) {
        HFM_CUDA(cudaMemcpyAsync(indeg.get(), indeg0.get(), N * sizeof(int), cudaMemcpyDeviceToDevice, s));
        acc.zero(s);
        sens.zero(s);
        counters.zero(s);
        rounds.zero(s);
        HFM_CUDA(cudaMemsetAsync(queue.get(), 0xff, N * sizeof(int), s));  // empty slots read -1
        // std::map::insert keeps the first weight of a repeated point
        std::vector<double> hacc_w;
        std::vector<long long> hacc_i;
        for (size_t k = 0; k < p.adjoint_index[gi].size(); ++k) {
            const long long x = p.adjoint_index[gi][k];
            if (std::find(hacc_i.begin(), hacc_i.end(), x) != hacc_i.end()) continue;
            hacc_i.push_back(x);
            hacc_w.push_back(p.adjoint_weight[gi][k]);
        }
        for (size_t k = 0; k < hacc_i.size(); ++k)
            HFM_CUDA(cudaMemcpyAsync(acc.get() + hacc_i[k], &hacc_w[k], sizeof(double), cudaMemcpyHostToDevice, s));
        HFM_CUDA(cudaStreamSynchronize(s));
        launch(adjoint_roots_kernel, nblocks(N, 256), 256, 0, s, A);
        void *args[] = {&A};
        count_launch();
        {
            std::lock_guard<std::mutex> coop(cooperative_mutex());
            HFM_CUDA(cudaLaunchCooperativeKernel((void *)adjoint_kernel,
                                                 dim3(std::max(1, nsm * per_sm / std::max(1, solver_share()))),
                                                 dim3(256), args, 0, s));
            check_status(status, "adjoint");
        }
        AdjointResult ar;
        ar.sensitivity.resize((size_t)N * vdim);
        sens.download(ar.sensitivity.data(), (size_t)N * vdim, s);
        unsigned hc[8];
        counters.download(hc, 8, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        const unsigned nseed = std::min(hc[3], seed_cap);
        std::vector<long long> si(nseed);
        std::vector<double> sw(nseed);
        seed_idx.download(si.data(), nseed, s);
        seed_w.download(sw.data(), nseed, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        std::vector<size_t> order(nseed);
        for (size_t k = 0; k < nseed; ++k) order[k] = k;
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            const double va = hvals[si[a]], vb = hvals[si[b]];
            return va != vb ? va > vb : si[a] > si[b];
        });
        for (size_t k : order) { ar.seed_index.push_back(si[k]); ar.seed_weight.push_back(sw[k]); }
        res.adjoints.push_back(std::move(ar));
    }
}

// Forward first variation (FirstVariation.h:389-429): cells in upwind-to-downwind order, each
// pulling result(x, k) = result(x, k) + var(x) cost(x, k) + sum_j w_j result(y_j, k) over its
// normalised flow, in the flow's order (so the sums are those of the reference, whatever the
// schedule). A cell is ready once the cells it reads are done: a counter of pending upwind cells,
// decremented through the reverse adjacency; rounds of ready lists in one cooperative launch.
struct FwdDev {
    long long N;
    int nvar;
    const int *fidx;
    const double *fw;
    const double *var;
    const uint8_t *nflow;
    const long long *rptr;
    const int *rx;
    const double *cost;  // [N][nvar][var_dim] or null
    int var_dim;         // components of var per cell
    double *res;         // [N][nvar]: seed value variations on entry
    int *cnt;            // upwind cells not yet done
    int *list[3];
    unsigned *count[3];
    unsigned *bar_count;
    unsigned *bar_gen;
    unsigned *status;
    unsigned long long *processed;  // cells processed (diagnostics)
};

__global__ void forward_roots_kernel(FwdDev F) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool want = x < F.N && F.cnt[x] == 0;
    const unsigned bal = __ballot_sync(0xffffffffu, want);
    if (!bal) return;
    unsigned base = 0;
    if (lane == __ffs(bal) - 1) base = atomicAdd(F.count[0], (unsigned)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, __ffs(bal) - 1);
    if (want) F.list[0][base + __popc(bal & ((1u << lane) - 1u))] = (int)x;
}

__global__ void forward_kernel(FwdDev F) {
    const int lane = threadIdx.x & 31;
    int *q = F.list[0];
    unsigned long long processed = 0;
    while (true) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(F.count[1], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((long long)base >= F.N) break;
        const long long i = (long long)base + lane;
        bool pending = i < F.N;
        unsigned long long idle = 0;
        while (__any_sync(0xffffffffu, pending)) {
            int x = -1;
            if (pending) x = ((volatile int *)q)[i];
            if (x >= F.N) {  // a queued cell is a cell of the grid
                atomicOr(F.status, (unsigned)kErrIndexRange);
                x = -1;
                pending = false;
            }
            const bool ready = pending && x >= 0;
            if (!__any_sync(0xffffffffu, ready)) {
                if (!__any_sync(0xffffffffu, pending)) break;
                if (++idle > kQueuePolls) {
                    if (lane == 0) atomicOr(F.status, (unsigned)kErrBarrierTimeout);
                    return;
                }
                __nanosleep(32);
                continue;
            }
            idle = 0;
            __threadfence();  // the upwind results written before this cell was queued
            long long e = 0, ee = 0;
            if (ready) {
                const int nf = F.nflow[x];
                const int vd = F.var_dim;
                for (int k = 0; k < F.nvar; ++k) {
                    double acc = __ldcg(F.res + (long long)x * F.nvar + k);
                    // the local derivative paired with the cost variation (DiffHelper::Scal)
                    double sc = 0.0;
                    for (int v = 0; v < vd; ++v)
                        sc = __dadd_rn(sc, __dmul_rn(F.var[(long long)x * vd + v],
                                                     F.cost ? F.cost[((long long)x * F.nvar + k) * vd + v] : 0.0));
                    acc = __dadd_rn(acc, sc);
                    for (int j = 0; j < nf; ++j) {
                        const long long y = F.fidx[j * F.N + x];
                        acc = __dadd_rn(acc, __dmul_rn(F.fw[j * F.N + x], __ldcg(F.res + y * F.nvar + k)));
                    }
                    __stcg(F.res + (long long)x * F.nvar + k, acc);
                }
                __threadfence();
                e = F.rptr[x];
                ee = F.rptr[x + 1];
                ++processed;
            }
            // downwind cells whose last pending input this was join the queue
            while (__any_sync(0xffffffffu, e < ee)) {
                bool want = false;
                int z = 0;
                if (e < ee) {
                    z = F.rx[e];
                    if ((unsigned)z < (unsigned)F.N) want = atomicSub(F.cnt + z, 1) == 1;
                    else atomicOr(F.status, (unsigned)kErrIndexRange);
                    ++e;
                }
                queue_push(q, F.count[0], want, z, lane);
            }
            if (ready) pending = false;
        }
    }
    if (processed) atomicAdd(F.processed, processed);
}

__global__ void nflow_to_count_kernel(long long N, const uint8_t *nflow, int *cnt) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < N) cnt[x] = nflow[x];
}

template <typename Real, int NFWD, int NSYM, int KIND>
void run_forward(const Dev<Real> &P, long long N, const EulerProblem &p, EulerResult &res,
                 DeviceBuffer<unsigned> &status, cudaStream_t s, FlowGraph &G) {
    const int nvar = p.fwd_nvar;
    DeviceBuffer<double> cost, out((size_t)N * nvar);
    out.zero(s);
    for (size_t i = 0; i < p.fwd_seed_cell.size(); ++i)
        HFM_CUDA(cudaMemcpyAsync(out.get() + p.fwd_seed_cell[i] * nvar, p.fwd_seed_value.data() + i * nvar,
                                 nvar * sizeof(double), cudaMemcpyHostToDevice, s));
    const int vdim = P.var_dim > 1 ? P.var_dim : 1;
    if (!p.fwd_cost.empty()) {
        cost.alloc((size_t)N * nvar * vdim);
        cost.upload(p.fwd_cost.data(), (size_t)N * nvar * vdim, s);
    }
    DeviceBuffer<int> cnt(N), queue(N);
    DeviceBuffer<unsigned> counters(8);
    DeviceBuffer<unsigned long long> rounds(1);
    counters.zero(s);
    rounds.zero(s);
    HFM_CUDA(cudaMemsetAsync(queue.get(), 0xff, N * sizeof(int), s));  // empty slots read -1
    launch(nflow_to_count_kernel, nblocks(N, 256), 256, 0, s, N, G.nflow.get(), cnt.get());
    FwdDev F{};
    F.N = N;
    F.nvar = nvar;
    F.fidx = G.fidx.get();
    F.fw = G.fw.get();
    F.var = G.var.get();
    F.nflow = G.nflow.get();
    F.rptr = G.rptr.get();
    F.rx = G.rx.get();
    F.cost = p.fwd_cost.empty() ? nullptr : cost.get();
    F.var_dim = vdim;
    F.res = out.get();
    F.cnt = cnt.get();
    for (int i = 0; i < 3; ++i) { F.list[i] = queue.get(); F.count[i] = counters.get() + i; }
    F.bar_count = counters.get() + 4;
    F.bar_gen = counters.get() + 5;
    F.status = status.get();
    F.processed = rounds.get();
    int dev = 0, nsm = 0, per_sm = 0;
    HFM_CUDA(cudaGetDevice(&dev));
    HFM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    HFM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_kernel, 256, 0));
    if (per_sm < 1) throw Error(HFM_ERR_CUDA, "forward variation kernel cannot be resident");
    launch(forward_roots_kernel, nblocks(N, 256), 256, 0, s, F);
    void *args[] = {&F};
    count_launch();
    {
        std::lock_guard<std::mutex> coop(cooperative_mutex());
        HFM_CUDA(cudaLaunchCooperativeKernel((void *)forward_kernel,
                                             dim3(std::max(1, nsm * per_sm / std::max(1, solver_share()))), dim3(256),
                                             args, 0, s));
        check_status(status, "forward variation");
    }
    res.value_variation.resize((size_t)N * nvar);
    out.download(res.value_variation.data(), (size_t)N * nvar, s);
    HFM_CUDA(cudaStreamSynchronize(s));
}

// The device state that the reverse sweep reads (RetainedSolve of a single-instance solve).
template <typename Real, int NFWD, int NSYM, int KIND>
struct Retained final : RetainedSolve {
    Dev<Real> P{};
    long long N = 0;
    DeviceBuffer<Inst> dinst;
    DeviceBuffer<int> tile_inst;
    DeviceBuffer<unsigned> status, code, vis;
    DeviceBuffer<Real> values, weight, mult, cls_w;
    DeviceBuffer<int8_t> cls_off, cls_ang;
    DeviceBuffer<int> cls_d2;
    DeviceBuffer<TTICell> tti;
    DeviceBuffer<double> diag;  // per-axis speeds of a Diagonal model (P.diag_src points here)
    void adjoint(const EulerProblem &p, EulerResult &res) override {
        cudaStream_t s = current_stream();
        // arrival times (RowMajor, FP64) for the ordering of the sensitive seeds
        std::vector<Real> v(N);
        values.download(v.data(), N, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        res.values.assign(v.begin(), v.end());
        EulerProblem q;
        q.adjoint_index = p.adjoint_index;
        q.adjoint_weight = p.adjoint_weight;
        status.zero(s);
        EventTimer tm;
        tm.start(s);
        run_adjoint<Real, NFWD, NSYM, KIND>(P, N, q, res, status, s);
        res.t_adjoint_ms = tm.stop(s);
        HFM_CUDA(cudaStreamSynchronize(s));
    }
};

template <typename Real, int NFWD, int NSYM, int KIND>
void run_batch_impl(const std::vector<const EulerProblem *> &probs, std::vector<EulerResult> &results) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    constexpr int NB = NFWD + 2 * NSYM;
    const auto wall_t0 = std::chrono::steady_clock::now();
    cudaStream_t s = current_stream();
    const int ninst = (int)probs.size();
    results.assign(ninst, EulerResult());
    const EulerProblem &p0 = *probs[0];

    // ---- batch layout: instance table, global tile space
    std::vector<Inst> hinst(ninst);
    long long ntile = 0, ncells = 0, nclass = 0, nmetric = 0, nmult = 0;
    bool any_walls = false, want_active = false, want_stencils = false;
    for (int i = 0; i < ninst; ++i) {
        const EulerProblem &p = *probs[i];
        Inst &I = hinst[i];
        std::memset(&I, 0, sizeof(I));
        I.g = make_geom(p.ndim, p.dims, p.periodic, p.tile_shift[0] >= 0 ? p.tile_shift : nullptr);
        I.tile0 = ntile;
        I.cell0 = ncells;
        I.cls0 = nclass;
        I.metric0 = nmetric;
        for (int a = 0; a < 3; ++a) I.h[a] = p.h[a];
        I.dual = p.dual;
        I.metric_const = p.metric_constant;
        I.has_walls = (!p.walls.empty() || p.d_walls || p.walls_f64) ? 1 : 0;
        ntile += I.g.ntile;
        ncells += I.g.ncells;
        nclass += SHARE ? p.nclass : 0;
        if (!SHARE) nmetric += p.metric_constant ? 1 : I.g.ncells;
        I.mult0 = nmult;
        I.mult_depth = p.mult_depth;
        I.mult_inverse = p.mult_inverse ? 1 : 0;
        I.nth = p.sphere_nth;
        I.nph = p.sphere_nph;
        if ((KIND == kKindShareS2) != (p.sphere_nth > 0))
            throw Error(HFM_ERR_VALUE, "R^3 x S^2 grids take the sphere-bundle stencil family");
        if (SHARE) {
            // multiplier over the whole grid, the angular part (theta for the curvature models,
            // (theta, phi) for ReedsShepp3), the spatial part, or a constant
            const long long nang = I.nth > 0 ? (long long)I.nth * I.nph : 0;
            const long long nm[4] = {1, nang ? nang : I.g.dims[2],
                                     (long long)I.g.dims[0] * I.g.dims[1] * (nang ? I.g.dims[2] / nang : 1),
                                     I.g.ncells};
            nmult += nm[std::min(3, std::max(0, p.mult_depth))];
        }
        any_walls |= I.has_walls != 0;
        want_active |= p.want_active;
        want_stencils |= p.want_stencils;
    }
    if (ntile >= (1ll << 31)) throw Error(HFM_ERR_UNSUPPORTED, "batch too large");
    if (ninst > 1)
        for (const EulerProblem *q : probs)
            if (!q->adjoint_index.empty()) throw Error(HFM_ERR_UNSUPPORTED, "the adjoint runs on single solves");
    const long long N = ncells, ntc = ntile * 64, nt = ntile;
    Dev<Real> P{};
    P.ninst = ninst;
    P.ncells = N;
    P.ntile = nt;
    P.ntc = ntc;
    P.sstride = ntc;
    DeviceBuffer<Inst> dinst;
    dinst.upload(hinst, s);
    P.inst = dinst.get();
    std::vector<int> htile_inst(nt);
    for (int i = 0; i < ninst; ++i)
        std::fill(htile_inst.begin() + hinst[i].tile0, htile_inst.begin() + hinst[i].tile0 + hinst[i].g.ntile, i);
    DeviceBuffer<int> tile_inst;
    tile_inst.upload(htile_inst, s);
    P.tile_inst = tile_inst.get();
    DeviceBuffer<unsigned> status(1);
    status.zero(s);
    P.status = status.get();
    DeviceBuffer<Real> values(N);
    P.values = values.get();
    launch(fill_kernel<Real>, nblocks(N, 256) > 4096 ? 4096 : nblocks(N, 256), 256, 0, s, values.get(), N,
           Arith<Real>::inf());
    EventTimer tm;

    // ---- stencils
    tm.start(s);
    DeviceBuffer<unsigned> code, vis, maxw(ninst);
    DeviceBuffer<Real> weight, mult, cls_w;
    DeviceBuffer<int8_t> cls_off, cls_ang, plain_off;
    DeviceBuffer<int> cls_d2;
    DeviceBuffer<uint8_t> cls_en;
    DeviceBuffer<double> metric, plain_w, mult_rm, kscale;
    DeviceBuffer<TTICell> ttibuf;
    DeviceBuffer<double> fac_val, fac_grad;
    DeviceBuffer<uint8_t> fac_mask;
    std::vector<double> hscale;
    maxw.zero(s);
    std::vector<unsigned> hmaxw(ninst, 0);
    if (!SHARE) {
        code.alloc(ND * ntc);
        code.zero(s);
        weight.alloc(ND * ntc);
        weight.zero(s);
        P.code = code.get();
        P.weight = weight.get();
        const int NS = KIND == kKindTTI ? 14 : p0.diagonal ? p0.ndim : p0.ndim * (p0.ndim + 1) / 2;
        const double *metric_ptr = nullptr;
        if (ninst == 1 && p0.d_metric) {
            metric_ptr = p0.d_metric;
        } else if (ninst == 1 && p0.metric_ptr) {
            metric.upload(p0.metric_ptr, p0.metric_len, s);
            metric_ptr = metric.get();
        } else {
            metric.alloc((size_t)nmetric * NS);
            for (int i = 0; i < ninst; ++i) {
                const EulerProblem &p = *probs[i];
                const size_t rows = p.metric_constant ? 1 : (size_t)hinst[i].g.ncells;
                const size_t bytes = rows * NS * sizeof(double);
                double *dst = metric.get() + hinst[i].metric0 * NS;
                if (p.d_metric) HFM_CUDA(cudaMemcpyAsync(dst, p.d_metric, bytes, cudaMemcpyDeviceToDevice, s));
                else staged_upload(dst, p.metric_ptr ? p.metric_ptr : p.metric.data(), bytes, s);
            }
            metric_ptr = metric.get();
        }
        if (want_stencils && KIND != kKindTTI) {
            plain_off.alloc(N * ND * 3);
            plain_w.alloc(N * ND);
        }
        if constexpr (KIND == kKindTTI) {
            ttibuf.alloc(ntc);
            ttibuf.zero(s);
            P.tti = ttibuf.get();
            if (p0.has_factoring()) {  // the static factor of a single instance
                if (ninst > 1) throw Error(HFM_ERR_UNSUPPORTED, "static factoring runs on single solves");
                fac_val.upload(p0.fac_values, s);
                fac_grad.upload(p0.fac_grads, s);
                fac_mask.upload(p0.fac_mask, s);
                P.fac_val = fac_val.get();
                P.fac_grad = fac_grad.get();
                P.fac_mask = fac_mask.get();
                for (int a = 0; a < 3; ++a) {
                    P.fac_lo[a] = p0.fac_lo[a];
                    P.fac_dims[a] = p0.fac_dims[a];
                }
                P.fac_sub = p0.fac_subdomain ? 1 : 0;
                // the corrected update is not monotone: cells rise and fall a few times on the way
                // to the fixed point, so a tile gets a larger budget of increases
                P.up_budget = 64 * kUpBudget;
            }
            launch(tti_setup_kernel<NSYM, Real>, nblocks(N, 128), 128, 0, s, P, metric_ptr);
        } else if (p0.diagonal) {
            launch(diagonal_stencil_kernel<Real>, nblocks(N, 128), 128, 0, s, P, p0.ndim, metric_ptr, plain_off.get(),
                   plain_w.get());
            if (ninst == 1) {  // first variations read the speeds again (the metric buffer lives on)
                P.diag_src = metric_ptr;
                P.diag_inverse = p0.mult_inverse ? 1 : 0;
                P.var_dim = p0.ndim;
            }
        } else if (p0.ndim == 2) {
            launch(riemann_stencil_kernel<2, Real>, nblocks(N, 128), 128, 0, s, P, metric_ptr, plain_off.get(),
                   plain_w.get());
        } else {
            launch(riemann_stencil_kernel<3, Real>, nblocks(N, 128), 128, 0, s, P, metric_ptr, plain_off.get(),
                   plain_w.get());
        }
        HFM_CUDA(cudaGetLastError());
        launch(width_kernel<Real, NSYM>, nblocks(N, 256), 256, 0, s, P, maxw.get());
        maxw.download(hmaxw.data(), ninst, s);
        if (ninst > 1 && p0.ordered && !p0.diagonal) {
            kscale.alloc(ninst);
            kscale.zero(s);
            if (KIND == kKindTTI)
                launch(tti_scale_kernel<Real>, nblocks(N, 256), 256, 0, s, P, metric_ptr, kscale.get());
            else if (p0.ndim == 2)
                launch(metric_scale_kernel<2, Real>, nblocks(N, 256), 256, 0, s, P, metric_ptr, kscale.get());
            else
                launch(metric_scale_kernel<3, Real>, nblocks(N, 256), 256, 0, s, P, metric_ptr, kscale.get());
            hscale.resize(ninst);
            kscale.download(hscale.data(), ninst, s);
        }
        HFM_CUDA(cudaStreamSynchronize(s));
    } else {
        std::vector<Real> hw;
        std::vector<int8_t> ho, ha;
        std::vector<int> hd2;
        std::vector<uint8_t> he;
        mult_rm.alloc(std::max(1ll, nmult));
        for (int i = 0; i < ninst; ++i) {
            const EulerProblem &p = *probs[i];
            for (double w : p.cls_w) hw.push_back((Real)w);
            ho.insert(ho.end(), p.cls_off.begin(), p.cls_off.end());
            if (KIND == kKindShareS2) {
                if (p.cls_ang.size() != (size_t)p.nclass * ND * 2)
                    throw Error(HFM_ERR_VALUE, "sphere-bundle stencils need their angular steps");
                ha.insert(ha.end(), p.cls_ang.begin(), p.cls_ang.end());
                // third-coordinate step of each slot of a class (theta, phi) = (cl / nphi, cl % nphi):
                // s dz ntheta nphi plus the periodized angular step (the same for every z)
                const int nth = hinst[i].nth, nph = hinst[i].nph;
                for (int cl = 0; cl < p.nclass; ++cl)
                    for (int k = 0; k < ND; ++k)
                        for (int si = 0; si < (k < NFWD ? 1 : 2); ++si) {
                            const int sg = si ? -1 : 1;
                            const int8_t *o = &p.cls_off[(cl * ND + k) * 3];
                            const int8_t *a = &p.cls_ang[(cl * ND + k) * 2];
                            int th = cl / nph + sg * a[0], ph = cl % nph + sg * a[1];
                            s2_wrap(nth, nph, th, ph);
                            hd2.push_back(sg * o[2] * nth * nph + (th * nph + ph) - cl);
                        }
            }
            he.insert(he.end(), p.cls_enabled.begin(), p.cls_enabled.end());
            const long long len = (i + 1 < ninst ? hinst[i + 1].mult0 : nmult) - hinst[i].mult0;
            const double *msrc = p.mult_ptr ? p.mult_ptr : p.mult.data();
            if (!p.mult_ptr && (long long)p.mult.size() < len)
                throw Error(HFM_ERR_VALUE, "speed multiplier field too short");
            staged_upload(mult_rm.get() + hinst[i].mult0, msrc, len * sizeof(double), s);
            if (ninst > 1 && p0.ordered) {  // time scale = mean cost over the (uniform) broadcast field
                double t = 0.0;
                for (long long k = 0; k < len; ++k) {
                    const double m = msrc[k];
                    t += p.mult_inverse ? m : (m > 0.0 ? 1.0 / m : 0.0);
                }
                hscale.push_back(t / (double)len * (double)hinst[i].g.ncells);
            }
            // width over the class tables, from each class centre (HFM_StencilShare.hxx:152-175)
            int mw = 0;
            for (int cl = 0; cl < p.nclass; ++cl)
                for (int k = 0; k < ND; ++k) {
                    if (p.cls_w[cl * ND + k] == 0.0) continue;
                    const int8_t *o = &p.cls_off[(cl * ND + k) * 3];
                    for (int si = 0; si < (k < NFWD ? 1 : 2); ++si) {
                        const int slot = k < NFWD ? k : NFWD + 2 * (k - NFWD) + si;
                        if (!p.cls_enabled[cl * NB + slot]) continue;
                        int l1 = std::abs(o[0]) + std::abs(o[1]) + std::abs(o[2]);
                        if (KIND == kKindShareS2)
                            l1 += std::abs(p.cls_ang[(cl * ND + k) * 2]) + std::abs(p.cls_ang[(cl * ND + k) * 2 + 1]);
                        mw = std::max(mw, l1);
                    }
                }
            hmaxw[i] = (unsigned)mw;
        }
        cls_w.upload(hw, s);
        cls_off.upload(ho, s);
        cls_en.upload(he, s);
        maxw.upload(hmaxw, s);
        P.cls_w = cls_w.get();
        P.cls_off = cls_off.get();
        if (KIND == kKindShareS2) {
            cls_ang.upload(ha, s);
            P.cls_ang = cls_ang.get();
            cls_d2.upload(hd2, s);
            P.cls_d2 = cls_d2.get();
        }
        mult.alloc(ntc);
        mult.zero(s);
        P.mult = mult.get();
        launch(mult_layout_kernel<Real>, nblocks(N, 256), 256, 0, s, P, mult_rm.get());
        vis.alloc(ntc);
        vis.zero(s);
        P.vis = vis.get();
    }
    for (int i = 0; i < ninst; ++i) results[i].max_stencil_width = (int)hmaxw[i];
    if (!hscale.empty()) {
        // key scale: 1 / (domain diameter x mean norm scale), a common progress measure of the
        // instances' fronts for the value-ordered scheduling of a batch
        for (int i = 0; i < ninst; ++i) {
            const GridGeom &g = hinst[i].g;
            const int nphys = SHARE && probs[i]->angular ? 2 : probs[i]->ndim;
            double d2 = 0.0;
            for (int a = 0; a < nphys; ++a) d2 += (g.dims[a] * hinst[i].h[a]) * (g.dims[a] * hinst[i].h[a]);
            const double t = std::sqrt(d2) * hscale[i] / (double)g.ncells;
            hscale[i] = (t > 0.0 && t < 1e300) ? 1.0 / t : 1.0;
        }
        kscale.upload(hscale, s);
        P.kscale = kscale.get();
    }

    // ---- walls and visibility
    DeviceBuffer<uint8_t> walls;
    DeviceBuffer<int> wdist;
    DeviceBuffer<int8_t> wd8;
    if (any_walls) {
        const uint8_t *walls_ptr = nullptr;
        if (ninst == 1 && p0.d_walls) {
            walls_ptr = p0.d_walls;
        } else {
            walls.alloc(N);
            walls.zero(s);
            for (int i = 0; i < ninst; ++i) {
                const EulerProblem &p = *probs[i];
                if (p.d_walls)
                    HFM_CUDA(cudaMemcpyAsync(walls.get() + hinst[i].cell0, p.d_walls, hinst[i].g.ncells,
                                             cudaMemcpyDeviceToDevice, s));
                else if (!p.walls.empty())
                    staged_upload(walls.get() + hinst[i].cell0, p.walls.data(), hinst[i].g.ncells, s);
                else if (p.walls_f64) {
                    DeviceBuffer<double> wf(hinst[i].g.ncells);
                    staged_upload(wf.get(), p.walls_f64, hinst[i].g.ncells * sizeof(double), s);
                    launch(walls_from_f64_kernel, nblocks(hinst[i].g.ncells, 256), 256, 0, s, hinst[i].g.ncells,
                           wf.get(), walls.get() + hinst[i].cell0);
                }
            }
            walls_ptr = walls.get();
        }
        wdist.alloc(N);
        wd8.alloc(N);
        launch(wall_init_kernel, nblocks(N, 256), 256, 0, s, N, walls_ptr, wdist.get());
        for (int i = 0; i < ninst; ++i) {
            if (!hinst[i].has_walls) continue;
            const GridGeom &g = hinst[i].g;
            for (int a = 0; a < 3; ++a) {
                if (g.dims[a] == 1) continue;
                const long long nl = g.ncells / g.dims[a];
                launch(wall_scan_kernel, nblocks(nl, 128), 128, 0, s, g, a, wdist.get() + hinst[i].cell0);
            }
        }
        launch(wall_cap_kernel<Real>, nblocks(N, 256), 256, 0, s, P, wdist.get(), maxw.get(), wd8.get());
        HFM_CUDA(cudaGetLastError());
    }
    launch(visibility_kernel<Real, NFWD, NSYM, KIND>, nblocks(ntc, 128), 128, 0, s, P, wd8.get(), cls_en.get());
    HFM_CUDA(cudaGetLastError());
    wdist.release();

    // ---- seeds (global cell indices) and their tiles
    std::vector<long long> hsi;
    std::vector<double> hsv;
    std::vector<int> st;
    std::vector<unsigned long long> sm;
    for (int i = 0; i < ninst; ++i) {
        const EulerProblem &p = *probs[i];
        const GridGeom &g = hinst[i].g;
        for (size_t k = 0; k < p.seed_index.size(); ++k) {
            const long long x = p.seed_index[k];
            hsi.push_back(hinst[i].cell0 + x);
            hsv.push_back(p.seed_value[k]);
            const int x2 = (int)(x % g.dims[2]);
            const long long rr = x / g.dims[2];
            const int x1 = (int)(rr % g.dims[1]), x0 = (int)(rr / g.dims[1]);
            const int T = (int)(hinst[i].tile0 + g.tile_of(x0, x1, x2));
            const int b = g.local_of(x0, x1, x2);
            if (st.empty() || st.back() != T) {
                auto it = std::find(st.begin(), st.end(), T);
                if (it == st.end()) { st.push_back(T); sm.push_back(1ull << b); continue; }
                sm[it - st.begin()] |= 1ull << b;
            } else {
                sm.back() |= 1ull << b;
            }
        }
    }
    const int ns = (int)hsi.size();
    DeviceBuffer<long long> sidx;
    DeviceBuffer<double> sval;
    if (ns) {
        sidx.upload(hsi, s);
        sval.upload(hsv, s);
        launch(seeds_kernel<Real, KIND>, nblocks(ns, 128), 128, 0, s, P, sidx.get(), sval.get(), ns);
    }

    // ---- tile dependency graph (reverse CSR over the global tile space)
    DeviceBuffer<unsigned> dcnt(nt);
    auto deps_pass = [&](bool large, int pass, const long long *offs, int *src, int *dst, unsigned long long *msk,
                         unsigned long long *dmsk) {
        if (large)
            launch(deps_kernel<Real, NFWD, NSYM, KIND, kDepCapLarge, kDepWarpsLarge>, nblocks(nt, kDepWarpsLarge),
                   kDepWarpsLarge * 32, 0, s, P, pass, dcnt.get(), offs, src, dst, msk, dmsk);
        else
            launch(deps_kernel<Real, NFWD, NSYM, KIND, kDepCapSmall, kDepWarpsSmall>, nblocks(nt, kDepWarpsSmall),
                   kDepWarpsSmall * 32, 0, s, P, pass, dcnt.get(), offs, src, dst, msk, dmsk);
        HFM_CUDA(cudaGetLastError());
    };
    bool large_deps = false;
    deps_pass(false, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
    {
        unsigned st = 0;
        status.download(&st, 1, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        if (st & kErrTableOverflow) {  // some tile reads more distinct tiles than the small table holds
            const unsigned keep = st & ~(unsigned)kErrTableOverflow;
            HFM_CUDA(cudaMemcpyAsync(status.get(), &keep, sizeof(unsigned), cudaMemcpyHostToDevice, s));
            large_deps = true;
            deps_pass(true, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
        }
    }
    DeviceBuffer<long long> doff(nt + 1), rptr(nt + 1);
    std::vector<unsigned> hc(nt);
    dcnt.download(hc.data(), nt, s);
    HFM_CUDA(cudaStreamSynchronize(s));
    std::vector<long long> ho(nt + 1, 0);
    long long tot = 0;
    for (long long t = 0; t < nt; ++t) { ho[t] = tot; tot += hc[t]; }
    ho[nt] = tot;
    doff.upload(ho, s);
    const long long nE = tot;
    DeviceBuffer<int> rtile(nE);
    DeviceBuffer<unsigned long long> rmask(nE), rdmask(nE);
    {
        DeviceBuffer<int> esrc(nE), edst(nE);
        DeviceBuffer<unsigned long long> emsk(nE), edmsk(nE);
        if (nE) deps_pass(large_deps, 1, doff.get(), esrc.get(), edst.get(), emsk.get(), edmsk.get());
        DeviceBuffer<unsigned> rcnt(nt), cursor(nt);
        rcnt.zero(s);
        cursor.zero(s);
        if (nE) launch(dep_count_kernel, nblocks(nE, 256), 256, 0, s, nE, esrc.get(), rcnt.get());
        std::vector<unsigned> hr(nt);
        rcnt.download(hr.data(), nt, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        std::vector<long long> hrp(nt + 1, 0);
        tot = 0;
        for (long long t = 0; t < nt; ++t) { hrp[t] = tot; tot += hr[t]; }
        hrp[nt] = tot;
        rptr.upload(hrp, s);
        if (nE)
            launch(dep_scatter_kernel, nblocks(nE, 256), 256, 0, s, nE, esrc.get(), edst.get(), emsk.get(),
                   edmsk.get(), rptr.get(), cursor.get(), rtile.get(), rmask.get(), rdmask.get());
        HFM_CUDA(cudaGetLastError());
    }
    P.dep_ptr = rptr.get();
    P.dep_tile = rtile.get();
    P.dep_mask = rmask.get();
    P.dep_dmask = rdmask.get();
    DeviceBuffer<unsigned long long> key(nt), rstat(32), maxval(nt);
    DeviceBuffer<DirtyWake> dirty(nt);
    DeviceBuffer<unsigned> tile_up(nt);
    tile_up.zero(s);
    P.tile_up = tile_up.get();
    launch(fill_kernel<DirtyWake>, nblocks(nt, 256), 256, 0, s, dirty.get(), nt, DirtyWake{0ull, kInfWake});
    P.dirty = dirty.get();
    P.skip_settled = true;
    launch(fill_kernel<unsigned long long>, nblocks(nt, 256), 256, 0, s, key.get(), nt, 0x7ff0000000000000ull);
    launch(fill_kernel<unsigned long long>, nblocks(nt, 256), 256, 0, s, maxval.get(), nt, 0x7ff0000000000000ull);

    {
        unsigned long long h[32];
        for (int i = 0; i < 8; ++i) { h[4 * i] = 0x7ff0000000000000ull; h[4 * i + 1] = 0; h[4 * i + 2] = 0; h[4 * i + 3] = 0; }
        rstat.upload(h, 32, s);
    }
    P.key = key.get();
    P.rstat = rstat.get();
    P.maxval = maxval.get();
    const float t_stencil = tm.stop(s);
    check_status(status, "stencil");

    // ---- solve
    DeviceBuffer<int> lists(3 * nt);
    DeviceBuffer<unsigned> counters(16), flags(3 * nt);
    counters.zero(s);
    flags.zero(s);
    DeviceBuffer<unsigned long long> stats(4);
    stats.zero(s);
    for (int i = 0; i < 3; ++i) {
        P.list[i] = lists.get() + i * nt;
        P.flag[i] = flags.get() + i * nt;
        P.count[i] = counters.get() + i;
        P.claim[i] = counters.get() + 3 + i;
    }
    P.bar_count = counters.get() + 6;
    P.bar_gen = counters.get() + 7;
    P.stats = stats.get();
    P.max_rounds = p0.max_rounds;
    P.sweeps = p0.sweeps_per_tile;
    DeviceBuffer<int> stile;
    DeviceBuffer<unsigned long long> smask;
    const bool bypass = ninst == 1 && p0.bypass;
    if (bypass) {  // the arrival times are given: no solve
        if ((long long)p0.bypass_values.size() != N) throw Error(HFM_ERR_VALUE, "values have inconsistent dims");
        DeviceBuffer<double> bv(N);
        staged_upload(bv.get(), p0.bypass_values.data(), N * sizeof(double), s);
        launch(from_double_kernel<Real>, std::min<unsigned>(nblocks(N, 256), 4096), 256, 0, s,
               (const double *)bv.get(), values.get(), N);
        HFM_CUDA(cudaStreamSynchronize(s));
    }
    tm.start(s);
    std::unique_lock<std::mutex> coop(cooperative_mutex(), std::defer_lock);
    if (!st.empty() && !bypass) {
        stile.upload(st, s);
        smask.upload(sm, s);
        launch(init_lists_kernel<Real>, nblocks((long long)st.size() * 32, 128), 128, 0, s, P, stile.get(),
               smask.get(), (int)st.size());
        HFM_CUDA(cudaGetLastError());
        int dev = 0, nsm = 0, per_sm = 0;
        HFM_CUDA(cudaGetDevice(&dev));
        HFM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        HFM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fim_kernel<Real, NFWD, NSYM, KIND>,
                                                               kWarpsPerCta * 32, 0));
        if (per_sm < 1) throw Error(HFM_ERR_CUDA, "solver kernel cannot be resident");
        const int grid = std::max(1, nsm * per_sm / std::max(1, solver_share()));
        const double nwarps = (double)grid * kWarpsPerCta;
        const bool ordered = p0.ordered;
        P.order_lo = ordered ? (unsigned)std::max(1.0, p0.band_lo * nwarps) : 0u;
        P.order_hi = ordered ? (unsigned)std::max(2.0, p0.band_hi * nwarps) : 0u;
        void *args[] = {&P};
        count_launch();
        coop.lock();
        HFM_CUDA(cudaLaunchCooperativeKernel((void *)fim_kernel<Real, NFWD, NSYM, KIND>, dim3(grid),
                                             dim3(kWarpsPerCta * 32), args, 0, s));
    }
    const float t_solve = tm.stop(s);
    if (coop.owns_lock()) coop.unlock();
    check_status(status, "solver");
    unsigned long long hs[4] = {0, 0, 0, 0};
    stats.download(hs, 4, s);
    Stopped<Real> stopped;
    bool stopping = false;
    if (ninst == 1 && p0.has_stopping()) {
        apply_stopping<Real, NFWD, NSYM, KIND>(P, N, p0, values.get(), stopped, s);
        stopping = true;
    }
    DeviceBuffer<unsigned long long> nacc(ninst);
    nacc.zero(s);
    launch(count_finite_kernel<Real>, nblocks(N, 256), 256, 0, s, P, nacc.get());
    std::vector<unsigned long long> hn(ninst);
    nacc.download(hn.data(), ninst, s);

    // ---- outputs per instance
    DeviceBuffer<double> vd;
    if (!std::is_same<Real, double>::value) {
        vd.alloc(N);
        launch(to_double_kernel<Real>, std::min<unsigned>(nblocks(N, 256), 4096), 256, 0, s, values.get(), vd.get(), N);
    }
    const double *vsrc = std::is_same<Real, double>::value ? reinterpret_cast<const double *>(values.get()) : vd.get();
    DeviceBuffer<unsigned long long> act;
    if (want_active) {
        act.alloc(N);
        launch(active_kernel<Real, NFWD, NSYM, KIND>, nblocks(N, 128), 128, 0, s, P, act.get());
        if (stopped.on) {  // cells not accepted: the neighbours that were accepted
            DeviceBuffer<unsigned long long> act2(N);
            Dev<Real> PM = P;
            PM.values = stopped.vmask.get();
            launch(active_kernel<Real, NFWD, NSYM, KIND>, nblocks(N, 128), 128, 0, s, PM, act2.get());
            launch(stop_select_kernel, nblocks(N, 256), 256, 0, s, N, (const uint8_t *)stopped.acc.get(),
                   (const unsigned long long *)act2.get(), act.get());
            HFM_CUDA(cudaStreamSynchronize(s));
        }
    }
    for (int i = 0; i < ninst; ++i) {
        const EulerProblem &p = *probs[i];
        EulerResult &res = results[i];
        const long long n = hinst[i].g.ncells, off = hinst[i].cell0;
        if (p.d_values_out) {
            HFM_CUDA(cudaMemcpyAsync(p.d_values_out, vsrc + off, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        } else {
            double *dst = p.h_values_out;
            if (!dst) {
                res.values.resize(n);
                dst = res.values.data();
            }
            if (n * sizeof(double) >= kStagedMin) staged_download(dst, vsrc + off, n * sizeof(double), s);
            else HFM_CUDA(cudaMemcpyAsync(dst, vsrc + off, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        if (p.want_active) {
            res.active.resize(n);
            HFM_CUDA(cudaMemcpyAsync(res.active.data(), act.get() + off, n * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, s));
        }
        if (p.want_stencils && !SHARE) {
            res.stencil_off.resize(n * ND * 3);
            res.stencil_w.resize(n * ND);
            HFM_CUDA(cudaMemcpyAsync(res.stencil_off.data(), plain_off.get() + off * ND * 3, n * ND * 3,
                                     cudaMemcpyDeviceToHost, s));
            HFM_CUDA(cudaMemcpyAsync(res.stencil_w.data(), plain_w.get() + off * ND, n * ND * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
        }
        res.n_accepted = stopping ? (int64_t)stopped.count : (int64_t)hn[i];
        res.rounds = (long long)hs[0];
        res.tile_activations = (long long)hs[1];
        res.local_solves = (long long)hs[2];
        res.tile_carries = (long long)hs[3];
        res.t_stencil_ms = t_stencil;
        res.t_solve_ms = t_solve;
    }
    HFM_CUDA(cudaStreamSynchronize(s));
    run_geodesics<Real, NFWD, NSYM, KIND>(P, hinst, probs, results, any_walls ? wd8.get() : nullptr, s);
    if (ninst == 1 && (!p0.adjoint_index.empty() || p0.fwd_nvar > 0)) {
        tm.start(s);
        FlowGraph G;
        build_flow_graph<Real, NFWD, NSYM, KIND>(P, N, G, s);
        if (!p0.adjoint_index.empty()) run_adjoint<Real, NFWD, NSYM, KIND>(P, N, p0, results[0], status, s, &G);
        if (p0.fwd_nvar > 0) run_forward<Real, NFWD, NSYM, KIND>(P, N, p0, results[0], status, s, G);
        results[0].t_adjoint_ms = tm.stop(s);
    }
    HFM_CUDA(cudaStreamSynchronize(s));
    HFM_CUDA(cudaGetLastError());
    // A Diagonal model's speeds stay in the metric buffer, which the retained state then owns.
    if (ninst == 1 && p0.retain && (!p0.diagonal || !p0.d_metric)) {
        auto r = std::make_shared<Retained<Real, NFWD, NSYM, KIND>>();
        r->P = P;
        r->N = N;
        r->dinst = std::move(dinst);
        r->tile_inst = std::move(tile_inst);
        r->status = std::move(status);
        r->code = std::move(code);
        r->vis = std::move(vis);
        r->values = std::move(values);
        r->weight = std::move(weight);
        r->mult = std::move(mult);
        r->cls_w = std::move(cls_w);
        r->cls_off = std::move(cls_off);
        r->cls_ang = std::move(cls_ang);
        r->cls_d2 = std::move(cls_d2);
        r->tti = std::move(ttibuf);
        if (p0.diagonal) r->diag = std::move(metric);
        results[0].retained = r;
    }
    const double total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall_t0).count();
    for (EulerResult &r : results) r.t_total_ms = total;
}

#include "resident.cuh"

}  // namespace detail

using detail::run_batch_impl;

std::string resident_family_key(const EulerProblem &p) {
    const bool plain = p.adjoint_index.empty() && p.fwd_nvar == 0 && !p.has_stopping() && !p.bypass && !p.want_active &&
                       !p.want_stencils && !p.retain && p.geo_tips.empty() && p.geo_tips_unoriented.empty() &&
                       !p.want_geodesic_flow && !p.d_metric && !p.d_walls && !p.d_values_out;
    if (!plain) return "";
    const char *prec = p.fp64 ? "f64" : "f32";
    if (p.kind == StencilKind::RiemannPerCell && !p.diagonal && (p.ndim == 2 || p.ndim == 3))
        return std::string("riemann") + std::to_string(p.ndim) + "/" + prec;
    if (p.kind == StencilKind::SharedByTheta && p.angular && p.nfwd == 0 && p.nsym == 4)
        return std::string("reedsshepp2/") + prec;
    return "";
}

std::unique_ptr<ResidentFamily> make_resident_family(const EulerProblem &p) {
    using namespace detail;
    if (p.kind == StencilKind::RiemannPerCell && p.ndim == 2)
        return p.fp64 ? make_resident_impl<double, 0, 3, kKindRiemann>(p) : make_resident_impl<float, 0, 3, kKindRiemann>(p);
    if (p.kind == StencilKind::RiemannPerCell && p.ndim == 3)
        return p.fp64 ? make_resident_impl<double, 0, 6, kKindRiemann>(p) : make_resident_impl<float, 0, 6, kKindRiemann>(p);
    if (p.kind == StencilKind::SharedByTheta && p.nfwd == 0 && p.nsym == 4)
        return p.fp64 ? make_resident_impl<double, 0, 4, kKindShare>(p) : make_resident_impl<float, 0, 4, kKindShare>(p);
    throw Error(HFM_ERR_UNSUPPORTED, "no resident solver for this model family");
}

std::unique_ptr<StagedInputs> stage_resident_inputs(const EulerProblem &p) { return detail::stage_inputs_impl(p); }

void solve_eulerian_batch(const std::vector<const EulerProblem *> &probs, std::vector<EulerResult> &results) {
    if (probs.empty()) {
        results.clear();
        return;
    }
    const EulerProblem &p = *probs[0];
    for (const EulerProblem *q : probs) {
        if (q->kind != p.kind || q->ndim != p.ndim || q->nfwd != p.nfwd || q->nsym != p.nsym || q->fp64 != p.fp64 ||
            q->diagonal != p.diagonal || q->nmax != p.nmax || (q->sphere_nth > 0) != (p.sphere_nth > 0))
            throw Error(HFM_ERR_VALUE, "a batch must hold instances of one model family and one precision");
    }
    if (p.kind == StencilKind::TTI) {
        if (p.ndim != 3 || !p.fp64 || p.nsym != kTTISlots)
            throw Error(HFM_ERR_UNSUPPORTED, "TTI3 is solved in FP64 on 3D grids");
        run_batch_impl<double, 0, kTTISlots, detail::kKindTTI>(probs, results);
    } else if (p.kind == StencilKind::RiemannPerCell && p.diagonal) {
        if (p.ndim == 2) {
            if (p.fp64) run_batch_impl<double, 0, 2, detail::kKindRiemann>(probs, results);
            else run_batch_impl<float, 0, 2, detail::kKindRiemann>(probs, results);
        } else if (p.ndim == 3) {
            if (p.fp64) run_batch_impl<double, 0, 3, detail::kKindRiemann>(probs, results);
            else run_batch_impl<float, 0, 3, detail::kKindRiemann>(probs, results);
        } else {
            throw Error(HFM_ERR_UNSUPPORTED, "Diagonal models support dimensions 2 and 3");
        }
    } else if (p.kind == StencilKind::RiemannPerCell) {
        if (p.ndim == 2) {
            if (p.fp64) run_batch_impl<double, 0, 3, detail::kKindRiemann>(probs, results);
            else run_batch_impl<float, 0, 3, detail::kKindRiemann>(probs, results);
        } else if (p.ndim == 3) {
            if (p.fp64) run_batch_impl<double, 0, 6, detail::kKindRiemann>(probs, results);
            else run_batch_impl<float, 0, 6, detail::kKindRiemann>(probs, results);
        } else {
            throw Error(HFM_ERR_UNSUPPORTED, "Riemann models support dimensions 2 and 3");
        }
    } else {
        if (p.nfwd == 0 && p.nsym == 4) {
            if (p.fp64) run_batch_impl<double, 0, 4, detail::kKindShare>(probs, results);
            else run_batch_impl<float, 0, 4, detail::kKindShare>(probs, results);
        } else if (p.nfwd == 0 && p.nsym == 2) {
            if (p.fp64) run_batch_impl<double, 0, 2, detail::kKindShare>(probs, results);
            else run_batch_impl<float, 0, 2, detail::kKindShare>(probs, results);
        } else if (p.nfwd == 0 && p.nsym == 3) {
            if (p.fp64) run_batch_impl<double, 0, 3, detail::kKindShare>(probs, results);
            else run_batch_impl<float, 0, 3, detail::kKindShare>(probs, results);
        } else if (p.nfwd == 3 && p.nsym == 1) {
            if (p.fp64) run_batch_impl<double, 3, 1, detail::kKindShare>(probs, results);
            else run_batch_impl<float, 3, 1, detail::kKindShare>(probs, results);
        } else if (p.nfwd == 27 && p.nsym == 0) {
            if (p.fp64) run_batch_impl<double, 27, 0, detail::kKindShare>(probs, results);
            else run_batch_impl<float, 27, 0, detail::kKindShare>(probs, results);
        } else if (p.nfwd == 12 && p.nsym == 0 && p.nmax == 2) {
            if (p.fp64) run_batch_impl<double, 12, 0, detail::kKindShare2>(probs, results);
            else run_batch_impl<float, 12, 0, detail::kKindShare2>(probs, results);
        } else if (p.nfwd == 0 && p.nsym == 8 && p.sphere_nth > 0) {
            if (p.fp64) run_batch_impl<double, 0, 8, detail::kKindShareS2>(probs, results);
            else run_batch_impl<float, 0, 8, detail::kKindShareS2>(probs, results);
        } else if (p.nfwd == 6 && p.nsym == 2 && p.sphere_nth > 0) {
            if (p.fp64) run_batch_impl<double, 6, 2, detail::kKindShareS2>(probs, results);
            else run_batch_impl<float, 6, 2, detail::kKindShareS2>(probs, results);
        } else {
            throw Error(HFM_ERR_UNSUPPORTED, "unsupported shared stencil shape");
        }
    }
}

void default_schedule(EulerProblem &p) {
    if (p.kind == StencilKind::TTI) { p.sweeps_per_tile = 1; p.band_lo = 1; p.band_hi = 4; }
    else if (p.sphere_nth > 0) {
        // ReedsShepp3: 8 x 8 x 1 tiles (one (z, theta, phi) column of 64 (x, y) cells) and one sweep
        // per activation measured 11-19 % faster than 4 x 4 x 4 with two sweeps
        p.sweeps_per_tile = 1; p.band_lo = 4; p.band_hi = 16;
        if (p.tile_shift[0] < 0) { p.tile_shift[0] = 3; p.tile_shift[1] = 3; p.tile_shift[2] = 0; }
    }
    else if (p.kind == StencilKind::SharedByTheta && p.angular && p.nfwd + p.nsym > 4) { p.sweeps_per_tile = 2; p.band_lo = 4; p.band_hi = 16; }
    else if (p.kind == StencilKind::SharedByTheta && p.angular) { p.sweeps_per_tile = 4; p.band_lo = 2; p.band_hi = 8; }
    else if (p.ndim == 3) { p.sweeps_per_tile = 2; p.band_lo = 0.5; p.band_hi = 4; }
    else { p.sweeps_per_tile = 3; p.band_lo = 2; p.band_hi = 8; }
}

void solve_eulerian(const EulerProblem &p, EulerResult &r) {
    std::vector<EulerResult> rs;
    solve_eulerian_batch({&p}, rs);
    r = std::move(rs[0]);
}

}  // namespace hfm
