/* CPU restatement of the reference fast-marching solve path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): linked by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py as the checker. The product path never calls into this file.
 *
 * Compiled with -ffp-contract=off: every multiply and add rounds separately, as in the reference's
 * scalar x86-64 build, so that the operation order written here reproduces its results.
 * Paths in citations are relative to the reference repository root.
 */
#include "fm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FMO_INF (1.0 / 0.0)

/* ------------------------------------------------------------------------------------------ */
/* Symmetric matrix helpers, packed as data[i*(i+1)/2 + j] for j <= i
 * (JMM_CPPLibs/JMM_CPPLibs/LinearAlgebra/Implementation/SymmetricMatrixType.hxx:11-16). */

static inline int sym_index(int i, int j) {
    if (i < j) { int t = i; i = j; j = t; }
    return (i * (i + 1)) / 2 + j;
}

/* ScalarProduct(u, v) = sum_i u_i (sum_j m_ij v_j), accumulated from 0 in index order
 * (SymmetricMatrixType.hxx:18-30). Integer vectors are converted to double. */
static double sym_scal_int(int n, const double *m, const int *u, const int *v) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) {
        double sumi = 0.0;
        for (int j = 0; j < n; ++j) sumi += m[sym_index(i, j)] * (double)v[j];
        sum += (double)u[i] * sumi;
    }
    return sum;
}

/* Trace accumulated from 0 (SymmetricMatrixType.hxx:189-196). */
static double sym_trace(int n, const double *m) {
    double r = 0.0;
    for (int i = 0; i < n; ++i) r += m[sym_index(i, i)];
    return r;
}

/* Determinant (SymmetricMatrixType.hxx:199-218). */
static double sym_det(int n, const double *m) {
#define C(i, j) m[sym_index(i, j)]
    if (n == 2) return C(0, 0) * C(1, 1) - C(1, 0) * C(0, 1);
    return C(0, 0) * (C(1, 1) * C(2, 2) - C(1, 2) * C(2, 1))
         + C(0, 1) * (2.0 * C(1, 2) * C(2, 0) - C(1, 0) * C(2, 2))
         - C(0, 2) * (C(1, 1) * C(2, 0));
#undef C
}

/* Inverse = Comatrix()/Determinant(), the division applied as a product with the rounded
 * reciprocal (SymmetricMatrixType.hxx:220-243, VectorType.h:37-42). */
static void sym_inverse(int n, const double *m, double *out) {
#define C(i, j) m[sym_index(i, j)]
    double co[6];
    if (n == 2) {
        co[0] = C(1, 1); co[1] = -C(1, 0); co[2] = C(0, 0);
    } else {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j <= i; ++j) {
                const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                co[sym_index(i, j)] = C(i1, j1) * C(i2, j2) - C(i1, j2) * C(i2, j1);
            }
    }
#undef C
    const double b = 1.0 / sym_det(n, m);
    const int ns = n * (n + 1) / 2;
    for (int k = 0; k < ns; ++k) out[k] = co[k] * b;
}

/* ------------------------------------------------------------------------------------------ */
/* Selling's algorithm: obtuse superbase from the canonical one, at most 200 sweeps
 * (JMM_CPPLibs/JMM_CPPLibs/LinearAlgebra/Implementation/BasisReduction.hpp:12-15, 65-99;
 *  maxIt BasisReduction.h:72). */
static int obtuse_superbase(int n, const double *m, int sb[4][3]) {
    if (sym_det(n, m) <= 0.0 || sym_trace(n, m) <= 0.0) return -1;
    for (int i = 0; i <= n; ++i)
        for (int j = 0; j < n; ++j) sb[i][j] = (i < n) ? (i == j) : -1;
    int reduced = 1;
    for (int it = 0; reduced && it < 200; ++it) {
        reduced = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j <= n; ++j) {
                if (sym_scal_int(n, m, sb[i], sb[j]) > 0.0) {
                    reduced = 1;
                    if (n == 2) {
                        const int k = 3 - i - j;
                        for (int c = 0; c < 2; ++c) sb[k][c] = sb[i][c] - sb[j][c];
                    } else {
                        int kl[2], r = 0;
                        for (int k = 0; k <= 3; ++k) if (k != i && k != j) kl[r++] = k;
                        for (int c = 0; c < 3; ++c) { sb[kl[0]][c] += sb[i][c]; sb[kl[1]][c] += sb[i][c]; }
                    }
                    for (int c = 0; c < n; ++c) sb[i][c] = -sb[i][c];
                }
            }
    }
    return reduced ? -1 : 0;
}

/* TensorDecomposition: 2D offsets Perp(sb_i), weights -<sb_j, D sb_k>; 3D offsets
 * Cross(sb_k, sb_l), weights -<sb_i, D sb_j> over pairs i<j in lexicographic order
 * (BasisReduction.hpp:102-157; Perp/Cross VectorType.h:98-113). Offsets are written with
 * 3 components (unused ones zero). */
static int tensor_decomposition(int n, const double *d, int off[6][3], double w[6]) {
    int sb[4][3];
    if (obtuse_superbase(n, d, sb)) return -1;
    if (n == 2) {
        for (int i = 0; i < 3; ++i) {
            const int j = (i + 1) % 3, k = (i + 2) % 3;
            off[i][0] = -sb[i][1]; off[i][1] = sb[i][0]; off[i][2] = 0;
            w[i] = -sym_scal_int(2, d, sb[j], sb[k]);
        }
    } else {
        int r = 0;
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) {
                int rem[2], q = 0;
                for (int k = 0; k < 4; ++k) if (k != i && k != j) rem[q++] = k;
                const int *u = sb[rem[0]], *v = sb[rem[1]];
                for (int c = 0; c < 3; ++c) {
                    const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
                    off[r][c] = u[c1] * v[c2] - u[c2] * v[c1];
                }
                w[r] = -sym_scal_int(3, d, sb[i], sb[j]);
                ++r;
            }
    }
    return 0;
}

/* Voronoi1Mat: weights below 1000*eps*Tr(D) set to zero (Headers/Specializations/CommonTraits.h:82-105). */
int fmo_selling_mat(int ndim, const double *d, int8_t *offsets, double *weights) {
    if (ndim != 2 && ndim != 3) return -1;
    int off[6][3];
    double w[6];
    if (tensor_decomposition(ndim, d, off, w)) return -1;
    const double atol = (1000.0 * DBL_EPSILON) * sym_trace(ndim, d);
    const int nk = ndim == 2 ? 3 : 6;
    for (int k = 0; k < nk; ++k) {
        weights[k] = w[k] < atol ? 0.0 : w[k];
        for (int c = 0; c < 3; ++c) offsets[3 * k + c] = (int8_t)off[k][c];
    }
    return 0;
}

/* StencilRiemann::SetStencil / Rescale<true>: D = (dual ? M : M^-1) o (1/(h_i h_j))
 * (Headers/Specializations/Riemannian.h:41-71). */
int fmo_riemann_stencil(int ndim, const double *metric, int dual, const double *h,
                        int8_t *offsets, double *weights) {
    const int ns = ndim * (ndim + 1) / 2;
    double m[6], d[6];
    if (dual) memcpy(m, metric, ns * sizeof(double));
    else sym_inverse(ndim, metric, m);
    for (int i = 0; i < ndim; ++i)
        for (int j = 0; j <= i; ++j) {
            const double g = h[i] * h[j];          /* RankOneTensor(h) (SymmetricMatrixType.hxx:74-81) */
            d[sym_index(i, j)] = m[sym_index(i, j)] * (1.0 / g);
        }
    return fmo_selling_mat(ndim, d, offsets, weights);
}

int fmo_riemann_stencils(int ndim, int64_t n, const double *metric, int dual, const double *h,
                         int8_t *offsets, double *weights) {
    const int ns = ndim * (ndim + 1) / 2, nk = ndim == 2 ? 3 : 6;
    for (int64_t x = 0; x < n; ++x)
        if (fmo_riemann_stencil(ndim, metric + x * ns, dual, h, offsets + x * nk * 3, weights + x * nk))
            return -1;
    return 0;
}

/* Voronoi1Vec (CommonTraits.h:118-161): decompose (1-eps^2) v v^T + eps^2 |v|^2 Id, drop weights
 * below |v|^2 * 1000 eps or offsets too far from the direction, orient offsets so that <v,e> <= 0. */
int fmo_voronoi1vec(int ndim, const double *v, double eps, int8_t *offsets, double *weights) {
    double relaxed[6];
    double sq = 0.0;
    for (int i = 0; i < ndim; ++i) sq += v[i] * v[i];
    const double e2 = eps * eps;
    const double s1 = 1.0 - e2;
    for (int i = 0; i < ndim; ++i)
        for (int j = 0; j <= i; ++j) {
            const double exact = v[i] * v[j];
            const double id = (double)(i == j) * sq * e2;
            relaxed[sym_index(i, j)] = exact * s1 + id;
        }
    int off[6][3];
    double w[6];
    if (tensor_decomposition(ndim, relaxed, off, w)) return -1;
    const double angleTol = 1.0 / sqrt((double)(ndim - 1));
    const double wTol = sq * (1000.0 * DBL_EPSILON);
    const double angTol = (1.0 + angleTol * angleTol) / sq;
    const int nk = ndim == 2 ? 3 : 6;
    for (int k = 0; k < nk; ++k) {
        double o[3] = {0, 0, 0};
        for (int c = 0; c < ndim; ++c) o[c] = (double)off[k][c];
        double scal = 0.0, on = 0.0;
        for (int c = 0; c < ndim; ++c) scal += v[c] * o[c];
        for (int c = 0; c < ndim; ++c) on += o[c] * o[c];
        weights[k] = (w[k] < wTol || (scal * scal) * angTol < on) ? 0.0 : w[k];
        for (int c = 0; c < 3; ++c) offsets[3 * k + c] = (int8_t)(c < ndim ? (scal <= 0 ? off[k][c] : -off[k][c]) : 0);
    }
    return 0;
}

static const double kPi = 3.141592653589793238462643383279502884;

/* StencilReedsShepp2::SetStencil (Headers/Specializations/Curvature2.h:48-66): per angle index,
 * Voronoi1Vec of (cos t, sin t)/h (3 symmetric), plus the angular difference (0,0,1) with weight
 * 1/(xi dtheta)^2, dtheta = (projective ? pi : 2 pi)/ntheta. */
int fmo_reedsshepp2_table(int ntheta, double h, double xi, double eps, int projective,
                          int8_t *offsets, double *weights) {
    const double ds = (projective ? kPi : 2.0 * kPi) / (double)ntheta;
    const double ih = 1.0 / h;  /* Vector /= scalar multiplies by the reciprocal (VectorType.h:37-42) */
    for (int t = 0; t < ntheta; ++t) {
        const double theta = (double)t * ds;
        const double v[2] = {cos(theta) * ih, sin(theta) * ih};
        if (fmo_voronoi1vec(2, v, eps, offsets + t * 12, weights + t * 4)) return -1;
        int8_t *o = offsets + t * 12 + 9;
        o[0] = 0; o[1] = 0; o[2] = 1;
        const double xd = xi * ds;
        weights[t * 4 + 3] = 1.0 / (xd * xd);
    }
    return 0;
}

/* StencilReedsSheppForward2::SetStencil (Curvature2.h:86-100): 3 forward differences from the
 * 2D Voronoi1Vec of (cos, sin)(theta) / h, then one symmetric angular difference, offset (0,0,-1),
 * weight 1/(xi dtheta)^2. Layout per angle: forward first, then the symmetric one. */
int fmo_reedssheppforward2_table(int ntheta, double h, double xi, double eps,
                                 int8_t *offsets, double *weights) {
    const double ds = (2.0 * kPi) / (double)ntheta;
    const double ih = 1.0 / h;
    for (int t = 0; t < ntheta; ++t) {
        const double theta = (double)t * ds;
        const double v[2] = {cos(theta) * ih, sin(theta) * ih};
        if (fmo_voronoi1vec(2, v, eps, offsets + t * 12, weights + t * 4)) return -1;
        int8_t *o = offsets + t * 12 + 9;
        o[0] = 0; o[1] = 0; o[2] = -1;
        const double xd = xi * ds;
        weights[t * 4 + 3] = 1.0 / (xd * xd);
    }
    return 0;
}

/* StencilDubins2::SetStencil (Curvature2.h:119-140): per angle two stencils of 6 forward
 * differences, the first from the 3D Voronoi1Vec of (cos/h, sin/h, 1/(xi dtheta)), the second the
 * same with the angular component of each offset negated. Layout per angle: 12 forward
 * differences, stencil 0 then stencil 1. */
int fmo_dubins2_table(int ntheta, double h, double xi, double eps, int8_t *offsets, double *weights) {
    const double ds = (2.0 * kPi) / (double)ntheta;
    for (int t = 0; t < ntheta; ++t) {
        const double theta = (double)t * ds;
        const double v[3] = {cos(theta) / h, sin(theta) / h, 1. / (xi * ds)};
        int8_t *O = offsets + t * 36;
        double *W = weights + t * 12;
        if (fmo_voronoi1vec(3, v, eps, O, W)) return -1;
        for (int i = 0; i < 6; ++i) {
            W[6 + i] = W[i];
            O[(6 + i) * 3 + 0] = O[i * 3 + 0];
            O[(6 + i) * 3 + 1] = O[i * 3 + 1];
            O[(6 + i) * 3 + 2] = (int8_t)(-O[i * 3 + 2]);
        }
    }
    return 0;
}

/* StencilElastica2<5>::SetStencil (Curvature2.h:178-234): Fejer quadrature over 5 points; for
 * l = 0,1 a 3D Voronoi1Vec (6 offsets) and its mirror in theta, then a 2D one (3 offsets). */
int fmo_elastica2_table(int ntheta, double h, double xi, double eps,
                        int8_t *offsets, double *weights) {
    static const double fejer[5] = {0.167781, 0.525552, 0.613333, 0.525552, 0.167781};
    const int nF = 5;
    const double ds = (2.0 * kPi) / (double)ntheta;
    for (int t = 0; t < ntheta; ++t) {
        int8_t *O = offsets + t * 27 * 3;
        double *W = weights + t * 27;
        const double theta = (2.0 * kPi * (double)t) / (double)ntheta;
        for (int l = 0; l < nF / 2; ++l) {
            const double phi = kPi * (l + 0.5) / nF;
            const double v[3] = {sin(phi) * cos(theta) / h, sin(phi) * sin(theta) / h,
                                 cos(phi) / (xi * ds)};
            const int s0 = 2 * l, s1 = 2 * l + 1;
            if (fmo_voronoi1vec(3, v, eps, O + 6 * s0 * 3, W + 6 * s0)) return -1;
            for (int i = 0; i < 6; ++i) {
                W[6 * s0 + i] *= fejer[l];
                W[6 * s1 + i] = W[6 * s0 + i];
                for (int c = 0; c < 3; ++c) O[(6 * s1 + i) * 3 + c] = O[(6 * s0 + i) * 3 + c];
                O[(6 * s1 + i) * 3 + 2] = (int8_t)(-O[(6 * s1 + i) * 3 + 2]);
            }
        }
        const double v2[2] = {cos(theta) / h, sin(theta) / h};
        const int s = nF - 1;
        if (fmo_voronoi1vec(2, v2, eps, O + 6 * s * 3, W + 6 * s)) return -1;
        for (int i = 0; i < 3; ++i) W[6 * s + i] *= fejer[nF / 2];
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Grid helpers: closed axes reject out-of-range indices, periodic axes wrap
 * (Headers/Base/Implementation/PeriodicGrid.hxx:120-187). */

static inline int periodize(const fmo_problem *p, int64_t *idx) {
    for (int a = 0; a < p->ndim; ++a) {
        const int64_t n = p->dims[a];
        if (p->periodic[a]) {
            int64_t r = idx[a] % n;
            if (r < 0) r += n;
            idx[a] = r;
        } else if (idx[a] < 0 || idx[a] >= n) {
            return 0;
        }
    }
    return 1;
}

static inline int64_t linear_of(const fmo_problem *p, const int64_t *idx) {
    int64_t r = 0;
    for (int a = 0; a < p->ndim; ++a) r = r * p->dims[a] + idx[a];
    return r;
}

static inline void index_of(const fmo_problem *p, int64_t lin, int64_t *idx) {
    for (int a = p->ndim - 1; a >= 0; --a) { idx[a] = lin % p->dims[a]; lin /= p->dims[a]; }
}

static inline int64_t ncells(const fmo_problem *p) {
    int64_t n = 1;
    for (int a = 0; a < p->ndim; ++a) n *= p->dims[a];
    return n;
}

static inline int64_t stencil_id(const fmo_problem *p, const int64_t *idx, int64_t lin) {
    return p->share ? idx[p->ndim - 1] : lin;
}

/* ------------------------------------------------------------------------------------------ */
/* Wall distance: multi-source breadth-first search over the 2d axis neighbours, capped at the
 * maximal stencil width; 127 (int8 max) marks "far" (Headers/ExtraAlgorithms/WallObstructionTest.h:39-91). */
static int8_t *wall_distance(const fmo_problem *p, int maxDist) {
    const int64_t N = ncells(p);
    int8_t *wd = (int8_t *)malloc(N);
    int64_t *q = (int64_t *)malloc(N * sizeof(int64_t));
    if (!wd || !q) { free(wd); free(q); return NULL; }
    int64_t head = 0, tail = 0;
    for (int64_t x = 0; x < N; ++x) {
        wd[x] = 127;
        if (p->walls[x]) { wd[x] = 0; q[tail++] = x; }
    }
    int64_t idx[3], nb[3];
    while (head < tail) {
        const int64_t x = q[head++];
        const int nbd = wd[x] + 1;
        if (nbd > maxDist) continue;
        index_of(p, x, idx);
        for (int a = 0; a < p->ndim; ++a)
            for (int s = -1; s <= 1; s += 2) {
                memcpy(nb, idx, sizeof(nb));
                nb[a] += s;
                if (!periodize(p, nb)) continue;
                const int64_t y = linear_of(p, nb);
                if (wd[y] <= nbd) continue;
                wd[y] = (int8_t)nbd;
                q[tail++] = y;
            }
    }
    free(q);
    return wd;
}

/* Visible(base, v, sum): discrete line walk from base toward sum = base + v
 * (WallObstructionTest.h:95-150). */
static int wall_visible(const fmo_problem *p, const int8_t *wd, const int64_t *base,
                        const int *v, const int64_t *sum) {
    int w = wd[linear_of(p, sum)];
    if (w == 127) return 1;
    if (w == 0) return 0;
    int vSign[3] = {0, 0, 0};
    int vSum = 0, vProd = 1, vMax = 0;
    for (int i = 0; i < p->ndim; ++i) {
        const int vi = v[i];
        if (vi != 0) {
            vSign[i] = vi > 0 ? 1 : -1;
            const int avi = abs(vi);
            vSum += avi;
            vProd *= avi;
            if (avi > vMax) vMax = avi;
        }
    }
    if (vSum <= w) return 1;
    int64_t pos[3] = {base[0], base[1], base[2]};
    long long vNext[3], vInc[3];
    for (int i = 0; i < p->ndim; ++i) {
        vNext[i] = v[i] == 0 ? (long long)2147483647 : (long long)(vProd / abs(v[i]));
        vInc[i] = 2 * vNext[i];
    }
    for (int i = 1; i < vMax; ++i) {
        const long long threshold = (2LL * i * vProd) / vMax;
        for (int j = 0; j < p->ndim; ++j) {
            if (v[j] != 0 && vNext[j] <= threshold) {
                vNext[j] += vInc[j];
                --vSum;
                pos[j] += vSign[j];
            }
        }
        int64_t per[3] = {pos[0], pos[1], pos[2]};
        periodize(p, per);
        w = wd[linear_of(p, per)];
        if (vSum <= w) return 1;
        if (w == 0) return 0;
    }
    return 1;
}

/* ------------------------------------------------------------------------------------------ */
/* Reversed offsets: for every stencil, offsets of non-zero weight whose target lies in the domain,
 * keyed by the (periodized) target, sorted and deduplicated
 * (Headers/Base/Implementation/HFM_StencilRecompute.hxx:81-124, HFM_StencilShare.hxx:132-181).
 * With shared stencils the domain test is made from the central point of each class. */
typedef struct { int64_t key; int8_t o[3]; } rev_pair;

static int rev_cmp(const void *a, const void *b) {
    const rev_pair *x = (const rev_pair *)a, *y = (const rev_pair *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    for (int c = 0; c < 3; ++c)
        if (x->o[c] != y->o[c]) return x->o[c] < y->o[c] ? -1 : 1;
    return 0;
}

typedef struct { int64_t *split; int8_t (*off)[3]; int64_t nkeys; } rev_csr;

static int build_reversed(const fmo_problem *p, rev_csr *rc, int *maxWidth) {
    const int nd = p->nfwd + p->nsym;
    const int64_t N = ncells(p);
    const int64_t nst = p->share ? p->dims[p->ndim - 1] : N;
    const int64_t nkeys = nst;
    const int64_t cap = nst * (int64_t)(p->nfwd + 2 * p->nsym);
    rev_pair *pairs = (rev_pair *)malloc((cap ? cap : 1) * sizeof(rev_pair));
    if (!pairs) return -1;
    int64_t np = 0;
    int64_t idx[3], acc[3];
    for (int64_t s = 0; s < nst; ++s) {
        if (p->share) {
            for (int a = 0; a < p->ndim; ++a) idx[a] = p->dims[a] / 2;
            idx[p->ndim - 1] = s;
        } else {
            index_of(p, s, idx);
        }
        const int8_t *O = p->off + s * nd * 3;
        const double *W = p->w + s * nd;
        for (int k = 0; k < nd; ++k) {
            if (W[k] == 0.0) continue;
            for (int sg = 1; sg >= -1; sg -= 2) {
                if (sg == -1 && k < p->nfwd) break;
                for (int a = 0; a < p->ndim; ++a) acc[a] = idx[a] + sg * O[3 * k + a];
                if (!periodize(p, acc)) continue;
                rev_pair rp;
                rp.key = p->share ? acc[p->ndim - 1] : linear_of(p, acc);
                for (int c = 0; c < 3; ++c) rp.o[c] = (int8_t)(sg * O[3 * k + c]);
                pairs[np++] = rp;
            }
        }
    }
    qsort(pairs, np, sizeof(rev_pair), rev_cmp);
    int64_t nu = 0;
    for (int64_t i = 0; i < np; ++i)
        if (nu == 0 || rev_cmp(&pairs[nu - 1], &pairs[i]) != 0) pairs[nu++] = pairs[i];
    rc->nkeys = nkeys;
    rc->split = (int64_t *)calloc(nkeys + 1, sizeof(int64_t));
    rc->off = (int8_t(*)[3])malloc((nu ? nu : 1) * 3);
    if (!rc->split || !rc->off) { free(pairs); return -1; }
    int mw = 0;
    for (int64_t i = 0; i < nu; ++i) {
        rc->split[pairs[i].key + 1]++;
        memcpy(rc->off[i], pairs[i].o, 3);
        const int l1 = abs(pairs[i].o[0]) + abs(pairs[i].o[1]) + abs(pairs[i].o[2]);
        if (l1 > mw) mw = l1;
    }
    for (int64_t k = 0; k < nkeys; ++k) rc->split[k + 1] += rc->split[k];
    free(pairs);
    *maxWidth = mw;
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Binary heap with libstdc++'s push_heap/pop_heap algorithms, ordered as the reference's
 * QueueElement (Headers/Base/Implementation/HamiltonFastMarching.hxx:51-56): smallest value on top. */
typedef struct { int64_t idx; double val; } qelem;
typedef struct { qelem *a; int64_t n, cap; } heap_t;

static inline int heap_less(const qelem *x, const qelem *y) { return x->val > y->val; }

static void heap_push_hole(qelem *a, int64_t hole, int64_t top, qelem v) {
    int64_t parent = (hole - 1) / 2;
    while (hole > top && heap_less(&a[parent], &v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

static int heap_push(heap_t *h, qelem v) {
    if (h->n == h->cap) {
        int64_t nc = h->cap ? 2 * h->cap : 1024;
        qelem *na = (qelem *)realloc(h->a, nc * sizeof(qelem));
        if (!na) return -1;
        h->a = na; h->cap = nc;
    }
    h->a[h->n++] = v;
    heap_push_hole(h->a, h->n - 1, 0, v);
    return 0;
}

static qelem heap_pop(heap_t *h) {
    qelem *a = h->a;
    const qelem top = a[0];
    const int64_t len = h->n - 1;  /* pop_heap on [0, n): moves last into place */
    if (len > 0) {
        const qelem v = a[len];
        a[len] = a[0];
        int64_t hole = 0, second = 0;
        while (second < (len - 1) / 2) {
            second = 2 * (second + 1);
            if (heap_less(&a[second], &a[second - 1])) second--;
            a[hole] = a[second];
            hole = second;
        }
        if ((len & 1) == 0 && second == (len - 2) / 2) {
            second = 2 * (second + 1);
            a[hole] = a[second - 1];
            hole = second - 1;
        }
        heap_push_hole(a, hole, 0, v);
    }
    h->n--;
    return top;
}

/* ------------------------------------------------------------------------------------------ */
/* Incremental quadratic of the Eulerian scheme (Headers/Base/EulerianStencil.h:117-133,
 * Implementation/EulerianStencil.hxx:30-72). */
typedef struct { double minVal, a, b, c; int used; } quad_t;

static inline void quad_add(quad_t *q, double value, double weight) {
    const double w = weight, v = value - q->minVal;
    const double wv = w * v, wv2 = (w * v) * v;
    q->a += w; q->b += wv; q->c += wv2;
}

static inline double quad_solve(const quad_t *q) {
    if (q->a == 0.0) return q->minVal + FMO_INF;
    const double delta2 = q->b * q->b - q->a * q->c;
    const double delta = sqrt(0.0 < delta2 ? delta2 : 0.0);
    const double res = (q->b + delta) / q->a;
    return q->minVal + res;
}

static inline double diff_weight(const fmo_problem *p, double base, int64_t cell) {
    if (!p->mult) return base;
    const double m = p->mult[cell];
    return base * (m * m);   /* EulerianDifference::Weight (EulerianStencil.h:80-96) */
}

int64_t fmo_fast_marching(const fmo_problem *p, double *values, uint64_t *active,
                          int *max_stencil_width) {
    const int64_t N = ncells(p);
    const int nd = p->nfwd + p->nsym;
    rev_csr rc = {0};
    int maxWidth = 0;
    if (build_reversed(p, &rc, &maxWidth)) return -1;
    if (max_stencil_width) *max_stencil_width = maxWidth;
    int8_t *wd = NULL;
    if (p->walls) { wd = wall_distance(p, maxWidth); if (!wd) return -1; }

    uint8_t *accepted = (uint8_t *)calloc(N, 1);
    uint64_t *act = active ? active : (uint64_t *)calloc(N, sizeof(uint64_t));
    const int nq = p->nmax == 2 ? 2 : 1;
    if (nq == 2 && (p->nsym != 0 || p->nfwd % 2)) return -1;
    quad_t *quads = (quad_t *)calloc(N * nq, sizeof(quad_t));
    heap_t heap = {0};
    if (!accepted || !act || !quads) return -1;
    if (active) memset(active, 0, N * sizeof(uint64_t));
    for (int64_t x = 0; x < N; ++x) values[x] = FMO_INF;

    /* RunInit (HamiltonFastMarching.hxx:65-84): seeds in increasing index order */
    for (int s = 0; s < p->nseeds; ++s) {
        values[p->seed_index[s]] = p->seed_value[s];
        heap_push(&heap, (qelem){p->seed_index[s], p->seed_value[s]});
    }
    int64_t nAccepted = 0;
    int64_t aidx[3], uidx[3];
    /* stopWhenAllAccepted sets: targets not yet accepted (duplicates count once) */
    uint8_t *all_left = NULL, *all_left_u = NULL;
    int64_t n_all = 0, n_all_u = 0;
    if (p->nstop_all > 0) {
        all_left = (uint8_t *)calloc(N, 1);
        for (int i = 0; i < p->nstop_all; ++i)
            if (!all_left[p->stop_all[i]]) { all_left[p->stop_all[i]] = 1; ++n_all; }
    }
    if (p->nstop_all_u > 0) {
        all_left_u = (uint8_t *)calloc(p->dims[0] * p->dims[1], 1);
        for (int i = 0; i < p->nstop_all_u; ++i)
            if (!all_left_u[p->stop_all_u[i]]) { all_left_u[p->stop_all_u[i]] = 1; ++n_all_u; }
    }
    while (heap.n > 0) {
        /* RunOnce (HamiltonFastMarching.hxx:86-112) */
        const qelem top = heap_pop(&heap);
        if (accepted[top.idx]) continue;
        ++nAccepted;
        index_of(p, top.idx, aidx);
        /* CommonStoppingCriteria::PostProcess (CommonStoppingCriteria.h:58-93): the cell that
         * triggers a criterion is counted but not accepted */
        {
            int stop = p->n_max_accepted > 0 && nAccepted >= p->n_max_accepted;
            for (int i = 0; !stop && i < p->nstop_any; ++i) stop = p->stop_any[i] == top.idx;
            if (!stop && all_left && all_left[top.idx]) { all_left[top.idx] = 0; stop = --n_all == 0; }
            const int64_t xy = aidx[0] * p->dims[1] + aidx[1];
            for (int i = 0; !stop && i < p->nstop_any_u; ++i) stop = p->stop_any_u[i] == xy;
            if (!stop && all_left_u && all_left_u[xy]) { all_left_u[xy] = 0; stop = --n_all_u == 0; }
            if (!stop && p->has_stop_at_distance && values[top.idx] > p->stop_at_distance) stop = 1;
            if (stop) break;
        }
        accepted[top.idx] = 1;
        const int64_t key = p->share ? aidx[p->ndim - 1] : top.idx;
        for (int64_t r = rc.split[key]; r < rc.split[key + 1]; ++r) {
            const int8_t *e = rc.off[r];
            /* ConditionalUpdate (HamiltonFastMarching.hxx:136-154) */
            for (int a = 0; a < p->ndim; ++a) uidx[a] = aidx[a] - e[a];
            if (!periodize(p, uidx)) continue;
            if (wd) {
                int v[3] = {-e[0], -e[1], -e[2]};
                if (!wall_visible(p, wd, aidx, v, uidx)) continue;
            }
            const int64_t u = linear_of(p, uidx);
            if (accepted[u]) continue;
            if (act[u] == 0 && values[u] != FMO_INF) continue;
            if (values[u] <= top.val) continue;
            /* Update + HopfLaxUpdate (HFM_StencilRecompute.hxx:48-57, HFM_StencilShare.hxx:74-84,
             * EulerianStencil.hxx:104-153) */
            quad_t *q = &quads[u * nq];
            if (!q->used) {
                for (int i = 0; i < nq; ++i) { q[i].used = 1; q[i].minVal = top.val; q[i].a = 0; q[i].b = 0; q[i].c = -1; }
            }
            const int64_t sid = stencil_id(p, uidx, u);
            const int8_t *O = p->off + sid * nd * 3;
            const double *W = p->w + sid * nd;
            int bit = 0;
            for (int k = 0; k < p->nfwd; ++k, ++bit) {
                const int8_t *o = O + 3 * k;
                if (o[0] == e[0] && o[1] == e[1] && o[2] == e[2]) {
                    act[u] |= (1ULL << bit);
                    quad_add(q + (nq == 2 && k >= p->nfwd / 2), top.val, diff_weight(p, W[k], u));
                }
            }
            for (int k = p->nfwd; k < nd; ++k, bit += 2) {
                const int8_t *o = O + 3 * k;
                if (o[0] == e[0] && o[1] == e[1] && o[2] == e[2]) {
                    if (!(act[u] & (1ULL << (bit + 1)))) {
                        act[u] |= (1ULL << bit);
                        quad_add(q, top.val, diff_weight(p, W[k], u));
                    }
                }
                if (o[0] == -e[0] && o[1] == -e[1] && o[2] == -e[2]) {
                    if (!(act[u] & (1ULL << bit))) {
                        act[u] |= (1ULL << (bit + 1));
                        quad_add(q, top.val, diff_weight(p, W[k], u));
                    }
                }
            }
            double val;
            if (nq == 2) {
                /* QuadraticMax<., 2>::Solve (EulerianStencil.hxx:30-50): the smaller root, the first
                 * stencil on ties; SetIMax records it in the bit after the differences */
                int imin = 0;
                double res = FMO_INF;
                for (int i = 0; i < 2; ++i) {
                    if (q[i].a == 0.0) continue;
                    const double delta2 = q[i].b * q[i].b - q[i].a * q[i].c;
                    const double r = (q[i].b + sqrt(0.0 < delta2 ? delta2 : 0.0)) / q[i].a;
                    if (r >= res) continue;
                    imin = i;
                    res = r;
                }
                val = q[0].minVal + res;
                if (imin) act[u] |= (1ULL << p->nfwd);
                else act[u] &= ~(1ULL << p->nfwd);
            } else {
                val = quad_solve(q);
            }
            values[u] = val;
            heap_push(&heap, (qelem){u, val});
        }
    }
    free(heap.a);
    free(quads);
    free(accepted);
    free(all_left);
    free(all_left_u);
    if (!active) free(act);
    free(wd);
    free(rc.split);
    free(rc.off);
    return nAccepted;
}

int fmo_visibility(const fmo_problem *p, int max_width, uint8_t *visible) {
    const int64_t N = ncells(p);
    const int nd = p->nfwd + p->nsym, nb = p->nfwd + 2 * p->nsym;
    int8_t *wd = p->walls ? wall_distance(p, max_width) : NULL;
    if (p->walls && !wd) return -1;
    int64_t idx[3], nbh[3];
    for (int64_t x = 0; x < N; ++x) {
        index_of(p, x, idx);
        const int64_t sid = stencil_id(p, idx, x);
        const int8_t *O = p->off + sid * nd * 3;
        int b = 0;
        for (int k = 0; k < nd; ++k)
            for (int sg = 1; sg >= -1; sg -= 2) {
                if (sg == -1 && k < p->nfwd) break;
                int e[3] = {sg * O[3 * k], sg * O[3 * k + 1], sg * O[3 * k + 2]};
                for (int a = 0; a < p->ndim; ++a) nbh[a] = idx[a] + e[a];
                int ok = periodize(p, nbh);
                if (ok && wd) {
                    int v[3] = {-e[0], -e[1], -e[2]};
                    ok = wall_visible(p, wd, nbh, v, idx);
                }
                visible[x * nb + b++] = (uint8_t)ok;
            }
    }
    free(wd);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Reverse first variation (Headers/ExtraAlgorithms/FirstVariation.h:198-251 ValueVariation for
 * Eulerian schemes, :341-385 BackwardVariation). The reference keeps the pending points in a
 * std::map keyed by (value, index); here a max-heap keyed the same way plus a per-cell slot
 * gives the same visiting order. */
typedef struct { double val; int64_t idx; } bkey;

static inline int bkey_less(const bkey *x, const bkey *y) {
    return x->val < y->val || (x->val == y->val && x->idx < y->idx);
}

typedef struct { bkey *a; int64_t n, cap; } bheap_t;

static int bheap_push(bheap_t *h, bkey k) {
    if (h->n == h->cap) {
        int64_t nc = h->cap ? 2 * h->cap : 1024;
        bkey *na = (bkey *)realloc(h->a, nc * sizeof(bkey));
        if (!na) return -1;
        h->a = na; h->cap = nc;
    }
    int64_t i = h->n++;
    while (i > 0) {
        int64_t par = (i - 1) / 2;
        if (!bkey_less(&h->a[par], &k)) break;
        h->a[i] = h->a[par];
        i = par;
    }
    h->a[i] = k;
    return 0;
}

static bkey bheap_pop(bheap_t *h) {
    bkey top = h->a[0];
    bkey last = h->a[--h->n];
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        const bkey *best = &last;
        if (l < h->n && bkey_less(best, &h->a[l])) { m = l; best = &h->a[l]; }
        if (r < h->n && bkey_less(best, &h->a[r])) { m = r; best = &h->a[r]; }
        if (m == i) break;
        h->a[i] = h->a[m];
        i = m;
    }
    if (h->n > 0) h->a[i] = last;
    return top;
}

/* ValueVariation for Eulerian stencils (FirstVariation.h:198-251): the active neighbours in
 * stencil order with weights w max(0, value - u_neighbour) normalised by their sum, and the local
 * derivative (sum of w valueDiff) / sum (times the speed multiplier of shared stencils). */
/* The differences of a Recompute (EulerianStencil.hxx:155-229): every active one, or with two
 * stencils (nmax = 2) the active ones of the stencil named by bit nfwd (GetIMax). */
static inline uint64_t recompute_active(const fmo_problem *p, uint64_t act) {
    if (p->nmax != 2) return act;
    const int half = p->nfwd / 2;
    const int imax = (int)((act >> p->nfwd) & 1ULL);
    return act & (((1ULL << half) - 1ULL) << (imax * half));
}

static void eul_value_variation(const fmo_problem *p, const double *values, const uint64_t *active, int64_t x,
                                int64_t *nb_idx, double *nb_w, int *nn_out, double *var) {
    const int nd = p->nfwd + p->nsym;
    const int vd = p->var_dim > 1 ? p->var_dim : 1;
    int64_t idx[3], nidx[3];
    index_of(p, x, idx);
    const double value = values[x];
    const int64_t sid = stencil_id(p, idx, x);
    const int8_t *O = p->off + sid * nd * 3;
    const double *W = p->w + sid * nd;
    const uint64_t act = recompute_active(p, active[x]);
    double weightSum = 0.0;
    for (int i = 0; i < vd; ++i) var[i] = 0.0;
    int nn = 0;
    int bit = 0;
    for (int k2 = 0; k2 < nd; ++k2) {
        for (int sg = 1; sg >= -1; sg -= 2) {
            if (sg == -1 && k2 < p->nfwd) break;
            const int b = (k2 < p->nfwd) ? bit : bit + (sg == 1 ? 0 : 1);
            if (act & (1ULL << b)) {
                for (int a = 0; a < p->ndim; ++a) nidx[a] = idx[a] + sg * O[3 * k2 + a];
                periodize(p, nidx);
                const int64_t y = linear_of(p, nidx);
                const double d = value - values[y];
                const double valueDiff = 0.0 < d ? d : 0.0;
                const double w = diff_weight(p, W[k2], x) * valueDiff;
                weightSum += w;
                nb_idx[nn] = y; nb_w[nn] = w; ++nn;
                /* DiffHelper::Elem: the component of the difference's multiplier (its axis for the
                 * diagonal models, whose difference k is along axis k) */
                var[vd > 1 ? k2 : 0] += w * valueDiff;
            }
        }
        bit += (k2 < p->nfwd) ? 1 : 2;
    }
    *nn_out = nn;
    if (weightSum == 0.0) return;
    const double inv = 1.0 / weightSum;
    for (int j = 0; j < nn; ++j) nb_w[j] *= inv;
    if (vd > 1) {
        for (int i = 0; i < vd; ++i) var[i] = inv * (p->mult_vec[x * vd + i] * var[i]);
    } else {
        var[0] = p->mult ? inv * (p->mult[x] * var[0]) : inv * var[0];
    }
}

int64_t fmo_backward_variation(const fmo_problem *p, const double *values, const uint64_t *active,
                               int npts, const int64_t *pt_index, const double *pt_weight,
                               double *sensitivity, int64_t max_seeds, int64_t *seed_out_index,
                               double *seed_out_weight) {
    const int64_t N = ncells(p);
    /* pending weight per cell; in_map marks membership of (values[x], x) in the ordered set */
    double *pend = (double *)calloc(N, sizeof(double));
    uint8_t *in_map = (uint8_t *)calloc(N, 1);
    bheap_t h = {0};
    if (!pend || !in_map) return -1;
    const int vd = p->var_dim > 1 ? p->var_dim : 1;
    for (int64_t x = 0; x < N * vd; ++x) sensitivity[x] = 0.0;
    for (int i = 0; i < npts; ++i) {
        const int64_t x = pt_index[i];
        if (x < 0 || x >= N) continue;
        if (in_map[x]) continue;  /* std::map::insert keeps the first weight */
        in_map[x] = 1; pend[x] = pt_weight[i];
        bheap_push(&h, (bkey){values[x], x});
    }
    int64_t nseeds = 0;
    int64_t nb_idx[64];
    double nb_w[64];
    while (h.n > 0) {
        const bkey k = bheap_pop(&h);
        const int64_t x = k.idx;
        if (!in_map[x]) continue;
        in_map[x] = 0;
        const double weight = pend[x];
        pend[x] = 0.0;
        if (weight == 0.0) continue;
        int nn = 0;
        double var[3];
        eul_value_variation(p, values, active, x, nb_idx, nb_w, &nn, var);
        if (nn == 0) {
            if (nseeds < max_seeds) { seed_out_index[nseeds] = x; seed_out_weight[nseeds] = weight; }
            ++nseeds;
        }
        for (int i = 0; i < vd; ++i) sensitivity[x * vd + i] = weight * var[i];
        for (int j = 0; j < nn; ++j) {
            const int64_t y = nb_idx[j];
            if (in_map[y]) pend[y] += nb_w[j] * weight;
            else { in_map[y] = 1; pend[y] = nb_w[j] * weight; bheap_push(&h, (bkey){values[y], y}); }
        }
    }
    free(h.a);
    free(pend);
    free(in_map);
    return nseeds;
}

/* ========================================================================================== */
/* TTI3: tilted transversely anisotropic norm, semi-Lagrangian (Lag2) scheme.
 * Norm: JMM_CPPLibs/JMM_CPPLibs/LinearAlgebra/TTINorm.h:19-28, Implementation/TTINorm.hxx:46-265.
 * Selling path: JMM_CPPLibs/JMM_CPPLibs/LinearAlgebra/Implementation/BasisReduction.hpp:207-287.
 * Local solve and neighbours: Headers/Experimental/Implementation/TTI.hpp:24-47, 67-92, 190-318.
 * Fast marching with the Lag2 policy: a cell is re-solved from all its accepted neighbours
 * whenever one of its path neighbours is accepted (Headers/Base/Implementation/
 * HamiltonFastMarching.hxx:136-183, HFM_StencilLag2.hxx). */

/* value, first and second derivative in t (the reference's Diff1 / AD2 types) */
typedef struct { double v, d, dd; } dual2;
static inline dual2 d2c(double v) { dual2 r = {v, 0.0, 0.0}; return r; }
static inline dual2 d2add(dual2 a, dual2 b) { dual2 r = {a.v + b.v, a.d + b.d, a.dd + b.dd}; return r; }
static inline dual2 d2sub(dual2 a, dual2 b) { dual2 r = {a.v - b.v, a.d - b.d, a.dd - b.dd}; return r; }
static inline dual2 d2scale(dual2 a, double s) { dual2 r = {a.v * s, a.d * s, a.dd * s}; return r; }
static inline dual2 d2mul(dual2 a, dual2 b) {
    dual2 r = {a.v * b.v, a.d * b.v + a.v * b.d, a.dd * b.v + 2.0 * (a.d * b.d) + a.v * b.dd};
    return r;
}
static inline dual2 d2div(dual2 a, dual2 b) {
    const double q = a.v / b.v;
    const double qd = (a.d - q * b.d) / b.v;
    const double qdd = (a.dd - 2.0 * qd * b.d - q * b.dd) / b.v;
    dual2 r = {q, qd, qdd};
    return r;
}
static inline dual2 d2sqrt(dual2 a) {
    const double s = sqrt(a.v);
    const double sd = a.d / (2.0 * s);
    const double sdd = (a.dd - 2.0 * sd * sd) / (2.0 * s);
    dual2 r = {s, sd, sdd};
    return r;
}

typedef struct {
    double l0, l1, q00, q01, q11;   /* linear and quadratic coefficients */
    double D0[6], D1[6];            /* packed symmetric matrices of the extremal ellipsoids */
    double tmin, tmax;
    int dir;                        /* optimDirection: -1 inf over t, +1 sup over t */
} tti_norm;

/* smallest positive s with 0.5 q s^2 + l s - 1 = 0 (TTINorm.hxx:46-60) */
static double tti_spr(double l, double q) {
    if (q == 0.0) return 1.0 / l;
    const double delta = l * l + 2. * q;
    const double sdelta = sqrt(delta);
    const double rm = (-l - sdelta) / q, rp = (-l + sdelta) / q;
    const double rmin = rm < rp ? rm : rp, rmax = rm < rp ? rp : rm;
    return rmin > 0 ? rmin : rmax;
}

/* MakeNorm (TTI.hpp:24-34: transform columns scaled by the grid scales), the extremal matrices
 * of Selling (TTINorm.hxx:89-97, Matrix::Inverse MatrixType.hxx:250-316) and Props
 * (TTINorm.hxx:62-87). */
static int tti_setup(const double *m, const double *h, tti_norm *n) {
    n->l0 = m[0]; n->l1 = m[1];
    n->q00 = m[2]; n->q01 = m[3]; n->q11 = m[4];
    /* the reference reads the transform row by row (element 5 + 3 i + j is its transform(i, j));
     * T holds it transposed, T(i, j) = element 5 + i + 3 j, and MakeNorm's scaling of column j by
     * h_j is a scaling of row i of T by h_i (pinned against the reference executable, non-uniform
     * grid scales included) */
    double T[3][3], B[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[i][j] = m[5 + i + 3 * j] * h[i];
    double det = 0.0;
    for (int i = 0; i < 3; ++i)
        det += T[i][0] * T[(i + 1) % 3][1] * T[(i + 2) % 3][2] - T[i][2] * T[(i + 1) % 3][1] * T[(i + 2) % 3][0];
    if (!(det != 0.0)) return -1;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            B[j][i] = T[(i + 1) % 3][(j + 1) % 3] * T[(i + 2) % 3][(j + 2) % 3] -
                      T[(i + 1) % 3][(j + 2) % 3] * T[(i + 2) % 3][(j + 1) % 3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] = B[i][j] / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j) {
            n->D0[sym_index(i, j)] = B[0][i] * B[0][j] + B[1][i] * B[1][j];
            n->D1[sym_index(i, j)] = B[2][i] * B[2][j];
        }
    if (!(n->l0 >= 0 && n->l1 >= 0 && n->l0 + n->l1 > 0)) return -1;
    const double root0 = tti_spr(n->l0, n->q00), root1 = tti_spr(n->l1, n->q11);
    const double a0 = n->l0 + n->q00 * root0, a1 = n->l1 + n->q01 * root0;
    const double b0 = n->l0 + n->q01 * root1, b1 = n->l1 + n->q11 * root1;
    double tmin = a1 / (a0 + a1), tmax = b1 / (b0 + b1);
    if (tmin < tmax) {
        n->dir = -1;
    } else {
        const double s = tmin; tmin = tmax; tmax = s;
        n->dir = 1;
    }
    n->tmin = tmin; n->tmax = tmax;
    return (tmin == tmin && tmax == tmax) ? 0 : -1;
}

/* Multiplier(t): beta such that diag(1-t,t)/beta is tangent to the dual unit ball
 * (TTINorm.hxx:165-226, general branch). */
static dual2 tti_multiplier(const tti_norm *n, dual2 t) {
    if (n->q00 == 0.0 && n->q01 == 0.0 && n->q11 == 0.0) return d2c(1. / (n->l0 + n->l1));
    const double Q00 = n->q11, Q01 = -n->q01, Q11 = n->q00;   /* comatrix */
    const double l0 = n->l0, l1 = n->l1;
    const double Ql0 = Q00 * l0 + Q01 * l1, Ql1 = Q01 * l0 + Q11 * l1;
    const double detQ = Q00 * Q11 - Q01 * Q01;
    const double lQl = l0 * Ql0 + l1 * Ql1;
    const dual2 v0 = d2sub(d2c(1.0), t), v1 = t;
    const dual2 Qv0 = d2add(d2scale(v0, Q00), d2scale(v1, Q01));
    const dual2 Qv1 = d2add(d2scale(v0, Q01), d2scale(v1, Q11));
    const dual2 detVL = d2sub(d2scale(v0, l1), d2scale(v1, l0));
    const dual2 lQv = d2add(d2scale(Qv0, l0), d2scale(Qv1, l1));
    const dual2 vQv = d2add(d2mul(v0, Qv0), d2mul(v1, Qv1));
    const dual2 num = d2add(d2mul(detVL, detVL), d2scale(vQv, 2.0));
    const double signNum = num.v > 0 ? 1.0 : -1.0;
    const dual2 delta = d2scale(vQv, 2 * detQ + lQl);
    if (delta.v < 1e-10) return d2c(tti_spr(n->l0, n->q00) * v0.v);
    const dual2 den = d2add(d2scale(d2sqrt(delta), signNum), lQv);
    return d2div(num, den);
}

typedef struct {
    int sb[4][3];
    int off[6][3];
    double w0[6], w1[6];
} tti_path;

static void tti_path_weights(const tti_norm *n, tti_path *P) {
    for (int i = 0, r = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j, ++r) {
            P->w0[r] = -sym_scal_int(3, n->D0, P->sb[i], P->sb[j]);
            P->w1[r] = -sym_scal_int(3, n->D1, P->sb[i], P->sb[j]);
        }
}

static void tti_cross(const int *u, const int *v, int *o) {
    for (int c = 0; c < 3; ++c) {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        o[c] = u[c1] * v[c2] - u[c2] * v[c1];
    }
}

static void tti_complement(int i, int j, int *k, int *l) {
    int r = 0, kl[2] = {0, 0};
    for (int q = 0; q < 4; ++q) if (q != i && q != j) kl[r++] = q;
    *k = kl[0]; *l = kl[1];
}

static int tti_lin(int i, int j) {  /* LinearizeIndices (BasisReduction.hpp:181-192), i < j */
    if (i > j) { const int s = i; i = j; j = s; }
    int r = j - i - 1;
    if (i == 1) r += 3;
    else if (i == 2) r += 5;
    return r;
}

/* SellingPath(D0, D1, t) (BasisReduction.hpp:213-233) */
static int tti_path_init(const tti_norm *n, double t, tti_path *P) {
    double D[6];
    for (int k = 0; k < 6; ++k) D[k] = (1. - t) * n->D0[k] + t * n->D1[k];
    if (obtuse_superbase(3, D, P->sb)) return -1;
    tti_path_weights(n, P);
    for (int i = 0, r = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j, ++r) {
            int k, l;
            tti_complement(i, j, &k, &l);
            tti_cross(P->sb[k], P->sb[l], P->off[r]);
        }
    return 0;
}

/* NextStep (BasisReduction.hpp:235-259): t receives the next breakpoint (inf if none). */
static void tti_next_step(const tti_path *P, double *t, int *in, int *jn) {
    *t = FMO_INF; *in = -1; *jn = -1;
    for (int i = 0, r = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j, ++r) {
            const double s0 = P->w0[r], s1 = P->w1[r];
            if (s1 >= s0) continue;
            if (0 >= s0) continue;
            const double tr = s0 / (s0 - s1);
            if (tr >= *t) continue;
            *t = tr; *in = i; *jn = j;
        }
}

/* MakeStep (BasisReduction.hpp:261-285) */
static void tti_make_step(const tti_norm *n, tti_path *P, int i, int j) {
    int k, l;
    tti_complement(i, j, &k, &l);
    for (int c = 0; c < 3; ++c) {
        P->sb[k][c] += P->sb[i][c];
        P->sb[l][c] += P->sb[i][c];
        P->sb[i][c] = -P->sb[i][c];
    }
    tti_cross(P->sb[k], P->sb[l], P->off[tti_lin(i, j)]);
    int tmp[3];
    memcpy(tmp, P->off[tti_lin(i, k)], sizeof tmp);
    memcpy(P->off[tti_lin(i, k)], P->off[tti_lin(i, l)], sizeof tmp);
    memcpy(P->off[tti_lin(i, l)], tmp, sizeof tmp);
    tti_path_weights(n, P);
}

/* UpdateValue (TTINorm.hxx:99-163): sorted-prefix solve of a x^2 - 2 b x + c = 0 with weights
 * interpolated at t; the scalar pass fixes the prefix, the derivative pass recomputes on it. */
static dual2 tti_update_value(const tti_norm *n, dual2 t, const double *val, const tti_path *P, int with_ad) {
    int idx[6];
    for (int i = 0; i < 6; ++i) idx[i] = i;
    for (int i = 1; i < 6; ++i) {   /* stable insertion sort by value */
        const int x = idx[i];
        int k = i - 1;
        while (k >= 0 && val[idx[k]] > val[x]) { idx[k + 1] = idx[k]; --k; }
        idx[k + 1] = x;
    }
    const double valMin = val[idx[0]];
    if (valMin == FMO_INF) return d2c(FMO_INF);
    const dual2 mult = tti_multiplier(n, t);
    double a = 0, b = 0, c = -mult.v, sol = FMO_INF;
    int r = 0;
    for (; r < 6; ++r) {
        const int i = idx[r];
        const double v = val[i] - valMin;
        if (v >= sol) break;
        const double w_ = P->w0[i] + t.v * (P->w1[i] - P->w0[i]);
        const double w = w_ > 0 ? w_ : 0.0, wv = w * v, wvv = wv * v;
        a += w; b += wv; c += wvv;
        if (a <= mult.v * 1e-10) continue;
        const double delta = b * b - a * c;
        sol = (b + sqrt(delta > 0 ? delta : 0.0)) / a;
    }
    if (!with_ad) return d2c(valMin + sol);
    if (sol == FMO_INF) return d2c(FMO_INF);
    dual2 A = d2c(0), B = d2c(0), C = d2scale(mult, -1.0);
    for (int q = 0; q < r; ++q) {
        const int i = idx[q];
        const double v = val[i] - valMin;
        const dual2 w = d2add(d2c(P->w0[i]), d2scale(t, P->w1[i] - P->w0[i]));
        const dual2 wv = d2scale(w, v), wvv = d2scale(wv, v);
        A = d2add(A, w); B = d2add(B, wv); C = d2add(C, wvv);
    }
    const dual2 delta = d2sub(d2mul(B, B), d2mul(A, C));
    const dual2 s = d2div(d2add(B, d2sqrt(delta)), A);
    return d2add(d2c(valMin), s);
}

/* Neighbour value of the Lag2 scheme: the accepted value, or +inf (TTI.hpp:203-211). */
typedef double (*tti_getter)(void *ctx, int64_t cell, const int *off);

/* HopfLaxUpdate with nmix = 0 (TTI.hpp:142-276): extremum over t in [tmin, tmax] of the
 * Riemannian updates of the Selling path, interval by interval, with endpoint tests and a
 * safeguarded Newton search inside. Returns the value; *t_active, *interior describe the
 * extremum. Returns +inf if no neighbour is available. */
static double tti_local_solve(const tti_norm *n, int64_t cell, tti_getter get, void *ctx, double *t_active,
                              int *interior) {
    tti_path P;
    if (tti_path_init(n, n->tmin, &P)) return FMO_INF;
    double values[6];
    for (int r = 0; r < 6; ++r) values[r] = -FMO_INF;
    double t0 = n->tmin;
    const double objSign = -(double)n->dir;
    double updateValue = FMO_INF, tAct = FMO_INF;
    int isInt = 0;
    for (int guard = 0; guard < 1000; ++guard) {
        double t1;
        int ni, nj;
        tti_next_step(&P, &t1, &ni, &nj);
        if (t1 > n->tmax) t1 = n->tmax;
        do {
            for (int r = 0; r < 6; ++r) {
                if (values[r] == -FMO_INF) {
                    int mo[3] = {-P.off[r][0], -P.off[r][1], -P.off[r][2]};
                    const double vp = get(ctx, cell, P.off[r]), vm = get(ctx, cell, mo);
                    values[r] = vp < vm ? vp : vm;
                }
            }
            dual2 tt = {t0, 1.0, 0.0};
            const dual2 val0 = d2scale(tti_update_value(n, tt, values, &P, 1), objSign);
            if (val0.d >= 0 && val0.v < FMO_INF) {
                if (val0.v < updateValue) { updateValue = val0.v; tAct = t0; isInt = 0; }
                break;
            }
            tt.v = t1;
            const dual2 val1 = d2scale(tti_update_value(n, tt, values, &P, 1), objSign);
            if (val1.d <= 0 && val1.v < FMO_INF) {
                if (val1.v < updateValue) { updateValue = val1.v; tAct = t1; isInt = 0; }
                break;
            }
            if (isinf(val0.v) && isinf(val1.v)) break;
            double x0 = t0, x1 = t1, x = (val1.d * t0 - val0.d * t1) / (val1.d - val0.d), xOld = FMO_INF;
            for (int it = 0; fabs(xOld - x) > 100 * DBL_EPSILON && it < 200; ++it) {
                xOld = x;
                dual2 tx = {x, 1.0, 0.0};
                const dual2 v = d2scale(tti_update_value(n, tx, values, &P, 1), objSign);
                if (v.d <= 0) x0 = x;
                else x1 = x;
                if (v.dd > 0) {
                    x -= v.d / v.dd;
                    if (x0 < x && x < x1) continue;
                }
                x = (x0 + x1) / 2.;
            }
            const double v = objSign * tti_update_value(n, d2c(x), values, &P, 0).v;
            if (v < updateValue) { updateValue = v; tAct = x; isInt = 1; }
        } while (0);
        if (t1 == n->tmax) break;
        t0 = t1;
        if (ni < 0) break;
        tti_make_step(n, &P, ni, nj);
        const int r = tti_lin(ni, nj);
        values[r] = -FMO_INF;
        int k, l;
        tti_complement(ni, nj, &k, &l);
        const double s = values[tti_lin(ni, k)];
        values[tti_lin(ni, k)] = values[tti_lin(ni, l)];
        values[tti_lin(ni, l)] = s;
    }
    if (t_active) *t_active = tAct;
    if (interior) *interior = isInt;
    return objSign * updateValue;
}

/* SetNeighbors (TTI.hpp:67-92): the Selling offsets at tmin and every offset entering along the
 * path up to tmax (each with its opposite). Returns the number of offsets written (<= cap). */
static int tti_neighbors(const tti_norm *n, int (*out)[3], int cap) {
    tti_path P;
    if (tti_path_init(n, n->tmin, &P)) return -1;
    int cnt = 0;
#define PUSH(o)                                                              \
    do {                                                                     \
        if (cnt + 2 > cap) return -1;                                        \
        for (int c_ = 0; c_ < 3; ++c_) { out[cnt][c_] = (o)[c_]; out[cnt + 1][c_] = -(o)[c_]; } \
        cnt += 2;                                                            \
    } while (0)
    for (int r = 0; r < 6; ++r) PUSH(P.off[r]);
    if (n->tmax == n->tmin) return cnt;
    double t = n->tmin;
    for (int guard = 0; guard < 1000; ++guard) {
        int i, j;
        tti_next_step(&P, &t, &i, &j);
        if (t >= n->tmax) break;
        tti_make_step(n, &P, i, j);
        PUSH(P.off[tti_lin(i, j)]);
    }
#undef PUSH
    return cnt;
}

typedef struct {
    const int64_t *dims;
    const double *values;
    const uint8_t *accepted;
    const fmo_problem *fac;   /* static factoring (fac_values), or NULL */
} tti_fm_ctx;

/* StaticFactoring::Correction with order 1 (StaticFactoring.hxx:33-57) at cell x for the offset
 * e: 0 unless x lies in the box and its mask; then <grad(x), e> + (value(x) - value(x + e)), the
 * parenthesis dropped (Correction 0) when x + e leaves a subdomain box. */
static double tti_fac_correction(const fmo_problem *f, int64_t x0, int64_t x1, int64_t x2, const int *off) {
    const int64_t b[3] = {x0 - f->fac_lo[0], x1 - f->fac_lo[1], x2 - f->fac_lo[2]};
    for (int a = 0; a < 3; ++a)
        if (b[a] < 0 || b[a] >= f->fac_dims[a]) return 0.0;
    const int64_t bi = (b[0] * f->fac_dims[1] + b[1]) * f->fac_dims[2] + b[2];
    if (!f->fac_mask[bi]) return 0.0;
    const int64_t e[3] = {b[0] + off[0], b[1] + off[1], b[2] + off[2]};
    for (int a = 0; a < 3; ++a)
        if (e[a] < 0 || e[a] >= f->fac_dims[a]) return 0.0;  /* subdomain; a whole-domain box holds x + e */
    const int64_t ei = (e[0] * f->fac_dims[1] + e[1]) * f->fac_dims[2] + e[2];
    double deriv = 0.0;
    for (int a = 0; a < 3; ++a) deriv += f->fac_grads[3 * bi + a] * (double)off[a];
    return deriv + (f->fac_values[bi] - f->fac_values[ei]);
}

static double tti_fm_get(void *vctx, int64_t cell, const int *off) {
    const tti_fm_ctx *c = (const tti_fm_ctx *)vctx;
    const int64_t n1 = c->dims[1], n2 = c->dims[2];
    const int64_t x0 = cell / (n1 * n2), x1 = (cell / n2) % n1, x2 = cell % n2;
    const int64_t y0 = x0 + off[0], y1 = x1 + off[1], y2 = x2 + off[2];
    if (y0 < 0 || y0 >= c->dims[0] || y1 < 0 || y1 >= n1 || y2 < 0 || y2 >= n2) return FMO_INF;
    const int64_t y = (y0 * n1 + y1) * n2 + y2;
    if (!c->accepted[y]) return FMO_INF;
    double r = c->values[y];  /* GetNeighborValue (HamiltonFastMarching.hxx:357-359) */
    if (c->fac && c->fac->fac_values) r += tti_fac_correction(c->fac, x0, x1, x2, off);
    return r;
}

int fmo_tti_norm(const double *metric, const double *h, double *out) {
    tti_norm n;
    if (tti_setup(metric, h, &n)) return -1;
    out[0] = n.tmin; out[1] = n.tmax; out[2] = n.dir;
    const dual2 m0 = tti_multiplier(&n, d2c(n.tmin)), m1 = tti_multiplier(&n, d2c(n.tmax));
    out[3] = m0.v; out[4] = m1.v;
    return 0;
}

int64_t fmo_tti_fast_marching_stop(const int64_t *dims, const double *h, const double *metric, int nseeds,
                                   const int64_t *seed_index, const double *seed_value, double *values,
                                   double *t_active, const fmo_problem *stop);

int64_t fmo_tti_fast_marching(const int64_t *dims, const double *h, const double *metric, int nseeds,
                              const int64_t *seed_index, const double *seed_value, double *values,
                              double *t_active) {
    return fmo_tti_fast_marching_stop(dims, h, metric, nseeds, seed_index, seed_value, values, t_active, NULL);
}

/* With the stopping criteria of `stop` (its stop_* fields only; NULL: none), as the Eulerian loop. */
int64_t fmo_tti_fast_marching_stop(const int64_t *dims, const double *h, const double *metric, int nseeds,
                                   const int64_t *seed_index, const double *seed_value, double *values,
                                   double *t_active, const fmo_problem *stop) {
    const int64_t N = dims[0] * dims[1] * dims[2];
    uint8_t *all_left = NULL;
    int64_t n_all = 0;
    tti_norm *norms = (tti_norm *)malloc(N * sizeof(tti_norm));
    uint8_t *accepted = (uint8_t *)calloc(N, 1), *seed = (uint8_t *)calloc(N, 1);
    enum { CAP = 64 };
    int (*nb)[3] = (int (*)[3])malloc(sizeof(int) * 3 * CAP);
    int64_t *rcount = (int64_t *)calloc(N + 1, sizeof(int64_t));
    int64_t ret = -1;
    heap_t h_ = {0};
    int64_t *rcell = NULL;
    if (!norms || !accepted || !seed || !nb || !rcount) goto done;
    for (int64_t x = 0; x < N; ++x)
        if (tti_setup(metric + 14 * x, h, &norms[x])) goto done;
    /* reversed neighbours: y is re-solved when x = y + o is accepted */
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            for (int64_t x = 0; x < N; ++x) rcount[x + 1] += rcount[x];
            rcell = (int64_t *)malloc((rcount[N] + 1) * sizeof(int64_t));
            if (!rcell) goto done;
        }
        int64_t *cursor = pass == 1 ? (int64_t *)calloc(N, sizeof(int64_t)) : NULL;
        for (int64_t y = 0; y < N; ++y) {
            const int k = tti_neighbors(&norms[y], nb, CAP);
            if (k < 0) { free(cursor); goto done; }
            const int64_t y0 = y / (dims[1] * dims[2]), y1 = (y / dims[2]) % dims[1], y2 = y % dims[2];
            for (int q = 0; q < k; ++q) {
                const int64_t x0 = y0 + nb[q][0], x1 = y1 + nb[q][1], x2 = y2 + nb[q][2];
                if (x0 < 0 || x0 >= dims[0] || x1 < 0 || x1 >= dims[1] || x2 < 0 || x2 >= dims[2]) continue;
                const int64_t x = (x0 * dims[1] + x1) * dims[2] + x2;
                if (pass == 0) rcount[x + 1]++;
                else rcell[rcount[x] + cursor[x]++] = y;
            }
        }
        free(cursor);
    }
    for (int64_t x = 0; x < N; ++x) { values[x] = FMO_INF; if (t_active) t_active[x] = FMO_INF; }
    for (int s = 0; s < nseeds; ++s) {
        values[seed_index[s]] = seed_value[s];
        seed[seed_index[s]] = 1;
        qelem q = {seed_index[s], seed_value[s]};
        if (heap_push(&h_, q)) goto done;
    }
    tti_fm_ctx ctx = {dims, values, accepted, stop};
    int64_t nacc = 0;
    if (stop && stop->nstop_all > 0) {
        all_left = (uint8_t *)calloc(N, 1);
        if (!all_left) goto done;
        for (int i = 0; i < stop->nstop_all; ++i)
            if (!all_left[stop->stop_all[i]]) { all_left[stop->stop_all[i]] = 1; ++n_all; }
    }
    while (h_.n > 0) {
        const qelem top = heap_pop(&h_);
        if (accepted[top.idx] || top.val != values[top.idx]) continue;
        ++nacc;
        if (stop) {  /* CommonStoppingCriteria::PostProcess (CommonStoppingCriteria.h:58-93) */
            int halt = stop->n_max_accepted > 0 && nacc >= stop->n_max_accepted;
            for (int i = 0; !halt && i < stop->nstop_any; ++i) halt = stop->stop_any[i] == top.idx;
            if (!halt && all_left && all_left[top.idx]) { all_left[top.idx] = 0; halt = --n_all == 0; }
            if (!halt && stop->has_stop_at_distance && values[top.idx] > stop->stop_at_distance) halt = 1;
            if (halt) break;
        }
        accepted[top.idx] = 1;
        for (int64_t k = rcount[top.idx]; k < rcount[top.idx + 1]; ++k) {
            const int64_t y = rcell[k];
            if (accepted[y] || seed[y]) continue;
            if (values[y] <= top.val) continue;  /* ConditionalUpdate, HamiltonFastMarching.hxx:151 */
            double ta = FMO_INF;
            int interior = 0;
            const double v = tti_local_solve(&norms[y], y, tti_fm_get, &ctx, &ta, &interior);
            if (v < values[y]) {
                values[y] = v;
                if (t_active) t_active[y] = interior ? ta : -ta;
                qelem q = {y, v};
                if (heap_push(&h_, q)) goto done;
            }
        }
    }
    ret = nacc;
done:
    free(norms); free(accepted); free(seed); free(nb); free(rcount); free(rcell); free(h_.a); free(all_left);
    return ret;
}

/* Order-independent restatement of the factored TTI update, for the fixed-point check of the
 * parallel solvers: at each cell of `values` (a finished fast marching), the smallest of the local
 * solves triggered, in fast marching, by the acceptance of each stencil neighbour y = x + e, taken in
 * increasing value while below the result so far; each solve reads the neighbours of value at most
 * that of y (the ones accepted by then), with the corrections. Seeds keep their values. */
typedef struct {
    tti_fm_ctx base;
    double theta;
} tti_prefix_ctx;

static double tti_prefix_get(void *vctx, int64_t cell, const int *off) {
    const tti_prefix_ctx *c = (const tti_prefix_ctx *)vctx;
    const int64_t n1 = c->base.dims[1], n2 = c->base.dims[2];
    const int64_t x0 = cell / (n1 * n2), x1 = (cell / n2) % n1, x2 = cell % n2;
    const int64_t y0 = x0 + off[0], y1 = x1 + off[1], y2 = x2 + off[2];
    if (y0 < 0 || y0 >= c->base.dims[0] || y1 < 0 || y1 >= n1 || y2 < 0 || y2 >= n2) return FMO_INF;
    const double v = c->base.values[(y0 * n1 + y1) * n2 + y2];
    if (!(v <= c->theta)) return FMO_INF;
    double r = v;
    if (c->base.fac && c->base.fac->fac_values) r += tti_fac_correction(c->base.fac, x0, x1, x2, off);
    return r;
}

int fmo_tti_prefix_solve(const int64_t *dims, const double *h, const double *metric, const double *values,
                         const uint8_t *is_seed, const fmo_problem *fac, double *out) {
    const int64_t N = dims[0] * dims[1] * dims[2];
    enum { CAP = 64 };
    int nb[CAP][3];
    for (int64_t x = 0; x < N; ++x) {
        if (is_seed[x]) { out[x] = values[x]; continue; }
        tti_norm n;
        if (tti_setup(metric + 14 * x, h, &n)) return -1;
        const int k = tti_neighbors(&n, nb, CAP);
        if (k < 0) return -1;
        const int64_t x0 = x / (dims[1] * dims[2]), x1 = (x / dims[2]) % dims[1], x2 = x % dims[2];
        double th[CAP];
        int nth = 0;
        for (int q = 0; q < k; ++q) {
            const int64_t y0 = x0 + nb[q][0], y1 = x1 + nb[q][1], y2 = x2 + nb[q][2];
            if (y0 < 0 || y0 >= dims[0] || y1 < 0 || y1 >= dims[1] || y2 < 0 || y2 >= dims[2]) continue;
            const double v = values[(y0 * dims[1] + y1) * dims[2] + y2];
            if (!(v < FMO_INF)) continue;
            int i = nth++;
            while (i > 0 && th[i - 1] > v) { th[i] = th[i - 1]; --i; }
            th[i] = v;
        }
        double best = FMO_INF;
        tti_prefix_ctx ctx = {{dims, values, NULL, fac}, 0.0};
        for (int q = 0; q < nth; ++q) {
            if (q > 0 && th[q] == th[q - 1]) continue;
            if (!(th[q] < best)) break;
            ctx.theta = th[q];
            double ta = FMO_INF;
            int in = 0;
            const double v = tti_local_solve(&n, x, tti_prefix_get, &ctx, &ta, &in);
            if (v < best) best = v;
        }
        out[x] = best;
    }
    return 0;
}

/* The fixed point of that form reached by Jacobi iteration from the seeds (the parallel solvers'
 * result): values holds the seed values (and +inf elsewhere) on entry and the fixed point on exit.
 * Returns the number of sweeps, or -1 (no fixed point within max_sweeps, or an invalid norm). */
int fmo_tti_prefix_fixed_point(const int64_t *dims, const double *h, const double *metric, double *values,
                               const uint8_t *is_seed, const fmo_problem *fac, int max_sweeps) {
    const int64_t N = dims[0] * dims[1] * dims[2];
    double *nv = (double *)malloc(N * sizeof(double));
    if (!nv) return -1;
    int it = 0;
    for (; it < max_sweeps; ++it) {
        if (fmo_tti_prefix_solve(dims, h, metric, values, is_seed, fac, nv)) { it = -1; break; }
        int same = 1;
        for (int64_t x = 0; x < N; ++x)
            if (nv[x] != values[x]) { same = 0; break; }
        memcpy(values, nv, N * sizeof(double));
        if (same) break;
    }
    free(nv);
    return it < max_sweeps ? it : -1;
}

/* _HopfLaxRecompute at the stored extremum t (TTI.hpp:278-389, order 1): Riemannian update of the
 * Selling decomposition at t, its value and the discrete flow (offset * sign, (sol - v) w). */
static double tti_recompute(const tti_norm *n, const int64_t *dims, const double *values, int64_t x, double t,
                            int64_t *nb, double *nbw, int *nn, double *width) {
    tti_path P;
    *nn = 0;
    if (tti_path_init(n, t, &P)) return FMO_INF;
    const int64_t n1 = dims[1], n2 = dims[2];
    const int64_t x0 = x / (n1 * n2), x1 = (x / n2) % n1, x2 = x % n2;
    double val[6];
    int64_t cell[6];
    for (int r = 0; r < 6; ++r) {
        double vs[2] = {FMO_INF, FMO_INF};
        int64_t cs[2] = {-1, -1};
        for (int sg = 0; sg < 2; ++sg) {
            const int s = sg ? -1 : 1;
            const int64_t y0 = x0 + s * P.off[r][0], y1 = x1 + s * P.off[r][1], y2 = x2 + s * P.off[r][2];
            if (y0 < 0 || y0 >= dims[0] || y1 < 0 || y1 >= n1 || y2 < 0 || y2 >= n2) continue;
            cs[sg] = (y0 * n1 + y1) * n2 + y2;
            vs[sg] = values[cs[sg]];
        }
        if (vs[0] < vs[1]) { val[r] = vs[0]; cell[r] = cs[0]; }
        else { val[r] = vs[1]; cell[r] = cs[1]; }
    }
    int idx[6];
    for (int i = 0; i < 6; ++i) idx[i] = i;
    for (int i = 1; i < 6; ++i) {
        const int q = idx[i];
        int k = i - 1;
        while (k >= 0 && val[idx[k]] > val[q]) { idx[k + 1] = idx[k]; --k; }
        idx[k + 1] = q;
    }
    const double valMin = val[idx[0]];
    if (!(valMin < FMO_INF)) return FMO_INF;
    double a = 0, b = 0, c = -tti_multiplier(n, d2c(t)).v, sol = FMO_INF;
    int r = 0;
    for (; r < 6; ++r) {
        const int i = idx[r];
        const double v = val[i] - valMin;
        if (v >= sol) break;
        const double w = (1 - t) * P.w0[i] + t * P.w1[i];
        const double wv = w * v, wvv = wv * v;
        a += w; b += wv; c += wvv;
        if (a <= 100 * fabs(c) * DBL_EPSILON) continue;
        const double delta = b * b - a * c;
        sol = (b + sqrt(delta)) / a;
    }
    double wsum = 0.0, wd = 0.0;
    for (int q = 0; q < r; ++q) {
        const int i = idx[q];
        const double v = val[i] - valMin;
        const double w0 = (1 - t) * P.w0[i] + t * P.w1[i];
        const double d = (sol - v) * w0;
        wsum += w0;
        nb[*nn] = cell[i];
        nbw[*nn] = d > 0 ? d : 0.0;
        wd += nbw[*nn];
        ++*nn;
    }
    if (width) *width = wd / wsum;  /* TTI.hpp:372-388 */
    return sol + valMin;
}

int64_t fmo_tti_backward_variation(const int64_t *dims, const double *h, const double *metric,
                                   const double *values, const double *t_active, int npts,
                                   const int64_t *pt_index, const double *pt_weight, double *sensitivity,
                                   int64_t max_seeds, int64_t *seed_out_index, double *seed_out_weight) {
    const int64_t N = dims[0] * dims[1] * dims[2];
    double *pend = (double *)calloc(N, sizeof(double));
    uint8_t *in_map = (uint8_t *)calloc(N, 1);
    bheap_t hp = {0};
    if (!pend || !in_map) { free(pend); free(in_map); return -1; }
    for (int64_t x = 0; x < N; ++x) sensitivity[x] = 0.0;
    for (int i = 0; i < npts; ++i) {
        const int64_t x = pt_index[i];
        if (x < 0 || x >= N || in_map[x]) continue;
        in_map[x] = 1; pend[x] = pt_weight[i];
        bheap_push(&hp, (bkey){values[x], x});
    }
    int64_t nseeds = 0, nb[6];
    double nbw[6];
    while (hp.n > 0) {
        const bkey k = bheap_pop(&hp);
        const int64_t x = k.idx;
        if (!in_map[x]) continue;
        in_map[x] = 0;
        const double weight = pend[x];
        pend[x] = 0.0;
        if (weight == 0.0) continue;
        /* ValueVariation, semi-Lagrangian branch (FirstVariation.h:169-196); Recompute returns the
         * stored value and no flow where no update was recorded (HamiltonFastMarching.hxx:194-195) */
        int nn = 0;
        double rec = values[x];
        if (t_active[x] < FMO_INF) {
            tti_norm n;
            if (tti_setup(metric + 14 * x, h, &n)) { nn = 0; }
            else rec = tti_recompute(&n, dims, values, x, fabs(t_active[x]), nb, nbw, &nn, NULL);
        }
        double ws = 0.0;
        for (int j = 0; j < nn; ++j) ws += nbw[j];
        double valueDiff = rec;
        for (int j = 0; j < nn; ++j) {
            nbw[j] = nbw[j] / ws;
            valueDiff -= nbw[j] * values[nb[j]];
        }
        if (nn == 0) {
            if (nseeds < max_seeds) { seed_out_index[nseeds] = x; seed_out_weight[nseeds] = weight; }
            ++nseeds;
        }
        sensitivity[x] = weight * valueDiff;
        for (int j = 0; j < nn; ++j) {
            const int64_t y = nb[j];
            if (in_map[y]) pend[y] += nbw[j] * weight;
            else { in_map[y] = 1; pend[y] = nbw[j] * weight; bheap_push(&hp, (bkey){values[y], y}); }
        }
    }
    free(hp.a); free(pend); free(in_map);
    return nseeds;
}

/* Number of distinct offsets (up to sign) of SetNeighbors for each cell; -1 if invalid. */
int fmo_tti_neighbor_counts(int64_t n, const double *metric, const double *h, int *counts) {
    int nb[64][3];
    for (int64_t x = 0; x < n; ++x) {
        tti_norm nm;
        if (tti_setup(metric + 14 * x, h, &nm)) { counts[x] = -1; continue; }
        const int k = tti_neighbors(&nm, nb, 64);
        if (k < 0) { counts[x] = -1; continue; }
        int distinct = 0;
        for (int q = 0; q < k; q += 2) {
            int dup = 0;
            for (int r = 0; r < q; r += 2)
                if ((nb[r][0] == nb[q][0] && nb[r][1] == nb[q][1] && nb[r][2] == nb[q][2]) ||
                    (nb[r][0] == -nb[q][0] && nb[r][1] == -nb[q][1] && nb[r][2] == -nb[q][2])) dup = 1;
            distinct += !dup;
        }
        counts[x] = distinct;
    }
    return 0;
}

/* ========================================================================================== */
/* Geodesic backtracking and the geodesic flow.
 * Discrete solver: Headers/Base/Implementation/GeodesicDiscreteSolver.hxx:41-211 (Run with its
 * restarts, GeodesicDiscrete); flow: HamiltonFastMarching.hxx:187-272 (Recompute, order 1) with
 * EulerianStencil.hxx:157-229 (HopfLaxRecompute) and :363-378 (GeodesicFlow). Points are in the
 * reference's dimensionless coordinates (cell i spans [i, i+1)); the caller applies ReDim. */

#define GEO_MAXF 64

typedef int (*geo_flow_fn)(void *ctx, int64_t x, int (*off)[3], double *fw, double *value, double *width);

/* Order-1 Recompute at cell x for Eulerian stencils: the active differences in stencil order (the
 * forward ones, then the +e and -e sides of each symmetric one), the quadratic update over them and
 * the flow weights w_i max(0, value - u_i); width = sum of flow weights / sum of w_i. */
typedef struct { const fmo_problem *p; const double *values; const uint64_t *active; } eul_ctx;

static int eul_recompute(void *vctx, int64_t x, int (*off)[3], double *fw, double *value, double *width) {
    const eul_ctx *E = (const eul_ctx *)vctx;
    const fmo_problem *p = E->p;
    const int nd = p->nfwd + p->nsym;
    const uint64_t act = recompute_active(p, E->active[x]);
    *width = 0.0;
    *value = E->values[x];
    if (act == 0) return 0;
    int64_t idx[3], nidx[3];
    index_of(p, x, idx);
    const int64_t sid = stencil_id(p, idx, x);
    const int8_t *O = p->off + sid * nd * 3;
    const double *W = p->w + sid * nd;
    double nv[GEO_MAXF], wts[GEO_MAXF];
    int n = 0, bit = 0;
    for (int k = 0; k < nd; ++k) {
        for (int sg = 1; sg >= -1; sg -= 2) {
            if (sg == -1 && k < p->nfwd) break;
            const int b = k < p->nfwd ? bit : bit + (sg == 1 ? 0 : 1);
            if (!(act & (1ULL << b)) || n >= GEO_MAXF) continue;
            for (int a = 0; a < 3; ++a) off[n][a] = a < p->ndim ? sg * O[3 * k + a] : 0;
            for (int a = 0; a < p->ndim; ++a) nidx[a] = idx[a] + off[n][a];
            periodize(p, nidx);
            nv[n] = E->values[linear_of(p, nidx)];
            wts[n] = diff_weight(p, W[k], x);
            ++n;
        }
        bit += k < p->nfwd ? 1 : 2;
    }
    quad_t q = {FMO_INF, 0.0, 0.0, -1.0, 1};  /* QuadraticMax<ScalarType, 1>: a = b = 0, c = -1 */
    for (int i = 0; i < n; ++i) q.minVal = nv[i] < q.minVal ? nv[i] : q.minVal;
    for (int i = 0; i < n; ++i) quad_add(&q, nv[i], wts[i]);
    const double val = quad_solve(&q);
    double wsum = 0.0;
    for (int i = 0; i < n; ++i) {
        const double d = val - nv[i];
        fw[i] = wts[i] * (0.0 < d ? d : 0.0);
        *width += fw[i];
    }
    for (int i = 0; i < n; ++i) wsum += wts[i];
    if (wsum > 0) *width /= wsum;
    *value = val;
    return n;
}

/* TTI3 (Lag2) Recompute at the stored extremum t: offsets of the used Selling-path cells. */
typedef struct { const int64_t *dims; const double *h; const double *metric; const double *values;
                 const double *t_active; } tti_ctx;

static int tti_flow(void *vctx, int64_t x, int (*off)[3], double *fw, double *value, double *width) {
    const tti_ctx *T = (const tti_ctx *)vctx;
    *width = 0.0;
    *value = T->values[x];
    if (!(T->t_active[x] < FMO_INF)) return 0;
    tti_norm nm;
    if (tti_setup(T->metric + 14 * x, T->h, &nm)) return 0;
    int64_t nb[6];
    double nbw[6];
    int nn = 0;
    *value = tti_recompute(&nm, T->dims, T->values, x, fabs(T->t_active[x]), nb, nbw, &nn, width);
    const int64_t n1 = T->dims[1], n2 = T->dims[2];
    const int64_t x0 = x / (n1 * n2), x1 = (x / n2) % n1, x2 = x % n2;
    for (int j = 0; j < nn; ++j) {
        const int64_t y = nb[j];
        off[j][0] = (int)(y / (n1 * n2) - x0);
        off[j][1] = (int)((y / n2) % n1 - x1);
        off[j][2] = (int)(y % n2 - x2);
        fw[j] = nbw[j];
    }
    return nn;
}

typedef struct { double val; int64_t ind[3]; double w; } geo_entry;

typedef struct {
    const fmo_problem *p;   /* grid (dims, periodic axes) */
    const double *values;
    geo_flow_fn flow;
    void *ctx;
    double step, threshold;
    double *pts;            /* [cap][ndim] */
    int64_t n, cap;
    int overflow;
} geo_run;

static void geo_push(geo_run *G, const double *pt) {
    const int D = G->p->ndim;
    if (G->n >= G->cap) { G->overflow = 1; return; }
    for (int a = 0; a < D; ++a) G->pts[G->n * D + a] = pt[a];
    ++G->n;
}

/* weightSum, indexSum and covSum of the entries (UpdateSums, GeodesicDiscreteSolver.hxx:71-76) */
typedef struct { double ws, is[3], cs[3][3]; } geo_sums;

static void geo_add(geo_sums *S, int D, double w, const int64_t *ind) {
    S->ws += w;
    for (int i = 0; i < D; ++i) S->is[i] += w * (double)ind[i];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j <= i; ++j) S->cs[i][j] += w * ((double)ind[i] * (double)ind[j]);
}

static int geo_greater(const geo_entry *a, const geo_entry *b, int D) {
    if (a->val != b->val) return a->val > b->val;
    for (int i = 0; i < D; ++i)
        if (a->ind[i] != b->ind[i]) return a->ind[i] > b->ind[i];
    return 0;
}

/* One pass of GeodesicDiscrete from the last point; returns 1 if a restart is needed, -1 on
 * allocation failure. */
static int geo_discrete_pass(geo_run *G, double vbound) {
    const fmo_problem *p = G->p;
    const int D = p->ndim;
    geo_entry *set = NULL;
    int64_t ns = 0, scap = 0;
    double *sv = NULL, (*sd)[3] = NULL;
    int64_t nst = 0, stcap = 0;
    geo_sums S;
    memset(&S, 0, sizeof(S));
    double avg[3] = {0, 0, 0}, base[3] = {0, 0, 0}, stepNorm = 0.0;
    int ret = 0;
    double tip[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) tip[a] = G->pts[(G->n - 1) * D + a];
    int64_t ref[3];
    double pref[3];
    for (int a = 0; a < D; ++a) { ref[a] = (int64_t)floor(tip[a]); pref[a] = (double)ref[a] + 0.5; }
    /* unit mass split among the 2^D grid neighbours of the tip */
    for (int i = 0; i < (1 << D); ++i) {
        double weight = 1.0;
        int64_t ind[3] = {0, 0, 0}, per[3];
        for (int j = 0; j < D; ++j) {
            const double diff = tip[j] - pref[j];
            ind[j] = ref[j];
            if (i & (1 << j)) { ind[j] += diff > 0 ? 1 : -1; weight *= fabs(diff); }
            else weight *= 1. - fabs(diff);
        }
        for (int j = 0; j < D; ++j) per[j] = ind[j];
        if (!periodize(p, per)) continue;
        if (ns == scap) { scap = scap ? 2 * scap : 64; set = (geo_entry *)realloc(set, scap * sizeof(geo_entry)); if (!set) return -1; }
        set[ns].val = G->values[linear_of(p, per)];
        for (int j = 0; j < 3; ++j) set[ns].ind[j] = ind[j];
        set[ns].w = weight;
        ++ns;
        geo_add(&S, D, weight, ind);
    }
    if (S.ws == 0) goto done;
    /* vector / scalar multiplies by the reciprocal (FriendOperators.h:35, VectorType.h:37-41) */
    { const double iw = 1.0 / S.ws; for (int a = 0; a < D; ++a) { avg[a] = S.is[a] * iw; base[a] = avg[a]; } }
    while (ns > 0 && S.ws > 1e-5) {
        int64_t best = 0;
        for (int64_t k = 1; k < ns; ++k)
            if (geo_greater(&set[k], &set[best], D)) best = k;
        const geo_entry e = set[best];
        set[best] = set[--ns];
        if (e.w == 0) continue;
        geo_add(&S, D, -e.w, e.ind);
        int64_t per[3] = {e.ind[0], e.ind[1], e.ind[2]};
        periodize(p, per);
        int off[GEO_MAXF][3];
        double fw[GEO_MAXF], rval, rwidth;
        const int nf = G->flow(G->ctx, linear_of(p, per), off, fw, &rval, &rwidth);
        double wSum = 0;
        for (int f = 0; f < nf; ++f) wSum += fw[f];
        if (wSum == 0) continue;
        for (int f = 0; f < nf; ++f) {
            const double w = e.w * fw[f] / wSum;
            int64_t ind[3] = {0, 0, 0}, q[3];
            for (int a = 0; a < D; ++a) { ind[a] = e.ind[a] + off[f][a]; q[a] = ind[a]; }
            periodize(p, q);
            const double val = G->values[linear_of(p, q)];
            int64_t k = -1;
            for (int64_t m = 0; m < ns; ++m) {
                int same = set[m].val == val;
                for (int a = 0; a < D && same; ++a) same = set[m].ind[a] == ind[a];
                if (same) { k = m; break; }
            }
            if (k < 0) {
                if (w < S.ws * G->threshold) continue;
                if (ns == scap) { scap = scap ? 2 * scap : 64; set = (geo_entry *)realloc(set, scap * sizeof(geo_entry)); if (!set) return -1; }
                set[ns].val = val;
                for (int a = 0; a < 3; ++a) set[ns].ind[a] = ind[a];
                set[ns].w = w;
                ++ns;
            } else {
                set[k].w += w;
            }
            geo_add(&S, D, w, ind);
        }
        if (S.ws <= 0) {
            double pt[3];
            for (int a = 0; a < D; ++a) pt[a] = avg[a] + 0.5;
            geo_push(G, pt);
            goto done;
        }
        double step[3] = {0, 0, 0}, sq = 0.0;
        const double iw = 1.0 / S.ws;
        for (int a = 0; a < D; ++a) {
            const double old = avg[a];
            avg[a] = S.is[a] * iw;
            step[a] = avg[a] - old;
        }
        for (int a = 0; a < D; ++a) sq += step[a] * step[a];
        if (nst == stcap) {
            stcap = stcap ? 2 * stcap : 64;
            sv = (double *)realloc(sv, stcap * sizeof(double));
            sd = (double (*)[3])realloc(sd, stcap * sizeof(*sd));
            if (!sv || !sd) { ret = -1; goto done; }
        }
        sv[nst] = e.val;
        for (int a = 0; a < 3; ++a) sd[nst][a] = step[a];
        ++nst;
        stepNorm += sqrt(sq);
        if (ns == 1) {  /* mass concentrated at one point (seed or wall corner) */
            if (nf == 0) break;
            double pt[3];
            for (int a = 0; a < D; ++a) { pt[a] = avg[a] + 0.5; base[a] = avg[a]; }
            geo_push(G, pt);
            stepNorm = 0; nst = 0;
            continue;
        }
        if (stepNorm < G->step && ns > 1) continue;
        const double valInc = sv[0] - e.val;
        if (valInc <= 0) continue;
        const double delta = valInc / D;
        const double rden = 1.0 / (valInc + delta);
        double pt[3];
        for (int a = 0; a < D; ++a) pt[a] = base[a];
        for (int64_t k = 0; k < nst; ++k)
            for (int a = 0; a < D; ++a) pt[a] += (sd[k][a] * (sv[k] - e.val + delta)) * rden;
        for (int a = 0; a < D; ++a) { pt[a] += 0.5; base[a] = avg[a]; }
        geo_push(G, pt);
        stepNorm = 0; nst = 0;
        /* spread of the mass: det(covariance + Id) against the squared volume bound */
        double V[3][3];
        for (int i = 0; i < D; ++i)
            for (int j = 0; j <= i; ++j) {
                V[i][j] = S.cs[i][j] * iw - (S.is[i] * iw) * (S.is[j] * iw) + (i == j ? 1.0 : 0.0);
                V[j][i] = V[i][j];
            }
        double det;
        if (D == 2) det = V[0][0] * V[1][1] - V[1][0] * V[0][1];
        else det = V[0][0] * (V[1][1] * V[2][2] - V[1][2] * V[2][1]) - V[0][1] * (V[1][0] * V[2][2] - V[1][2] * V[2][0]) +
                   V[0][2] * (V[1][0] * V[2][1] - V[1][1] * V[2][0]);
        if (det > vbound * vbound) {
            for (int a = 0; a < D; ++a) pt[a] = avg[a] + 0.5;
            geo_push(G, pt);
            ret = 1;
            goto done;
        }
    }
done:
    free(set); free(sv); free(sd);
    return ret;
}

/* Run (GeodesicDiscreteSolver.hxx:41-55): restarts from the last point while the mass spreads too
 * much; after 5 restarts the volume bound grows by 1.3 per restart; 50 restarts mean failure. */
static int64_t geo_discrete_all(const fmo_problem *grid, const double *values, geo_flow_fn flow, void *ctx,
                                int ntips, const double *tips, double step, double threshold, double volume_bound,
                                int64_t max_points, double *points, int64_t *lengths, int *failed) {
    const int D = grid->ndim;
    int64_t total = 0;
    for (int t = 0; t < ntips; ++t) {
        geo_run G = {grid, values, flow, ctx, step, threshold, points + total * D, 0, max_points - total, 0};
        geo_push(&G, tips + (int64_t)t * D);
        int restarts = 0;
        double vb = volume_bound;
        while (restarts < 50 && !G.overflow) {
            const int r = geo_discrete_pass(&G, vb);
            if (r < 0) return -1;
            if (!r) break;
            ++restarts;
            if (restarts >= 5) vb *= 1.3;
        }
        if (G.overflow) return -2;
        lengths[t] = G.n;
        failed[t] = restarts == 50;
        total += G.n;
    }
    return total;
}

int64_t fmo_geodesic_discrete(const fmo_problem *p, const double *values, const uint64_t *active, int ntips,
                              const double *tips, double step, double threshold, double volume_bound,
                              int64_t max_points, double *points, int64_t *lengths, int *failed) {
    eul_ctx E = {p, values, active};
    return geo_discrete_all(p, values, eul_recompute, &E, ntips, tips, step, threshold, volume_bound, max_points,
                            points, lengths, failed);
}

int64_t fmo_tti_geodesic_discrete(const int64_t *dims, const double *h, const double *metric, const double *values,
                                  const double *t_active, int ntips, const double *tips, double step,
                                  double threshold, double volume_bound, int64_t max_points, double *points,
                                  int64_t *lengths, int *failed) {
    fmo_problem g;
    memset(&g, 0, sizeof(g));
    g.ndim = 3;
    for (int a = 0; a < 3; ++a) g.dims[a] = dims[a];
    tti_ctx T = {dims, h, metric, values, t_active};
    return geo_discrete_all(&g, values, tti_flow, &T, ntips, tips, step, threshold, volume_bound, max_points, points,
                            lengths, failed);
}

/* GeodesicFlow at every cell: flow[x] = sum of weight * offset over the Recompute flow (dimensionless;
 * the export is -ReDim of it), value and width of the Recompute. */
static void geo_flow_all(const fmo_problem *grid, geo_flow_fn flow, void *ctx, double *out, double *value,
                         double *width) {
    const int D = grid->ndim;
    const int64_t N = ncells(grid);
    int off[GEO_MAXF][3];
    double fw[GEO_MAXF];
    for (int64_t x = 0; x < N; ++x) {
        double v, wd;
        const int nf = flow(ctx, x, off, fw, &v, &wd);
        for (int a = 0; a < D; ++a) {
            double s = 0.0;
            for (int f = 0; f < nf; ++f) s += fw[f] * (double)off[f][a];
            out[x * D + a] = s;
        }
        if (value) value[x] = v;
        if (width) width[x] = wd;
    }
}

int fmo_geodesic_flow(const fmo_problem *p, const double *values, const uint64_t *active, double *flow,
                      double *value, double *width) {
    eul_ctx E = {p, values, active};
    geo_flow_all(p, eul_recompute, &E, flow, value, width);
    return 0;
}

int fmo_tti_geodesic_flow(const int64_t *dims, const double *h, const double *metric, const double *values,
                          const double *t_active, double *flow, double *value, double *width) {
    fmo_problem g;
    memset(&g, 0, sizeof(g));
    g.ndim = 3;
    for (int a = 0; a < 3; ++a) g.dims[a] = dims[a];
    tti_ctx T = {dims, h, metric, values, t_active};
    geo_flow_all(&g, tti_flow, &T, flow, value, width);
    return 0;
}


/* ========================================================================================== */
/* Forward first variation (Headers/ExtraAlgorithms/FirstVariation.h:389-429, inputs :103-124):
 * cells in increasing (value, index) order; result(x, k) += ValueVariation(x) * costVariation(x, k),
 * then += w_i result(neighbour_i, k) over the normalised flow. `result` [N][nvar] holds the seed
 * value variations on entry (zero elsewhere); cost_var [N][nvar] may be NULL (no cost variation). */
typedef struct { double val; int64_t idx; } vkey;

static int vkey_cmp(const void *a, const void *b) {
    const vkey *x = (const vkey *)a, *y = (const vkey *)b;
    if (x->val < y->val) return -1;
    if (x->val > y->val) return 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx ? 1 : 0);
}

static vkey *sorted_cells(const double *values, int64_t N) {
    vkey *o = (vkey *)malloc((size_t)N * sizeof(vkey));
    if (!o) return NULL;
    for (int64_t x = 0; x < N; ++x) { o[x].val = values[x]; o[x].idx = x; }
    qsort(o, (size_t)N, sizeof(vkey), vkey_cmp);
    return o;
}

int fmo_forward_variation(const fmo_problem *p, const double *values, const uint64_t *active, int nvar,
                          const double *cost_var, double *result) {
    const int64_t N = ncells(p);
    vkey *order = sorted_cells(values, N);
    if (!order) return -1;
    int64_t nb_idx[64];
    double nb_w[64];
    for (int64_t i = 0; i < N; ++i) {
        const int64_t x = order[i].idx;
        int nn = 0;
        double var[3];
        eul_value_variation(p, values, active, x, nb_idx, nb_w, &nn, var);
        const int vd = p->var_dim > 1 ? p->var_dim : 1;
        for (int k = 0; k < nvar; ++k) {
            double r = result[x * nvar + k];
            /* DiffHelper::Scal: sum of the products of the components */
            double sc = 0.0;
            for (int i = 0; i < vd; ++i) sc += var[i] * (cost_var ? cost_var[(x * nvar + k) * vd + i] : 0.0);
            r += sc;
            for (int j = 0; j < nn; ++j) r += nb_w[j] * result[nb_idx[j] * nvar + k];
            result[x * nvar + k] = r;
        }
    }
    free(order);
    return 0;
}

int fmo_tti_forward_variation(const int64_t *dims, const double *h, const double *metric, const double *values,
                              const double *t_active, int nvar, const double *cost_var, double *result) {
    const int64_t N = dims[0] * dims[1] * dims[2];
    vkey *order = sorted_cells(values, N);
    if (!order) return -1;
    int64_t nb[6];
    double nbw[6];
    for (int64_t i = 0; i < N; ++i) {
        const int64_t x = order[i].idx;
        /* semi-Lagrangian ValueVariation (FirstVariation.h:169-196), as in the backward sweep */
        int nn = 0;
        double rec = values[x];
        if (t_active[x] < FMO_INF) {
            tti_norm n;
            if (!tti_setup(metric + 14 * x, h, &n)) rec = tti_recompute(&n, dims, values, x, fabs(t_active[x]), nb, nbw, &nn, NULL);
        }
        double ws = 0.0;
        for (int j = 0; j < nn; ++j) ws += nbw[j];
        double var = rec;
        for (int j = 0; j < nn; ++j) {
            nbw[j] = nbw[j] / ws;
            var -= nbw[j] * values[nb[j]];
        }
        for (int k = 0; k < nvar; ++k) {
            double r = result[x * nvar + k];
            r += var * (cost_var ? cost_var[x * nvar + k] : 0.0);
            for (int j = 0; j < nn; ++j) r += nbw[j] * result[nb[j] * nvar + k];
            result[x * nvar + k] = r;
        }
    }
    free(order);
    return 0;
}

/* ========================================================================================== */
/* ODE geodesic solver (Headers/Base/Implementation/GeodesicODESolver.hxx): a midpoint scheme on
 * the geodesic flow interpolated from the 2^D cells around the point, stopping when the L-infinity
 * distance to the seeds (capped at 6) stops decreasing, or failing when a cell is revisited too
 * often (stationarity). For unit offsets the wall test of VisibleOffset reduces to "the target is
 * not a wall" (WallObstructionTest.h:95-150 with vMax = 1). */

typedef struct { int64_t key; int count; double flow[3], value, width; } ode_slot;
typedef struct { ode_slot *a; int64_t cap, n; } ode_map;

static ode_slot *ode_find(ode_map *m, int64_t key, int *fresh) {
    if (2 * (m->n + 1) > m->cap) {
        const int64_t nc = m->cap ? 2 * m->cap : 1024;
        ode_slot *na = (ode_slot *)malloc((size_t)nc * sizeof(ode_slot));
        if (!na) return NULL;
        for (int64_t i = 0; i < nc; ++i) na[i].key = -1;
        for (int64_t i = 0; i < m->cap; ++i) {
            if (m->a[i].key < 0) continue;
            int64_t h = (m->a[i].key * 0x9E3779B97F4A7C15ULL) & (nc - 1);
            while (na[h].key >= 0) h = (h + 1) & (nc - 1);
            na[h] = m->a[i];
        }
        free(m->a);
        m->a = na;
        m->cap = nc;
    }
    int64_t h = (key * 0x9E3779B97F4A7C15ULL) & (m->cap - 1);
    while (m->a[h].key >= 0 && m->a[h].key != key) h = (h + 1) & (m->cap - 1);
    *fresh = m->a[h].key < 0;
    if (*fresh) { m->a[h].key = key; m->a[h].count = 0; ++m->n; }
    return &m->a[h];
}

/* LInfDistance (GeodesicODESolver.hxx:225-258): breadth-first distance over the 3^D - 1 neighbours
 * through visible offsets, capped: cells at the cap are reached but not expanded. */
static int16_t *linf_distance(const fmo_problem *p, const int64_t *seeds, int nseeds, int cap) {
    const int64_t N = ncells(p);
    int16_t *d = (int16_t *)malloc((size_t)N * sizeof(int16_t));
    int64_t *q = (int64_t *)malloc((size_t)N * sizeof(int64_t));
    if (!d || !q) { free(d); free(q); return NULL; }
    for (int64_t x = 0; x < N; ++x) d[x] = 32767;
    int64_t head = 0, tail = 0;
    for (int s = 0; s < nseeds; ++s) {
        if (d[seeds[s]] != 0) { d[seeds[s]] = 0; q[tail++] = seeds[s]; }
    }
    int64_t idx[3], nb[3];
    const int D = p->ndim;
    while (head < tail) {
        const int64_t x = q[head++];
        if (d[x] >= cap) continue;
        index_of(p, x, idx);
        int n3 = 1;
        for (int a = 0; a < D; ++a) n3 *= 3;
        for (int c = 0; c < n3; ++c) {
            int cc = c, zero = 1;
            for (int a = 0; a < D; ++a) { const int o = cc % 3 - 1; cc /= 3; nb[a] = idx[a] + o; zero &= o == 0; }
            if (zero || !periodize(p, nb)) continue;
            const int64_t y = linear_of(p, nb);
            if (p->walls && p->walls[y]) continue;
            if (d[y] <= d[x] + 1) continue;
            d[y] = (int16_t)(d[x] + 1);
            q[tail++] = y;
        }
    }
    free(q);
    return d;
}

typedef struct { double flow[3]; int nstat, tol; } ode_flow;

static int ode_flow_at(const fmo_problem *p, geo_flow_fn flow, void *ctx, const int16_t *target, ode_map *cache,
                       double causality, const double *pt, ode_flow *out) {
    const int D = p->ndim;
    int64_t pi[3] = {0, 0, 0};
    double w[3] = {0, 0, 0};
    int sg[3] = {0, 0, 0};
    for (int j = 0; j < D; ++j) {
        pi[j] = (int64_t)floor(pt[j]);
        w[j] = pt[j] - (double)pi[j] - 0.5;
        sg[j] = w[j] > 0 ? 1 : -1;
        w[j] = fabs(w[j]);
    }
    ode_slot *slots[8];
    double wt[8];
    int mintol = 2147483647, maxstat = 0;
    for (int i = 0; i < (1 << D); ++i) {
        slots[i] = NULL;
        wt[i] = 0.0;
        int64_t q[3] = {0, 0, 0};
        for (int j = 0; j < D; ++j) q[j] = pi[j] + (((i >> j) & 1) ? sg[j] : 0);
        if (!periodize(p, q)) continue;
        const int64_t y = linear_of(p, q);
        if (p->walls && p->walls[y]) continue;
        if (target[y] < mintol) mintol = target[y];
        int fresh = 0;
        ode_slot *s = ode_find(cache, y, &fresh);
        if (!s) return -1;
        if (fresh) {
            int off[GEO_MAXF][3];
            double fw[GEO_MAXF];
            const int nf = flow(ctx, y, off, fw, &s->value, &s->width);
            for (int a = 0; a < 3; ++a) {
                double acc = 0.0;
                for (int f = 0; f < nf; ++f) acc += fw[f] * (double)off[f][a];
                s->flow[a] = acc;
            }
        }
        double weight = 1;
        for (int j = 0; j < D; ++j) weight *= ((i >> j) & 1) ? w[j] : (1 - w[j]);
        slots[i] = s;
        wt[i] = weight;
        if (s->count > maxstat) maxstat = s->count;
        ++s->count;
    }
    out->nstat = maxstat;
    out->tol = mintol;
    out->flow[0] = out->flow[1] = out->flow[2] = 0.0;
    double minVal = FMO_INF;
    int imin = -1;
    for (int i = 0; i < (1 << D); ++i)
        if (wt[i] > 0 && slots[i]->value < minVal) { minVal = slots[i]->value; imin = i; }
    if (minVal == FMO_INF) return 0;
    const double thr = minVal + causality * slots[imin]->width;
    double ws = 0.0;
    for (int i = 0; i < (1 << D); ++i) {
        if (wt[i] <= 0) continue;
        if (slots[i]->value <= thr) {
            ws += wt[i];
            for (int a = 0; a < D; ++a) out->flow[a] += wt[i] * slots[i]->flow[a];
        }
    }
    if (ws > 0)
    {
        const double iw = 1.0 / ws;
        for (int a = 0; a < D; ++a) out->flow[a] *= iw;
    }
    return 0;
}

/* Run (GeodesicODESolver.hxx:159-212) for one tip; returns 0 (reached the seeds or a seed), 1
 * (stalled: the reference's failure), -1 on allocation failure, -2 if the output is full. */
static int ode_run(const fmo_problem *p, geo_flow_fn flow, void *ctx, const int16_t *target, double step,
                   double causality, double *pts, int64_t cap, int64_t *len) {
    const int D = p->ndim;
    ode_map cache = {NULL, 0, 0};
    const int nstat_max = (int)(6 * sqrt((double)D) / step);
    int nh = 0;
    for (int i = 0; i < sqrt((double)D) / step; ++i) ++nh;
    int *hist = (int *)malloc((size_t)(nh > 0 ? nh : 1) * sizeof(int));
    if (!hist) return -1;
    for (int i = 0; i < nh; ++i) hist[i] = 2147483647;
    int head = 0, ret = 0;
    for (;;) {
        const double *pt = pts + (*len - 1) * D;
        ode_flow fd;
        if (ode_flow_at(p, flow, ctx, target, &cache, causality, pt, &fd)) { ret = -1; break; }
        int old = 2147483647;
        if (nh > 0) { old = hist[head]; hist[head] = fd.tol; head = (head + 1) % nh; }
        else old = fd.tol;  /* an empty history compares the front of the pushed value */
        if (old < fd.tol) break;
        if (fd.nstat > nstat_max) { ret = 1; break; }
        double nrm = 0.0;
        for (int a = 0; a < D; ++a) nrm += fd.flow[a] * fd.flow[a];
        nrm = sqrt(nrm);
        if (nrm == 0) break;
        double q[3];
        const double inv = 1.0 / nrm;
        for (int a = 0; a < D; ++a) q[a] = pt[a] + (0.5 * step * fd.flow[a]) * inv;
        if (ode_flow_at(p, flow, ctx, target, &cache, causality, q, &fd)) { ret = -1; break; }
        nrm = 0.0;
        for (int a = 0; a < D; ++a) nrm += fd.flow[a] * fd.flow[a];
        nrm = sqrt(nrm);
        if (nrm == 0) break;
        if (*len >= cap) { ret = -2; break; }
        const double inv2 = 1.0 / nrm;
        for (int a = 0; a < D; ++a) pts[*len * D + a] = pt[a] + (step * fd.flow[a]) * inv2;
        ++*len;
    }
    free(hist);
    free(cache.a);
    return ret;
}

static int64_t ode_all(const fmo_problem *grid, geo_flow_fn flow, void *ctx, const int64_t *seeds, int nseeds,
                       int ntips, const double *tips, double step, double causality, int64_t max_points,
                       double *points, int64_t *lengths, int *failed) {
    const int D = grid->ndim;
    int16_t *target = linf_distance(grid, seeds, nseeds, 6);
    if (!target) return -1;
    int64_t total = 0;
    for (int t = 0; t < ntips; ++t) {
        if (total >= max_points) { free(target); return -2; }
        double *pts = points + total * D;
        for (int a = 0; a < D; ++a) pts[a] = tips[(int64_t)t * D + a];
        int64_t len = 1;
        const int r = ode_run(grid, flow, ctx, target, step, causality, pts, max_points - total, &len);
        if (r == -1 || r == -2) { free(target); return r; }
        lengths[t] = len;
        failed[t] = r == 1;
        total += len;
    }
    free(target);
    return total;
}

int64_t fmo_geodesic_ode(const fmo_problem *p, const double *values, const uint64_t *active, int ntips,
                         const double *tips, double step, double causality, int64_t max_points, double *points,
                         int64_t *lengths, int *failed) {
    eul_ctx E = {p, values, active};
    return ode_all(p, eul_recompute, &E, p->seed_index, p->nseeds, ntips, tips, step, causality, max_points, points,
                   lengths, failed);
}

int64_t fmo_tti_geodesic_ode(const int64_t *dims, const double *h, const double *metric, const double *values,
                             const double *t_active, int nseeds, const int64_t *seed_index, int ntips,
                             const double *tips, double step, double causality, int64_t max_points, double *points,
                             int64_t *lengths, int *failed) {
    fmo_problem g;
    memset(&g, 0, sizeof(g));
    g.ndim = 3;
    for (int a = 0; a < 3; ++a) g.dims[a] = dims[a];
    tti_ctx T = {dims, h, metric, values, t_active};
    return ode_all(&g, tti_flow, &T, seed_index, nseeds, ntips, tips, step, causality, max_points, points, lengths,
                   failed);
}

/* ------------------------------------------------------------------------------------------ */
/* ReedsShepp3 on R^3 x S^2 (Headers/Specializations/Curvature3.h:11-70): axes x, y, z closed,
 * theta Sphere2_0 and phi Sphere2_1 (PeriodicGrid.hxx:120-186); one stencil per (theta, phi)
 * index, shared by the spatial points (HFM_StencilShare.hxx); eight symmetric differences. */

#define RS3_NSYM 8

int fmo_rs3_stencil(int ntheta, int nphi, double h, double xi, double eps, int dual, int8_t *offsets,
                    double *weights) {
    /* param.Setup(that, 2 pi / dims.back()) (Curvature3.h:61, HFM_ParamDefault.hxx:19-34) */
    const double ds = (2.0 * 3.141592653589793238462643383279502884) / (double)nphi;
    const double e2 = eps * eps;
    for (int it = 0; it < ntheta; ++it)
        for (int ip = 0; ip < nphi; ++ip) {
            const int cls = it * nphi + ip;
            int8_t *O = offsets + (int64_t)cls * RS3_NSYM * 5;
            double *W = weights + (int64_t)cls * RS3_NSYM;
            const double theta = (it + 0.5) * ds, phi = ip * ds;
            const double v[3] = {cos(theta), sin(theta) * cos(phi), sin(theta) * sin(phi)};
            /* m = (1 - eps^2) v v^T + eps^2 Id, or (eps^2 - 1) v v^T + Id for the dual model,
             * then / gridScale^2 (Curvature3.h:50-55), a division that multiplies every component
             * by the reciprocal (Vector::operator/=, LinearAlgebra/VectorType.h:37-42) */
            double d[6];
            const double a = dual ? (e2 - 1.0) : (1.0 - e2), b = dual ? 1.0 : e2, rh2 = 1.0 / (h * h);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j <= i; ++j) {
                    const double r = v[i] * v[j];
                    d[sym_index(i, j)] = (a * r + (i == j ? b : 0.0)) * rh2;
                }
            int8_t o3[18];
            double w3[6];
            memset(O, 0, RS3_NSYM * 5);
            if (fmo_selling_mat(3, d, o3, w3)) return -1;
            for (int k = 0; k < 6; ++k) {
                for (int c = 0; c < 3; ++c) O[5 * k + c] = o3[3 * k + c];
                W[k] = w3[k];
            }
            O[5 * 6 + 3] = 1;
            W[6] = 1.0 / ((xi * ds) * (xi * ds));
            O[5 * 7 + 4] = 1;
            const double sx = sin(theta) * xi * ds;
            W[7] = 1.0 / (sx * sx);
        }
    return 0;
}

/* PeriodizeNoBase on indices (PeriodicGrid.hxx:120-160): closed axes reject, theta reflects at
 * the poles into [0, ntheta) while phi turns by nphi / 2, phi wraps. Returns 0 outside. */
static int rs3_periodize(const int64_t *dims, int64_t *x, int *flip) {
    *flip = 0;
    for (int a = 0; a < 3; ++a)
        if (x[a] < 0 || x[a] >= dims[a]) return 0;
    const int64_t nt = dims[3], np = dims[4];
    int64_t t = x[3] % (2 * nt);
    if (t < 0) t += 2 * nt;
    if (t >= nt) {
        t = 2 * nt - t - 1;
        *flip = 1;
        x[4] += np / 2;
    }
    x[3] = t;
    int64_t ph = x[4] % np;
    if (ph < 0) ph += np;
    x[4] = ph;
    return 1;
}

static inline int64_t rs3_linear(const int64_t *dims, const int64_t *x) {
    int64_t r = 0;
    for (int a = 0; a < 5; ++a) r = r * dims[a] + x[a];
    return r;
}

typedef struct { int64_t key; int8_t o[5]; } rs3_pair;

static int rs3_pair_cmp(const void *a, const void *b) {
    const rs3_pair *x = (const rs3_pair *)a, *y = (const rs3_pair *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    for (int c = 0; c < 5; ++c)
        if (x->o[c] != y->o[c]) return x->o[c] < y->o[c] ? -1 : 1;
    return 0;
}

/* ReedsSheppForward3 (Curvature3.h:72-107): per class, 6 forward differences of Voronoi1Vec of
 * v = (cos theta, sin theta cos phi, sin theta sin phi) / gridScale (theta = pi (it + 1/2) / ntheta,
 * phi = 2 pi ip / nphi; the division multiplies by the reciprocal), then the theta and phi steps
 * (symmetric) of weights 1 / (xi ds)^2 and 1 / (sin(theta) xi ds)^2, ds = 2 pi / nphi. */
int fmo_rsf3_stencil(int ntheta, int nphi, double h, double xi, double eps, int8_t *offsets, double *weights) {
    const double pi = 3.141592653589793238462643383279502884;
    const double ds = (2.0 * pi) / (double)nphi;
    const double ih = 1.0 / h;
    for (int it = 0; it < ntheta; ++it)
        for (int ip = 0; ip < nphi; ++ip) {
            const int cls = it * nphi + ip;
            int8_t *O = offsets + (int64_t)cls * 8 * 5;
            double *W = weights + (int64_t)cls * 8;
            const double theta = pi * (it + 0.5) / (double)ntheta, phi = (2.0 * pi * ip) / (double)nphi;
            const double v[3] = {cos(theta) * ih, sin(theta) * cos(phi) * ih, sin(theta) * sin(phi) * ih};
            int8_t o3[18];
            double w3[6];
            memset(O, 0, 8 * 5);
            if (fmo_voronoi1vec(3, v, eps, o3, w3)) return -1;
            for (int k = 0; k < 6; ++k) {
                for (int c = 0; c < 3; ++c) O[5 * k + c] = o3[3 * k + c];
                W[k] = w3[k];
            }
            O[5 * 6 + 3] = 1;
            W[6] = 1.0 / ((xi * ds) * (xi * ds));
            O[5 * 7 + 4] = 1;
            const double sx = sin(theta) * xi * ds;
            W[7] = 1.0 / (sx * sx);
        }
    return 0;
}

int64_t fmo_s2_fast_marching(const int64_t *dims, int nfwd, int nsym, const int8_t *offsets,
                             const double *weights, const double *mult, int nseeds, const int64_t *seed_index,
                             const double *seed_value, double *values, uint64_t *active,
                             int *max_stencil_width) {
    const int nd = nfwd + nsym;
    const int64_t nt = dims[3], np = dims[4], ncls = nt * np;
    int64_t N = 1;
    for (int a = 0; a < 5; ++a) N *= dims[a];
    /* Reversed offsets (HFM_StencilShare.hxx:132-181): from the centre point of each class, the
     * offsets of non-zero weight whose target lies in the domain, pulled back through the
     * reflection (Transform::PullVector, PeriodicGrid.hxx:19-25), keyed by the target's class,
     * sorted and deduplicated */
    rs3_pair *pairs = (rs3_pair *)malloc((size_t)ncls * 2 * nd * sizeof(rs3_pair));
    if (!pairs) return -1;
    int64_t npairs = 0;
    for (int64_t cl = 0; cl < ncls; ++cl) {
        const int8_t *O = offsets + cl * nd * 5;
        const double *W = weights + cl * nd;
        for (int k = 0; k < nd; ++k) {
            if (W[k] == 0.0) continue;
            for (int sg = 1; sg >= -1; sg -= 2) {
                if (sg == -1 && k < nfwd) break;
                int64_t y[5] = {dims[0] / 2, dims[1] / 2, dims[2] / 2, cl / np, cl % np};
                int8_t e[5];
                for (int c = 0; c < 5; ++c) { e[c] = (int8_t)(sg * O[5 * k + c]); y[c] += e[c]; }
                int flip;
                if (!rs3_periodize(dims, y, &flip)) continue;
                if (flip) e[3] = (int8_t)(-e[3]);
                rs3_pair rp;
                rp.key = y[3] * np + y[4];
                memcpy(rp.o, e, 5);
                pairs[npairs++] = rp;
            }
        }
    }
    qsort(pairs, npairs, sizeof(rs3_pair), rs3_pair_cmp);
    int64_t nu = 0;
    for (int64_t i = 0; i < npairs; ++i)
        if (nu == 0 || rs3_pair_cmp(&pairs[nu - 1], &pairs[i]) != 0) pairs[nu++] = pairs[i];
    int64_t *split = (int64_t *)calloc(ncls + 1, sizeof(int64_t));
    if (!split) { free(pairs); return -1; }
    int mw = 0;
    for (int64_t i = 0; i < nu; ++i) {
        split[pairs[i].key + 1]++;
        int l1 = 0;
        for (int c = 0; c < 5; ++c) l1 += abs(pairs[i].o[c]);
        if (l1 > mw) mw = l1;
    }
    for (int64_t k = 0; k < ncls; ++k) split[k + 1] += split[k];
    if (max_stencil_width) *max_stencil_width = mw;

    uint8_t *accepted = (uint8_t *)calloc(N, 1);
    uint64_t *act = active ? active : (uint64_t *)calloc(N, sizeof(uint64_t));
    quad_t *quads = (quad_t *)calloc(N, sizeof(quad_t));
    heap_t heap = {0};
    if (!accepted || !act || !quads) return -1;
    if (active) memset(active, 0, N * sizeof(uint64_t));
    for (int64_t x = 0; x < N; ++x) values[x] = FMO_INF;
    for (int s = 0; s < nseeds; ++s) {
        values[seed_index[s]] = seed_value[s];
        heap_push(&heap, (qelem){seed_index[s], seed_value[s]});
    }
    int64_t nAccepted = 0;
    while (heap.n > 0) {
        /* RunOnce (HamiltonFastMarching.hxx:86-112) */
        const qelem top = heap_pop(&heap);
        if (accepted[top.idx]) continue;
        ++nAccepted;
        accepted[top.idx] = 1;
        int64_t aidx[5], r = top.idx;
        for (int a = 4; a >= 0; --a) { aidx[a] = r % dims[a]; r /= dims[a]; }
        const int64_t key = aidx[3] * np + aidx[4];
        for (int64_t ri = split[key]; ri < split[key + 1]; ++ri) {
            /* ConditionalUpdate (HamiltonFastMarching.hxx:136-154): updated = accepted - e, and the
             * offset pulled back through that periodization is the updated cell's own */
            int8_t e[5];
            memcpy(e, pairs[ri].o, 5);
            int64_t uidx[5];
            for (int a = 0; a < 5; ++a) uidx[a] = aidx[a] - e[a];
            int flip;
            if (!rs3_periodize(dims, uidx, &flip)) continue;
            if (flip) e[3] = (int8_t)(-e[3]);
            const int64_t u = rs3_linear(dims, uidx);
            if (accepted[u]) continue;
            if (act[u] == 0 && values[u] != FMO_INF) continue;
            if (values[u] <= top.val) continue;
            /* Update + HopfLaxUpdate (HFM_StencilShare.hxx:74-84, EulerianStencil.hxx:104-153) */
            quad_t *q = &quads[u];
            if (!q->used) { q->used = 1; q->minVal = top.val; q->a = 0; q->b = 0; q->c = -1; }
            const int64_t cl = uidx[3] * np + uidx[4];
            const int8_t *O = offsets + cl * nd * 5;
            const double *W = weights + cl * nd;
            const double m = mult ? mult[u] : 1.0;
            int bit = 0;
            for (int k = 0; k < nfwd; ++k, ++bit) {
                const int8_t *o = O + 5 * k;
                int pos = 1;
                for (int c = 0; c < 5; ++c) pos &= o[c] == e[c];
                if (pos) { act[u] |= 1ULL << bit; quad_add(q, top.val, mult ? W[k] * (m * m) : W[k]); }
            }
            for (int k = nfwd; k < nd; ++k, bit += 2) {
                const int8_t *o = O + 5 * k;
                int pos = 1, neg = 1;
                for (int c = 0; c < 5; ++c) { pos &= o[c] == e[c]; neg &= o[c] == -e[c]; }
                const double w = mult ? W[k] * (m * m) : W[k];
                if (pos && !(act[u] & (1ULL << (bit + 1)))) { act[u] |= 1ULL << bit; quad_add(q, top.val, w); }
                if (neg && !(act[u] & (1ULL << bit))) { act[u] |= 1ULL << (bit + 1); quad_add(q, top.val, w); }
            }
            values[u] = quad_solve(q);
            heap_push(&heap, (qelem){u, values[u]});
        }
    }
    free(heap.a);
    free(quads);
    free(accepted);
    if (!active) free(act);
    free(split);
    free(pairs);
    return nAccepted;
}
