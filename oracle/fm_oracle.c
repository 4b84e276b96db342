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
    quad_t *quads = (quad_t *)calloc(N, sizeof(quad_t));
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
    while (heap.n > 0) {
        /* RunOnce (HamiltonFastMarching.hxx:86-112) */
        const qelem top = heap_pop(&heap);
        if (accepted[top.idx]) continue;
        ++nAccepted;
        accepted[top.idx] = 1;
        index_of(p, top.idx, aidx);
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
            quad_t *q = &quads[u];
            if (!q->used) { q->used = 1; q->minVal = top.val; q->a = 0; q->b = 0; q->c = -1; }
            const int64_t sid = stencil_id(p, uidx, u);
            const int8_t *O = p->off + sid * nd * 3;
            const double *W = p->w + sid * nd;
            int bit = 0;
            for (int k = 0; k < p->nfwd; ++k, ++bit) {
                const int8_t *o = O + 3 * k;
                if (o[0] == e[0] && o[1] == e[1] && o[2] == e[2]) {
                    act[u] |= (1ULL << bit);
                    quad_add(q, top.val, diff_weight(p, W[k], u));
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
            const double val = quad_solve(q);
            values[u] = val;
            heap_push(&heap, (qelem){u, val});
        }
    }
    free(heap.a);
    free(quads);
    free(accepted);
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

int64_t fmo_backward_variation(const fmo_problem *p, const double *values, const uint64_t *active,
                               int npts, const int64_t *pt_index, const double *pt_weight,
                               double *sensitivity, int64_t max_seeds, int64_t *seed_out_index,
                               double *seed_out_weight) {
    const int64_t N = ncells(p);
    const int nd = p->nfwd + p->nsym;
    /* pending weight per cell; in_map marks membership of (values[x], x) in the ordered set */
    double *pend = (double *)calloc(N, sizeof(double));
    uint8_t *in_map = (uint8_t *)calloc(N, 1);
    bheap_t h = {0};
    if (!pend || !in_map) return -1;
    for (int64_t x = 0; x < N; ++x) sensitivity[x] = 0.0;
    for (int i = 0; i < npts; ++i) {
        const int64_t x = pt_index[i];
        if (x < 0 || x >= N) continue;
        if (in_map[x]) continue;  /* std::map::insert keeps the first weight */
        in_map[x] = 1; pend[x] = pt_weight[i];
        bheap_push(&h, (bkey){values[x], x});
    }
    int64_t nseeds = 0;
    int64_t idx[3], nidx[3];
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
        /* ValueVariation */
        index_of(p, x, idx);
        const double value = values[x];
        const int64_t sid = stencil_id(p, idx, x);
        const int8_t *O = p->off + sid * nd * 3;
        const double *W = p->w + sid * nd;
        const uint64_t act = active[x];
        double var = 0.0, weightSum = 0.0;
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
                    var += w * valueDiff;
                }
            }
            bit += (k2 < p->nfwd) ? 1 : 2;
        }
        if (nn == 0) {
            if (nseeds < max_seeds) { seed_out_index[nseeds] = x; seed_out_weight[nseeds] = weight; }
            ++nseeds;
        }
        if (weightSum != 0.0) {
            const double inv = 1.0 / weightSum;
            for (int j = 0; j < nn; ++j) nb_w[j] *= inv;
            var = p->mult ? inv * (p->mult[x] * var) : inv * var;
        }
        sensitivity[x] = weight * var;
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
