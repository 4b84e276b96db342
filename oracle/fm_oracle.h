/* CPU restatement of the reference solve path (test infrastructure, never shipped).
 *
 * This oracle restates, in plain C99, the arithmetic of the reference's sequential fast-marching
 * path for Eulerian schemes so that tests can check the CUDA path against it in-process:
 *   - Selling / Voronoi stencil construction (2D and 3D), Riemann metric rescaling, the
 *     relaxed rank-one (Voronoi1Vec) stencils of the curvature models;
 *   - wall distance and line-of-sight visibility;
 *   - Dijkstra-ordered fast marching with the incremental Hopf-Lax quadratic solve, using the
 *     same binary-heap algorithm as libstdc++'s std::priority_queue so that tie order matches;
 *   - the reverse-mode first variation (costSensitivity).
 * Each function cites the reference file:line it follows. Compiled with -ffp-contract=off.
 */
#ifndef HFM_FM_ORACLE_H
#define HFM_FM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Selling decomposition of a packed SPD matrix (xx,xy,yy[,xz,yz,zz]) into 3 (2D) or 6 (3D)
 * integer offsets and weights, including the 1000*eps*Tr tolerance. Returns 0, or -1 if the
 * matrix is rejected (non positive determinant/trace) or Selling did not terminate. */
int fmo_selling_mat(int ndim, const double *d, int8_t *offsets, double *weights);

/* Riemann stencil at one point: packed metric (or dual metric), grid scales h[ndim]. */
int fmo_riemann_stencil(int ndim, const double *metric, int dual, const double *h,
                        int8_t *offsets, double *weights);

/* Voronoi1Vec: relaxed rank-one decomposition with reorientation (<v,e> <= 0). */
int fmo_voronoi1vec(int ndim, const double *v, double eps, int8_t *offsets, double *weights);

/* Per-angle stencil tables of the curvature models, nd = 3 components per offset.
 * ReedsShepp2: 4 symmetric differences per angle. Elastica2<5>: 27 forward differences. */
int fmo_reedsshepp2_table(int ntheta, double h, double xi, double eps, int projective,
                          int8_t *offsets, double *weights);
int fmo_elastica2_table(int ntheta, double h, double xi, double eps,
                        int8_t *offsets, double *weights);
/* ReedsSheppForward2: 3 forward differences then 1 symmetric (angular) per angle.
 * Dubins2: 12 forward differences per angle, two stencils of 6 (nmax = 2). */
int fmo_dubins2_table(int ntheta, double h, double xi, double eps, int8_t *offsets, double *weights);
int fmo_reedssheppforward2_table(int ntheta, double h, double xi, double eps,
                                 int8_t *offsets, double *weights);

typedef struct {
    int ndim;
    int64_t dims[3];
    int periodic[3];
    int nfwd, nsym;            /* differences per stencil: forward first, then symmetric */
    int share;                 /* 0: one stencil per cell, 1: one stencil per index of the last axis */
    const int8_t *off;         /* [nstencil][nfwd+nsym][3] */
    const double *w;           /* [nstencil][nfwd+nsym] base weights */
    const double *mult;        /* [N] speed multiplier (weights scale by mult^2) or NULL */
    const uint8_t *walls;      /* [N] or NULL */
    int nseeds;
    const int64_t *seed_index; /* row-major linear indices */
    const double *seed_value;
    /* stopping criteria (Headers/ExtraAlgorithms/CommonStoppingCriteria.h:58-93); a zeroed field
     * is no criterion: stop_at_distance is used when has_stop_at_distance, n_max_accepted when > 0;
     * stop_any / stop_all are cells, the _u variants (x, y) pairs packed as x * dims[1] + y. */
    int has_stop_at_distance;
    double stop_at_distance;
    int64_t n_max_accepted;
    int nstop_any, nstop_all, nstop_any_u, nstop_all_u;
    const int64_t *stop_any, *stop_all, *stop_any_u, *stop_all_u;
    /* Diagonal models: the first variation is per axis (a speed vector per cell): var_dim = ndim
     * and mult_vec[N][var_dim] the speeds; 0 (or 1) and NULL otherwise. */
    int var_dim;
    const double *mult_vec;
    /* nmax = 2: the forward differences form two stencils of nfwd / 2 each and the value is the
     * smaller of their two solutions (EulerianStencil<.., nMax = 2>, EulerianStencil.hxx:13-50,
     * 104-153); activeNeighs bit nfwd records which one, and a Recompute (geodesics, first
     * variations) uses that stencil only. 0 or 1: one stencil. */
    int nmax;
    /* Static factoring of TTI3 (StaticFactoring.hxx:33-64): over the box of cells
     * [fac_lo, fac_lo + fac_dims), factor values, adimensional gradients [3] and mask; a neighbour
     * value u(x + e) read by the update of a masked cell x of the box becomes
     * u(x + e) + <grad(x), e> + (value(x) - value(x + e)), the parenthesis 0 when x + e leaves a
     * subdomain box. fac_values NULL: none. Read by fmo_tti_fast_marching_stop. */
    const double *fac_values, *fac_grads;
    const uint8_t *fac_mask;
    int fac_lo[3], fac_dims[3];
    int fac_subdomain;
} fmo_problem;

/* Fast marching. values[N] out; active[N] out (bitset, forward bits then symmetric +/- pairs,
 * as the reference's ActiveNeighFlagType) may be NULL. Returns the number of cells popped from the
 * queue and examined (the reference's nAccepted: with a stopping criterion this counts the cell
 * that stopped the run, which is not accepted), or -1. */
int64_t fmo_fast_marching(const fmo_problem *p, double *values, uint64_t *active,
                          int *max_stencil_width);

/* Reverse first variation from weighted points (linear indices). sensitivity[N][max(1, var_dim)] out;
 * seed_out_index/seed_out_weight receive up to max_seeds sensitive seeds. Returns the number of
 * sensitive seeds, or -1. */
int64_t fmo_backward_variation(const fmo_problem *p, const double *values, const uint64_t *active,
                               int npts, const int64_t *pt_index, const double *pt_weight,
                               double *sensitivity, int64_t max_seeds, int64_t *seed_out_index,
                               double *seed_out_weight);

/* Wall distance (capped BFS) and visibility, exposed for tests of the visibility kernel.
 * visible[N][nfwd + 2*nsym] receives 1 if the neighbour (x+e) may update x. */
int fmo_visibility(const fmo_problem *p, int max_width, uint8_t *visible);

/* TTI3 (semi-Lagrangian, nmix = 0): metric[N][14] = linear(2), quadratic (xx,xy,yy), transform
 * 3x3 read row by row (transform(i, j) at element 5 + 3 i + j); h[3] grid scales. values[N] out, t_active[N] (may be NULL) receives the
 * reference's activeNeighs encoding (t of the extremum, negative at an interval endpoint).
 * Returns the accepted count, or -1. */
int64_t fmo_tti_fast_marching(const int64_t *dims, const double *h, const double *metric, int nseeds,
                              const int64_t *seed_index, const double *seed_value, double *values,
                              double *t_active);
/* The same with stopping criteria: the stop_* fields of `stop` (NULL: none). */
int64_t fmo_tti_fast_marching_stop(const int64_t *dims, const double *h, const double *metric, int nseeds,
                                   const int64_t *seed_index, const double *seed_value, double *values,
                                   double *t_active, const fmo_problem *stop);
/* Reverse first variation of the TTI3 solve (semi-Lagrangian ValueVariation), from the values and
 * t_active of fmo_tti_fast_marching. Returns the number of sensitive seeds, or -1. */
int64_t fmo_tti_backward_variation(const int64_t *dims, const double *h, const double *metric,
                                   const double *values, const double *t_active, int npts,
                                   const int64_t *pt_index, const double *pt_weight, double *sensitivity,
                                   int64_t max_seeds, int64_t *seed_out_index, double *seed_out_weight);
/* Properties of one TTI norm: out = {tmin, tmax, optimDirection, Multiplier(tmin), Multiplier(tmax)}. */
int fmo_tti_norm(const double *metric, const double *h, double *out);
/* Fixed-point form of the (factored) TTI update over finished values; see fm_oracle.c. */
int fmo_tti_prefix_solve(const int64_t *dims, const double *h, const double *metric, const double *values,
                         const uint8_t *is_seed, const fmo_problem *fac, double *out);
int fmo_tti_prefix_fixed_point(const int64_t *dims, const double *h, const double *metric, double *values,
                               const uint8_t *is_seed, const fmo_problem *fac, int max_sweeps);

/* Discrete geodesic backtracking from ntips tips (dimensionless coordinates: cell i spans [i, i+1)),
 * from the values and activeNeighs of fmo_fast_marching. points[max_points][ndim] receive the
 * concatenated geodesics (dimensionless), lengths[ntips] their lengths, failed[ntips] 1 where the
 * restart limit was reached. Returns the total number of points, -1 on allocation failure, -2 if
 * max_points is too small. */
int64_t fmo_geodesic_discrete(const fmo_problem *p, const double *values, const uint64_t *active, int ntips,
                              const double *tips, double step, double threshold, double volume_bound,
                              int64_t max_points, double *points, int64_t *lengths, int *failed);
int64_t fmo_tti_geodesic_discrete(const int64_t *dims, const double *h, const double *metric, const double *values,
                                  const double *t_active, int ntips, const double *tips, double step,
                                  double threshold, double volume_bound, int64_t max_points, double *points,
                                  int64_t *lengths, int *failed);
/* Geodesic flow per cell (sum of Recompute weight * offset, dimensionless) with the Recompute value
 * and width (value, width may be NULL). */
int fmo_geodesic_flow(const fmo_problem *p, const double *values, const uint64_t *active, double *flow,
                      double *value, double *width);
/* Forward first variation: result [N][nvar] holds the seed value variations on entry and the
 * valueVariation on return; cost_var [N][nvar][max(1, var_dim)] or NULL. Returns 0, or -1 on
 * allocation failure. */
int fmo_forward_variation(const fmo_problem *p, const double *values, const uint64_t *active, int nvar,
                          const double *cost_var, double *result);
int fmo_tti_forward_variation(const int64_t *dims, const double *h, const double *metric, const double *values,
                              const double *t_active, int nvar, const double *cost_var, double *result);
/* ODE geodesic solver (midpoint scheme on the interpolated flow) from the same inputs as
 * fmo_geodesic_discrete; causality = geodesicCausalityTolerance. failed[t] = 1 where the solver
 * stalled. Returns the total number of points, -1 on allocation failure, -2 if max_points is too
 * small. The TTI variant takes the seed cells explicitly. */
int64_t fmo_geodesic_ode(const fmo_problem *p, const double *values, const uint64_t *active, int ntips,
                         const double *tips, double step, double causality, int64_t max_points, double *points,
                         int64_t *lengths, int *failed);
int64_t fmo_tti_geodesic_ode(const int64_t *dims, const double *h, const double *metric, const double *values,
                             const double *t_active, int nseeds, const int64_t *seed_index, int ntips,
                             const double *tips, double step, double causality, int64_t max_points, double *points,
                             int64_t *lengths, int *failed);
int fmo_tti_geodesic_flow(const int64_t *dims, const double *h, const double *metric, const double *values,
                          const double *t_active, double *flow, double *value, double *width);

/* ReedsShepp3 / ReedsSheppForward3 (Headers/Specializations/Curvature3.h:11-107) on dims
 * (x, y, z, theta, phi), RowMajor. The stencil builders fill, per class (theta, phi) =
 * it * nphi + ip, 8 differences: offsets [ncls][8][5] and weights [ncls][8] (ReedsShepp3: 8
 * symmetric; ReedsSheppForward3: 6 forward, then 2 symmetric). fmo_s2_fast_marching: mult [N]
 * (speed; weights scale by its square) or NULL; seeds as increasing unique row-major indices.
 * Returns nAccepted, or -1. */
int fmo_rs3_stencil(int ntheta, int nphi, double h, double xi, double eps, int dual, int8_t *offsets,
                    double *weights);
int fmo_rsf3_stencil(int ntheta, int nphi, double h, double xi, double eps, int8_t *offsets, double *weights);
int64_t fmo_s2_fast_marching(const int64_t *dims, int nfwd, int nsym, const int8_t *offsets,
                             const double *weights, const double *mult, int nseeds, const int64_t *seed_index,
                             const double *seed_value, double *values, uint64_t *active,
                             int *max_stencil_width);

#ifdef __cplusplus
}
#endif
#endif
