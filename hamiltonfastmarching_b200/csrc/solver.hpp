// Host interface of the GPU solve path for Eulerian schemes (Riemann, ReedsShepp2, Elastica2).
//
// The host orchestration (run.cpp) turns hfmIn keys into an EulerProblem; solve_eulerian builds the
// stencils on the GPU, computes wall visibility, runs the tiled fast-iterative solver to the
// upwind fixed point of the reference's fast marching, and returns the arrival times.
#pragma once

#include <cstdint>
#include <string>
#include <memory>
#include <utility>
#include <vector>

namespace hfm {

enum class StencilKind {
    RiemannPerCell,   // Selling stencil of a metric at every cell (Recomp policy)
    SharedByTheta,    // one stencil per index of the last axis times a speed multiplier (Share policy)
    TTI,              // TTI3 norm per cell, semi-Lagrangian Selling-path update (Lag2 policy); metric has 14 values
};

// Stencil slots of a TTI3 cell: the distinct offsets of its Selling path (at most 8 were met on
// Thomsen media with eps, delta <= 0.2; a longer path is reported as an error).
constexpr int kTTISlots = 10;

struct EulerProblem {
    int ndim = 2;
    int dims[3] = {1, 1, 1};
    int periodic[3] = {0, 0, 0};
    bool fp64 = true;
    StencilKind kind = StencilKind::RiemannPerCell;

    // RiemannPerCell: packed metric (xx,xy,yy[,xz,yz,zz]) RowMajor, one per cell or a single one.
    std::vector<double> metric;
    const double *metric_ptr = nullptr;  // used instead of `metric` when set (host, not owned)
    size_t metric_len = 0;
    bool metric_constant = false;
    bool dual = false;
    // Diagonal2/3: `metric` holds ndim speeds (or costs, mult_inverse) per cell instead of a
    // packed matrix; the stencil is one symmetric difference per axis.
    bool diagonal = false;
    double h[3] = {1, 1, 1};

    // SharedByTheta: nclass stencils of nfwd forward + nsym symmetric differences, one per index of
    // the last axis; `angular` when that axis is an angle (curvature models; the isotropic models
    // repeat one axis-aligned stencil on every index of the last axis).
    bool angular = true;
    int nfwd = 0, nsym = 0, nclass = 0;
    int nmax = 1;                      // 2: two groups of nfwd/2 forward differences (Dubins2)
    std::vector<int8_t> cls_off;       // [nclass][nfwd+nsym][3]
    std::vector<double> cls_w;         // [nclass][nfwd+nsym]
    std::vector<uint8_t> cls_enabled;  // [nclass][nfwd+2*nsym] slot reachable from the class centre
    // ReedsShepp3 (R^3 x S^2): the grid (x, y, z, theta, phi) is held as the 3-D grid
    // (x, y, (z * sphere_nth + theta) * sphere_nph + phi); the classes are the (theta, phi) pairs
    // and cls_ang [nclass][nsym][2] holds the theta and phi steps of each difference (cls_off the
    // x, y, z steps). 0: no sphere bundle.
    int sphere_nth = 0, sphere_nph = 0;
    std::vector<int8_t> cls_ang;
    // Speed multiplier of the shared stencils, given compactly as in the reference's lifted scalar
    // fields (HFMInterface.hxx:23-32): depth 0 (one value), 1 (per angle), 2 (per physical point
    // x,y) or 3 (per cell), RowMajor at mult_ptr (host, not owned, or `mult` when null); the cost
    // form (mult_inverse) is turned into a speed 1/cost on the device (DataSource_Inverse).
    std::vector<double> mult;
    const double *mult_ptr = nullptr;
    int mult_depth = 3;
    bool mult_inverse = false;

    std::vector<uint8_t> walls;        // [N] or empty
    const double *walls_f64 = nullptr; // [N] host view of a full walls field (nonzero = wall), instead of `walls`
    // Device-resident alternatives (zero-copy path): used instead of `metric` / `walls` when set,
    // and `d_values_out` receives the FP64 arrival times instead of EulerResult::values.
    const double *d_metric = nullptr;
    const uint8_t *d_walls = nullptr;
    double *d_values_out = nullptr;
    double *h_values_out = nullptr;   // host destination of the arrival times instead of EulerResult::values
    std::vector<int64_t> seed_index;   // sorted, unique
    std::vector<double> seed_value;

    // Static factoring (TTI3): over the box of cells [fac_lo, fac_lo + fac_dims), the factor values
    // and their adimensional gradients; a neighbour value u(x + e) read by the update of a cell x of
    // the box (and of the mask) becomes u(x + e) + <grad(x), e> + value(x) - value(x + e), the last
    // two terms from the box (0 when x + e leaves a subdomain box), StaticFactoring.hxx:33-64.
    std::vector<double> fac_values;    // [box cells] RowMajor
    std::vector<double> fac_grads;     // [box cells][3]
    std::vector<uint8_t> fac_mask;     // [box cells]
    int fac_lo[3] = {0, 0, 0}, fac_dims[3] = {0, 0, 0};
    bool fac_subdomain = false;
    bool has_factoring() const { return !fac_values.empty(); }

    bool want_active = false;          // export the activeNeighs bitsets
    // Reverse first variation: groups of (linear index, weight) points (inspectSensitivity).
    std::vector<std::vector<int64_t>> adjoint_index;
    std::vector<std::vector<double>> adjoint_weight;
    bool want_stencils = false;        // export per-cell offsets/weights (RiemannPerCell)
    bool retain = false;               // keep the device state for later reverse sweeps (single instance)
    // Geodesic backtracking (tips, tips_Unoriented) from the solved arrival times, in dimensionless
    // coordinates (cell i spans [i, i+1) on every axis): geo_tips [n][ndim]; geo_tips_unoriented
    // [n][2] (x, y) whose angle is chosen on the device; the discrete solver's parameters.
    std::vector<double> geo_tips, geo_tips_unoriented;
    double geo_step = 0.25, geo_threshold = 1e-3, geo_volume_bound = 8.45;
    bool geo_ode = false;              // geodesicSolver 'ODE' instead of 'Discrete'
    double geo_causality = 4.0;        // geodesicCausalityTolerance (ODE)
    bool want_geodesic_flow = false;   // exportGeodesicFlow
    // Forward first variation (costVariation, seedValueVariation): fwd_nvar variations; fwd_cost
    // [N][nvar] RowMajor or empty; seed cells and their value variations [n][nvar], later entries
    // overwriting earlier ones.
    // Stopping criteria (stopAtDistance, nMaxAccepted, stopWhenAny/AllAccepted; the _Unoriented
    // forms give (x, y) columns packed as x * dims[1] + y); single instances of Eulerian models.
    bool has_stop_distance = false;
    double stop_distance = 0.0;
    int64_t stop_n_max = 0;
    std::vector<int64_t> stop_any, stop_all, stop_any_u, stop_all_u;
    bool has_stopping() const {
        return has_stop_distance || stop_n_max > 0 || !stop_any.empty() || !stop_all.empty() ||
               !stop_any_u.empty() || !stop_all_u.empty();
    }
    // Bypass of the solve (values and activeNeighs given, HFMInterface.hxx:399-427): the arrival
    // times are taken as given [N] (geodesics and first variations are computed from them).
    bool bypass = false;
    std::vector<double> bypass_values;
    int fwd_nvar = 0;
    std::vector<double> fwd_cost;
    std::vector<int64_t> fwd_seed_cell;
    std::vector<double> fwd_seed_value;
    int tile_shift[3] = {-1, -1, -1};  // log2 tile extents per axis (sum 6); -1: 8x8 / 4x4x4
    int sweeps_per_tile = 4;           // local Jacobi sweeps before a tile re-queues itself
    int max_rounds = 1 << 20;
    // Value-ordered scheduling: a round solves the tiles whose wake-up key is within a band above
    // the smallest key; the band adapts to keep [band_lo, band_hi] x (resident warps) tiles per round.
    bool ordered = true;
    double band_lo = 2.0, band_hi = 8.0;
};

// FirstVariation::BackwardVariation output for one group of inspected points.
struct AdjointResult {
    std::vector<double> sensitivity;   // costSensitivity, RowMajor
    std::vector<int64_t> seed_index;   // sensitive seeds, by decreasing (value, index)
    std::vector<double> seed_weight;
};

struct EulerResult;

// Device state of a solve kept for later reverse sweeps (EulerProblem::retain): the stencils and
// arrival times stay in device memory, so a sensitivity for new inspection weights costs one
// reverse sweep instead of a new solve.
struct RetainedSolve {
    virtual ~RetainedSolve() = default;
    // Reverse first variation of the retained solve for the groups of p.adjoint_index.
    virtual void adjoint(const EulerProblem &p, EulerResult &res) = 0;
};

struct EulerResult {
    std::vector<double> values;        // RowMajor, +inf where unreached
    std::vector<uint64_t> active;      // activeNeighs bitsets (if requested)
    std::vector<int8_t> stencil_off;   // [N][K][3] (if requested)
    std::vector<double> stencil_w;     // [N][K]
    int64_t n_accepted = 0;
    int max_stencil_width = 0;
    std::vector<AdjointResult> adjoints;
    // Geodesics of geo_tips ([0]) and geo_tips_unoriented ([1]): concatenated dimensionless points,
    // the length, status bits (1: restart limit reached; 2, 4: overflow; 8: iteration limit;
    // 16: index range) and restarts of each.
    std::vector<double> geo_points[2];
    std::vector<int64_t> geo_lengths[2];
    std::vector<int> geo_status[2], geo_restarts[2];
    std::vector<double> geodesic_flow;  // [N][ndim] sum of Recompute weight * offset (dimensionless)
    std::vector<double> value_variation;  // [N][fwd_nvar] forward first variation
    double t_stencil_ms = 0, t_solve_ms = 0, t_adjoint_ms = 0, t_geodesic_ms = 0, t_total_ms = 0;
    long long rounds = 0, tile_activations = 0, local_solves = 0;
    long long tile_carries = 0;  // list entries passed on to the next round (key above the band)
    std::shared_ptr<RetainedSolve> retained;  // set when EulerProblem::retain (single instance)
};

void solve_eulerian(const EulerProblem &p, EulerResult &r);
// Default schedule of a family (local sweeps per activation and band limits), measured on B200:
// Riemann3 2 sweeps, band [1,4]; Riemann2 3, [2,8]; ReedsShepp2 4, [2,8]; Elastica2 2, [4,16];
// TTI3 1, [1,4]. Callers override it with tileSweeps / bandLo / bandHi (or the autotuner).
void default_schedule(EulerProblem &p);
// One launch sequence for many instances of one model family and precision (a global tile space
// over all instances, one persistent solver launch). Results are in the order of `probs`.
void solve_eulerian_batch(const std::vector<const EulerProblem *> &probs, std::vector<EulerResult> &results);

// Device copies of a request's large inputs (metric or speed multiplier, walls), uploaded ahead of
// its admission by another thread while the solver runs (stage_resident_inputs).
struct StagedInputs {
    virtual ~StagedInputs() = default;
    virtual size_t bytes() const = 0;
};
// Issues the uploads on the calling thread's current stream and returns once the host sources have
// been read; admission waits for the copies on its own stream.
std::unique_ptr<StagedInputs> stage_resident_inputs(const EulerProblem &p);

// Resident solver of one model family for the serving loop (resident.cuh): admitted instances live
// in a device arena and one persistent solver runs them in slices; each instance is released as
// soon as its own tiles drain. All calls come from one thread. The slice runs on the thread's
// current stream; prepare() and finish() take their own stream and may run while a slice of this
// family is in flight: they only touch arena ranges that the running solver does not read.
class ResidentFamily {
public:
    enum Admit { kPrepared, kNoSlot, kNeedsGrow };
    virtual ~ResidentFamily() = default;
    // Builds `p` in the arena on stream `s` (stencils, walls, visibility, seeds, tile
    // dependencies, slot) from the staged inputs when given; it joins the solver's lists at the
    // next activate(). kNeedsGrow: the arena is full and `may_grow` is false (a slice is running).
    // Throws Error for an invalid instance (nothing of it stays resident).
    virtual Admit prepare(const EulerProblem &p, int64_t ticket, const StagedInputs *staged, bool may_grow,
                          cudaStream_t s, int *max_width) = 0;
    // Seed tiles of the prepared instances into the lists (no slice running).
    virtual void activate() = 0;
    // Launches a slice: the solver runs until an instance converges, every tile is done, the
    // attention word (device view of host memory, may be null) is raised after min_ms, or max_ms
    // (0: no limit) has passed. slice_done() polls it; slice_end() waits for it and throws Error
    // when the solver failed.
    virtual void slice_begin(const volatile unsigned *attn_dev, double min_ms, double max_ms) = 0;
    virtual bool slice_done() = 0;
    virtual void slice_end() = 0;
    // Converged instances (no slice running): they leave the lists; their tickets are appended.
    virtual void collect(std::vector<int64_t> &done) = 0;
    // Result of a collected instance (values, nAccepted, MaxStencilWidth, times), copied out on
    // stream `s` into its output field; then its arena range and slot are free.
    virtual void finish(int64_t ticket, EulerResult &res, cudaStream_t s) = 0;
    // Drops every instance (prepared, running or collected) after a failure of the solver; their
    // tickets are appended.
    virtual void abandon(std::vector<int64_t> &tickets) = 0;
    virtual bool has_work() const = 0;     // instances in the lists
    virtual bool has_pending() const = 0;  // prepared instances waiting for activate()
    virtual int resident() const = 0;
    virtual size_t arena_bytes() const = 0;
};
// A store's request parsed for the serving loop (the part of Run before the solver loop), and the
// exports that finish it (run.cu): the same keys, defaults, messages and usage report as hfm_run.
struct PreparedRun {
    virtual ~PreparedRun() = default;
    virtual EulerProblem &problem() = 0;
    virtual bool skip() const = 0;    // no seeds and nothing cached: nothing to solve
    // Exports a solve's results into the store and closes the request (usage report).
    virtual void finish(const EulerResult &r) = 0;
    // Closes a failed request: drops a partly created output field.
    virtual void fail() = 0;
};

}  // namespace hfm
struct hfm_io;
namespace hfm {
std::unique_ptr<PreparedRun> prepare_run(hfm_io *io);

// Family of a problem for the resident solver ("" when it is solved through the batch path:
// other models, or outputs beyond the arrival times), and a new resident solver for it.
std::string resident_family_key(const EulerProblem &p);
std::unique_ptr<ResidentFamily> make_resident_family(const EulerProblem &p);

// Curvature model stencil tables built on the host with the C library's cos/sin
// (Headers/Specializations/Curvature2.h:48-66, 86-100, 178-234, CommonTraits.h:118-161).
void reedsshepp2_table(int ntheta, double h, double xi, double eps, bool projective,
                       std::vector<int8_t> &off, std::vector<double> &w);
// ReedsShepp3 classes (theta, phi) = it * nphi + ip: x, y, z steps [ncls][8][3], theta and phi
// steps [ncls][8][2], weights [ncls][8].
void reedsshepp3_table(int nth, int nph, double h, double xi, double eps, bool dual, std::vector<int8_t> &off,
                       std::vector<int8_t> &ang, std::vector<double> &w);
// ReedsSheppForward3: the same layout, 6 forward differences then the 2 angular ones.
void reedssheppforward3_table(int nth, int nph, double h, double xi, double eps, std::vector<int8_t> &off,
                              std::vector<int8_t> &ang, std::vector<double> &w);
void elastica2_table(int ntheta, double h, double xi, double eps, std::vector<int8_t> &off,
                     std::vector<double> &w);
void reedssheppforward2_table(int ntheta, double h, double xi, double eps, std::vector<int8_t> &off,
                              std::vector<double> &w);
void dubins2_table(int ntheta, double h, double xi, double eps, std::vector<int8_t> &off, std::vector<double> &w);

}  // namespace hfm
