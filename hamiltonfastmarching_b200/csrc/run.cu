// hfm_run: the reference's Run(IO&) for the GPU solve path, and the C ABI of include/hfm_b200.h.
//
// Orchestration mirrors HFMInterface<T>::Run (Headers/Base/Implementation/HFMInterface.hxx:296-579):
// set up IO (verbosity, arrayOrdering), read the model's fields (Riemannian.h:46-61,
// Curvature2.h:61-66 and 219-224, HFM_StencilShare.hxx:61-71), place seeds (StaticFactoring.hxx:242-393),
// solve, export values / activeNeighs / sensitivities, then IO::UsageReport (BaseIO.hxx:64-104).
// Options outside the GPU path fail with HFM_ERR_UNSUPPORTED instead of being ignored.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <limits>
#include <set>
#include <sstream>
#include <thread>

#include "common.cuh"
#include "io.hpp"
#include "selling.cuh"
#include "store_handle.hpp"
#include "solver.hpp"


namespace hfm {
namespace {

const double kPi = 3.141592653589793238462643383279502884;

struct Param {
    int ndim = 2;
    int dims[5] = {1, 1, 1, 1, 1};
    int periodic[5] = {0, 0, 0, 0, 0};
    double origin[5] = {0, 0, 0, 0, 0};
    double scale[5] = {1, 1, 1, 1, 1};  // grid scale per axis (dependScale on the angular axes)
    int sphere = -1;  // axis of a Sphere2_0 / Sphere2_1 pair (theta, phi: ReedsShepp3), or -1
    // point -> index (HFM_ParamDefault.hxx ADim + BaseGrid::IndexFromPoint + PeriodizeNoBase,
    // PeriodicGrid.hxx:120-160: closed axes reject, theta reflects at the poles while phi turns by
    // half a circle, periodic axes wrap)
    bool index_of(const double *p, int64_t *lin) const {
        long long idx[5];
        for (int a = 0; a < ndim; ++a) idx[a] = (long long)std::floor((p[a] - origin[a]) / scale[a]);
        int64_t r = 0;
        for (int a = 0; a < ndim; ++a) {
            long long i = idx[a];
            if (a == sphere) {
                const long long n2 = 2LL * dims[a];
                i %= n2;
                if (i < 0) i += n2;
                if (i >= dims[a]) {
                    i = n2 - i - 1;
                    idx[a + 1] += dims[a + 1] / 2;
                }
            } else if (periodic[a] || (sphere >= 0 && a == sphere + 1)) {
                i %= dims[a];
                if (i < 0) i += dims[a];
            } else if (i < 0 || i >= dims[a]) {
                return false;
            }
            r = r * dims[a] + i;
        }
        *lin = r;
        return true;
    }
};

std::vector<int> read_dims(Store &io, int ndim) {
    int64_t n = 0;
    std::vector<double> d = io.get_vector("dims", 1, &n);
    if ((int)n != ndim)
        throw Error(HFM_ERR_VALUE, "dims must have " + std::to_string(ndim) + " entries, found " + std::to_string(n));
    std::vector<int> out(ndim);
    for (int a = 0; a < ndim; ++a) {
        out[a] = (int)d[a];
        if (out[a] <= 0) throw Error(HFM_ERR_VALUE, "BaseGrid error : domain size must be positive");
    }
    return out;
}

std::vector<double> read_point(Store &io, const std::string &key, int n, const std::vector<double> &def) {
    if (!io.has_field(key)) {
        std::ostringstream o;
        o << "{";
        for (int i = 0; i < n; ++i) o << (i ? "," : "") << def[i];
        o << "}";
        if (io.verbosity >= 1) io.msg("Field " + key + " defaults to " + o.str() + "\n");
        io.get_scalar(key, 0.0, 99);  // record as defaulted (message already printed)
        return def;
    }
    const RawElement &r = io.raw(key);
    if (r.dims.size() != 1 || r.dims[0] != n)
        throw Error(HFM_ERR_VALUE, "Field " + key + " must be a vector of " + std::to_string(n) + " entries");
    return std::vector<double>(r.ptr(), r.ptr() + r.count());
}

void reject_unsupported(Store &io) {
    static const char *keys[] = {"speed_times", "cost_times", "metric_times", "dualMetric_times",
                                 "euclideanScale", "seedFlags"};
    for (const char *k : keys)
        if (io.has_field(k))
            throw Error(HFM_ERR_UNSUPPORTED, std::string("option '") + k + "' is not supported by the GPU solve path");
    if (io.has_field("order") && io.get_scalar("order") != 1)
        throw Error(HFM_ERR_UNSUPPORTED, "only order=1 is supported by the GPU solve path");
    if (io.get_scalar("exportActiveOffsets", 0.0, 3) != 0)
        throw Error(HFM_ERR_UNSUPPORTED, "exportActiveOffsets is not supported by the GPU solve path");
    if (io.get_scalar("refineStencilAtWallBoundary", 0.0, 3) != 0)
        throw Error(HFM_ERR_UNSUPPORTED, "refineStencilAtWallBoundary is not supported by the GPU solve path");
}

// Distance guess of the seed spreading (StaticFactoring.hxx:285-346): the model's norm at a cell,
// or interpolated at a point over its 2^D grid neighbours with the reference's unnormalised
// weights (BaseGrid.h:79-101, PeriodicGrid.hxx Neighbors, MapWeightedSum.h): a symmetric matrix
// in grid units for Riemann metrics (Riemannian.h:62-71: the metric, inverted if dual, times
// h_i h_j), a diagonal d_i = h_i / speed_i for the isotropic and diagonal models (Isotropic.h),
// the 14 TTI3 metric elements with the transform's columns scaled by h_j (TTI.hpp:22-46).
struct SeedGuess {
    const EulerProblem &p;
    const Param &pm;
    int ns() const {
        if (p.kind == StencilKind::TTI) return 14;
        return p.kind == StencilKind::RiemannPerCell && !p.diagonal ? pm.ndim * (pm.ndim + 1) / 2 : pm.ndim;
    }
    // raw model data at a cell: packed metric, speed vector (diagonal) or speed (isotropic)
    void raw(int64_t cell, double *out) const {
        const int D = pm.ndim;
        if (p.kind == StencilKind::TTI) {
            const double *src = p.metric_ptr ? p.metric_ptr : p.metric.data();
            const double *m = src + (p.metric_constant ? 0 : cell * 14);
            for (int k = 0; k < 14; ++k) out[k] = m[k];
        } else if (p.kind == StencilKind::RiemannPerCell) {
            const int n = ns();
            const double *src = p.metric_ptr ? p.metric_ptr : p.metric.data();
            const double *m = src + (p.metric_constant ? 0 : cell * n);
            for (int k = 0; k < n; ++k) out[k] = (p.diagonal && p.mult_inverse) ? 1.0 / m[k] : m[k];
        } else {
            const double *src = p.mult_ptr ? p.mult_ptr : p.mult.data();
            const double v = src[p.mult_depth == 0 ? 0 : cell];
            out[0] = p.mult_inverse ? 1.0 / v : v;
            (void)D;
        }
    }
    // the norm from interpolated or cell data: Riemann matrices rescaled to grid units
    void finish(const double *in, double *norm) const {
        const int D = pm.ndim;
        if (p.kind == StencilKind::TTI) {  // linear (2), quadratic (3), transform(i, j) at 5 + 3 i + j
            for (int k = 0; k < 14; ++k) norm[k] = in[k];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) norm[5 + 3 * i + j] *= pm.scale[j];
        } else if (p.kind == StencilKind::RiemannPerCell && !p.diagonal) {
            double m[6];
            for (int k = 0; k < ns(); ++k) m[k] = in[k];
            if (p.dual) {  // Inverse = Comatrix / Determinant (SymmetricMatrixType.hxx:201-242)
                auto c = [&](int i, int j) { return i >= j ? m[i * (i + 1) / 2 + j] : m[j * (j + 1) / 2 + i]; };
                double co[6], det;
                if (D == 2) {
                    co[0] = c(1, 1); co[1] = -c(1, 0); co[2] = c(0, 0);
                    det = c(0, 0) * c(1, 1) - c(1, 0) * c(0, 1);
                } else {
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j <= i; ++j) {
                            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                            co[i * (i + 1) / 2 + j] = c(i1, j1) * c(i2, j2) - c(i1, j2) * c(i2, j1);
                        }
                    det = c(0, 0) * (c(1, 1) * c(2, 2) - c(1, 2) * c(2, 1)) +
                          c(0, 1) * (2. * c(1, 2) * c(2, 0) - c(1, 0) * c(2, 2)) - c(0, 2) * (c(1, 1) * c(2, 0));
                }
                const double idet = 1. / det;  // matrix / scalar multiplies by the reciprocal
                for (int k = 0; k < ns(); ++k) m[k] = co[k] * idet;
            }
            for (int i = 0; i < D; ++i)
                for (int j = 0; j <= i; ++j) m[i * (i + 1) / 2 + j] *= pm.scale[i] * pm.scale[j];
            for (int k = 0; k < ns(); ++k) norm[k] = m[k];
        } else if (p.diagonal) {
            for (int i = 0; i < D; ++i) norm[i] = pm.scale[i] / in[i];
        } else {
            for (int i = 0; i < D; ++i) norm[i] = pm.scale[i] / in[0];
        }
    }
    double apply(const double *norm, const double *v) const {
        const int D = pm.ndim;
        if (p.kind == StencilKind::TTI) return tti_norm(norm, v);
        if (p.kind == StencilKind::RiemannPerCell && !p.diagonal) {  // sqrt(<v, M v>)
            auto c = [&](int i, int j) { return i >= j ? norm[i * (i + 1) / 2 + j] : norm[j * (j + 1) / 2 + i]; };
            double sum = 0.;
            for (int i = 0; i < D; ++i) {
                double si = 0.;
                for (int j = 0; j < D; ++j) si += c(i, j) * v[j];
                sum += v[i] * si;
            }
            return std::sqrt(sum);
        }
        double s = 0.;
        for (int i = 0; i < D; ++i) s += (norm[i] * v[i]) * (norm[i] * v[i]);
        return std::sqrt(s);
    }
    // TTINorm::Norm (TTINorm.hxx:331-336) = <Gradient(v), v>, the gradient from the optimized
    // variant of TTINorm::Gradient (TTINorm.hxx:268-329): in the plane (|(Av)_xy|, (Av)_z) of the
    // transformed vector, maximise <q, p> subject to the level 1 - <l, (x^2, y^2)> - 1/2 <(x^2, y^2),
    // Q (x^2, y^2)> >= 0 by 8 steps of sequential quadratic programming (AD2::SQP, AD2.h:124-140:
    // h = lambda H^-1 q - H^-1 g, lambda = -sqrt((<H^-1 g, g> - 2 f) / <H^-1 q, q>)), the first one
    // in closed form; then map back through the transposed transform. Sums start from 0 and
    // divisions of vectors and matrices multiply by the reciprocal, as in the reference's algebra.
    static double tti_norm(const double *m, const double *v) {
        if (v[0] == 0. && v[1] == 0. && v[2] == 0.) return 0.;
        double g[3];
        tti_gradient(m, v, g);
        double norm = 0.;
        for (int i = 0; i < 3; ++i) norm += g[i] * v[i];
        return norm;
    }
    // TTINorm::Gradient (TTINorm.hxx:268-329) at a non-zero vector v.
    static void tti_gradient(const double *m, const double *v, double *grad) {
        const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4];
        auto A = [&](int i, int j) { return m[5 + 3 * i + j]; };  // the guess reads the transform row by row
        double q1[3];
        for (int i = 0; i < 3; ++i) {
            q1[i] = 0.;
            for (int j = 0; j < 3; ++j) q1[i] += A(i, j) * v[j];
        }
        const double q[2] = {std::sqrt(q1[0] * q1[0] + q1[1] * q1[1]), q1[2]};
        const double q0a = q[0] / a, q1b = q[1] / b;
        const double r0 = 1. / std::sqrt(q[0] * q0a + q[1] * q1b);
        double pp[2] = {q0a * r0, q1b * r0};
        for (int it = 1; it < 8; ++it) {
            const double x = pp[0], y = pp[1];
            const double x2 = x * x, y2 = y * y, cx2 = c * x2, ey2 = e * y2, dx2 = d * x2, dy2 = d * y2;
            const double f = 1. - (a * x2 + b * y2 + 0.5 * (cx2 * x2 + 2. * dx2 * y2 + ey2 * y2));
            const double g[2] = {-2. * (x * (a + cx2 + dy2)), -2. * (y * (b + dx2 + ey2))};
            const double h[3] = {-2. * (a + 3. * cx2 + dy2), -2. * (2. * d * x * y), -2. * (b + dx2 + 3. * ey2)};
            const double det = h[0] * h[2] - h[1] * h[1];
            const double idet = 1. / det;  // Comatrix / Determinant
            const double hi[3] = {h[2] * idet, -h[1] * idet, h[0] * idet};
            double hg[2], hq[2];
            for (int i = 0; i < 2; ++i) {
                hg[i] = 0.;
                hq[i] = 0.;
                for (int j = 0; j < 2; ++j) {
                    const double hij = hi[i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i];
                    hg[i] += hij * g[j];
                    hq[i] += hij * q[j];
                }
            }
            double num = 0., den = 0.;
            for (int i = 0; i < 2; ++i) { num += hg[i] * g[i]; den += hq[i] * q[i]; }
            num -= 2. * f;
            const double lambda = -std::sqrt(num / den);
            for (int i = 0; i < 2; ++i) pp[i] += lambda * hq[i] - hg[i];
        }
        const double n01 = q[0];
        const double w[3] = {n01 == 0. ? 0. : pp[0] * q1[0] / n01, n01 == 0. ? 0. : pp[0] * q1[1] / n01, pp[1]};
        for (int i = 0; i < 3; ++i) {
            double gi = 0.;
            for (int j = 0; j < 3; ++j) gi += A(j, i) * w[j];
            grad[i] = gi;
        }
    }
    bool cell_of(const int64_t *idx, int64_t *lin) const {
        int64_t r = 0;
        for (int a = 0; a < pm.ndim; ++a) {
            if (idx[a] < 0 || idx[a] >= pm.dims[a]) return false;
            r = r * pm.dims[a] + idx[a];
        }
        *lin = r;
        return true;
    }
    void at_cell(const int64_t *idx, double *norm) const {
        int64_t lin;
        cell_of(idx, &lin);
        double d[14];
        raw(lin, d);
        finish(d, norm);
    }
    void at_point(const double *q, double *norm) const {
        const int D = pm.ndim, n = ns();
        int64_t nearest[3];
        int dir[3];
        double w[3];
        for (int i = 0; i < D; ++i) {
            nearest[i] = (int64_t)std::floor(q[i]);
            const double diff = q[i] - nearest[i] - 0.5;
            dir[i] = diff > 0 ? 1 : -1;
            w[i] = std::abs(diff);
        }
        double acc[14] = {};
        for (int i = 0; i < (1 << D); ++i) {
            int64_t idx[3];
            double wt = 1.;
            for (int j = 0; j < D; ++j) {
                idx[j] = nearest[j];
                if ((i >> j) & 1) { wt *= w[j]; idx[j] += dir[j]; }
                else wt *= 1. - w[j];
            }
            int64_t lin = 0;
            const bool inside = cell_of(idx, &lin);
            if (!inside) wt = 0.;
            if (i > 0 && wt == 0) continue;  // the first term is always evaluated (MapWeightedSum.h)
            double d[14] = {};
            if (inside) raw(lin, d);
            for (int k = 0; k < n; ++k) acc[k] = i == 0 ? wt * d[k] : acc[k] + wt * d[k];
        }
        finish(acc, norm);
    }
};

// Reversed offsets of a cell x of a Riemann model (HFM_StencilRecompute.hxx:85-124): the offsets e,
// sorted and without repeats, such that e or -e is a difference of nonzero weight of the Selling
// stencil of y = x - e, y in the domain (no walls, no periodic axes here). The stencils scanned are
// those of the cells within `width` (the largest offset component of the domain's stencils) of x.
void riemann_cell_stencil(const EulerProblem &p, const Param &pm, int64_t lin, int off[6][3], double w[6]) {
    SeedGuess G{p, pm};
    double m[6];
    G.raw(lin, m);
    const bool ok = pm.ndim == 2 ? riemann_stencil<2>(m, p.dual, p.h, off, w) : riemann_stencil<3>(m, p.dual, p.h, off, w);
    if (!ok) throw Error(HFM_ERR_VALUE, "Error : metric is not positive definite");
}

// Largest offset component over every cell's stencil (the search box of the reversed offsets).
// The width is needed before any device work; the cells are split among host threads, since one
// Selling decomposition per cell of a large grid takes seconds on one core.
int riemann_max_width(const EulerProblem &p, const Param &pm) {
    int64_t ncell = 1;
    for (int a = 0; a < pm.ndim; ++a) ncell *= pm.dims[a];
    if (p.metric_constant) ncell = 1;
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw, ncell / 65536));
    std::vector<int> widths(nt, 0);
    std::vector<std::exception_ptr> errors(nt);
    auto work = [&](int t) {
        try {
            int width = 0;
            for (int64_t lin = ncell * t / nt; lin < ncell * (t + 1) / nt; ++lin) {
                int off[6][3];
                double w[6];
                riemann_cell_stencil(p, pm, lin, off, w);
                for (int k = 0; k < (pm.ndim == 2 ? 3 : 6); ++k)
                    for (int a = 0; a < pm.ndim; ++a) width = std::max(width, std::abs(off[k][a]));
            }
            widths[t] = width;
        } catch (...) {
            errors[t] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (std::thread &th : pool) th.join();
    for (const std::exception_ptr &e : errors)
        if (e) std::rethrow_exception(e);
    return *std::max_element(widths.begin(), widths.end());
}

std::vector<std::array<int, 3>> reversed_offsets(const EulerProblem &p, const Param &pm, const int64_t *x, int width) {
    const int D = pm.ndim;
    SeedGuess G{p, pm};
    const int nk = D == 2 ? 3 : 6;
    for (int a = 0; a < D; ++a)
        if (x[a] < 0 || x[a] >= pm.dims[a])
            throw Error(HFM_ERR_UNSUPPORTED, "seedRadius < 0 with a seed closer to the domain boundary than the radius "
                                             "is not supported by the GPU solve path");
    std::set<std::array<int, 3>> out;
    const int side = 2 * width + 1;
    int64_t box = 1;
    for (int a = 0; a < D; ++a) box *= side;
    for (int64_t b = 0; b < box; ++b) {
        int64_t y[3] = {0, 0, 0}, r = b;
        bool inside = true;
        for (int a = D - 1; a >= 0; --a) {
            y[a] = x[a] + (r % side) - width;
            r /= side;
            inside = inside && y[a] >= 0 && y[a] < pm.dims[a];
        }
        if (!inside) continue;
        int64_t lin = 0;
        G.cell_of(y, &lin);
        int off[6][3];
        double w[6];
        riemann_cell_stencil(p, pm, lin, off, w);
        for (int k = 0; k < nk; ++k) {
            if (w[k] == 0.) continue;
            for (int sgn = 1; sgn >= -1; sgn -= 2) {
                std::array<int, 3> e = {0, 0, 0};
                bool hit = true;
                for (int a = 0; a < D; ++a) {
                    e[a] = sgn * off[k][a];
                    hit = hit && y[a] + e[a] == x[a];
                }
                if (hit) out.insert(e);
            }
        }
    }
    return std::vector<std::array<int, 3>>(out.begin(), out.end());
}

// Seeds: points -> unique indices (first value kept), sorted; with seedRadius > 0 each seed is
// spread to the cells whose centre lies within that many cells of it (StaticFactoring.hxx:242-346).

void read_seeds(Store &io, const Param &pm, EulerProblem &p, bool unoriented_allowed, double default_radius) {
    std::map<int64_t, double> seeds;
    std::vector<double> pts;
    int64_t n = 0;
    if (io.has_field("seeds")) {
        pts = io.get_vector("seeds", pm.ndim, &n);
        std::vector<double> vals(n, 0.0);
        if (io.has_field("seedValues")) {
            int64_t nv = 0;
            vals = io.get_vector("seedValues", 1, &nv);
            if (nv != n) throw Error(HFM_ERR_VALUE, "Error : Inconsistent size of seedValues.");
        }
        // seedRadius < 0: spread to |seedRadius|, then one step of the reversed stencils
        const double radius_in = io.get_scalar("seedRadius", default_radius);
        const bool stencil_step = radius_in < 0;
        const double radius = std::abs(radius_in);
        const bool shared_axes = p.diagonal || (p.kind == StencilKind::SharedByTheta && !p.angular);
        if (stencil_step) {
            if (p.kind != StencilKind::RiemannPerCell && !shared_axes)
                throw Error(HFM_ERR_UNSUPPORTED, "seedRadius < 0 (stencil-step spreading) is supported for the Riemann, "
                                                 "Isotropic and Diagonal models only");
            if (io.has_field("walls") || pm.periodic[0] || pm.periodic[1] || pm.periodic[2])
                throw Error(HFM_ERR_UNSUPPORTED, "seedRadius < 0 with walls or periodic axes is not supported by the GPU solve path");
        }
        if (radius > 0) {
            const bool guessable = p.kind == StencilKind::RiemannPerCell || p.kind == StencilKind::TTI ||
                                   (p.kind == StencilKind::SharedByTheta && !p.angular);
            if (!guessable)
                throw Error(HFM_ERR_UNSUPPORTED, "seedRadius > 0 is supported for the Riemann, Isotropic, Diagonal and TTI3 models only");
            const int D = pm.ndim;
            SeedGuess G{p, pm};
            std::vector<double> npts, nvals;
            const int bd = 1 + (int)std::ceil(radius);
            const int side = 1 + 2 * bd;
            int64_t box = 1;
            for (int a = 0; a < D; ++a) box *= side;
            int width = -1;  // largest stencil offset component, computed on first use
            for (int64_t i = 0; i < n; ++i) {
                double q[3];
                for (int a = 0; a < D; ++a) q[a] = (pts[i * D + a] - pm.origin[a]) / pm.scale[a];  // ADim
                std::set<std::vector<int64_t>> seen;
                double distp[14];
                G.at_point(q, distp);
                auto insert = [&](const int64_t *index, double rad) {
                    double v[3], nn = 0.;
                    for (int a = 0; a < D; ++a) { v[a] = q[a] - ((double)index[a] + 0.5); nn += v[a] * v[a]; }
                    if (std::sqrt(nn) >= rad) return;
                    if (!seen.insert(std::vector<int64_t>(index, index + D)).second) return;
                    int64_t lin;
                    if (!G.cell_of(index, &lin)) return;
                    double distq[14];
                    G.at_cell(index, distq);
                    for (int a = 0; a < D; ++a) npts.push_back(((double)index[a] + 0.5) * pm.scale[a] + pm.origin[a]);
                    nvals.push_back(vals[i] + 0.5 * (G.apply(distp, v) + G.apply(distq, v)));
                };
                int64_t pidx[3];
                for (int a = 0; a < D; ++a) pidx[a] = (int64_t)std::floor(q[a]);
                insert(pidx, std::numeric_limits<double>::infinity());
                for (int64_t k = 0; k < box; ++k) {  // the box of offsets, RowMajor
                    int64_t idx[3], r = k;
                    for (int a = D - 1; a >= 0; --a) { idx[a] = pidx[a] + (r % side) - bd; r /= side; }
                    insert(idx, radius);
                }
                if (stencil_step) {  // every index seen so far, in index order, plus its reversed offsets
                    // Isotropic and Diagonal models share one stencil, +-e_i with nonzero base weights,
                    // whose reversed offsets the reference takes once, from the domain's centre
                    // (HFM_StencilShare.hxx:104-180): the same sorted list for every cell.
                    std::vector<std::array<int, 3>> shared;
                    if (shared_axes) {
                        std::set<std::array<int, 3>> acc;
                        for (int a = 0; a < D; ++a)
                            for (int sgn = -1; sgn <= 1; sgn += 2) {
                                const int64_t c = pm.dims[a] / 2 + sgn;
                                if (c < 0 || c >= pm.dims[a]) continue;
                                std::array<int, 3> e = {0, 0, 0};
                                e[a] = sgn;
                                acc.insert(e);
                            }
                        shared.assign(acc.begin(), acc.end());
                    } else if (width < 0) {
                        width = riemann_max_width(p, pm);
                    }
                    const std::set<std::vector<int64_t>> base = seen;
                    for (const std::vector<int64_t> &x : base) {
                        for (const std::array<int, 3> &e : shared_axes ? shared : reversed_offsets(p, pm, x.data(), width)) {
                            int64_t idx[3];
                            for (int a = 0; a < D; ++a) idx[a] = x[a] + e[a];
                            insert(idx, std::numeric_limits<double>::infinity());
                        }
                    }
                }
            }
            io.set_vector("spreadedSeeds", (int64_t)nvals.size(), D, npts.data());
            io.set_vector("spreadedSeedValues", (int64_t)nvals.size(), 1, nvals.data());
            pts.swap(npts);
            vals.swap(nvals);
            n = (int64_t)vals.size();
        }
        for (int64_t i = 0; i < n; ++i) {
            int64_t lin;
            if (!pm.index_of(&pts[i * pm.ndim], &lin)) {
                std::ostringstream o;
                o << "Error : seed {";
                for (int a = 0; a < pm.ndim; ++a) o << (a ? "," : "") << pts[i * pm.ndim + a];
                o << "} is out of range.\n";
                io.warn(o.str());
                continue;
            }
            seeds.emplace(lin, vals[i]);
        }
    }
    int64_t nu = 0;
    if (unoriented_allowed && io.has_field("seeds_Unoriented")) {
        std::vector<double> up = io.get_vector("seeds_Unoriented", 2, &nu);
        std::vector<double> uv(nu, 0.0);
        if (io.has_field("seedValues_Unoriented")) {
            int64_t nv = 0;
            uv = io.get_vector("seedValues_Unoriented", 1, &nv);
            if (nv != nu) throw Error(HFM_ERR_VALUE, "Error : Inconsistent size of seedValues_Unoriented.");
        }
        for (int64_t i = 0; i < nu; ++i)
            for (int t = 0; t < pm.dims[2]; ++t) {
                const double q[3] = {up[2 * i], up[2 * i + 1], pm.origin[2] + (t + 0.5) * pm.scale[2]};
                int64_t lin;
                if (!pm.index_of(q, &lin)) continue;
                seeds.emplace(lin, uv[i]);
            }
    }
    if (seeds.empty() && (n + nu) > 0) throw Error(HFM_ERR_VALUE, "Error : seeds incorrectly set");
    for (const auto &kv : seeds) {
        p.seed_index.push_back(kv.first);
        p.seed_value.push_back(kv.second);
    }
}

// A scalar field over the lifted grid given with depth 0 (constant), 3 (full), 2 (physical x,y)
// or 1 (angle only) (HFMInterface.hxx:23-32), kept compact: the solver expands it on the device.
// Returns the depth; `f` holds the field (a view into the store when no reordering is needed).
int read_lifted_scalar(Store &io, const std::string &key, const int *dims, Field &f) {
    const std::vector<int64_t> dd = io.field_domain_dims(key, 1);
    const int depth = (int)dd.size();
    if (depth > 3) throw Error(HFM_ERR_VALUE, "Field " + key + " has incorrect depth.\n");
    f = io.get_field(key, depth, 1);
    if ((depth == 3 && (f.dims[0] != dims[0] || f.dims[1] != dims[1] || f.dims[2] != dims[2])) ||
        (depth == 2 && (f.dims[0] != dims[0] || f.dims[1] != dims[1])) || (depth == 1 && f.dims[0] != dims[2]))
        throw Error(HFM_ERR_VALUE, "Error : Field " + key + " has inconsistent dimensions.");
    return depth;
}

// Walls (GetIntegralField<bool>: (bool)double). A full RowMajor field stored in the store is
// handed to the solver as a view (converted on the device); other shapes are converted here.
void read_walls(Store &io, const Param &pm, bool lifted, EulerProblem &p) {
    std::vector<uint8_t> &w = p.walls;
    w.clear();
    p.walls_f64 = nullptr;
    if (!io.has_field("walls")) return;
    const int64_t N = (int64_t)pm.dims[0] * pm.dims[1] * pm.dims[2];
    if (lifted) {
        w.resize(N);
        Field f;
        const int depth = read_lifted_scalar(io, "walls", pm.dims, f);
        const double *v = f.ptr();
        const int64_t nt = pm.dims[2];
        for (int64_t i = 0; i < N; ++i) {
            const int64_t k = depth == 3 ? i : depth == 2 ? i / nt : depth == 1 ? i % nt : 0;
            w[i] = v[k] != 0.0;
        }
        return;
    }
    const std::vector<int64_t> dd = io.field_domain_dims("walls", 1);
    Field f = io.get_field("walls", dd.empty() ? 0 : pm.ndim, 1);
    if (f.constant()) {
        w.assign(N, f.ptr()[0] != 0.0);
        return;
    }
    for (int a = 0; a < pm.ndim; ++a)
        if (f.dims[a] != pm.dims[a]) throw Error(HFM_ERR_VALUE, "Error : walls have inconsistent dims");
    if (f.view) {
        p.walls_f64 = f.view;
        return;
    }
    w.resize(N);
    const double *v = f.ptr();
    for (int64_t i = 0; i < N; ++i) w[i] = v[i] != 0.0;
}

void set_common_solver_options(Store &io, EulerProblem &p) {
    const std::string prec = io.get_string("solverPrecision", "float64", 2);
    if (prec == "float64") p.fp64 = true;
    else if (prec == "float32") p.fp64 = false;
    else throw Error(HFM_ERR_VALUE, "solverPrecision must be float64 or float32");
    default_schedule(p);
    p.sweeps_per_tile = (int)io.get_scalar("tileSweeps", p.sweeps_per_tile, 3);
    if (p.sweeps_per_tile < 1 || p.sweeps_per_tile > 1024) throw Error(HFM_ERR_VALUE, "tileSweeps out of range");
    p.max_rounds = (int)io.get_scalar("maxRounds", (double)(1 << 20), 3);
    p.ordered = io.get_scalar("tileOrdering", 1.0, 3) != 0;
    p.band_lo = io.get_scalar("bandLo", p.band_lo, 3);
    p.band_hi = io.get_scalar("bandHi", p.band_hi, 3);
    if (!(p.band_lo > 0) || !(p.band_hi > p.band_lo)) throw Error(HFM_ERR_VALUE, "bandLo/bandHi must satisfy 0 < bandLo < bandHi");
    if (io.has_field("tileShape")) {
        // tile extents per axis (x, y[, z|theta]): powers of two whose product is 64
        int64_t n = 0;
        const std::vector<double> e = io.get_vector("tileShape", 1, &n);
        if (n != p.ndim) throw Error(HFM_ERR_VALUE, "tileShape must give one extent per axis");
        int sum = 0;
        for (int a = 0; a < p.ndim; ++a) {
            const int v = (int)e[a];
            if (v < 1 || v != e[a] || (v & (v - 1))) throw Error(HFM_ERR_VALUE, "tileShape extents must be powers of two");
            int sh = 0;
            while ((1 << sh) < v) ++sh;
            p.tile_shift[a] = sh;
            sum += sh;
        }
        if (sum != 6) throw Error(HFM_ERR_VALUE, "tileShape must hold 64 cells");
    }
}

// ------------------------------------------------------------------------------------------
void setup_riemann(Store &io, int ndim, Param &pm, EulerProblem &p) {
    const std::vector<int> dims = read_dims(io, ndim);
    pm.ndim = ndim;
    for (int a = 0; a < ndim; ++a) pm.dims[a] = dims[a];
    const std::vector<double> origin = read_point(io, "origin", ndim, std::vector<double>(ndim, 0.0));
    std::vector<double> hs(ndim);
    if (io.has_field("gridScales")) {
        hs = read_point(io, "gridScales", ndim, hs);
    } else {
        const double h = io.get_scalar("gridScale");
        std::fill(hs.begin(), hs.end(), h);
    }
    for (int a = 0; a < ndim; ++a) {
        if (!(hs[a] > 0)) throw Error(HFM_ERR_VALUE, "Parametrization error : gridscales should be positive");
        pm.origin[a] = origin[a];
        pm.scale[a] = hs[a];
        p.h[a] = hs[a];
        p.dims[a] = dims[a];
    }
    p.ndim = ndim;
    p.kind = StencilKind::RiemannPerCell;
    const int ns = ndim * (ndim + 1) / 2;
    std::string key = "metric";
    if (io.has_field("dualMetric")) {
        if (io.has_field("metric")) throw Error(HFM_ERR_VALUE, "Error: both primal and dual metric provided");
        key = "dualMetric";
        p.dual = true;
    }
    const std::vector<int64_t> dd = io.field_domain_dims(key, ns);
    Field f = io.get_field(key, dd.empty() ? 0 : ndim, ns);
    if (!f.constant()) {
        for (int a = 0; a < ndim; ++a)
            if (f.dims[a] != dims[a]) throw Error(HFM_ERR_VALUE, "Error : Field " + key + " has inconsistent dimensions.");
    }
    p.metric_constant = f.constant();
    if (f.view) {
        p.metric_ptr = f.view;
        p.metric_len = f.size();
    } else {
        p.metric = std::move(f.data);
    }
}

// TTI3 (Headers/Experimental/TTI.h:18-33, Implementation/TTI.hpp:11-21): a 14-component metric
// per point (linear 2, quadratic 3, transform 9), grid scales as for Riemann3, `nmix` (0: the
// Newton-like optimisation, the only one on the GPU path).
void setup_tti(Store &io, Param &pm, EulerProblem &p) {
    const int ndim = 3;
    const std::vector<int> dims = read_dims(io, ndim);
    pm.ndim = ndim;
    for (int a = 0; a < ndim; ++a) pm.dims[a] = dims[a];
    const std::vector<double> origin = read_point(io, "origin", ndim, std::vector<double>(ndim, 0.0));
    std::vector<double> hs(ndim);
    if (io.has_field("gridScales")) {
        hs = read_point(io, "gridScales", ndim, hs);
    } else {
        const double h = io.get_scalar("gridScale");
        std::fill(hs.begin(), hs.end(), h);
    }
    for (int a = 0; a < ndim; ++a) {
        if (!(hs[a] > 0)) throw Error(HFM_ERR_VALUE, "Parametrization error : gridscales should be positive");
        pm.origin[a] = origin[a];
        pm.scale[a] = hs[a];
        p.h[a] = hs[a];
        p.dims[a] = dims[a];
    }
    if (io.has_field("nmix") && io.get_scalar("nmix") != 0)
        throw Error(HFM_ERR_UNSUPPORTED, "TTI3 with nmix > 0 (finite envelope) is not supported by the GPU solve path");
    if (io.has_field("walls"))
        throw Error(HFM_ERR_UNSUPPORTED, "TTI3 with walls is not supported by the GPU solve path");
    p.ndim = ndim;
    p.kind = StencilKind::TTI;
    p.nfwd = 0;
    p.nsym = kTTISlots;
    const std::vector<int64_t> dd = io.field_domain_dims("metric", 14);
    Field f = io.get_field("metric", dd.empty() ? 0 : ndim, 14);
    if (!f.constant()) {
        for (int a = 0; a < ndim; ++a)
            if (f.dims[a] != dims[a]) throw Error(HFM_ERR_VALUE, "Error : Field metric has inconsistent dimensions.");
    }
    p.metric_constant = f.constant();
    if (f.view) {
        p.metric_ptr = f.view;
        p.metric_len = f.size();
    } else {
        p.metric = std::move(f.data);
    }
}

// Isotropic2 / Isotropic3 (Headers/Specializations/Isotropic.h:11-59): one symmetric difference
// per axis, base weight 1 / h_i^2, times the squared speed of the cell (speed, or 1 / cost). Solved
// as a shared stencil (the same table on every index of the last axis) with the speed as the
// per-cell multiplier, so that activeNeighs, sensitivities and variations follow the reference's
// multiplier semantics.
void setup_isotropic(Store &io, int ndim, Param &pm, EulerProblem &p) {
    const std::vector<int> dims = read_dims(io, ndim);
    pm.ndim = ndim;
    p.ndim = ndim;
    const std::vector<double> origin = read_point(io, "origin", ndim, std::vector<double>(ndim, 0.0));
    std::vector<double> hs(ndim);
    if (io.has_field("gridScales")) {
        hs = read_point(io, "gridScales", ndim, hs);
    } else {
        const double h = io.get_scalar("gridScale");
        std::fill(hs.begin(), hs.end(), h);
    }
    for (int a = 0; a < ndim; ++a) {
        if (!(hs[a] > 0)) throw Error(HFM_ERR_VALUE, "Parametrization error : gridscales should be positive");
        pm.dims[a] = p.dims[a] = dims[a];
        pm.origin[a] = origin[a];
        pm.scale[a] = p.h[a] = hs[a];
    }
    p.kind = StencilKind::SharedByTheta;
    p.angular = false;
    p.nfwd = 0;
    p.nsym = ndim;
    p.nclass = ndim == 3 ? dims[2] : 1;
    p.cls_off.assign((size_t)p.nclass * ndim * 3, 0);
    p.cls_w.assign((size_t)p.nclass * ndim, 0.0);
    p.cls_enabled.assign((size_t)p.nclass * 2 * ndim, 1);
    for (int c = 0; c < p.nclass; ++c)
        for (int i = 0; i < ndim; ++i) {
            p.cls_off[(c * ndim + i) * 3 + i] = 1;
            p.cls_w[c * ndim + i] = 1. / (hs[i] * hs[i]);
        }
    const bool has_speed = io.has_field("speed");
    const char *key = has_speed ? "speed" : "cost";
    const std::vector<int64_t> dd = io.field_domain_dims(key, 1);
    Field f = io.get_field(key, dd.empty() ? 0 : ndim, 1);
    if (!f.constant())
        for (int a = 0; a < ndim; ++a)
            if (f.dims[a] != dims[a]) throw Error(HFM_ERR_VALUE, std::string("Error : Field ") + key + " has inconsistent dimensions.");
    p.mult_depth = f.constant() ? 0 : 3;
    p.mult_inverse = !has_speed;
    if (f.view) {
        p.mult_ptr = f.view;
    } else {
        p.mult = std::move(f.data);
        p.mult_ptr = nullptr;
    }
}

// Diagonal2 / Diagonal3 (Headers/Specializations/Isotropic.h:61-115): a speed (or cost) vector
// per point, one symmetric difference per axis of weight speed_i^2 / h_i^2.
void setup_diagonal(Store &io, int ndim, Param &pm, EulerProblem &p) {
    const std::vector<int> dims = read_dims(io, ndim);
    pm.ndim = ndim;
    p.ndim = ndim;
    const std::vector<double> origin = read_point(io, "origin", ndim, std::vector<double>(ndim, 0.0));
    std::vector<double> hs(ndim);
    if (io.has_field("gridScales")) {
        hs = read_point(io, "gridScales", ndim, hs);
    } else {
        const double h = io.get_scalar("gridScale");
        std::fill(hs.begin(), hs.end(), h);
    }
    for (int a = 0; a < ndim; ++a) {
        if (!(hs[a] > 0)) throw Error(HFM_ERR_VALUE, "Parametrization error : gridscales should be positive");
        pm.dims[a] = p.dims[a] = dims[a];
        pm.origin[a] = origin[a];
        pm.scale[a] = p.h[a] = hs[a];
    }
    p.kind = StencilKind::RiemannPerCell;
    p.diagonal = true;
    const bool has_speed = io.has_field("speed");
    const std::string key = has_speed ? "speed" : "cost";
    const std::vector<int64_t> dd = io.field_domain_dims(key, ndim);
    Field f = io.get_field(key, dd.empty() ? 0 : ndim, ndim);
    if (!f.constant())
        for (int a = 0; a < ndim; ++a)
            if (f.dims[a] != dims[a]) throw Error(HFM_ERR_VALUE, "Error : Field " + key + " has inconsistent dimensions.");
    p.metric_constant = f.constant();
    p.mult_inverse = !has_speed;
    if (f.view) {
        p.metric_ptr = f.view;
        p.metric_len = f.size();
    } else {
        p.metric = std::move(f.data);
    }
}

void setup_curvature(Store &io, const std::string &model, Param &pm, EulerProblem &p) {
    const std::vector<int> dims = read_dims(io, 3);
    pm.ndim = 3;
    p.ndim = 3;
    for (int a = 0; a < 3; ++a) pm.dims[a] = p.dims[a] = dims[a];
    pm.periodic[2] = p.periodic[2] = 1;
    const bool rs = model == "ReedsShepp2";
    const double eps = io.get_scalar("eps", 0.1);
    const double xi = io.get_scalar("xi", 1.0);
    const bool projective = rs ? io.get_scalar("projective", 0.0) != 0 : false;
    const double h = io.get_scalar("gridScale");
    if (!(h > 0)) throw Error(HFM_ERR_VALUE, "Parametrization error : gridscale should be positive");
    const double ds = ((projective ? kPi : 2.0 * kPi)) / (double)dims[2];
    const std::vector<double> origin = read_point(io, "origin", 2, {0.0, 0.0});
    pm.origin[0] = origin[0];
    pm.origin[1] = origin[1];
    pm.origin[2] = -ds / 2.0;
    pm.scale[0] = pm.scale[1] = h;
    pm.scale[2] = ds;
    p.h[0] = p.h[1] = h;  // the class tables carry the scales; h only sizes the domain
    p.h[2] = ds;
    p.kind = StencilKind::SharedByTheta;
    p.nclass = dims[2];
    if (rs) {
        p.nfwd = 0;
        p.nsym = 4;
        reedsshepp2_table(dims[2], h, xi, eps, projective, p.cls_off, p.cls_w);
    } else if (model == "ReedsSheppForward2") {
        p.nfwd = 3;
        p.nsym = 1;
        reedssheppforward2_table(dims[2], h, xi, eps, p.cls_off, p.cls_w);
    } else if (model == "Dubins2") {
        p.nfwd = 12;
        p.nsym = 0;
        p.nmax = 2;
        dubins2_table(dims[2], h, xi, eps, p.cls_off, p.cls_w);
    } else {
        p.nfwd = 27;
        p.nsym = 0;
        elastica2_table(dims[2], h, xi, eps, p.cls_off, p.cls_w);
    }
    // Slots reachable from each class centre (dims/2, dims/2, theta) (HFM_StencilShare.hxx:114-175).
    const int ND = p.nfwd + p.nsym, NB = p.nfwd + 2 * p.nsym;
    p.cls_enabled.assign((size_t)p.nclass * NB, 0);
    for (int c = 0; c < p.nclass; ++c)
        for (int k = 0; k < ND; ++k) {
            const int8_t *o = &p.cls_off[(c * ND + k) * 3];
            for (int si = 0; si < (k < p.nfwd ? 1 : 2); ++si) {
                const int s = si ? -1 : 1;
                const int slot = k < p.nfwd ? k : p.nfwd + 2 * (k - p.nfwd) + si;
                const int y0 = dims[0] / 2 + s * o[0], y1 = dims[1] / 2 + s * o[1];
                p.cls_enabled[c * NB + slot] = (y0 >= 0 && y0 < dims[0] && y1 >= 0 && y1 < dims[1]) ? 1 : 0;
            }
        }
    // speed, or cost inverted on the device (DataSource_Inverse, HFMInterface.hxx:131-150)
    const bool has_speed = io.has_field("speed");
    Field f;
    p.mult_depth = read_lifted_scalar(io, has_speed ? "speed" : "cost", dims.data(), f);
    p.mult_inverse = !has_speed;
    if (f.view) {
        p.mult_ptr = f.view;
    } else {
        p.mult = std::move(f.data);
        p.mult_ptr = nullptr;
    }
}

// ReedsShepp3 and ReedsSheppForward3 on R^3 x S^2 (Headers/Specializations/Curvature3.h:29-107):
// the grid (x, y, z, theta, phi), theta in (0, pi) at (i + 1/2) ds and phi at j ds, ds = 2 pi / nphi
// (nphi = 2 ntheta, or 4 ntheta for the projective ReedsShepp3), Sphere2 boundary conditions on
// (theta, phi). The solver holds it as the 3-D grid (x, y, (z * ntheta + theta) * nphi + phi) with
// one shared stencil per (theta, phi); the speed (or cost) is a constant or a field over the whole
// grid, (x, y, z) or (theta, phi) (SpecializationsDefault::GetField, HFMInterface.hxx:23-32).
void setup_reedsshepp3(Store &io, Param &pm, EulerProblem &p, bool forward) {
    const std::vector<int> dims = read_dims(io, 5);
    const double eps = io.get_scalar("eps", 0.1);
    const double xi = io.get_scalar("xi", 1.0);
    const bool dual = forward ? false : io.get_scalar("dual", 0.0) != 0;
    const bool projective = forward ? false : io.get_scalar("projective", 0.0) != 0;
    const double h = io.get_scalar("gridScale");
    if (!(h > 0)) throw Error(HFM_ERR_VALUE, "Parametrization error : gridscale should be positive");
    const std::string name = forward ? "ReedsSheppForward3" : "ReedsShepp3";
    if (projective && dims[4] != 4 * dims[3])
        throw Error(HFM_ERR_VALUE, name + " setup error : inconsistent bundle dimensions (projective : nPhi=4*nTheta).");
    if (!projective && dims[4] != 2 * dims[3])
        throw Error(HFM_ERR_VALUE, name + " setup error : inconsistent bundle dimensions (expected : nPhi=2*nTheta).");
    const long long nw = (long long)dims[2] * dims[3] * dims[4];
    if (nw >= (1ll << 30) || (long long)dims[0] * dims[1] * nw >= (1ll << 40))
        throw Error(HFM_ERR_UNSUPPORTED, "ReedsShepp3 grid too large for the GPU solve path");
    const double ds = (2.0 * kPi) / (double)dims[4];
    pm.ndim = 5;
    for (int a = 0; a < 5; ++a) pm.dims[a] = dims[a];
    const std::vector<double> origin = read_point(io, "origin", 3, {0.0, 0.0, 0.0});
    for (int a = 0; a < 3; ++a) {
        pm.origin[a] = origin[a];
        pm.scale[a] = h;
    }
    pm.origin[3] = 0.0;
    pm.origin[4] = -ds / 2.0;  // HFM_ParamDefault.hxx:25
    pm.scale[3] = pm.scale[4] = ds;
    pm.sphere = 3;
    p.ndim = 3;
    p.dims[0] = dims[0];
    p.dims[1] = dims[1];
    p.dims[2] = (int)nw;
    p.h[0] = p.h[1] = p.h[2] = h;  // the class tables carry the scales; h only sizes the domain
    p.kind = StencilKind::SharedByTheta;
    p.angular = true;
    p.nfwd = forward ? 6 : 0;
    p.nsym = forward ? 2 : 8;
    p.nclass = dims[3] * dims[4];
    p.sphere_nth = dims[3];
    p.sphere_nph = dims[4];
    if (forward) reedssheppforward3_table(dims[3], dims[4], h, xi, eps, p.cls_off, p.cls_ang, p.cls_w);
    else reedsshepp3_table(dims[3], dims[4], h, xi, eps, dual, p.cls_off, p.cls_ang, p.cls_w);
    // slots reachable from each class centre (dims / 2 on x, y, z; the sphere steps always land
    // in the domain) (HFM_StencilShare.hxx:132-175)
    const int NB = p.nfwd + 2 * p.nsym;
    p.cls_enabled.assign((size_t)p.nclass * NB, 0);
    for (int c = 0; c < p.nclass; ++c)
        for (int k = 0; k < 8; ++k)
            for (int si = 0; si < (k < p.nfwd ? 1 : 2); ++si) {
                const int s = si ? -1 : 1;
                const int slot = k < p.nfwd ? k : p.nfwd + 2 * (k - p.nfwd) + si;
                bool in = true;
                for (int a = 0; a < 3; ++a) {
                    const int y = dims[a] / 2 + s * p.cls_off[(c * 8 + k) * 3 + a];
                    in = in && y >= 0 && y < dims[a];
                }
                p.cls_enabled[c * NB + slot] = in ? 1 : 0;
            }
    const bool has_speed = io.has_field("speed");
    const std::string key = has_speed ? "speed" : "cost";
    const std::vector<int64_t> dd = io.field_domain_dims(key, 1);
    const int depth = (int)dd.size();
    if (depth != 0 && depth != 2 && depth != 3 && depth != 5)
        throw Error(HFM_ERR_VALUE, "Field " + key + " has incorrect depth.\n");
    Field f = io.get_field(key, depth, 1);
    const int first = depth == 2 ? 3 : 0;
    for (int a = 0; a < depth; ++a)
        if (f.dims[a] != dims[first + a])
            throw Error(HFM_ERR_VALUE, "Error : Field " + key + " has inconsistent dimensions.");
    p.mult_depth = depth == 5 ? 3 : depth == 3 ? 2 : depth == 2 ? 1 : 0;
    p.mult_inverse = !has_speed;
    if (f.view) {
        p.mult_ptr = f.view;
    } else {
        p.mult = std::move(f.data);
        p.mult_ptr = nullptr;
    }
    // the GPU solve path covers the arrival times (values, activeNeighs, nAccepted and the stencil
    // width) of this model
    static const char *kRefused[] = {"walls",        "seeds_Unoriented",     "stopWhenAnyAccepted_Unoriented",
                                     "stopWhenAllAccepted_Unoriented", "tips", "tips_Unoriented",
                                     "inspectSensitivity", "costVariation", "seedValueVariation",
                                     "values",       "activeNeighs"};
    for (const char *k : kRefused)
        if (io.has_field(k))
            throw Error(HFM_ERR_UNSUPPORTED, name + " with " + k + " is not supported by the GPU solve path");
    if (io.has_field("seedRadius") && io.get_scalar("seedRadius") != 0)
        throw Error(HFM_ERR_UNSUPPORTED, name + " with seedRadius is not supported by the GPU solve path");
    if (io.get_scalar("exportGeodesicFlow", 0.0, 3) != 0 || io.get_scalar("retainState", 0.0, 3) != 0)
        throw Error(HFM_ERR_UNSUPPORTED, name + " geodesic flow and retained state are not supported by the GPU solve path");
}

// inspectSensitivity groups (FirstVariation::Finally, FirstVariation.h:60-102): weighted points.
void read_inspect(Store &io, const Param &pm, EulerProblem &p) {
    p.adjoint_index.clear();
    p.adjoint_weight.clear();
    // FirstVariation::Finally (FirstVariation.h:60-102): groups of weighted points
    int64_t n = 0;
    const std::vector<double> pts = io.get_vector("inspectSensitivity", pm.ndim, &n);
    std::vector<double> lengths(n, 1.0);
    if (io.has_field("inspectSensitivityLengths")) {
        int64_t nl = 0;
        lengths = io.get_vector("inspectSensitivityLengths", 1, &nl);
        double tot = 0;
        for (double l : lengths) tot += l;
        if (tot != (double)n) throw Error(HFM_ERR_VALUE, "Error : inconsistent inspectSensitivityLengths");
    }
    std::vector<double> weights(n, 1.0);
    if (io.has_field("inspectSensitivityWeights")) {
        int64_t nw = 0;
        weights = io.get_vector("inspectSensitivityWeights", 1, &nw);
        if (nw != n) throw Error(HFM_ERR_VALUE, "Error: Inconsistent inspectSensitivityWeights size");
    }
    int64_t pos = 0;
    for (size_t gi = 0; gi < lengths.size(); ++gi) {
        std::vector<int64_t> idx;
        std::vector<double> wts;
        for (int64_t k = 0; k < (int64_t)lengths[gi]; ++k, ++pos) {
            int64_t lin;
            if (!pm.index_of(&pts[pos * pm.ndim], &lin))
                throw Error(HFM_ERR_VALUE, "Error : inspectSensitivity data points are out of range");
            idx.push_back(lin);
            wts.push_back(weights[pos]);
        }
        p.adjoint_index.push_back(std::move(idx));
        p.adjoint_weight.push_back(std::move(wts));
    }
}

// Geodesic keys (HFMInterface.hxx:452-523, GeodesicDiscreteSolver.hxx:8-15): tips and, on the
// lifted models, tips_Unoriented, made dimensionless; the discrete solver's parameters. Returns
// which of the two tip keys are present.
void read_geodesics(Store &io, const Param &pm, bool lifted, EulerProblem &p, bool has[2]) {
    has[0] = io.has_field("tips");
    has[1] = lifted && io.has_field("tips_Unoriented");
    if (has[0] || has[1]) {
        const std::string solver = io.get_string("geodesicSolver", "Discrete");
        if (solver != "Discrete" && solver != "ODE")
            throw Error(HFM_ERR_VALUE, "Error : Unrecognized geodesic solver " + solver + ".\n");
        p.geo_ode = solver == "ODE";
        p.geo_step = io.get_scalar("geodesicStep", 0.25);
        if (!(p.geo_step > 0)) throw Error(HFM_ERR_VALUE, "geodesicStep must be positive");
        if (p.geo_ode) {
            // GeodesicODESolver.hxx:17-23; the target tolerance is read but the distances to the
            // seeds are capped at 6 when the solver is built, before the keys are read
            p.geo_causality = io.get_scalar("geodesicCausalityTolerance", 4.0);
            io.get_scalar("geodesicTargetTolerance", 6.0);
        } else {
            p.geo_threshold = io.get_scalar("geodesicWeightThreshold", 0.001);
            p.geo_volume_bound = io.get_scalar("geodesicVolumeBound", 5. * std::pow(1.3, pm.ndim));
        }
    }
    if (has[0]) {
        int64_t n = 0;
        const std::vector<double> t = io.get_vector("tips", pm.ndim, &n);
        p.geo_tips.resize(n * pm.ndim);
        for (int64_t i = 0; i < n; ++i)
            for (int a = 0; a < pm.ndim; ++a)
                p.geo_tips[i * pm.ndim + a] = (t[i * pm.ndim + a] - pm.origin[a]) / pm.scale[a];  // ADim
    }
    if (has[1]) {
        int64_t n = 0;
        const std::vector<double> t = io.get_vector("tips_Unoriented", 2, &n);
        p.geo_tips_unoriented.resize(n * 2);
        for (int64_t i = 0; i < n; ++i)
            for (int a = 0; a < 2; ++a) p.geo_tips_unoriented[i * 2 + a] = (t[i * 2 + a] - pm.origin[a]) / pm.scale[a];
    }
    p.want_geodesic_flow = io.get_scalar("exportGeodesicFlow", 0.0, 2) != 0;
}

// costVariation (dims + (nVar,), the store's ordering applied to all axes) and seedValueVariation
// ((nVar, nSeeds), RowMajor whatever the ordering) of the forward first variation
// (FirstVariation.h:103-124, 389-396).
void read_forward_variation(Store &io, const Param &pm, EulerProblem &p) {
    const bool cost = io.has_field("costVariation"), seed = io.has_field("seedValueVariation");
    if (!cost && !seed) return;
    int64_t ncells = 1;
    for (int a = 0; a < pm.ndim; ++a) ncells *= pm.dims[a];
    int kc = 0, ks = 0;
    if (cost) {
        // one component per axis for the Diagonal models (their multiplier is a speed vector)
        const int comp = p.diagonal ? pm.ndim : 1;
        const Field f = io.get_field("costVariation", pm.ndim + 1, comp);
        bool ok = (int)f.dims.size() == pm.ndim + 1;
        for (int a = 0; ok && a < pm.ndim; ++a) ok = f.dims[a] == pm.dims[a];
        if (!ok) throw Error(HFM_ERR_VALUE, "Forward variation error : inconsistent input sizes");
        kc = (int)f.dims[pm.ndim];
        p.fwd_cost.assign(f.ptr(), f.ptr() + ncells * kc * comp);
    }
    if (seed) {
        const RawElement &r = io.raw("seedValueVariation");
        if (r.is_string() || r.dims.size() != 2)
            throw Error(HFM_ERR_VALUE, "IO::GetArray error : Field seedValueVariation has depth " +
                                           std::to_string(r.dims.size()) + " instead of expected 2.");
        int64_t ns = 0;
        const std::vector<double> pts = io.get_vector("seeds", pm.ndim, &ns);
        if (ns != r.dims[1]) throw Error(HFM_ERR_VALUE, "Error : Inconsistent size of seedValueVariation");
        ks = (int)r.dims[0];
        const double *sv = r.ptr();
        for (int64_t i = 0; i < ns; ++i) {
            int64_t lin;
            if (!pm.index_of(&pts[i * pm.ndim], &lin)) continue;
            p.fwd_seed_cell.push_back(lin);
            for (int k = 0; k < ks; ++k) p.fwd_seed_value.push_back(sv[k * ns + i]);
        }
    }
    if (cost && seed && kc != ks) throw Error(HFM_ERR_VALUE, "Forward variation error : inconsistent input sizes");
    p.fwd_nvar = cost ? kc : ks;
    if (p.fwd_nvar <= 0) throw Error(HFM_ERR_VALUE, "Forward variation error : inconsistent input sizes");
}

// Stopping criteria (CommonStoppingCriteria.h:95-147): targets out of range are dropped with the
// reference's warning; the _Unoriented forms exist on the lifted models only.
void read_stopping(Store &io, const Param &pm, bool lifted, EulerProblem &p) {
    if (io.has_field("nMaxAccepted")) p.stop_n_max = (int64_t)io.get_scalar("nMaxAccepted");
    auto targets = [&](const char *key, std::vector<int64_t> &out) {
        if (!io.has_field(key)) return;
        int64_t n = 0;
        const std::vector<double> pts = io.get_vector(key, pm.ndim, &n);
        for (int64_t i = 0; i < n; ++i) {
            int64_t lin;
            if (pm.index_of(&pts[i * pm.ndim], &lin)) out.push_back(lin);
            else io.msg("Warning : target is out of range.");
        }
    };
    targets("stopWhenAnyAccepted", p.stop_any);
    targets("stopWhenAllAccepted", p.stop_all);
    auto targets_u = [&](const char *key, std::vector<int64_t> &out) {
        if (!lifted || !io.has_field(key)) return;
        int64_t n = 0;
        const std::vector<double> pts = io.get_vector(key, 2, &n);
        for (int64_t i = 0; i < n; ++i) {
            const double q[3] = {pts[2 * i], pts[2 * i + 1], pm.origin[2] + 0.5 * pm.scale[2]};
            int64_t lin;
            if (pm.index_of(q, &lin)) out.push_back(lin / pm.dims[2]);
            else io.msg("Warning : unoriented target is out of range.");
        }
    };
    targets_u("stopWhenAnyAccepted_Unoriented", p.stop_any_u);
    targets_u("stopWhenAllAccepted_Unoriented", p.stop_all_u);
    if (io.has_field("stopAtDistance")) {
        p.has_stop_distance = true;
        p.stop_distance = io.get_scalar("stopAtDistance");
    }
}

// Static factoring keys (StaticFactoring.hxx:66-84): imported (factoringValues) or computed
// (factoringRadius != 0); either one makes seedRadius default to 2 (:270), the radius key alone too.
struct FactorKeys {
    bool import = false, compute = false, radius_key = false;
};

FactorKeys read_factor_keys(Store &io, const std::string &model) {
    FactorKeys k;
    k.import = io.has_field("factoringValues");
    k.radius_key = io.has_field("factoringRadius");
    k.compute = k.radius_key && io.get_scalar("factoringRadius") != 0;
    if (k.import && k.compute)
        throw Error(HFM_ERR_VALUE, "StaticFactoring error : factoringValues (import) and factoringRadius (compute) both specified.");
    if ((k.import || k.compute) && model != "TTI3")
        throw Error(HFM_ERR_UNSUPPORTED, "static factoring is supported for TTI3 only by the GPU solve path (the Eulerian "
                                         "models apply it through an acceptance-time recompute)");
    return k;
}

// ImportFactor (StaticFactoring.hxx:86-117): values, gradients (a co-vector: adimensionized by
// multiplying by the grid scales), an optional mask and an optional index shift (a subdomain box).
void import_factor(Store &io, const Param &pm, EulerProblem &p) {
    const Field fv = io.get_field("factoringValues", pm.ndim, 1);
    if (!io.has_field("factoringGradients"))
        throw Error(HFM_ERR_VALUE, "StaticFactoring error : factoringGradients are not provided");
    const Field fg = io.get_field("factoringGradients", pm.ndim, pm.ndim);
    Field fm;
    const bool has_mask = io.has_field("factoringMask");
    if (has_mask) fm = io.get_field("factoringMask", pm.ndim, 1);
    p.fac_subdomain = io.has_field("factoringIndexShift");
    if (p.fac_subdomain) {
        const std::vector<double> sh = read_point(io, "factoringIndexShift", pm.ndim, std::vector<double>(pm.ndim, 0.0));
        for (int a = 0; a < pm.ndim; ++a) p.fac_lo[a] = (int)sh[a];
    }
    size_t n = 1;
    for (int a = 0; a < pm.ndim; ++a) {
        const int64_t want = p.fac_subdomain ? fv.dims[a] : pm.dims[a];
        if (fv.dims[a] != want || fg.dims[a] != want || (has_mask && fm.dims[a] != want))
            throw Error(HFM_ERR_VALUE, "Static factoring error : inconsistent data dimension.");
        p.fac_dims[a] = (int)want;
        n *= (size_t)want;
    }
    p.fac_values.assign(fv.ptr(), fv.ptr() + n);
    p.fac_grads.assign(fg.ptr(), fg.ptr() + n * pm.ndim);
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < pm.ndim; ++a) p.fac_grads[i * pm.ndim + a] *= pm.scale[a];  // ReDim
    p.fac_mask.assign(n, 1);
    if (has_mask)
        for (size_t i = 0; i < n; ++i) p.fac_mask[i] = fm.ptr()[i] != 0.0;
}

// ComputeFactor with factoringPointChoice "Seed" (StaticFactoring.hxx:119-175): the distance from
// the single seed x0 in the norm at the seed (interpolated), value(x) = <g, x - x0> with
// g = -Gradient(x0 - x) (0 at the seed), on the cells of the box [floor(x0 - r), ceil(x0 + r)) clipped
// to the domain (the whole domain for r < 0), r truncated to an integer.
void compute_factor(Store &io, const Param &pm, EulerProblem &p) {
    int64_t ns = 0;
    const std::vector<double> pts = io.get_vector("seeds", pm.ndim, &ns);
    if (ns != 1)
        throw Error(HFM_ERR_VALUE, "Exactly one seed point must be specified for computing the factor, found " +
                                       std::to_string(ns) + ".");
    const std::string choice = io.get_string("factoringPointChoice", "Seed");
    if (choice == "Both")
        throw Error(HFM_ERR_UNSUPPORTED, "factoringPointChoice = 'Both' is not supported by the GPU solve path");
    if (choice != "Seed" && choice != "Key")
        throw Error(HFM_ERR_VALUE, "StaticFactoring error : Unsupported factoringPointChoice " + choice + ".");
    const int radius = (int)io.get_scalar("factoringRadius");
    const int D = pm.ndim;
    double seed[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) seed[a] = (pts[a] - pm.origin[a]) / pm.scale[a];
    p.fac_subdomain = radius >= 0;
    size_t n = 1;
    for (int a = 0; a < D; ++a) {
        if (p.fac_subdomain) {
            p.fac_lo[a] = std::max(0, (int)std::floor(seed[a] - radius));
            const int top = std::min(pm.dims[a] - 1, (int)std::ceil(seed[a] + radius));
            p.fac_dims[a] = std::max(0, top - p.fac_lo[a]);
        } else {
            p.fac_lo[a] = 0;
            p.fac_dims[a] = pm.dims[a];
        }
        n *= (size_t)p.fac_dims[a];
    }
    SeedGuess G{p, pm};
    double norm[14];
    G.at_point(seed, norm);
    p.fac_values.assign(n, 0.0);
    p.fac_grads.assign(n * D, 0.0);
    p.fac_mask.assign(n, 1);
    for (size_t i = 0; i < n; ++i) {
        int64_t idx[3], r = (int64_t)i;
        for (int a = D - 1; a >= 0; --a) { idx[a] = r % p.fac_dims[a]; r /= p.fac_dims[a]; }
        double v[3] = {0, 0, 0}, mv[3] = {0, 0, 0}, g[3] = {0, 0, 0};
        bool null = true;
        for (int a = 0; a < D; ++a) {
            v[a] = ((double)(idx[a] + p.fac_lo[a]) + 0.5) - seed[a];
            mv[a] = -v[a];
            null = null && v[a] == 0.0;
        }
        if (!null) {
            SeedGuess::tti_gradient(norm, mv, g);
            for (int a = 0; a < D; ++a) g[a] = -g[a];
        }
        double f = 0.0;
        for (int a = 0; a < D; ++a) f += g[a] * v[a];
        p.fac_values[i] = f;
        for (int a = 0; a < D; ++a) p.fac_grads[i * D + a] = g[a];
    }
    if (io.get_scalar("exportFactoring", 0.0) != 0) {
        const std::vector<int64_t> bd(p.fac_dims, p.fac_dims + D);
        io.set_field("factoringValues", bd, 1, p.fac_values.data());
        io.set_field("factoringGradients", bd, D, p.fac_grads.data());
        if (p.fac_subdomain) {
            const double sh[3] = {(double)p.fac_lo[0], (double)p.fac_lo[1], (double)p.fac_lo[2]};
            io.set_vector("factoringIndexShift", D, 1, sh);
        }
    }
}

// A model read from its store, ready to solve (the part of Run before the solver loop).
struct Prepared {
    Param pm;
    EulerProblem p;
    bool geo_keys[2] = {false, false};  // tips, tips_Unoriented present
    bool export_values = false, export_active = false, skip = false;
    bool get_stencils = false;          // getStencils given: the cells whose stencils are printed
    bool export_stencils = false;       // exportStencils: all Selling stencils as arrays
    std::vector<int64_t> stencil_cells;
    std::vector<int64_t> dims;
    double *values_dst = nullptr;
};

size_t n_cells(const std::vector<int64_t> &dims);

// getStencils (HFMInterface.hxx:360-375): the points are placed like seeds; a point out of range
// is skipped with the reference's warning. Riemann stencils are exported from the GPU's Selling
// arrays; the other models' stencils are their host tables.
void read_get_stencils(Store &io, Prepared &q) {
    if (!io.has_field("getStencils")) return;
    const Param &pm = q.pm;
    if (q.p.kind == StencilKind::TTI)
        throw Error(HFM_ERR_UNSUPPORTED, "getStencils on TTI3 is not supported by the GPU solve path");
    int64_t n = 0;
    const std::vector<double> pts = io.get_vector("getStencils", pm.ndim, &n);
    for (int64_t i = 0; i < n; ++i) {
        int64_t lin;
        if (!pm.index_of(&pts[i * pm.ndim], &lin)) {
            std::ostringstream o;
            o << "GetStencil error : point {";
            for (int a = 0; a < pm.ndim; ++a) o << (a ? "," : "") << pts[i * pm.ndim + a];
            o << "}is out of range.\n";
            io.warn(o.str());
            continue;
        }
        q.stencil_cells.push_back(lin);
    }
    q.get_stencils = true;
    if (q.p.kind == StencilKind::RiemannPerCell && !q.p.diagonal) q.p.want_stencils = true;
}

// exportStencils (an extension, Riemann models): every cell's Selling stencil as arrays,
// stencilOffsets (dims + (K, ndim)) and stencilWeights (dims + (K,)), K = 3 (2D) or 6 (3D), in the
// order and with the full FP64 weights the solver uses.
bool read_export_stencils(Store &io, Prepared &q) {
    if (io.get_scalar("exportStencils", 0.0, 3) == 0) return false;
    if (q.p.kind != StencilKind::RiemannPerCell || q.p.diagonal)
        throw Error(HFM_ERR_UNSUPPORTED, "exportStencils applies to the Riemann models");
    q.p.want_stencils = true;
    return true;
}

// The `stencils` string in the reference's print format: "{" then, per point, "{" index ","
// stencil "}," then "}"; a stencil prints as {"forward" -> {{diffs}},"symmetric" -> {{diffs}},}
// (EulerianStencil.hxx:76-87 with ExportArrayRecursiveArrow, ExportArrow.h:101-102) and a
// difference as {baseWeight,{offset}} with the stream's default 6 significant digits. The base
// weight excludes the speed multiplier (Isotropic, Diagonal and curvature models print 1/h^2 or
// their table weights whatever the speed or cost).
void export_stencils(Store &io, const Prepared &q, const EulerResult &r) {
    if (!q.get_stencils) return;
    const EulerProblem &p = q.p;
    const Param &pm = q.pm;
    const int D = pm.ndim;
    std::ostringstream o;
    // a difference's offset: its D components (the sphere bundle's are the x, y, z steps followed by
    // the theta and phi steps)
    auto diff = [&](double w, const int8_t *off, const int8_t *ang = nullptr) {
        o << "{" << w << ",{";
        for (int a = 0; a < D; ++a) o << (a ? "," : "") << (int)(a < 3 || !ang ? off[a] : ang[a - 3]);
        o << "}}";
    };
    o << "{";
    for (int64_t x : q.stencil_cells) {
        int64_t idx[5], rr = x;
        for (int a = D - 1; a >= 0; --a) { idx[a] = rr % pm.dims[a]; rr /= pm.dims[a]; }
        o << "{{";
        for (int a = 0; a < D; ++a) o << (a ? "," : "") << idx[a];
        o << "},{\"forward\" -> {{";
        if (p.kind == StencilKind::SharedByTheta) {
            const int ND = p.nfwd + p.nsym;
            const bool s2 = p.sphere_nth > 0;
            const int64_t cls = s2 ? idx[3] * p.sphere_nph + idx[4] : p.nclass > 1 ? idx[2] : 0;
            auto ang = [&](int k) { return s2 ? &p.cls_ang[(cls * ND + k) * 2] : nullptr; };
            for (int k = 0; k < p.nfwd; ++k) {
                if (k) o << ",";
                diff(p.cls_w[cls * ND + k], &p.cls_off[(cls * ND + k) * 3], ang(k));
            }
            o << "}},\"symmetric\" -> {{";
            for (int k = p.nfwd; k < ND; ++k) {
                if (k > p.nfwd) o << ",";
                diff(p.cls_w[cls * ND + k], &p.cls_off[(cls * ND + k) * 3], ang(k));
            }
        } else if (p.diagonal) {  // one difference per axis, base weight 1 / h_i^2
            o << "}},\"symmetric\" -> {{";
            for (int k = 0; k < D; ++k) {
                int8_t e[3] = {0, 0, 0};
                e[k] = 1;
                if (k) o << ",";
                diff(1. / (p.h[k] * p.h[k]), e);
            }
        } else {
            const int NK = D == 2 ? 3 : 6;
            if (r.stencil_off.size() < (size_t)(x + 1) * NK * 3)
                throw Error(HFM_ERR_VALUE, "stencils of the requested points were not exported");
            o << "}},\"symmetric\" -> {{";
            for (int k = 0; k < NK; ++k) {
                int8_t e[3];
                for (int a = 0; a < D; ++a) e[a] = r.stencil_off[((size_t)x * NK + k) * 3 + a];
                if (k) o << ",";
                diff(r.stencil_w[(size_t)x * NK + k], e);
            }
        }
        o << "}},}},";
    }
    o << "}";
    io.set_string("stencils", o.str());
}

void export_stencil_arrays(Store &io, const Prepared &q, const EulerResult &r) {
    if (!q.export_stencils) return;
    const int D = q.pm.ndim, NK = D == 2 ? 3 : 6;
    const size_t n = n_cells(q.dims);
    std::vector<double> off(n * NK * D);
    for (size_t x = 0; x < n; ++x)
        for (int k = 0; k < NK; ++k)
            for (int a = 0; a < D; ++a) off[(x * NK + k) * D + a] = (double)r.stencil_off[(x * NK + k) * 3 + a];
    std::vector<int64_t> od(q.dims);
    od.push_back(NK);
    io.set_field("stencilOffsets", od, D, off.data());
    io.set_field("stencilWeights", od, 1, r.stencil_w.data());
}

void prepare_model(Store &io, const std::string &model, Prepared &q) {
    Param &pm = q.pm;
    EulerProblem &p = q.p;
    // Run_SetupIO (HFMInterface.hxx:311-341)
    io.verbosity = (int)io.get_scalar("verbosity", io.verbosity);
    if (io.has_field("keyHelp")) io.get_string("keyHelp");
    const std::string ord = io.get_string("arrayOrdering", ordering_name(io.ordering()));
    Ordering o;
    if (!ordering_from_name(ord, &o)) throw Error(HFM_ERR_VALUE, "Error : unrecognized array ordering");
    io.set_ordering(o);
    reject_unsupported(io);

    const bool lifted = model == "ReedsShepp2" || model == "ReedsSheppForward2" || model == "Elastica2" ||
                        model == "Dubins2";
    if (model == "Riemann2") setup_riemann(io, 2, pm, p);
    else if (model == "Riemann3") setup_riemann(io, 3, pm, p);
    else if (model == "Isotropic2") setup_isotropic(io, 2, pm, p);
    else if (model == "Isotropic3") setup_isotropic(io, 3, pm, p);
    else if (model == "Diagonal2") setup_diagonal(io, 2, pm, p);
    else if (model == "Diagonal3") setup_diagonal(io, 3, pm, p);
    else if (lifted) setup_curvature(io, model, pm, p);
    else if (model == "ReedsShepp3" || model == "ReedsSheppForward3")
        setup_reedsshepp3(io, pm, p, model == "ReedsSheppForward3");
    else if (model == "TTI3") setup_tti(io, pm, p);
    else throw Error(HFM_ERR_UNSUPPORTED, "Unrecognized model : " + model);
    set_common_solver_options(io, p);
    read_walls(io, pm, lifted, p);
    // StaticFactoring::Setup (StaticFactoring.hxx:66-84): import, seeds, compute
    const FactorKeys fk = read_factor_keys(io, model);
    if (fk.import) import_factor(io, pm, p);
    read_seeds(io, pm, p, lifted, (fk.import || fk.radius_key) ? 2.0 : 0.0);
    if (fk.compute) compute_factor(io, pm, p);

    read_stopping(io, pm, lifted, p);
    read_geodesics(io, pm, lifted, p, q.geo_keys);
    q.export_values = io.get_scalar("exportValues", 0.0, 2) != 0;
    p.retain = io.get_scalar("retainState", 0.0, 3) != 0;
    q.export_active = io.get_scalar("exportActiveNeighs", 0.0, 3) != 0;
    const bool inspect = io.has_field("inspectSensitivity");
    p.want_active = q.export_active;

    q.dims.assign(pm.dims, pm.dims + pm.ndim);
    // values and activeNeighs given: the solve is bypassed (HFMInterface.hxx:399-427); the cells
    // without an active neighbour (the seeds of the run that produced them) are fixed, since the
    // reference's Recompute gives them no flow
    if (io.has_field("values") || io.has_field("activeNeighs")) {
        if (!(io.has_field("values") && io.has_field("activeNeighs")))
            throw Error(HFM_ERR_UNSUPPORTED, "values without activeNeighs (or the converse) is not supported by the GPU solve path");
        const Field fv = io.get_field("values", pm.ndim, 1), fa = io.get_field("activeNeighs", pm.ndim, 1);
        for (int a = 0; a < pm.ndim; ++a)
            if (fv.dims[a] != pm.dims[a] || fa.dims[a] != pm.dims[a])
                throw Error(HFM_ERR_VALUE, "values and activeNeighs must have the domain's dims");
        const size_t n = fv.size();
        p.bypass = true;
        p.bypass_values.assign(fv.ptr(), fv.ptr() + n);
        p.seed_index.clear();
        p.seed_value.clear();
        const double *act = fa.ptr();
        const bool tti = p.kind == StencilKind::TTI;
        for (size_t x = 0; x < n; ++x) {
            const bool none = tti ? !(act[x] < std::numeric_limits<double>::infinity()) : act[x] == 0.0;
            if (none && p.bypass_values[x] < std::numeric_limits<double>::infinity()) {
                p.seed_index.push_back((int64_t)x);
                p.seed_value.push_back(p.bypass_values[x]);
            }
        }
        if (io.verbosity >= 1) io.msg("Bypassing fast marching solver based on cached data.\n");
    }
    if (p.seed_index.empty() && !p.bypass) {
        io.warn("No seeds to run fast marching solver, and missing values or activeNeighs to compute geodesics.\n");
        q.skip = true;
        return;
    }
    read_get_stencils(io, q);
    q.export_stencils = read_export_stencils(io, q);
    if (inspect) read_inspect(io, pm, p);
    read_forward_variation(io, pm, p);
    // Dubins2 first variations and geodesics: an illegal memory access was met twice on the GPU on
    // a fixture with both (its cause is not found); they stay off the device until it is
    if (p.nmax == 2 && (inspect || p.fwd_nvar > 0 || !p.geo_tips.empty() || !p.geo_tips_unoriented.empty() ||
                        p.want_geodesic_flow))
        throw Error(HFM_ERR_UNSUPPORTED, "Dubins2 first variations and geodesics are not supported by the GPU solve path");
    if (p.has_factoring() && (inspect || p.fwd_nvar > 0 || p.has_stopping() || !p.geo_tips.empty() ||
                              p.want_geodesic_flow || p.bypass || p.retain))
        throw Error(HFM_ERR_UNSUPPORTED, "static factoring with first variations, geodesics, stopping criteria, cached "
                                         "values or retained state is not supported by the GPU solve path");
    // the arrival times are downloaded straight into the output field when no reordering is needed
    q.values_dst = q.export_values ? io.create_field("values", q.dims, 1) : nullptr;
    p.h_values_out = q.values_dst;
}

size_t n_cells(const std::vector<int64_t> &dims) {
    size_t n = 1;
    for (int64_t d : dims) n *= (size_t)d;
    return n;
}

// costSensitivity_i and seedSensitivity_i (point, weight) of each inspection group.
void export_sensitivities(Store &io, const Param &pm, const std::vector<int64_t> &dims,
                          const std::vector<AdjointResult> &adjoints) {
    for (size_t gi = 0; gi < adjoints.size(); ++gi) {
        const AdjointResult &ar = adjoints[gi];
        const int comp = (int)(ar.sensitivity.size() / std::max<size_t>(1, n_cells(dims)));
        io.set_field("costSensitivity_" + std::to_string(gi), dims, comp, ar.sensitivity.data());
        std::vector<double> ss;
        for (size_t k = 0; k < ar.seed_index.size(); ++k) {
            int64_t x = ar.seed_index[k];
            double q[3];
            for (int a = pm.ndim - 1; a >= 0; --a) {
                const int64_t i = x % pm.dims[a];
                x /= pm.dims[a];
                q[a] = (i + 0.5) * pm.scale[a] + pm.origin[a];  // ReDim(PointFromIndex)
            }
            for (int a = 0; a < pm.ndim; ++a) ss.push_back(q[a]);
            ss.push_back(ar.seed_weight[k]);
        }
        io.set_vector("seedSensitivity_" + std::to_string(gi), (int64_t)ar.seed_index.size(), pm.ndim + 1,
                      ss.data());
    }
}

// geodesicPoints / geodesicLengths (suffix _Unoriented for tips_Unoriented) in physical
// coordinates (ReDim), the reference's messages for failed tips (GeodesicDiscreteSolver.hxx:17-34),
// and geodesicFlow = -ReDim(flow) (HFMInterface.hxx:452-485, 541-553).
void export_geodesics(Store &io, const Prepared &q, const EulerResult &r) {
    const Param &pm = q.pm;
    const int D = pm.ndim;
    for (int gi = 0; gi < 2; ++gi) {
        if (!q.geo_keys[gi]) continue;
        const std::string suffix = gi ? "_Unoriented" : "";
        std::vector<double> pts(r.geo_points[gi]);
        for (size_t k = 0; k < pts.size(); ++k) pts[k] = pts[k] * pm.scale[k % D] + pm.origin[k % D];
        std::vector<double> lens(r.geo_lengths[gi].begin(), r.geo_lengths[gi].end());
        size_t first = 0;
        for (size_t t = 0; t < lens.size(); ++t) {
            std::ostringstream tip;
            tip << "{";
            for (int a = 0; a < D; ++a) tip << (a ? "," : "") << pts[first * D + a];
            tip << "}";
            const int st = r.geo_status[gi][t];
            if (io.verbosity < 1) {
            } else if ((st & 1) && q.p.geo_ode) {
                io.msg("Geodesic ODE solver seems to have failed for tip " + tip.str() + ".\n");
            } else if (st & 1) {
                io.msg("Geodesic extraction failed for tip " + tip.str() + "\n");
            } else if (r.geo_restarts[gi][t] > 5) {
                double vb = q.p.geo_volume_bound;
                for (int k = 5; k <= r.geo_restarts[gi][t]; ++k) vb *= 1.3;
                std::ostringstream m;
                m << "Tip " << tip.str() << " yields " << r.geo_restarts[gi][t] << " restarts, "
                  << "geodesicVolumeBound increased to " << vb << "\n";
                io.msg(m.str());
            }
            if (st & ~1)
                io.warn("Geodesic extraction for tip " + tip.str() + " stopped early (" +
                        ((st & 6) ? std::string("out of room") : (st & 8) ? std::string("iteration limit") : std::string("index range")) + ")\n");
            first += (size_t)lens[t];
        }
        io.set_vector("geodesicPoints" + suffix, (int64_t)(pts.size() / D), D, pts.data());
        io.set_vector("geodesicLengths" + suffix, (int64_t)lens.size(), 1, lens.data());
    }
    if (q.p.want_geodesic_flow && !r.geodesic_flow.empty()) {
        std::vector<double> f(r.geodesic_flow.size());
        for (size_t k = 0; k < f.size(); ++k) f[k] = -(r.geodesic_flow[k] * pm.scale[k % D]);
        io.set_field("geodesicFlow", q.dims, D, f.data());
    }
}

void finish_model(Store &io, const Prepared &q, const EulerResult &r) {
    const Param &pm = q.pm;
    const std::vector<int64_t> &dims = q.dims;
    // Outputs (Run_SetupSolver/Run_RunSolver/Run_ExportData, CommonStoppingCriteria::Finally)
    io.set_scalar("MaxStencilWidth", r.max_stencil_width);
    export_stencils(io, q, r);
    export_stencil_arrays(io, q, r);
    io.set_scalar("StencilCPUTime", r.t_stencil_ms * 1e-3);
    io.set_scalar("FMCPUTime", r.t_solve_ms * 1e-3);
    io.set_scalar("GeodesicCPUTime", r.t_geodesic_ms * 1e-3);
    io.set_scalar("GPUStencilTime", r.t_stencil_ms * 1e-3);
    io.set_scalar("GPUSolveTime", r.t_solve_ms * 1e-3);
    io.set_scalar("solverRounds", (double)r.rounds);
    io.set_scalar("tileActivations", (double)r.tile_activations);
    io.set_scalar("executedUpdates", (double)r.local_solves);
    io.set_scalar("tileCarries", (double)r.tile_carries);
    if (io.verbosity >= 1) {
        std::ostringstream m;
        m << "Fast marching solver completed in " << r.t_solve_ms * 1e-3 << " s.\n";
        io.msg(m.str());
    }
    if (q.export_values && !q.values_dst) io.set_field("values", dims, 1, r.values.data());
    if (q.export_active) {
        std::vector<double> a(r.active.size());
        if (q.p.kind == StencilKind::TTI)  // the extremum t, stored as the bits of a double
            std::memcpy(a.data(), r.active.data(), a.size() * sizeof(double));
        else
            for (size_t i = 0; i < a.size(); ++i) a[i] = (double)r.active[i];
        io.set_field("activeNeighs", dims, 1, a.data());
    }
    export_sensitivities(io, pm, dims, r.adjoints);
    if (q.p.fwd_nvar > 0) {
        std::vector<int64_t> vd(dims);
        vd.push_back(q.p.fwd_nvar);
        io.set_field("valueVariation", vd, 1, r.value_variation.data());
    }
    export_geodesics(io, q, r);
    io.set_scalar("nAccepted", (double)r.n_accepted);
}


// The device state of the last retainState solve of a store, with its grid description.
struct RetainedCtx {
    std::shared_ptr<RetainedSolve> solve;
    Param pm;
    std::vector<int64_t> dims;
};

void run_model(Store &io, const std::string &model, std::shared_ptr<void> *retained) {
    Prepared q;
    prepare_model(io, model, q);
    if (q.skip) return;
    EulerResult r;
    try {
        solve_eulerian(q.p, r);
    } catch (...) {
        if (q.values_dst) io.erase_field("values");
        throw;
    }
    finish_model(io, q, r);
    if (retained) {
        if (r.retained) {
            auto ctx = std::make_shared<RetainedCtx>();
            ctx->solve = r.retained;
            ctx->pm = q.pm;
            ctx->dims = q.dims;
            *retained = ctx;
        } else {
            retained->reset();
        }
    }
}

// Reverse first variation of the retained solve for the inspectSensitivity keys now in the store.
void run_sensitivity(Store &io, const std::shared_ptr<void> &retained) {
    if (!retained) throw Error(HFM_ERR_ARG, "no retained solve on this store (run it with retainState = 1)");
    const RetainedCtx &ctx = *static_cast<const RetainedCtx *>(retained.get());
    if (!io.has_field("inspectSensitivity")) throw Error(HFM_ERR_KEY, "BaseIO import error : field inspectSensitivity not found.");
    EulerProblem p;
    read_inspect(io, ctx.pm, p);
    EulerResult r;
    ctx.solve->adjoint(p, r);
    export_sensitivities(io, ctx.pm, ctx.dims, r.adjoints);
    io.set_scalar("GPUAdjointTime", r.t_adjoint_ms * 1e-3);
}

}  // namespace

namespace {
struct PreparedRunImpl final : PreparedRun {
    hfm_io *io;
    Prepared q;
    explicit PreparedRunImpl(hfm_io *h) : io(h) {}
    ~PreparedRunImpl() override { io->store.current_setter = Setter::User; }
    EulerProblem &problem() override { return q.p; }
    bool skip() const override { return q.skip; }
    void finish(const EulerResult &r) override {
        finish_model(io->store, q, r);
        io->store.usage_report();
    }
    void fail() override {
        if (q.values_dst) io->store.erase_field("values");
        q.values_dst = nullptr;
    }
};
}  // namespace

// Parses a store as hfm_run does; the store stays in the compute setter until the handle goes.
std::unique_ptr<PreparedRun> prepare_run(hfm_io *io) {
    auto r = std::make_unique<PreparedRunImpl>(io);
    Store &st = io->store;
    st.current_setter = Setter::Compute;
    const std::string model = st.get_string("model");
    prepare_model(st, model == "Elastica2_5" ? "Elastica2" : model, r->q);
    r->q.p.retain = false;
    return r;
}

}  // namespace hfm

// =============================================================================== C ABI
using hfm::Error;

template <typename F>
static int guarded(hfm_io *io, F f) {
    if (!io) return HFM_ERR_ARG;
    io->last_error.clear();
    try {
        f();
        return HFM_OK;
    } catch (const Error &e) {
        io->last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        io->last_error = "host allocation failure";
        return HFM_ERR_NOMEM;
    } catch (const std::exception &e) {
        io->last_error = e.what();
        return HFM_ERR_VALUE;
    }
}

extern "C" {

hfm_io *hfm_io_create(int default_ordering) {
    if (default_ordering < 0 || default_ordering > 3) return nullptr;
    try {
        return new hfm_io(static_cast<hfm::Ordering>(default_ordering));
    } catch (...) {
        return nullptr;
    }
}

void hfm_io_destroy(hfm_io *io) { delete io; }

int hfm_io_set_scalar(hfm_io *io, const char *key, double value) {
    return guarded(io, [&] {
        if (!key) throw Error(HFM_ERR_ARG, "null key");
        io->store.set_scalar(key, value);
    });
}

int hfm_io_set_string(hfm_io *io, const char *key, const char *value) {
    return guarded(io, [&] {
        if (!key || !value) throw Error(HFM_ERR_ARG, "null argument");
        io->store.set_string(key, value);
    });
}

int hfm_io_set_array(hfm_io *io, const char *key, const double *data, int ndim, const int64_t *shape) {
    return guarded(io, [&] {
        if (!key || ndim < 0 || (ndim > 0 && !shape)) throw Error(HFM_ERR_ARG, "null argument");
        std::vector<int64_t> dims(shape, shape + ndim);
        int64_t n = 1;
        for (int64_t d : dims) n *= d;
        if (n > 0 && !data) throw Error(HFM_ERR_ARG, "null data");
        io->store.set_array(key, data, dims);
    });
}

int hfm_io_set_array_view(hfm_io *io, const char *key, const double *data, int ndim, const int64_t *shape) {
    return guarded(io, [&] {
        if (!key || ndim < 0 || (ndim > 0 && !shape)) throw Error(HFM_ERR_ARG, "null argument");
        io->store.set_array_view(key, data, std::vector<int64_t>(shape, shape + ndim));
    });
}

int hfm_io_get_scalar(hfm_io *io, const char *key, double *value) {
    return guarded(io, [&] {
        if (!key || !value) throw Error(HFM_ERR_ARG, "null argument");
        *value = io->store.get_scalar(key);
    });
}

int hfm_io_get_string(hfm_io *io, const char *key, char *buf, size_t cap, size_t *len) {
    return guarded(io, [&] {
        if (!key) throw Error(HFM_ERR_ARG, "null key");
        const std::string s = io->store.get_string(key);
        if (len) *len = s.size();
        if (buf && cap) {
            const size_t n = std::min(cap - 1, s.size());
            std::memcpy(buf, s.data(), n);
            buf[n] = 0;
        }
    });
}

int hfm_io_get_array_info(hfm_io *io, const char *key, int *ndim, int64_t *shape, int max_ndim) {
    return guarded(io, [&] {
        if (!key || !ndim) throw Error(HFM_ERR_ARG, "null argument");
        const hfm::RawElement &r = io->store.raw(key, false);
        if (r.is_string()) throw Error(HFM_ERR_KEY, "PythonIO error : field " + std::string(key) + " is a string, not an array");
        *ndim = (int)r.dims.size();
        for (int i = 0; i < *ndim && i < max_ndim; ++i)
            if (shape) shape[i] = r.dims[i];
    });
}

int hfm_io_get_array(hfm_io *io, const char *key, double *out, size_t count) {
    return guarded(io, [&] {
        if (!key || (count && !out)) throw Error(HFM_ERR_ARG, "null argument");
        const hfm::RawElement &r = io->store.raw(key);
        if (r.is_string()) throw Error(HFM_ERR_KEY, "PythonIO error : field " + std::string(key) + " is a string, not an array");
        if (r.dims.empty()) throw Error(HFM_ERR_KEY, "PythonIO error : field " + std::string(key) + " is a scalar, not an array");
        if (count != r.count()) throw Error(HFM_ERR_ARG, "buffer size does not match field " + std::string(key));
        std::memcpy(out, r.ptr(), count * sizeof(double));
    });
}

int hfm_io_get_array_ptr(hfm_io *io, const char *key, const double **data, int *ndim, int64_t *shape,
                         int max_ndim) {
    return guarded(io, [&] {
        if (!key || !data || !ndim) throw Error(HFM_ERR_ARG, "null argument");
        const hfm::RawElement &r = io->store.raw(key);
        if (r.is_string()) throw Error(HFM_ERR_KEY, "PythonIO error : field " + std::string(key) + " is a string, not an array");
        *ndim = (int)r.dims.size();
        if (shape)
            for (int i = 0; i < *ndim && i < max_ndim; ++i) shape[i] = r.dims[i];
        *data = r.ptr();
    });
}

int hfm_io_has_field(hfm_io *io, const char *key) {
    if (!io || !key) return -HFM_ERR_ARG;
    return io->store.has_field(key) ? 1 : 0;
}

int hfm_io_erase_field(hfm_io *io, const char *key) {
    return guarded(io, [&] {
        if (!key) throw Error(HFM_ERR_ARG, "null key");
        if (!io->store.erase_field(key)) throw Error(HFM_ERR_KEY, "field " + std::string(key) + " not found");
    });
}

int hfm_io_computed_keys(hfm_io *io, char *buf, size_t cap, size_t *len) {
    return guarded(io, [&] {
        const std::string s = io->store.computed_keys();
        if (len) *len = s.size();
        if (buf && cap) {
            const size_t n = std::min(cap - 1, s.size());
            std::memcpy(buf, s.data(), n);
            buf[n] = 0;
        }
    });
}

int hfm_run(hfm_io *io, const char *expected_model) {
    return guarded(io, [&] {
        hfm::Store &st = io->store;
        const std::string model = st.get_string("model");
        if (expected_model && model != expected_model)
            throw Error(HFM_ERR_VALUE, std::string("Executable applies to ") + expected_model + ", not to " + model + ".");
        st.current_setter = hfm::Setter::Compute;
        struct Restore {
            hfm::Store &s;
            ~Restore() { s.current_setter = hfm::Setter::User; }
        } restore{st};
        hfm::run_model(st, model == "Elastica2_5" ? "Elastica2" : model, &io->retained);
        st.usage_report();
    });
}

int hfm_run_batch(hfm_io *const *ios, int n, const char *expected_model, int *codes) {
    if (n < 0 || (n > 0 && !ios)) return HFM_ERR_ARG;
    for (int i = 0; i < n; ++i)
        if (!ios[i]) return HFM_ERR_ARG;
    std::vector<int> rc(n, HFM_OK);
    std::vector<std::unique_ptr<hfm::Prepared>> qs(n);
    for (int i = 0; i < n; ++i) ios[i]->store.current_setter = hfm::Setter::Compute;
    // Reading: every instance on its own (errors stay with their instance).
    for (int i = 0; i < n; ++i) {
        rc[i] = guarded(ios[i], [&] {
            hfm::Store &st = ios[i]->store;
            const std::string model = st.get_string("model");
            if (expected_model && model != expected_model)
                throw Error(HFM_ERR_VALUE,
                            std::string("Executable applies to ") + expected_model + ", not to " + model + ".");
            auto q = std::make_unique<hfm::Prepared>();
            hfm::prepare_model(st, model == "Elastica2_5" ? "Elastica2" : model, *q);
            q->p.retain = false;  // device state is retained by hfm_run only
            qs[i] = std::move(q);
        });
    }
    // Solving: instances of one stencil family and precision share one launch sequence; first
    // variation requests (inspectSensitivity, costVariation, seedValueVariation) run on their own.
    std::vector<char> done(n, 0);
    for (int i = 0; i < n; ++i) {
        if (rc[i] != HFM_OK || done[i] || qs[i]->skip) continue;
        std::vector<int> grp{i};
        done[i] = 1;
        const hfm::EulerProblem &pi = qs[i]->p;
        if (pi.adjoint_index.empty() && pi.fwd_nvar == 0 && !pi.has_stopping() && !pi.bypass) {
            for (int j = i + 1; j < n; ++j) {
                if (rc[j] != HFM_OK || done[j] || qs[j]->skip) continue;
                const hfm::EulerProblem &pj = qs[j]->p;
                if (pj.adjoint_index.empty() && pj.fwd_nvar == 0 && !pj.has_stopping() && !pj.bypass &&
                    pj.kind == pi.kind && pj.diagonal == pi.diagonal && pj.ndim == pi.ndim && pj.nfwd == pi.nfwd &&
                    pj.nsym == pi.nsym && pj.fp64 == pi.fp64 && pj.sweeps_per_tile == pi.sweeps_per_tile &&
                    pj.max_rounds == pi.max_rounds) {
                    grp.push_back(j);
                    done[j] = 1;
                }
            }
        }
        std::vector<const hfm::EulerProblem *> probs;
        for (int j : grp) probs.push_back(&qs[j]->p);
        std::vector<hfm::EulerResult> res;
        hfm_io *lead = ios[grp[0]];
        int code = guarded(lead, [&] { hfm::solve_eulerian_batch(probs, res); });
        if (code != HFM_OK && code != HFM_ERR_CUDA && grp.size() > 1) {
            // an invalid instance (e.g. a non-SPD metric) fails its whole group: solve the members
            // one by one so that the error stays with its own store
            res.assign(grp.size(), hfm::EulerResult());
            for (size_t k = 0; k < grp.size(); ++k) {
                const int j = grp[k];
                rc[j] = guarded(ios[j], [&] { hfm::solve_eulerian(qs[j]->p, res[k]); });
                if (rc[j] != HFM_OK && qs[j]->values_dst) ios[j]->store.erase_field("values");
            }
            for (size_t k = 0; k < grp.size(); ++k) {
                const int j = grp[k];
                if (rc[j] == HFM_OK) rc[j] = guarded(ios[j], [&] { hfm::finish_model(ios[j]->store, *qs[j], res[k]); });
            }
            continue;
        }
        for (size_t k = 0; k < grp.size(); ++k) {
            const int j = grp[k];
            if (code != HFM_OK) {
                rc[j] = code;
                ios[j]->last_error = lead->last_error;
                if (qs[j]->values_dst) ios[j]->store.erase_field("values");
                continue;
            }
            rc[j] = guarded(ios[j], [&] { hfm::finish_model(ios[j]->store, *qs[j], res[k]); });
        }
    }
    int first = HFM_OK;
    for (int i = 0; i < n; ++i) {
        if (rc[i] == HFM_OK) rc[i] = guarded(ios[i], [&] { ios[i]->store.usage_report(); });
        ios[i]->store.current_setter = hfm::Setter::User;
        if (codes) codes[i] = rc[i];
        if (first == HFM_OK) first = rc[i];
    }
    return first;
}

int hfm_run_sensitivity(hfm_io *io) {
    return guarded(io, [&] {
        hfm::Store &st = io->store;
        st.current_setter = hfm::Setter::Compute;
        struct Restore {
            hfm::Store &s;
            ~Restore() { s.current_setter = hfm::Setter::User; }
        } restore{st};
        hfm::run_sensitivity(st, io->retained);
    });
}

const char *hfm_io_last_error(hfm_io *io) { return io ? io->last_error.c_str() : "null hfm_io"; }

const char *hfm_version(void) { return "hfm_b200 0.1 (sm_100a)"; }

int hfm_device_count(int *count) {
    if (!count) return HFM_ERR_ARG;
    const cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? HFM_OK : HFM_ERR_CUDA;
    }
    return HFM_OK;
}

}  // extern "C"
