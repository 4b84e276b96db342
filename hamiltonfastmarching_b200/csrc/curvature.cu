// Host-side stencil tables of the curvature-penalised models on the lifted grid (x, y, theta).
//
// There are only ntheta distinct stencils, so they are built once on the host with the C
// library's cos/sin, which is what the reference does (its Share policy builds one stencil per
// angle index, Headers/Base/Implementation/HFM_StencilShare.hxx:132-181). The arithmetic follows:
//   Voronoi1Vec (relaxed rank-one tensor, tolerances, reorientation)  CommonTraits.h:118-161
//   StencilReedsShepp2::SetStencil                                      Curvature2.h:48-66
//   StencilReedsSheppForward2::SetStencil                               Curvature2.h:86-100
//   StencilDubins2::SetStencil                                          Curvature2.h:113-140
//   StencilElastica2<5>::SetStencil and its Fejer weights               Curvature2.h:178-234
//   StencilReedsShepp3::SetStencil (R^3 x S^2, Voronoi1Mat)             Curvature3.h:37-58
//   StencilReedsSheppForward3::SetStencil (R^3 x S^2, Voronoi1Vec)      Curvature3.h:79-95
#include <cmath>

#include "selling.cuh"
#include "solver.hpp"

namespace hfm {

static const double kPi = 3.141592653589793238462643383279502884;

template <int D>
static void voronoi1vec(const double *v, double eps, int8_t *off, double *w) {
    double relaxed[6];
    double sq = 0.0;
    for (int i = 0; i < D; ++i) sq += v[i] * v[i];
    const double e2 = eps * eps;
    const double s1 = 1.0 - e2;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j <= i; ++j) {
            const double exact = v[i] * v[j];
            const double id = (double)(i == j) * sq * e2;
            relaxed[sym_idx(i, j)] = exact * s1 + id;
        }
    int o[6][3];
    double ww[6];
    if (!tensor_decomposition<D>(relaxed, o, ww))
        throw Error(HFM_ERR_VALUE, "ObtuseSuperbase error : input must be positive definite");
    const double angleTol = 1.0 / std::sqrt((double)(D - 1));
    const double wTol = sq * (1000.0 * 2.220446049250313080847e-16);
    const double angTol = (1.0 + angleTol * angleTol) / sq;
    const int nk = D == 2 ? 3 : 6;
    for (int k = 0; k < nk; ++k) {
        double scal = 0.0, on = 0.0;
        for (int c = 0; c < D; ++c) scal += v[c] * (double)o[k][c];
        for (int c = 0; c < D; ++c) on += (double)o[k][c] * (double)o[k][c];
        w[k] = (ww[k] < wTol || (scal * scal) * angTol < on) ? 0.0 : ww[k];
        for (int c = 0; c < 3; ++c) off[3 * k + c] = (int8_t)(c < D ? (scal <= 0 ? o[k][c] : -o[k][c]) : 0);
    }
}

void reedsshepp2_table(int ntheta, double h, double xi, double eps, bool projective, std::vector<int8_t> &off,
                       std::vector<double> &w) {
    off.assign((size_t)ntheta * 4 * 3, 0);
    w.assign((size_t)ntheta * 4, 0.0);
    const double ds = (projective ? kPi : 2.0 * kPi) / (double)ntheta;
    const double ih = 1.0 / h;
    for (int t = 0; t < ntheta; ++t) {
        const double theta = (double)t * ds;
        const double v[2] = {std::cos(theta) * ih, std::sin(theta) * ih};
        voronoi1vec<2>(v, eps, &off[t * 12], &w[t * 4]);
        off[t * 12 + 9] = 0;
        off[t * 12 + 10] = 0;
        off[t * 12 + 11] = 1;
        const double xd = xi * ds;
        w[t * 4 + 3] = 1.0 / (xd * xd);
    }
}

// Forward-only car: per angle, the 3 forward differences of the 2D Voronoi1Vec of (cos, sin)/h
// followed by one symmetric angular difference, offset (0, 0, -1), weight 1/(xi dtheta)^2.
void reedssheppforward2_table(int ntheta, double h, double xi, double eps, std::vector<int8_t> &off,
                              std::vector<double> &w) {
    off.assign((size_t)ntheta * 4 * 3, 0);
    w.assign((size_t)ntheta * 4, 0.0);
    const double ds = 2.0 * kPi / (double)ntheta;
    const double ih = 1.0 / h;
    const double xd = xi * ds;
    for (int t = 0; t < ntheta; ++t) {
        const double theta = (double)t * ds;
        const double v[2] = {std::cos(theta) * ih, std::sin(theta) * ih};
        voronoi1vec<2>(v, eps, &off[t * 12], &w[t * 4]);
        off[t * 12 + 9] = 0;
        off[t * 12 + 10] = 0;
        off[t * 12 + 11] = -1;
        w[t * 4 + 3] = 1.0 / (xd * xd);
    }
}

// Dubins car: per angle two stencils of 6 forward differences, the first the 3D Voronoi1Vec of
// (cos/h, sin/h, 1/(xi dtheta)), the second the same differences with the angular component of
// each offset negated (turning the other way). Layout per angle: 12 forward differences, stencil 0
// then stencil 1.
void dubins2_table(int ntheta, double h, double xi, double eps, std::vector<int8_t> &off, std::vector<double> &w) {
    off.assign((size_t)ntheta * 12 * 3, 0);
    w.assign((size_t)ntheta * 12, 0.0);
    const double ds = (2.0 * kPi) / (double)ntheta;
    for (int t = 0; t < ntheta; ++t) {
        int8_t *O = &off[(size_t)t * 36];
        double *W = &w[(size_t)t * 12];
        const double theta = (double)t * ds;
        const double v[3] = {std::cos(theta) / h, std::sin(theta) / h, 1. / (xi * ds)};
        voronoi1vec<3>(v, eps, O, W);
        for (int i = 0; i < 6; ++i) {
            W[6 + i] = W[i];
            O[(6 + i) * 3 + 0] = O[i * 3 + 0];
            O[(6 + i) * 3 + 1] = O[i * 3 + 1];
            O[(6 + i) * 3 + 2] = (int8_t)(-O[i * 3 + 2]);
        }
    }
}

void elastica2_table(int ntheta, double h, double xi, double eps, std::vector<int8_t> &off, std::vector<double> &w) {
    static const double fejer[5] = {0.167781, 0.525552, 0.613333, 0.525552, 0.167781};
    const int nF = 5;
    off.assign((size_t)ntheta * 27 * 3, 0);
    w.assign((size_t)ntheta * 27, 0.0);
    const double ds = (2.0 * kPi) / (double)ntheta;
    for (int t = 0; t < ntheta; ++t) {
        int8_t *O = &off[(size_t)t * 81];
        double *W = &w[(size_t)t * 27];
        const double theta = (2.0 * kPi * (double)t) / (double)ntheta;
        for (int l = 0; l < nF / 2; ++l) {
            const double phi = kPi * (l + 0.5) / nF;
            const double v[3] = {std::sin(phi) * std::cos(theta) / h, std::sin(phi) * std::sin(theta) / h,
                                 std::cos(phi) / (xi * ds)};
            const int s0 = 2 * l, s1 = 2 * l + 1;
            voronoi1vec<3>(v, eps, O + 6 * s0 * 3, W + 6 * s0);
            for (int i = 0; i < 6; ++i) {
                W[6 * s0 + i] *= fejer[l];
                W[6 * s1 + i] = W[6 * s0 + i];
                for (int c = 0; c < 3; ++c) O[(6 * s1 + i) * 3 + c] = O[(6 * s0 + i) * 3 + c];
                O[(6 * s1 + i) * 3 + 2] = (int8_t)(-O[(6 * s1 + i) * 3 + 2]);
            }
        }
        const double v2[2] = {std::cos(theta) / h, std::sin(theta) / h};
        voronoi1vec<2>(v2, eps, O + 6 * (nF - 1) * 3, W + 6 * (nF - 1));
        for (int i = 0; i < 3; ++i) W[6 * (nF - 1) + i] *= fejer[nF / 2];
    }
}

// ReedsShepp3: one stencil per (theta, phi), theta = (it + 1/2) ds, phi = ip ds, ds = 2 pi / nphi
// (param.Setup(that, 2 pi / dims.back())). The 3x3 matrix (1 - eps^2) v v^T + eps^2 Id (dual:
// (eps^2 - 1) v v^T + Id) of the direction v = (cos theta, sin theta cos phi, sin theta sin phi),
// scaled by the reciprocal of gridScale^2 (the reference's matrix / scalar multiplies by 1 / s),
// is decomposed by Selling with the 1000 eps Tr cut-off of Voronoi1Mat (CommonTraits.h:82-105);
// then the theta and phi steps of weights 1 / (xi ds)^2 and 1 / (sin(theta) xi ds)^2.
void reedsshepp3_table(int nth, int nph, double h, double xi, double eps, bool dual, std::vector<int8_t> &off,
                       std::vector<int8_t> &ang, std::vector<double> &w) {
    const int ncls = nth * nph;
    off.assign((size_t)ncls * 8 * 3, 0);
    ang.assign((size_t)ncls * 8 * 2, 0);
    w.assign((size_t)ncls * 8, 0.0);
    const double ds = (2.0 * kPi) / (double)nph;
    const double e2 = eps * eps;
    const double a = dual ? (e2 - 1.0) : (1.0 - e2), b = dual ? 1.0 : e2, rh2 = 1.0 / (h * h);
    for (int it = 0; it < nth; ++it)
        for (int ip = 0; ip < nph; ++ip) {
            const int c = it * nph + ip;
            const double theta = ((double)it + 0.5) * ds, phi = (double)ip * ds;
            const double v[3] = {std::cos(theta), std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi)};
            double d[6];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j <= i; ++j) d[sym_idx(i, j)] = (a * (v[i] * v[j]) + (i == j ? b : 0.0)) * rh2;
            int o[6][3];
            double ww[6];
            if (!tensor_decomposition<3>(d, o, ww))
                throw Error(HFM_ERR_VALUE, "ObtuseSuperbase error : input must be positive definite");
            const double atol = (1000.0 * 2.220446049250313080847e-16) * sym_trace<3>(d);
            for (int k = 0; k < 6; ++k) {
                w[c * 8 + k] = ww[k] < atol ? 0.0 : ww[k];
                for (int q = 0; q < 3; ++q) off[(c * 8 + k) * 3 + q] = (int8_t)o[k][q];
            }
            ang[(c * 8 + 6) * 2 + 0] = 1;
            w[c * 8 + 6] = 1.0 / ((xi * ds) * (xi * ds));
            ang[(c * 8 + 7) * 2 + 1] = 1;
            const double sx = std::sin(theta) * xi * ds;
            w[c * 8 + 7] = 1.0 / (sx * sx);
        }
}

// ReedsSheppForward3 (Curvature3.h:72-107): per (theta, phi), theta = pi (it + 1/2) / ntheta and
// phi = 2 pi ip / nphi, the 6 forward differences of Voronoi1Vec of
// v = (cos theta, sin theta cos phi, sin theta sin phi) / gridScale, then the theta and phi steps
// of weights 1 / (xi ds)^2 and 1 / (sin(theta) xi ds)^2, ds = 2 pi / nphi.
void reedssheppforward3_table(int nth, int nph, double h, double xi, double eps, std::vector<int8_t> &off,
                              std::vector<int8_t> &ang, std::vector<double> &w) {
    const int ncls = nth * nph;
    off.assign((size_t)ncls * 8 * 3, 0);
    ang.assign((size_t)ncls * 8 * 2, 0);
    w.assign((size_t)ncls * 8, 0.0);
    const double ds = (2.0 * kPi) / (double)nph;
    const double ih = 1.0 / h;
    for (int it = 0; it < nth; ++it)
        for (int ip = 0; ip < nph; ++ip) {
            const int c = it * nph + ip;
            const double theta = kPi * ((double)it + 0.5) / (double)nth, phi = (2.0 * kPi * (double)ip) / (double)nph;
            const double v[3] = {std::cos(theta) * ih, std::sin(theta) * std::cos(phi) * ih,
                                 std::sin(theta) * std::sin(phi) * ih};
            voronoi1vec<3>(v, eps, &off[c * 8 * 3], &w[c * 8]);
            ang[(c * 8 + 6) * 2 + 0] = 1;
            w[c * 8 + 6] = 1.0 / ((xi * ds) * (xi * ds));
            ang[(c * 8 + 7) * 2 + 1] = 1;
            const double sx = std::sin(theta) * xi * ds;
            w[c * 8 + 7] = 1.0 / (sx * sx);
        }
}

}  // namespace hfm
