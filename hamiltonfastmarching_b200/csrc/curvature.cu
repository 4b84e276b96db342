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

}  // namespace hfm
