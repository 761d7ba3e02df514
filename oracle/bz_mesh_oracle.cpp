// ORACLE — test infrastructure only (see oracle.hpp). FP64 restatement, on an arbitrary list of
// quadtree elements (the meshes of the adaptive smoother: per element its bounds and, for the
// error, its 16 resolved Bezier coefficients), of
//  * AdaptiveCGCubicBezierSmoother::compute_element_l2_error and estimate_element_error
//    (src/bathymetry/adaptive_cg_cubic_bezier_smoother.cpp:100-160): the squared misfit at the
//    ngauss x ngauss Gauss-Legendre points of [0,1]^2 (v outer, u inner), each point mapped to
//    physical coordinates and back as the smoother's evaluate(x, y) does, weighted by
//    w_i w_j; l2 = sqrt(sum x dx x dy), normalized = l2 / sqrt(dx dy);
//  * the element part of CGBezierSmootherBase::assemble_data_fitting_global
//    (src/bathymetry/cg_bezier_smoother_base.cpp:308-364) with gauss_legendre_01 (:28-58; four
//    points at most): per element the 16 x 16 block sum_q weight B_i B_j, the 16-vector
//    sum_q weight B_i d and sum_q weight d d, weight = w_qi w_qj dx dy relaxation, the points in
//    the order qi (u) outer, qj (v) inner.
// The Bernstein values are CubicBezierBasis2D::evaluate_bernstein_1d's recurrence
// (src/bathymetry/cubic_bezier_basis_2d.cpp:42-78), phi(i + 4 j) = Bu(i) Bv(j) (:133-145).
// zdata and relax hold ngauss x ngauss values per element, [e][qj][qi].
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle.hpp"

namespace orc {
namespace {

void bern3(double t, double B[4]) {
    const double s = 1.0 - t;
    double prev[4] = {1.0, 0.0, 0.0, 0.0};
    for (int deg = 1; deg <= 3; ++deg) {
        double cur[4];
        cur[0] = s * prev[0];
        for (int i = 1; i < deg; ++i) cur[i] = t * prev[i - 1] + s * prev[i];
        cur[deg] = t * prev[deg - 1];
        for (int i = 0; i <= deg; ++i) prev[i] = cur[i];
    }
    for (int i = 0; i < 4; ++i) B[i] = prev[i];
}

// gauss_legendre_01 (n >= 4 gives the 4-point rule)
int gl01(int n, double *pts, double *wts) {
    if (n == 1) {
        pts[0] = 0.5;
        wts[0] = 1.0;
        return 1;
    }
    if (n == 2) {
        pts[0] = 0.5 - 0.5 / std::sqrt(3.0);
        pts[1] = 0.5 + 0.5 / std::sqrt(3.0);
        wts[0] = wts[1] = 0.5;
        return 2;
    }
    if (n == 3) {
        pts[0] = 0.5 - 0.5 * std::sqrt(0.6);
        pts[1] = 0.5;
        pts[2] = 0.5 + 0.5 * std::sqrt(0.6);
        wts[0] = wts[2] = 5.0 / 18.0;
        wts[1] = 8.0 / 18.0;
        return 3;
    }
    const double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    const double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    pts[0] = 0.5 * (1.0 - b);
    pts[1] = 0.5 * (1.0 - a);
    pts[2] = 0.5 * (1.0 + a);
    pts[3] = 0.5 * (1.0 + b);
    const double wa = (18.0 + std::sqrt(30.0)) / 72.0, wb = (18.0 - std::sqrt(30.0)) / 72.0;
    wts[0] = wts[3] = 0.5 * wb;
    wts[1] = wts[2] = 0.5 * wa;
    return 4;
}

}  // namespace
}  // namespace orc

using namespace orc;

extern "C" {

// bounds: n x (xmin, ymin, xmax, ymax); coeffs: n x 16 (i + 4 j)
int orc_bz_mesh_element_errors(long n, const double *bounds, const double *coeffs, const double *zdata, int ng,
                               double *l2, double *nrm) {
    if (n < 0 || ng < 1) return -1;
    Vec gx, gw;
    gauss_legendre(ng, gx, gw);
    std::vector<double> gn(ng), gwt(ng);
    for (int i = 0; i < ng; ++i) {
        gn[i] = 0.5 * (gx[i] + 1.0);
        gwt[i] = 0.5 * gw[i];
    }
    for (long e = 0; e < n; ++e) {
        const double *bb = bounds + 4 * e, *c = coeffs + 16 * e;
        const double dx = bb[2] - bb[0], dy = bb[3] - bb[1];
        double err2 = 0.0;
        for (int j = 0; j < ng; ++j)
            for (int i = 0; i < ng; ++i) {
                const double px = bb[0] + gn[i] * dx, py = bb[1] + gn[j] * dy;
                const double u = std::clamp((px - bb[0]) / dx, 0.0, 1.0), v = std::clamp((py - bb[1]) / dy, 0.0, 1.0);
                double bu[4], bv[4];
                bern3(u, bu);
                bern3(v, bv);
                double z = 0.0;
                for (int b = 0; b < 4; ++b)
                    for (int a = 0; a < 4; ++a) z += c[a + 4 * b] * bu[a] * bv[b];
                const double w = gwt[i] * gwt[j];
                const double diff = zdata[(e * ng + j) * ng + i] - z;
                err2 += w * diff * diff;
            }
        l2[e] = std::sqrt(err2 * dx * dy);
        if (nrm) nrm[e] = l2[e] / std::sqrt(dx * dy);
    }
    return 0;
}

// BtWB: n x 256 (row i, column j), BtWd: n x 16, dTWd: n; relax may be null (factor 1). ng is
// 1..4 (gauss_legendre_01 gives the 4-point rule for every n >= 4, so callers pass min(n, 4)).
int orc_bz_mesh_data_fitting(long n, const double *bounds, const double *zdata, const double *relax, int ng,
                             double *BtWB, double *BtWd, double *dTWd) {
    if (n < 0 || ng < 1 || ng > 4) return -1;
    double pts[4], wts[4];
    const int nq = gl01(ng, pts, wts);
    for (long e = 0; e < n; ++e) {
        const double *bb = bounds + 4 * e;
        const double dx = bb[2] - bb[0], dy = bb[3] - bb[1], jac = dx * dy;
        double K[256] = {0.0}, r[16] = {0.0}, dd = 0.0;
        for (int qi = 0; qi < nq; ++qi)
            for (int qj = 0; qj < nq; ++qj) {
                const long q = (e * ng + qj) * ng + qi;
                const double rel = relax ? relax[q] : 1.0;
                const double weight = wts[qi] * wts[qj] * jac * rel;
                const double d = zdata[q];
                dd += weight * d * d;
                double bu[4], bv[4], B[16];
                bern3(pts[qi], bu);
                bern3(pts[qj], bv);
                for (int j = 0; j < 4; ++j)
                    for (int i = 0; i < 4; ++i) B[i + 4 * j] = bu[i] * bv[j];
                for (int i = 0; i < 16; ++i) {
                    for (int j = 0; j < 16; ++j) K[16 * i + j] += weight * B[i] * B[j];
                    r[i] += weight * B[i] * d;
                }
            }
        std::copy(K, K + 256, BtWB + 256 * e);
        std::copy(r, r + 16, BtWd + 16 * e);
        dTWd[e] = dd;
    }
    return 0;
}

}  // extern "C"
