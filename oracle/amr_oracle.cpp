// ORACLE — test infrastructure only (see oracle.hpp). FP64 restatement of
// DG3DIntegration::compute_rhs (src/dg/operators_3d.cpp:228-282) for the scalar conservation
// law u_t + div(a u) = 0 with a constant velocity a, on hexahedral LGL elements of one order
// N connected by the reference's face connections (FaceConnection,
// include/dg/face_connection.hpp:51):
//  * volume_integral (:81-122) with the integration's quadrature quad_(order, GaussLegendre)
//    (:162), i.e. N Gauss-Legendre points per direction (GaussQuadrature1D takes the point
//    count, src/dg/quadrature_3d.cpp:13-18), and the identity Jacobian of compute_rhs
//    (:249-250): rhs_i -= sum_q w_q grad(phi_i)(x_q) . a u(x_q);
//  * non-conforming faces: compute_interface_flux_nonconforming (:345) through the mortar,
//    once per coarse face (orc_mortar_apply);
//  * conforming and boundary faces are TODO in the reference (:262-268). Mode 1 ("complete")
//    adds the reference's own ConformingInterface::compute_flux (src/dg/mortar.cpp:320: +w F on
//    the left face, -w F on the right) and compute_boundary_flux (:393, Outflow: the exterior
//    state is the interior one), each lifted by interp_to_faceᵀ, with the (N+1) x (N+1) LGL
//    face weights of the collocated face nodes. (The reference builds those face rules as
//    FaceQuadrature(face, order), N points per direction, which does not match the (N+1)^2
//    face nodes the loops index.) Each element applies its own side of a conforming face from
//    its own outward normal, which is the reference's -F on the right side for these fluxes;
//  * mass_inv (:279): the diagonal LGL mass, 1 / (w_i w_j w_k) (src/dg/basis_hexahedron.cpp:393).
// Accumulation order per element: volume, its faces 0..5, then the mortar lifts in interface
// order; then the mass inverse.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "oracle.hpp"

extern "C" int orc_mortar_apply(int order, long n_if, const int *type, const long *coarse_elem,
                                const int *coarse_face, const long *fine_elem, const int *fine_face,
                                int flux_kind, const double *a, long n_elem, const double *U, double *rhs);

namespace orc {
namespace {

// volume node of face node (it, jt) of face f (build_face_interpolation,
// src/dg/basis_hexahedron.cpp:431): normal index at the boundary, tangential indices in axis order
int amr_face_node(int np, int f, int it, int jt) {
    const int axis = f / 2, b = (f % 2) ? np - 1 : 0;
    if (axis == 0) return b + np * (it + np * jt);
    if (axis == 1) return it + np * (b + np * jt);
    return it + np * (jt + np * b);
}

// the scalar fluxes of include/flux/numerical_flux.hpp: 0 central :244, 1 upwind :264,
// 2 Lax-Friedrichs :222 with speed |a.n|
double amr_flux(int kind, double uL, double uR, double vn) {
    if (kind == 0) return 0.5 * (vn * uL + vn * uR);
    if (kind == 1) return vn * (vn >= 0 ? uL : uR);
    if (kind == 2) return 0.5 * (vn * uL + vn * uR) - 0.5 * std::abs(vn) * (uR - uL);
    throw std::invalid_argument("amr: flux kind must be 0, 1 or 2");
}

}  // namespace
}  // namespace orc

using namespace orc;

extern "C" {

// rhs = M^-1 (volume + faces + mortar lifts) of DG3DIntegration::compute_rhs. mode 0: the
// reference's semantics (non-conforming faces only), 1: conforming and boundary faces too.
// conf: n_conf x (e1, f1, e2, f2); bnd: n_bnd x (e, f); interfaces as orc_mortar_apply.
// U, rhs: n_elem x (N+1)^3, element-major. Returns 0, or -1 on bad arguments.
int orc_amr_rhs(int order, long n_elem, int mode, int flux_kind, const double *a, long n_conf,
                const long *conf, long n_bnd, const long *bnd, long n_if, const int *type,
                const long *coarse_elem, const int *coarse_face, const long *fine_elem,
                const int *fine_face, const double *U, double *rhs) {
    try {
        if (order < 1 || order > 5 || n_elem < 0 || (mode != 0 && mode != 1)) return -1;
        const int np = order + 1, nd = np * np * np, nq = order;
        const Basis1D lgl = make_lgl(order);
        Vec gx, gw;
        gauss_legendre(nq, gx, gw);
        const Vec B = interpolation_matrix(lgl.nodes, gx);  // nq x np: phi_m(x_q)
        Vec Bd((size_t)nq * np, 0.0);                        // phi_m'(x_q) = sum_i phi_i(x_q) D[i][m]
        for (int q = 0; q < nq; ++q)
            for (int m = 0; m < np; ++m)
                for (int i = 0; i < np; ++i) Bd[q * np + m] += B[q * np + i] * lgl.D[i * np + m];
        // per element and face: 1 conforming (neighbour element and face), 2 boundary
        std::vector<long> nbe((size_t)n_elem * 6, -1);
        std::vector<int> nbf((size_t)n_elem * 6, -1), kind((size_t)n_elem * 6, 0);
        if (mode == 1) {
            for (long i = 0; i < n_conf; ++i) {
                const long e1 = conf[4 * i], f1 = conf[4 * i + 1], e2 = conf[4 * i + 2], f2 = conf[4 * i + 3];
                if (e1 < 0 || e1 >= n_elem || e2 < 0 || e2 >= n_elem || f1 < 0 || f1 > 5 || f2 < 0 || f2 > 5)
                    return -1;
                kind[e1 * 6 + f1] = 1; nbe[e1 * 6 + f1] = e2; nbf[e1 * 6 + f1] = (int)f2;
                kind[e2 * 6 + f2] = 1; nbe[e2 * 6 + f2] = e1; nbf[e2 * 6 + f2] = (int)f1;
            }
            for (long i = 0; i < n_bnd; ++i) {
                const long e = bnd[2 * i], f = bnd[2 * i + 1];
                if (e < 0 || e >= n_elem || f < 0 || f > 5) return -1;
                kind[e * 6 + f] = 2;
            }
        }
        std::vector<double> uq((size_t)nq * nq * nq);
        for (long e = 0; e < n_elem; ++e) {
            const double *u = U + e * nd;
            double *r = rhs + e * nd;
            // u at the quadrature points
            for (int q3 = 0; q3 < nq; ++q3)
                for (int q2 = 0; q2 < nq; ++q2)
                    for (int q1 = 0; q1 < nq; ++q1) {
                        double s = 0.0;
                        for (int k = 0; k < np; ++k)
                            for (int j = 0; j < np; ++j)
                                for (int i = 0; i < np; ++i)
                                    s += B[q1 * np + i] * B[q2 * np + j] * B[q3 * np + k] * u[i + np * (j + np * k)];
                        uq[q1 + nq * (q2 + nq * q3)] = s;
                    }
            // volume_integral: rhs_i -= w_q (grad phi_i . a) u_q
            for (int k = 0; k < np; ++k)
                for (int j = 0; j < np; ++j)
                    for (int i = 0; i < np; ++i) {
                        double s = 0.0;
                        for (int q3 = 0; q3 < nq; ++q3)
                            for (int q2 = 0; q2 < nq; ++q2)
                                for (int q1 = 0; q1 < nq; ++q1) {
                                    const double w = gw[q1] * gw[q2] * gw[q3];
                                    const double g = a[0] * Bd[q1 * np + i] * B[q2 * np + j] * B[q3 * np + k] +
                                                     a[1] * B[q1 * np + i] * Bd[q2 * np + j] * B[q3 * np + k] +
                                                     a[2] * B[q1 * np + i] * B[q2 * np + j] * Bd[q3 * np + k];
                                    s += w * g * uq[q1 + nq * (q2 + nq * q3)];
                                }
                        r[i + np * (j + np * k)] = -s;
                    }
            // conforming and boundary faces (complete mode)
            for (int f = 0; f < 6; ++f) {
                const int kd = kind[e * 6 + f];
                if (kd == 0) continue;
                const int axis = f / 2;
                const double vn = ((f % 2) ? 1.0 : -1.0) * a[axis];
                for (int jt = 0; jt < np; ++jt)
                    for (int it = 0; it < np; ++it) {
                        const int n = amr_face_node(np, f, it, jt);
                        const double uL = u[n];
                        const double uR =
                            kd == 1 ? U[nbe[e * 6 + f] * nd + amr_face_node(np, nbf[e * 6 + f], it, jt)] : uL;
                        r[n] += lgl.weights[it] * lgl.weights[jt] * amr_flux(flux_kind, uL, uR, vn);
                    }
            }
        }
        if (n_if > 0 &&
            orc_mortar_apply(order, n_if, type, coarse_elem, coarse_face, fine_elem, fine_face, flux_kind, a,
                             n_elem, U, rhs) != 0)
            return -1;
        for (long e = 0; e < n_elem; ++e)
            for (int k = 0; k < np; ++k)
                for (int j = 0; j < np; ++j)
                    for (int i = 0; i < np; ++i)
                        rhs[e * nd + i + np * (j + np * k)] *= 1.0 / (lgl.weights[i] * lgl.weights[j] * lgl.weights[k]);
        return 0;
    } catch (const std::exception &) {
        return -1;
    }
}

}  // extern "C"
