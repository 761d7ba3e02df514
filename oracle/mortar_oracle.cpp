// ORACLE — test infrastructure only (see oracle.hpp). FP64 restatement of the reference's
// mortar space for non-conforming faces (MortarSpace, src/dg/mortar.cpp:13-258) and of the
// non-conforming face flux of DG3DIntegration (compute_interface_flux_nonconforming,
// src/dg/operators_3d.cpp:345-390), with the reference's behaviour kept:
//  * mortar order = the (common) element order p, mortar basis = tensor LGL Lagrange, mortar
//    quadrature = (2p + 1)^2 Gauss-Legendre points on the coarse face (mortar.cpp:17-18);
//  * the fine-side coupling B_f sums the mortar quadrature points that lie in the CLOSED
//    sub-face rectangle with their full-face weights (mortar.cpp:176-200): a point on a split
//    line counts for both halves;
//  * the flux is scalar, evaluated at the mortar nodes after projection (mortar.cpp:212-248);
//  * coarse lift L_c M^-1 F, fine lifts -L_f M^-1 F (mortar.cpp:250-258).
// Face traces: face f has normal axis f / 2 on its positive side when f is odd; face node
// (it, jt) is volume node i + np (j + np k) with the normal index at the boundary and the two
// tangential indices in axis order (build_face_interpolation, src/dg/basis_hexahedron.cpp:431).
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "oracle.hpp"

namespace orc {
namespace {

// FaceConnectionType (include/dg/face_connection.hpp:15): SameLevel, Fine2x1, Fine1x2,
// Fine3_2plus1, Fine3_1plus2, Fine2x2
int num_fine(int type) {
    static const int n[6] = {1, 2, 2, 3, 3, 4};
    if (type < 0 || type > 5) throw std::invalid_argument("mortar: connection type must be 0..5");
    return n[type];
}

// sub-face rectangles (min t1, min t2, max t1, max t2) in the coarse face's [-1, 1]^2
// (MortarSpace::compute_subface_bounds, src/dg/mortar.cpp:27)
void subfaces(int type, double b[4][4]) {
    auto set = [&](int f, double a0, double a1, double c0, double c1) {
        b[f][0] = a0; b[f][1] = a1; b[f][2] = c0; b[f][3] = c1;
    };
    switch (type) {
    case 0: set(0, -1, -1, 1, 1); break;
    case 1: set(0, -1, -1, 0, 1); set(1, 0, -1, 1, 1); break;
    case 2: set(0, -1, -1, 1, 0); set(1, -1, 0, 1, 1); break;
    case 3: set(0, -1, -1, 0, 0); set(1, 0, -1, 1, 0); set(2, -1, 0, 1, 1); break;
    case 4: set(0, -1, -1, 0, 0); set(1, -1, 0, 0, 1); set(2, 0, -1, 1, 1); break;
    case 5: set(0, -1, -1, 0, 0); set(1, 0, -1, 1, 0); set(2, -1, 0, 0, 1); set(3, 0, 0, 1, 1); break;
    default: throw std::invalid_argument("mortar: connection type must be 0..5");
    }
}

void invert(const Vec &A, int n, Vec &Ainv) {
    Vec M = A, I((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(M[r * n + c]) > std::abs(M[piv * n + c])) piv = r;
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(M[c * n + k], M[piv * n + k]);
                std::swap(I[c * n + k], I[piv * n + k]);
            }
        const double d = 1.0 / M[c * n + c];
        for (int k = 0; k < n; ++k) { M[c * n + k] *= d; I[c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = M[r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) { M[r * n + k] -= f * M[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
        }
    }
    Ainv = I;
}

struct Ops {
    int np, nm, nf, nfine, nq1;
    Vec M, Minv, Pc, Lc, Pf[4], Lf[4];
};

Ops build_ops(int order, int type) {
    if (order < 1 || order > 8) throw std::invalid_argument("mortar: order must be 1..8");
    Ops o;
    o.np = order + 1;
    o.nm = o.nf = o.np * o.np;
    o.nfine = num_fine(type);
    o.nq1 = 2 * order + 1;
    const int np = o.np, nm = o.nm, nf = o.nf, nq1 = o.nq1, nq = nq1 * nq1;
    const Basis1D lgl = make_lgl(order);
    Vec gx, gw;
    gauss_legendre(nq1, gx, gw);
    // Phi(q, m) on the mortar quadrature, q = qi + nq1 qj, m = i + np j
    const Vec I1 = interpolation_matrix(lgl.nodes, gx);  // nq1 x np
    Vec Phi((size_t)nq * nm), W(nq);
    for (int qj = 0; qj < nq1; ++qj)
        for (int qi = 0; qi < nq1; ++qi) {
            const int q = qi + nq1 * qj;
            W[q] = gw[qi] * gw[qj];
            for (int j = 0; j < np; ++j)
                for (int i = 0; i < np; ++i) Phi[(size_t)q * nm + i + np * j] = I1[qi * np + i] * I1[qj * np + j];
        }
    o.M.assign((size_t)nm * nm, 0.0);
    for (int q = 0; q < nq; ++q)
        for (int a = 0; a < nm; ++a)
            for (int b = 0; b < nm; ++b) o.M[(size_t)a * nm + b] += W[q] * Phi[(size_t)q * nm + a] * Phi[(size_t)q * nm + b];
    invert(o.M, nm, o.Minv);
    auto mul = [&](const Vec &A, const Vec &B, int n, int k, int m) {  // (n x k)(k x m)
        Vec C((size_t)n * m, 0.0);
        for (int r = 0; r < n; ++r)
            for (int t = 0; t < k; ++t)
                for (int c = 0; c < m; ++c) C[(size_t)r * m + c] += A[(size_t)r * k + t] * B[(size_t)t * m + c];
        return C;
    };
    auto transpose = [](const Vec &A, int n, int m) {
        Vec T((size_t)n * m);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < m; ++c) T[(size_t)c * n + r] = A[(size_t)r * m + c];
        return T;
    };
    // coarse: B_c(m, j) = sum_q w_q Phi(q, m) psi_j(q) (the coarse basis equals the mortar basis)
    Vec Bc((size_t)nm * nf, 0.0);
    for (int q = 0; q < nq; ++q)
        for (int m = 0; m < nm; ++m)
            for (int j = 0; j < nf; ++j) Bc[(size_t)m * nf + j] += W[q] * Phi[(size_t)q * nm + m] * Phi[(size_t)q * nm + j];
    o.Pc = mul(o.Minv, Bc, nm, nm, nf);
    o.Lc = transpose(Bc, nm, nf);
    double sb[4][4];
    subfaces(type, sb);
    for (int f = 0; f < o.nfine; ++f) {
        Vec Bf((size_t)nm * nf, 0.0);
        for (int qj = 0; qj < nq1; ++qj)
            for (int qi = 0; qi < nq1; ++qi) {
                const double x0 = gx[qi], x1 = gx[qj];
                if (!(x0 >= sb[f][0] && x0 <= sb[f][2] && x1 >= sb[f][1] && x1 <= sb[f][3])) continue;
                const int q = qi + nq1 * qj;
                const Vec xf = {2.0 * (x0 - sb[f][0]) / (sb[f][2] - sb[f][0]) - 1.0};
                const Vec yf = {2.0 * (x1 - sb[f][1]) / (sb[f][3] - sb[f][1]) - 1.0};
                const Vec pt = interpolation_matrix(lgl.nodes, xf), ps = interpolation_matrix(lgl.nodes, yf);
                for (int m = 0; m < nm; ++m)
                    for (int jf = 0; jf < np; ++jf)
                        for (int i_f = 0; i_f < np; ++i_f)
                            Bf[(size_t)m * nf + i_f + np * jf] += W[q] * Phi[(size_t)q * nm + m] * pt[i_f] * ps[jf];
            }
        o.Pf[f] = mul(o.Minv, Bf, nm, nm, nf);
        o.Lf[f] = transpose(Bf, nm, nf);
    }
    return o;
}

// volume node of face node (it, jt) of face f
int face_node(int np, int f, int it, int jt) {
    const int axis = f / 2, b = (f % 2) ? np - 1 : 0;
    int i, j, k;
    if (axis == 0) { i = b; j = it; k = jt; }
    else if (axis == 1) { i = it; j = b; k = jt; }
    else { i = it; j = jt; k = b; }
    return i + np * (j + np * k);
}

// scalar numerical flux for u_t + div(a u) = 0 (include/flux/numerical_flux.hpp):
// 0 CentralFlux :244, 1 UpwindFlux :264, 2 LaxFriedrichsFlux :222 with speed |a.n|
double scalar_flux(int kind, double uL, double uR, double vn) {
    if (kind == 0) return 0.5 * (vn * uL + vn * uR);
    if (kind == 1) return vn * (vn >= 0 ? uL : uR);
    if (kind == 2) return 0.5 * (vn * uL + vn * uR) - 0.5 * std::abs(vn) * (uR - uL);
    throw std::invalid_argument("mortar: flux kind must be 0 (central), 1 (upwind) or 2 (LF)");
}

}  // namespace
}  // namespace orc

using namespace orc;

extern "C" {

// Operators of one connection type: M, M^-1 (nm x nm), P_c (nm x nf), L_c (nf x nm),
// P_f (nfine x nm x nf), L_f (nfine x nf x nm); any output may be null. Returns the number of
// fine faces, or -1 on error.
int orc_mortar_ops(int order, int type, double *M, double *Minv, double *Pc, double *Lc, double *Pf,
                   double *Lf) {
    try {
        const Ops o = build_ops(order, type);
        const size_t a = (size_t)o.nm * o.nm, b = (size_t)o.nm * o.nf;
        if (M) std::memcpy(M, o.M.data(), a * 8);
        if (Minv) std::memcpy(Minv, o.Minv.data(), a * 8);
        if (Pc) std::memcpy(Pc, o.Pc.data(), b * 8);
        if (Lc) std::memcpy(Lc, o.Lc.data(), b * 8);
        for (int f = 0; f < o.nfine; ++f) {
            if (Pf) std::memcpy(Pf + f * b, o.Pf[f].data(), b * 8);
            if (Lf) std::memcpy(Lf + f * b, o.Lf[f].data(), b * 8);
        }
        return o.nfine;
    } catch (const std::exception &) {
        return -1;
    }
}

// rhs += the mortar flux contributions of n_if interfaces, in list order (coarse side, then
// the fine faces in order). U, rhs: n_elem x np^3 (element-major). fine_elem / fine_face: 4 per
// interface (entries past the type's fine-face count are ignored).
int orc_mortar_apply(int order, long n_if, const int *type, const long *coarse_elem, const int *coarse_face,
                     const long *fine_elem, const int *fine_face, int flux_kind, const double *a,
                     long n_elem, const double *U, double *rhs) {
    try {
        const int np = order + 1, nd = np * np * np;
        std::vector<Ops> ops;
        for (int t = 0; t < 6; ++t) ops.push_back(build_ops(order, t));
        for (long i = 0; i < n_if; ++i) {
            const Ops &o = ops.at(type[i]);
            const int nm = o.nm, nf = o.nf;
            if (coarse_elem[i] < 0 || coarse_elem[i] >= n_elem) throw std::invalid_argument("bad element");
            Vec Uc(nf), Ucm(nm, 0.0), Ufm(nm, 0.0), F(nm), G(nm, 0.0);
            for (int jt = 0; jt < np; ++jt)
                for (int it = 0; it < np; ++it)
                    Uc[it + np * jt] = U[coarse_elem[i] * nd + face_node(np, coarse_face[i], it, jt)];
            for (int m = 0; m < nm; ++m)
                for (int j = 0; j < nf; ++j) Ucm[m] += o.Pc[(size_t)m * nf + j] * Uc[j];
            std::vector<Vec> Uf(o.nfine, Vec(nf));
            for (int f = 0; f < o.nfine; ++f) {
                const long e = fine_elem[4 * i + f];
                if (e < 0 || e >= n_elem) throw std::invalid_argument("bad element");
                for (int jt = 0; jt < np; ++jt)
                    for (int it = 0; it < np; ++it)
                        Uf[f][it + np * jt] = U[e * nd + face_node(np, fine_face[4 * i + f], it, jt)];
                Vec t(nm, 0.0);
                for (int m = 0; m < nm; ++m)
                    for (int j = 0; j < nf; ++j) t[m] += o.Pf[f][(size_t)m * nf + j] * Uf[f][j];
                for (int m = 0; m < nm; ++m) Ufm[m] += t[m];
            }
            const int axis = coarse_face[i] / 2;
            const double sgn = (coarse_face[i] % 2) ? 1.0 : -1.0, vn = sgn * a[axis];
            for (int m = 0; m < nm; ++m) F[m] = scalar_flux(flux_kind, Ucm[m], Ufm[m], vn);
            for (int m = 0; m < nm; ++m)
                for (int k = 0; k < nm; ++k) G[m] += o.Minv[(size_t)m * nm + k] * F[k];
            for (int j = 0; j < nf; ++j) {
                double s = 0.0;
                for (int m = 0; m < nm; ++m) s += o.Lc[(size_t)j * nm + m] * G[m];
                rhs[coarse_elem[i] * nd + face_node(np, coarse_face[i], j % np, j / np)] += s;
            }
            for (int f = 0; f < o.nfine; ++f) {
                const long e = fine_elem[4 * i + f];
                for (int j = 0; j < nf; ++j) {
                    double s = 0.0;
                    for (int m = 0; m < nm; ++m) s += o.Lf[f][(size_t)j * nm + m] * G[m];
                    rhs[e * nd + face_node(np, fine_face[4 * i + f], j % np, j / np)] += -s;
                }
            }
        }
        return 0;
    } catch (const std::exception &) {
        return -1;
    }
}

}  // extern "C"
