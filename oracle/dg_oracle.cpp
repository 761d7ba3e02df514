// ORACLE (test infrastructure, never linked into the product). FP64 CPU restatement of
// the DRIFTER DG path: basis/quadrature, compat element RHS and mode-split step (with the
// reference's quirks), fluxes, time steppers, and the physical split-explicit scheme.
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <thread>
#include <functional>

namespace orc {

// ============================================================================ basis
// src/dg/basis_hexahedron.hpp:23 legendre_poly_and_derivative (three-term recurrence)
void legendre(int n, double x, double &L, double &dL) {
    if (n == 0) { L = 1.0; dL = 0.0; return; }
    if (n == 1) { L = x; dL = 1.0; return; }
    double Lm2 = 1.0, Lm1 = x, dLm2 = 0.0, dLm1 = 1.0;
    for (int k = 2; k <= n; ++k) {
        L = (2.0 * k - 1.0) / k * x * Lm1 - (k - 1.0) / k * Lm2;
        dL = dLm2 + (2.0 * k - 1.0) * Lm1;
        Lm2 = Lm1; Lm1 = L; dLm2 = dLm1; dLm1 = dL;
    }
}

// src/dg/basis_hexahedron.cpp:14 compute_gauss_legendre_nodes
void gauss_legendre(int n, Vec &x, Vec &w) {
    x.assign(n, 0.0); w.assign(n, 0.0);
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; return; }
    if (n == 2) { x[0] = -std::sqrt(1.0 / 3.0); x[1] = -x[0]; w[0] = w[1] = 1.0; return; }
    for (int i = 0; i <= (n - 1) / 2; ++i) {
        double xi = -std::cos((2.0 * i + 1.0) / (2.0 * n) * M_PI), L, dL;
        for (int it = 0; it < 100; ++it) {
            double xo = xi;
            legendre(n, xi, L, dL);
            xi -= L / dL;
            if (std::abs(xi - xo) < 1e-15) break;
        }
        x[i] = xi; x[n - 1 - i] = -xi;
        legendre(n, xi, L, dL);
        w[i] = w[n - 1 - i] = 2.0 / ((1.0 - xi * xi) * dL * dL);
    }
    if (n % 2 == 1) {
        double L, dL;
        legendre(n, 0.0, L, dL);
        x[n / 2] = 0.0; w[n / 2] = 2.0 / (dL * dL);
    }
}

// src/dg/basis_hexahedron.cpp:70 compute_gauss_lobatto_nodes: Newton on P_{N+1} - P_{N-1}
// with the reference's initial guess; weights 2/(N(N+1) P_N^2).
void gauss_lobatto(int n, Vec &x, Vec &w) {
    if (n < 2) throw std::invalid_argument("LGL requires at least 2 nodes");
    x.assign(n, 0.0); w.assign(n, 0.0);
    if (n == 2) { x[0] = -1.0; x[1] = 1.0; w[0] = w[1] = 1.0; return; }
    x[0] = -1.0; x[n - 1] = 1.0;
    w[0] = w[n - 1] = 2.0 / (n * (n - 1));
    const int N = n - 1;
    for (int i = 1; i <= (n - 1) / 2; ++i) {
        double xi = -std::cos((0.25 + i) * M_PI / N - 3.0 / (8.0 * N * M_PI * (0.25 + i)));
        for (int it = 0; it < 100; ++it) {
            double xo = xi;
            double LNm1, dLNm1, LN, dLN;
            legendre(N - 1, xi, LNm1, dLNm1);
            legendre(N, xi, LN, dLN);
            const int k = N + 1;
            double LNp1 = (2.0 * k - 1.0) / k * xi * LN - (k - 1.0) / k * LNm1;
            double dLNp1 = dLNm1 + (2.0 * k - 1.0) * LN;
            xi -= (LNp1 - LNm1) / (dLNp1 - dLNm1);
            if (std::abs(xi - xo) < 1e-15) break;
        }
        x[i] = xi; x[n - 1 - i] = -xi;
        double LN, dLN;
        legendre(N, xi, LN, dLN);
        w[i] = w[n - 1 - i] = 2.0 / (N * (N + 1) * LN * LN);
    }
    if (n % 2 == 1) {
        double LN, dLN;
        legendre(N, 0.0, LN, dLN);
        x[n / 2] = 0.0; w[n / 2] = 2.0 / (N * (N + 1) * LN * LN);
    }
}

// src/dg/basis_hexahedron.cpp:152
Vec barycentric_weights(const Vec &x) {
    const int n = (int)x.size();
    Vec w(n);
    for (int j = 0; j < n; ++j) {
        double p = 1.0;
        for (int k = 0; k < n; ++k) if (k != j) p *= (x[j] - x[k]);
        w[j] = 1.0 / p;
    }
    return w;
}

// src/dg/basis_hexahedron.cpp:190 (negative-sum diagonal)
Vec derivative_matrix(const Vec &x) {
    const int n = (int)x.size();
    Vec bw = barycentric_weights(x), D(n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) if (i != j) {
            D[i * n + j] = (bw[j] / bw[i]) / (x[i] - x[j]);
            s += D[i * n + j];
        }
        D[i * n + i] = -s;
    }
    return D;
}

// src/dg/basis_hexahedron.cpp:218
Vec interpolation_matrix(const Vec &from, const Vec &to) {
    const int nf = (int)from.size(), nt = (int)to.size();
    Vec bw = barycentric_weights(from), I(nt * nf, 0.0);
    for (int i = 0; i < nt; ++i) {
        int at = -1;
        for (int j = 0; j < nf; ++j) if (std::abs(to[i] - from[j]) < 1e-15) { at = j; break; }
        if (at >= 0) { I[i * nf + at] = 1.0; continue; }
        double s = 0.0;
        Vec t(nf);
        for (int j = 0; j < nf; ++j) { t[j] = bw[j] / (to[i] - from[j]); s += t[j]; }
        for (int j = 0; j < nf; ++j) I[i * nf + j] = t[j] / s;
    }
    return I;
}

static void fill_S(Basis1D &b) {
    // S[k][m] = int_{-1}^{x_k} l_m(x) dx by (np+1)-point Gauss-Legendre on [-1, x_k] (exact).
    const int np = b.np();
    b.S.assign(np * np, 0.0);
    Vec gx, gw;
    gauss_legendre(np + 1, gx, gw);
    for (int k = 1; k < np; ++k) {
        const double a = -1.0, c = b.nodes[k], half = 0.5 * (c - a);
        Vec pts(np + 1);
        for (int q = 0; q <= np; ++q) pts[q] = a + half * (gx[q] + 1.0);
        Vec I = interpolation_matrix(b.nodes, pts);
        for (int m = 0; m < np; ++m) {
            double s = 0.0;
            for (int q = 0; q <= np; ++q) s += gw[q] * I[q * np + m];
            b.S[k * np + m] = half * s;
        }
    }
}

// Ainv = (D + e_0 e_0^T / w_0)^-1 by Gauss-Jordan elimination with partial pivoting.
static void fill_Ainv(Basis1D &b) {
    const int n = b.np();
    Vec A(b.D), I(n * n, 0.0);
    A[0] += 1.0 / b.weights[0];
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int pr = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(A[r * n + c]) > std::abs(A[pr * n + c])) pr = r;
        for (int k = 0; k < n; ++k) {
            std::swap(A[c * n + k], A[pr * n + k]);
            std::swap(I[c * n + k], I[pr * n + k]);
        }
        const double d = A[c * n + c];
        for (int k = 0; k < n; ++k) { A[c * n + k] /= d; I[c * n + k] /= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = A[r * n + c];
            for (int k = 0; k < n; ++k) { A[r * n + k] -= f * A[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
        }
    }
    b.Ainv = I;
    b.a0.assign(n, 0.0);
    for (int k = 0; k < n; ++k) b.a0[k] = I[k * n + 0] / b.weights[0];
}

Basis1D make_lgl(int order) {
    Basis1D b;
    b.order = order;
    gauss_lobatto(order + 1, b.nodes, b.weights);
    b.bary = barycentric_weights(b.nodes);
    b.D = derivative_matrix(b.nodes);
    fill_S(b);
    fill_Ainv(b);
    return b;
}
Basis1D make_gl(int order) {
    Basis1D b;
    b.order = order;
    gauss_legendre(order + 1, b.nodes, b.weights);
    b.bary = barycentric_weights(b.nodes);
    b.D = derivative_matrix(b.nodes);
    fill_S(b);
    return b;
}

void build_dense_3d(const Basis1D &b, Vec &Dxi, Vec &Deta, Vec &Dzeta) {
    const int np = b.np(), nd = np * np * np;
    Dxi.assign((size_t)nd * nd, 0.0); Deta = Dxi; Dzeta = Dxi;
    auto id = [np](int i, int j, int k) { return i + np * (j + np * k); };
    for (int k = 0; k < np; ++k) for (int j = 0; j < np; ++j) for (int i = 0; i < np; ++i) {
        const int r = id(i, j, k);
        for (int m = 0; m < np; ++m) {
            Dxi[(size_t)r * nd + id(m, j, k)] = b.D[i * np + m];
            Deta[(size_t)r * nd + id(i, m, k)] = b.D[j * np + m];
            Dzeta[(size_t)r * nd + id(i, j, m)] = b.D[k * np + m];
        }
    }
}

// ============================================================================ fluxes
void sw_physical_flux(const double U[3], double nx, double ny, double g, double F[3]) {
    double h = U[0] < 1e-10 ? 1e-10 : U[0];
    double u = U[1] / h, v = U[2] / h, un = u * nx + v * ny;
    F[0] = h * un;
    F[1] = h * u * un + 0.5 * g * h * h * nx;
    F[2] = h * v * un + 0.5 * g * h * h * ny;
}

// LF factory: src/flux/numerical_flux.cpp:134-180 + include/flux/numerical_flux.hpp:222
static void flux_lf(const double UL[3], const double UR[3], double nx, double ny, double g,
                    double F[3]) {
    auto phys = [g](const double U[3], double Fx[3], double Fy[3]) {
        double h = U[0] < 1e-10 ? 1e-10 : U[0];
        double u = U[1] / h, v = U[2] / h;
        Fx[0] = U[1]; Fx[1] = U[1] * u + 0.5 * g * h * h; Fx[2] = U[1] * v;
        Fy[0] = U[2]; Fy[1] = U[2] * u; Fy[2] = U[2] * v + 0.5 * g * h * h;
    };
    double FxL[3], FyL[3], FxR[3], FyR[3];
    phys(UL, FxL, FyL);
    phys(UR, FxR, FyR);
    double hL = std::max(UL[0], 1e-10), hR = std::max(UR[0], 1e-10);
    double unL = (UL[1] / hL) * nx + (UL[2] / hL) * ny, unR = (UR[1] / hR) * nx + (UR[2] / hR) * ny;
    double lam = std::max(std::abs(unL) + std::sqrt(g * hL), std::abs(unR) + std::sqrt(g * hR));
    for (int i = 0; i < 3; ++i) {
        double FnL = FxL[i] * nx + FyL[i] * ny, FnR = FxR[i] * nx + FyR[i] * ny;
        F[i] = 0.5 * (FnL + FnR) - 0.5 * lam * (UR[i] - UL[i]);
    }
}

// include/flux/numerical_flux.hpp:272-390 (HLLC with Einfeldt speeds)
static void flux_hllc(const double UL[3], const double UR[3], double nx, double ny, double g,
                      double F[3]) {
    double hL = UL[0] < 1e-10 ? 1e-10 : UL[0], hR = UR[0] < 1e-10 ? 1e-10 : UR[0];
    double huL = UL[1], hvL = UL[2], huR = UR[1], hvR = UR[2];
    double uL = huL / hL, vL = hvL / hL, uR = huR / hR, vR = hvR / hR;
    double unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
    double cL = std::sqrt(g * hL), cR = std::sqrt(g * hR);
    double SL = std::min(unL - cL, unR - cR), SR = std::max(unL + cL, unR + cR), Ss;
    double den = hL * (SL - unL) - hR * (SR - unR);
    if (std::abs(den) > 1e-10)
        Ss = (hL * unL * (SL - unL) - hR * unR * (SR - unR) + 0.5 * g * (hR * hR - hL * hL)) / den;
    else
        Ss = 0.5 * (unL + unR);
    auto phys = [&](double h, double u, double v, double out[3]) {
        double un = u * nx + v * ny;
        out[0] = h * un; out[1] = h * u * un + 0.5 * g * h * h * nx;
        out[2] = h * v * un + 0.5 * g * h * h * ny;
    };
    double FL[3], FR[3];
    phys(hL, uL, vL, FL);
    phys(hR, uR, vR, FR);
    if (SL >= 0) { for (int i = 0; i < 3; ++i) F[i] = FL[i]; return; }
    if (SR <= 0) { for (int i = 0; i < 3; ++i) F[i] = FR[i]; return; }
    if (Ss >= 0) {
        double hs = hL * (SL - unL) / (SL - Ss);
        double Us[3] = {hs, hs * (uL + (Ss - unL) * nx), hs * (vL + (Ss - unL) * ny)};
        double Uv[3] = {hL, huL, hvL};
        for (int i = 0; i < 3; ++i) F[i] = FL[i] + SL * (Us[i] - Uv[i]);
    } else {
        double hs = hR * (SR - unR) / (SR - Ss);
        double Us[3] = {hs, hs * (uR + (Ss - unR) * nx), hs * (vR + (Ss - unR) * ny)};
        double Uv[3] = {hR, huR, hvR};
        for (int i = 0; i < 3; ++i) F[i] = FR[i] + SR * (Us[i] - Uv[i]);
    }
}

// src/flux/numerical_flux.cpp:13-131 (Roe with Harten entropy fix, entropy_fix = 0.1)
static void flux_roe(const double UL[3], const double UR[3], double nx, double ny, double g,
                     double F[3]) {
    const double efix = 0.1;
    double hL = UL[0] < 1e-10 ? 1e-10 : UL[0], hR = UR[0] < 1e-10 ? 1e-10 : UR[0];
    double uL = UL[1] / hL, vL = UL[2] / hL, uR = UR[1] / hR, vR = UR[2] / hR;
    double unL = uL * nx + vL * ny, utL = -uL * ny + vL * nx;
    double unR = uR * nx + vR * ny, utR = -uR * ny + vR * nx;
    double sL = std::sqrt(hL), sR = std::sqrt(hR), den = sL + sR;
    double hr = 0.5 * (hL + hR), ur = (sL * uL + sR * uR) / den, vr = (sL * vL + sR * vR) / den;
    double unr = ur * nx + vr * ny, cr = std::sqrt(g * hr);
    double l1 = unr - cr, l2 = unr, l3 = unr + cr, delta = efix * cr;
    if (std::abs(l1) < delta) { l1 = (l1 * l1 + delta * delta) / (2.0 * delta); if (l1 < 0) l1 = -l1; }
    if (std::abs(l3) < delta) { l3 = (l3 * l3 + delta * delta) / (2.0 * delta); if (l3 < 0) l3 = -l3; }
    double dh = hR - hL, dun = unR - unL, dut = utR - utL;
    double a1 = 0.5 * (dh - hr / cr * dun), a2 = hr * dut, a3 = 0.5 * (dh + hr / cr * dun);
    double F1L = hL * unL, F2L = hL * uL * unL + 0.5 * g * hL * hL * nx, F3L = hL * vL * unL + 0.5 * g * hL * hL * ny;
    double F1R = hR * unR, F2R = hR * uR * unR + 0.5 * g * hR * hR * nx, F3R = hR * vR * unR + 0.5 * g * hR * hR * ny;
    double al1 = std::abs(l1), al2 = std::abs(l2), al3 = std::abs(l3);
    double r11 = a1, r12 = a1 * (ur - cr * nx), r13 = a1 * (vr - cr * ny);
    double r21 = 0.0, r22 = a2 * (-ny), r23 = a2 * nx;
    double r31 = a3, r32 = a3 * (ur + cr * nx), r33 = a3 * (vr + cr * ny);
    F[0] = 0.5 * (F1L + F1R) - 0.5 * (al1 * r11 + al2 * r21 + al3 * r31);
    F[1] = 0.5 * (F2L + F2R) - 0.5 * (al1 * r12 + al2 * r22 + al3 * r32);
    F[2] = 0.5 * (F3L + F3R) - 0.5 * (al1 * r13 + al2 * r23 + al3 * r33);
}

void sw_flux(int kind, const double UL[3], const double UR[3], double nx, double ny, double g,
             double F[3]) {
    if (kind == FLUX_HLLC) flux_hllc(UL, UR, nx, ny, g, F);
    else if (kind == FLUX_ROE) flux_roe(UL, UR, nx, ny, g, F);
    else flux_lf(UL, UR, nx, ny, g, F);
}

// ============================================================================ compat
static void matvec(const Vec &M, int n, const double *x, double *y) {
    for (int r = 0; r < n; ++r) {
        double s = 0.0;
        for (int c = 0; c < n; ++c) s += M[(size_t)r * n + c] * x[c];
        y[r] = s;
    }
}

// The element operator's tables, built once as DG3DElementOperator holds them
// (src/dg/operators_3d.cpp:14-45): LGL basis, dense 3D derivative matrices (quirk Q2) and the
// sigma weights (src/physics/mode_splitting.cpp:80-85).
struct CompatOps {
    Basis1D b;
    Vec Dx, Dy, Dz, sw;
    explicit CompatOps(int order) : b(make_lgl(order)) {
        build_dense_3d(b, Dx, Dy, Dz);
        sw.resize(b.np());
        for (int k = 0; k < b.np(); ++k) sw[k] = 0.5 * b.weights[k];
    }
};

// src/physics/primitive_equations.cpp:136-393 (element) and :428 (solver loop).
static void compat_rhs_elements(const CompatOps &ops, int nel, const double *const in[6],
                                const double *hh, const double *ff, const CompatParams &p,
                                double *const out[5]) {
    const Basis1D &b = ops.b;
    const Vec &Dx = ops.Dx, &Dy = ops.Dy, &Dz = ops.Dz, &sw = ops.sw;
    const int np = b.np(), nd = np * np * np, nh = np * np, nv = np;
    Vec H(nd), Hinv(nd), u(nd), v(nd), T(nd), S(nd), t1(nd), t2(nd), t3(nd), a(nd), c(nd);
    for (int e = 0; e < nel; ++e) {
        const size_t o = (size_t)e * nd;
        const double *Hu = in[0] + o, *Hv = in[1] + o, *eta = in[2] + o, *HT = in[3] + o,
                     *HS = in[4] + o, *om = in[5] + o, *h = hh + o, *f = ff + o;
        double *dHu = out[0] + o, *dHv = out[1] + o, *deta = out[2] + o, *dHT = out[3] + o,
               *dHS = out[4] + o;
        // PrimitiveState::update_derived :12
        for (int i = 0; i < nd; ++i) {
            H[i] = eta[i] + h[i];
            Hinv[i] = (H[i] > 1e-10) ? 1.0 / H[i] : 0.0;
            u[i] = Hu[i] * Hinv[i]; v[i] = Hv[i] * Hinv[i];
            T[i] = HT[i] * Hinv[i]; S[i] = HS[i] * Hinv[i];
        }
        auto divergence = [&](const double *q, const double *vx, const double *vy,
                              const double *vz, double *res) {
            Vec fx(nd), fy(nd), fz(nd), r1(nd), r2(nd), r3(nd);
            for (int i = 0; i < nd; ++i) { fx[i] = q[i] * vx[i]; fy[i] = q[i] * vy[i]; fz[i] = q[i] * vz[i]; }
            matvec(Dx, nd, fx.data(), r1.data());
            matvec(Dy, nd, fy.data(), r2.data());
            matvec(Dz, nd, fz.data(), r3.data());
            for (int i = 0; i < nd; ++i) res[i] = r1[i] + r2[i] + r3[i];
        };
        // momentum :154-199 — flux q*u uses Hu*u, Hu*v, Hu*omega
        {
            Vec advu(nd), advv(nd), dex(nd), dey(nd);
            {
                Vec fx(nd), fy(nd), fz(nd), r1(nd), r2(nd), r3(nd);
                for (int i = 0; i < nd; ++i) { fx[i] = Hu[i] * u[i]; fy[i] = Hu[i] * v[i]; fz[i] = Hu[i] * om[i]; }
                matvec(Dx, nd, fx.data(), r1.data()); matvec(Dy, nd, fy.data(), r2.data()); matvec(Dz, nd, fz.data(), r3.data());
                for (int i = 0; i < nd; ++i) advu[i] = r1[i] + r2[i] + r3[i];
                for (int i = 0; i < nd; ++i) { fx[i] = Hv[i] * u[i]; fy[i] = Hv[i] * v[i]; fz[i] = Hv[i] * om[i]; }
                matvec(Dx, nd, fx.data(), r1.data()); matvec(Dy, nd, fy.data(), r2.data()); matvec(Dz, nd, fz.data(), r3.data());
                for (int i = 0; i < nd; ++i) advv[i] = r1[i] + r2[i] + r3[i];
            }
            matvec(Dx, nd, eta, dex.data());
            matvec(Dy, nd, eta, dey.data());
            for (int i = 0; i < nd; ++i) {
                dHu[i] = 0.0 - advu[i];
                dHv[i] = 0.0 - advv[i];
                dHu[i] += f[i] * Hv[i];
                dHv[i] += -f[i] * Hu[i];
                dHu[i] += -p.g * H[i] * dex[i];
                dHv[i] += -p.g * H[i] * dey[i];
            }
            if (p.nu_h > 0.0) {
                Vec gx(nd), gy(nd), gxx(nd), gyy(nd), hx(nd), hy(nd), hxx(nd), hyy(nd);
                matvec(Dx, nd, u.data(), gx.data()); matvec(Dy, nd, u.data(), gy.data());
                matvec(Dx, nd, gx.data(), gxx.data()); matvec(Dy, nd, gy.data(), gyy.data());
                matvec(Dx, nd, v.data(), hx.data()); matvec(Dy, nd, v.data(), hy.data());
                matvec(Dx, nd, hx.data(), hxx.data()); matvec(Dy, nd, hy.data(), hyy.data());
                for (int i = 0; i < nd; ++i) {
                    dHu[i] += H[i] * (p.nu_h * gxx[i] + p.nu_h * gyy[i]);
                    dHv[i] += H[i] * (p.nu_h * hxx[i] + p.nu_h * hyy[i]);
                }
            }
            if (p.nu_v > 0.0) {
                Vec g1(nd), g2(nd), k1(nd), k2(nd);
                matvec(Dz, nd, u.data(), g1.data()); matvec(Dz, nd, g1.data(), g2.data());
                matvec(Dz, nd, v.data(), k1.data()); matvec(Dz, nd, k1.data(), k2.data());
                for (int i = 0; i < nd; ++i) {
                    dHu[i] += p.nu_v * g2[i] * Hinv[i];
                    dHv[i] += p.nu_v * k2[i] * Hinv[i];
                }
            }
        }
        // tracers :201-227
        divergence(HT, u.data(), v.data(), om, a.data());
        divergence(HS, u.data(), v.data(), om, c.data());
        for (int i = 0; i < nd; ++i) { dHT[i] = 0.0 - a[i]; dHS[i] = 0.0 - c[i]; }
        if (p.kappa_v_T > 0.0) {
            matvec(Dz, nd, T.data(), t1.data()); matvec(Dz, nd, t1.data(), t2.data());
            for (int i = 0; i < nd; ++i) dHT[i] += p.kappa_v_T * t2[i] * Hinv[i];
        }
        if (p.kappa_v_S > 0.0) {
            matvec(Dz, nd, S.data(), t1.data()); matvec(Dz, nd, t1.data(), t3.data());
            for (int i = 0; i < nd; ++i) dHS[i] += p.kappa_v_S * t3[i] * Hinv[i];
        }
        // eta :229-273 — column index i_h*n_vert + k (quirk Q1)
        Vec HUb(nh), HVb(nh);
        for (int ih = 0; ih < nh; ++ih) {
            double su = 0.0, sv = 0.0;
            for (int k = 0; k < nv; ++k) { su += sw[k] * Hu[ih * nv + k]; sv += sw[k] * Hv[ih * nv + k]; }
            HUb[ih] = su; HVb[ih] = sv;
        }
        for (int j = 0; j < np; ++j) for (int i = 0; i < np; ++i) {
            double dx = 0.0, dy = 0.0;
            for (int ii = 0; ii < np; ++ii) {
                dx += b.D[i * np + ii] * HUb[ii + j * np];
                dy += b.D[j * np + ii] * HVb[i + ii * np];
            }
            const double d2 = -(dx + dy);
            for (int k = 0; k < nv; ++k) deta[(i + j * np) * nv + k] = d2;
        }
    }
}

void compat_compute_rhs(int order, int nel, const double *const in[6], const double *hh,
                        const double *ff, const CompatParams &p, double *const out[5]) {
    const CompatOps ops(order);
    compat_rhs_elements(ops, nel, in, hh, ff, p, out);
}

// src/physics/mode_splitting.cpp:136-600 per element (quirks Q1, Q4, Q10 replicated).
void compat_modesplit_step(int order, int nel, double dt, int nsub, double *const st[12],
                           const double *hh, const double *ff, const CompatParams &p) {
    if (nsub < 1) throw std::invalid_argument("nsub must be >= 1");
    Basis1D b = make_lgl(order);
    const int np = b.np(), nd = np * np * np, nh = np * np, nv = np;
    Vec sw(nv);
    double swsum = 0.0;
    for (int k = 0; k < nv; ++k) sw[k] = 0.5 * b.weights[k];
    auto Dx2 = [&](const Vec &x, int ih) {
        int i = ih % np, j = ih / np; double s = 0.0;
        for (int ii = 0; ii < np; ++ii) s += b.D[i * np + ii] * x[ii + j * np];
        return s;
    };
    auto Dy2 = [&](const Vec &x, int ih) {
        int i = ih % np, j = ih / np; double s = 0.0;
        for (int ii = 0; ii < np; ++ii) s += b.D[j * np + ii] * x[i + ii * np];
        return s;
    };
    for (int e = 0; e < nel; ++e) {
        const size_t o = (size_t)e * nd;
        double *Hu = st[0] + o, *Hv = st[1] + o, *eta = st[2] + o, *HT = st[3] + o, *HS = st[4] + o,
               *H = st[5] + o, *u = st[6] + o, *v = st[7] + o, *T = st[8] + o, *S = st[9] + o,
               *om = st[10] + o, *rho = st[11] + o;
        const double *h = hh + o, *f = ff + o;
        auto depth_average = [&](const double *x3, Vec &out) {
            out.assign(nh, 0.0);
            for (int ih = 0; ih < nh; ++ih) {
                double s = 0.0, ws = 0.0;
                for (int k = 0; k < nv; ++k) { s += sw[k] * x3[ih * nv + k]; ws += sw[k]; }
                out[ih] = s / ws;
            }
        };
        auto depth_integrate = [&](const double *x3, const double *H3, Vec &out) {
            out.assign(nh, 0.0);
            for (int ih = 0; ih < nh; ++ih) {
                double s = 0.0;
                for (int k = 0; k < nv; ++k) s += sw[k] * H3[ih * nv + k] * x3[ih * nv + k];
                out[ih] = s;
            }
        };
        (void)swsum;
        // decompose :359
        Vec Ub, Vb, HUb, HVb, beta(nh), bH(nh);
        depth_average(u, Ub); depth_average(v, Vb);
        for (int i = 0; i < nh; ++i) { beta[i] = eta[i]; bH[i] = H[i]; }
        depth_integrate(u, H, HUb); depth_integrate(v, H, HVb);
        Vec up(nd), vp(nd), cHT(HT, HT + nd), cHS(HS, HS + nd), com(om, om + nd);
        for (int ih = 0; ih < nh; ++ih) for (int k = 0; k < nv; ++k) {
            up[ih * nv + k] = u[ih * nv + k] - Ub[ih];
            vp[ih * nv + k] = v[ih * nv + k] - Vb[ih];
        }
        // subcycle :319 with predictor-corrector :293 and barotropic_rhs :213
        auto rhs = [&](const Vec &E, const Vec &HU, const Vec &HV, const Vec &Hb, Vec &dE, Vec &dU,
                       Vec &dV) {
            dE.assign(nh, 0.0); dU.assign(nh, 0.0); dV.assign(nh, 0.0);
            for (int i = 0; i < nh; ++i) {
                dE[i] = -(Dx2(HU, i) + Dy2(HV, i));
                double pgx = -p.g * Hb[i] * Dx2(E, i), pgy = -p.g * Hb[i] * Dy2(E, i);
                double cx = f[i] * HV[i], cy = -f[i] * HU[i];
                dU[i] = pgx + cx + 0.0;
                dV[i] = pgy + cy + 0.0;
            }
        };
        const double dtb = dt / nsub;
        Vec eavg(nh, 0.0), dE, dU, dV, sE, sU, sV;
        for (int sub = 0; sub < nsub; ++sub) {
            rhs(beta, HUb, HVb, bH, dE, dU, dV);
            Vec Es(nh), Us(nh), Vs(nh), Hs(nh);
            for (int i = 0; i < nh; ++i) {
                Es[i] = beta[i] + dtb * dE[i]; Us[i] = HUb[i] + dtb * dU[i]; Vs[i] = HVb[i] + dtb * dV[i];
                Hs[i] = Es[i] + h[i];
            }
            rhs(Es, Us, Vs, Hs, sE, sU, sV);
            const double hdt = 0.5 * dtb;
            for (int i = 0; i < nh; ++i) {
                beta[i] += hdt * (dE[i] + sE[i]);
                HUb[i] += hdt * (dU[i] + sU[i]);
                HVb[i] += hdt * (dV[i] + sV[i]);
                bH[i] = beta[i] + h[i];
                double Hi = (bH[i] > 1e-10) ? 1.0 / bH[i] : 0.0;
                Ub[i] = HUb[i] * Hi; Vb[i] = HVb[i] * Hi;
                eavg[i] += beta[i];
            }
        }
        for (int i = 0; i < nh; ++i) eavg[i] /= (double)nsub;
        // update_baroclinic :487
        for (int ih = 0; ih < nh; ++ih) for (int k = 0; k < nv; ++k) eta[ih * nv + k] = eavg[ih];
        for (int ih = 0; ih < nh; ++ih) {
            double Hv_ = eavg[ih] + h[ih];
            for (int k = 0; k < nv; ++k) H[ih * nv + k] = Hv_;
        }
        Vec U2, V2;
        depth_average(u, U2); depth_average(v, V2);
        for (int ih = 0; ih < nh; ++ih) for (int k = 0; k < nv; ++k) {
            int idx = ih * nv + k;
            double ut = U2[ih] + up[idx], vt = V2[ih] + vp[idx];
            u[idx] = ut; v[idx] = vt;
            Hu[idx] = H[idx] * ut; Hv[idx] = H[idx] * vt;
        }
        for (int idx = 0; idx < nd; ++idx) {
            double Hi = (H[idx] > 1e-10) ? 1.0 / H[idx] : 0.0;
            T[idx] = cHT[idx] * Hi; S[idx] = cHS[idx] * Hi;
        }
        for (int idx = 0; idx < nd; ++idx) { cHT[idx] = H[idx] * T[idx]; cHS[idx] = H[idx] * S[idx]; }
        Vec HU2, HV2;
        depth_integrate(u, H, HU2); depth_integrate(v, H, HV2);
        for (int ih = 0; ih < nh; ++ih) {
            double div = Dx2(HU2, ih) + Dy2(HV2, ih);
            double Hval = H[ih * nv], Hi = (Hval > 1e-10) ? 1.0 / Hval : 0.0;
            for (int k = 0; k < nv; ++k) {
                double sf = (double)k / (double)(nv - 1);
                com[ih * nv + k] = -sf * div * Hi;
            }
        }
        for (int idx = 0; idx < nd; ++idx) {
            om[idx] = com[idx];
            rho[idx] = p.rho0 * (1.0 - p.alpha * (T[idx] - 10.0) + p.beta * (S[idx] - 35.0));
        }
        // recombine :398
        for (int ih = 0; ih < nh; ++ih) for (int k = 0; k < nv; ++k) {
            int idx = ih * nv + k;
            u[idx] = Ub[ih] + up[idx];
            v[idx] = Vb[ih] + vp[idx];
            eta[idx] = beta[ih];
        }
        for (int idx = 0; idx < nd; ++idx) { HT[idx] = cHT[idx]; HS[idx] = cHS[idx]; om[idx] = com[idx]; }
    }
    (void)ff;
}

void compat_ssprk3_step(int order, int nel, double dt, double *const st6[6], const double *hh,
                        const double *ff, const CompatParams &p, int nthreads) {
    const int np = order + 1, nd = np * np * np;
    const size_t per = (size_t)5 * nd, N = per * nel;
    // pack_state: [Hu, Hv, eta, HT, HS] per element
    Vec U(N), U1(N), U2(N), k(N);
    auto pack = [&](Vec &X) {
        for (int e = 0; e < nel; ++e)
            for (int v = 0; v < 5; ++v)
                for (int i = 0; i < nd; ++i) X[e * per + v * nd + i] = st6[v][(size_t)e * nd + i];
    };
    pack(U);
    Vec om(st6[5], st6[5] + (size_t)nel * nd);
    const CompatOps ops(order);  // the element operator, built once (not per element or stage)
    auto rhs = [&](const Vec &X, Vec &dX) {
        // unpack_state into per-element arrays, then the element loop in chunks
        const int nt = std::max(1, nthreads);
        auto work = [&](int e0, int e1) {
            Vec in[6], out[5];
            for (int e = e0; e < e1; ++e) {
                for (int v = 0; v < 5; ++v) in[v].assign(X.begin() + e * per + v * nd, X.begin() + e * per + (v + 1) * nd);
                in[5].assign(om.begin() + (size_t)e * nd, om.begin() + (size_t)(e + 1) * nd);
                for (int v = 0; v < 5; ++v) out[v].assign(nd, 0.0);
                const double *ip[6] = {in[0].data(), in[1].data(), in[2].data(), in[3].data(), in[4].data(), in[5].data()};
                double *op[5] = {out[0].data(), out[1].data(), out[2].data(), out[3].data(), out[4].data()};
                compat_rhs_elements(ops, 1, ip, hh + (size_t)e * nd, ff + (size_t)e * nd, p, op);
                for (int v = 0; v < 5; ++v) std::copy(out[v].begin(), out[v].end(), dX.begin() + e * per + v * nd);
            }
        };
        if (nt == 1) { work(0, nel); return; }
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) {
            const int e0 = (int)((long)nel * t / nt), e1 = (int)((long)nel * (t + 1) / nt);
            th.emplace_back(work, e0, e1);
        }
        for (auto &x : th) x.join();
    };
    rhs(U, k);
    for (size_t i = 0; i < N; ++i) U1[i] = U[i] + dt * k[i];
    rhs(U1, k);
    for (size_t i = 0; i < N; ++i) U2[i] = 0.75 * U[i] + 0.25 * (U1[i] + dt * k[i]);
    rhs(U2, k);
    for (size_t i = 0; i < N; ++i) U[i] = (1.0 / 3.0) * U[i] + (2.0 / 3.0) * (U2[i] + dt * k[i]);
    for (int e = 0; e < nel; ++e)
        for (int v = 0; v < 5; ++v)
            for (int i = 0; i < nd; ++i) st6[v][(size_t)e * nd + i] = U[e * per + v * nd + i];
}

// ============================================================================ time steppers
const double LSRK_A[5] = {0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257};
const double LSRK_B[5] = {0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488,
                          0.1530572479681};
const double LSRK_C[5] = {0.0, 0.1496590219993, 0.3704009573644, 0.6222557631345, 0.9582821306748};

// src/solver/time_stepper.cpp:13-240
void rk_step(int scheme, double t, double dt, Vec &U, const RHSFn &rhs) {
    const size_t n = U.size();
    Vec k1(n), k2(n), k3(n), k4(n), k5(n), k6(n), tmp(n);
    auto lin = [&](Vec &out, double a, const Vec &x, double b2, const Vec &y) {
        for (size_t i = 0; i < n; ++i) out[i] = a * x[i] + b2 * y[i];
    };
    switch (scheme) {
    case RK_EULER:
        rhs(t, U, k1);
        for (size_t i = 0; i < n; ++i) U[i] += dt * k1[i];
        break;
    case RK_MIDPOINT:
        rhs(t, U, k1);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + 0.5 * dt * k1[i];
        rhs(t + 0.5 * dt, tmp, k2);
        for (size_t i = 0; i < n; ++i) U[i] += dt * k2[i];
        break;
    case RK_SSP3: {
        Vec U1(n), U2(n);
        rhs(t, U, k1);
        for (size_t i = 0; i < n; ++i) U1[i] = U[i] + dt * k1[i];
        rhs(t + dt, U1, k1);
        for (size_t i = 0; i < n; ++i) U2[i] = 0.75 * U[i] + 0.25 * (U1[i] + dt * k1[i]);
        rhs(t + 0.5 * dt, U2, k1);
        for (size_t i = 0; i < n; ++i) U[i] = (1.0 / 3.0) * U[i] + (2.0 / 3.0) * (U2[i] + dt * k1[i]);
        break;
    }
    case RK_RK4:
        rhs(t, U, k1);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + 0.5 * dt * k1[i];
        rhs(t + 0.5 * dt, tmp, k2);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + 0.5 * dt * k2[i];
        rhs(t + 0.5 * dt, tmp, k3);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + dt * k3[i];
        rhs(t + dt, tmp, k4);
        for (size_t i = 0; i < n; ++i) U[i] += (dt / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
        break;
    case RK_LSRK45: {
        Vec res(n, 0.0);
        for (int s = 0; s < 5; ++s) {
            rhs(t + LSRK_C[s] * dt, U, tmp);
            for (size_t i = 0; i < n; ++i) res[i] = LSRK_A[s] * res[i] + dt * tmp[i];
            for (size_t i = 0; i < n; ++i) U[i] += LSRK_B[s] * res[i];
        }
        break;
    }
    case RK_DOPRI:
        rhs(t, U, k1);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + (dt / 5.0) * k1[i];
        rhs(t + dt / 5.0, tmp, k2);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + dt * (3.0 / 40.0 * k1[i] + 9.0 / 40.0 * k2[i]);
        rhs(t + 3.0 * dt / 10.0, tmp, k3);
        for (size_t i = 0; i < n; ++i) tmp[i] = U[i] + dt * (44.0 / 45.0 * k1[i] - 56.0 / 15.0 * k2[i] + 32.0 / 9.0 * k3[i]);
        rhs(t + 4.0 * dt / 5.0, tmp, k4);
        for (size_t i = 0; i < n; ++i)
            tmp[i] = U[i] + dt * (19372.0 / 6561.0 * k1[i] - 25360.0 / 2187.0 * k2[i] + 64448.0 / 6561.0 * k3[i] - 212.0 / 729.0 * k4[i]);
        rhs(t + 8.0 * dt / 9.0, tmp, k5);
        for (size_t i = 0; i < n; ++i)
            tmp[i] = U[i] + dt * (9017.0 / 3168.0 * k1[i] - 355.0 / 33.0 * k2[i] + 46732.0 / 5247.0 * k3[i] + 49.0 / 176.0 * k4[i] - 5103.0 / 18656.0 * k5[i]);
        rhs(t + dt, tmp, k6);
        for (size_t i = 0; i < n; ++i)
            U[i] += dt * (35.0 / 384.0 * k1[i] + 500.0 / 1113.0 * k3[i] + 125.0 / 192.0 * k4[i] - 2187.0 / 6784.0 * k5[i] + 11.0 / 84.0 * k6[i]);
        break;
    default:
        throw std::invalid_argument("unknown RK scheme");
    }
    (void)lin;
}

// ============================================================================ physical mode
// The coupled scheme the reference declares but leaves as stubs (face fluxes
// src/physics/primitive_equations.cpp:444-578, full-column omega src/physics/vertical_velocity.cpp:55,
// wind stress :695, bottom friction :716, mode split src/physics/mode_splitting.cpp:434):
// nodal strong-form DGSEM on LGL nodes, affine (x, y, sigma) elements, collocated lifting.
void PhysModel::init(const PhysParams &pp, const double *h2, const double *f2, const double *tx,
                     const double *ty) {
    p = pp;
    b = make_lgl(p.order);
    np = b.np(); np2 = np * np; np3 = np2 * np;
    ncol = p.nx * p.ny;
    n2 = (long)ncol * np2;
    n3 = (long)ncol * p.nz * np3;
    dx = p.Lx / p.nx; dy = p.Ly / p.ny; dsig = 1.0 / p.nz;
    h.assign(h2, h2 + n2); f.assign(f2, f2 + n2);
    taux.assign(tx, tx + n2); tauy.assign(ty, ty + n2);
    for (auto &q : Q) q.assign(n3, 0.0);
    eta.assign(n2, 0.0); HU.assign(n2, 0.0); HV.assign(n2, 0.0); eta_avg.assign(n2, 0.0);
    t = 0.0;
}

void PhysModel::set_state(const double *const q[4], const double *eta2) {
    for (int v = 0; v < 4; ++v) Q[v].assign(q[v], q[v] + n3);
    eta.assign(eta2, eta2 + n2);
    eta_avg = eta;
    column_integral(Q[0], HU);
    column_integral(Q[1], HV);
}

double PhysModel::tide(double time) const {
    return p.tide_amp * std::sin(2.0 * M_PI * time / p.tide_period);
}

void PhysModel::column_integral(const Vec &g3, Vec &out2) const {
    out2.assign(n2, 0.0);
    for (int c = 0; c < ncol; ++c)
        for (int a = 0; a < np2; ++a) {
            double s = 0.0;
            for (int ez = 0; ez < p.nz; ++ez)
                for (int k = 0; k < np; ++k)
                    s += 0.5 * dsig * b.weights[k] * g3[((size_t)c * p.nz + ez) * np3 + a + np2 * k];
            out2[(size_t)c * np2 + a] = s;
        }
}

// Runs fn(c0, c1) on contiguous ranges of the ncol water columns on the host's threads
// (ORACLE_THREADS in the environment caps them; 1 runs inline).
static void for_columns(int ncol, const std::function<void(int, int)> &fn) {
    int nt = (int)std::thread::hardware_concurrency();
    if (const char *e = std::getenv("ORACLE_THREADS")) nt = std::atoi(e);
    nt = std::max(1, std::min(nt, ncol / 4));
    if (nt <= 1) {
        fn(0, ncol);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back(fn, (int)((long)ncol * t / nt), (int)((long)ncol * (t + 1) / nt));
    for (auto &x : th) x.join();
}

// Hydrostatic pressure of the density anomaly, PressureGradientElement::hydrostatic_pressure
// (include/physics/pressure_gradient.hpp:232-249: p(k) = sum_{j>=k} w_j g rho H, a surface-down
// column sum) taken over the whole water column and integrated exactly per layer with the
// integration matrix S: p'/rho0 = g H B(sigma), B(sigma) = int_sigma^0 b dsigma'. The density
// is the reference's linear equation of state (src/physics/mode_splitting.cpp:589-598).
void PhysModel::baroclinic_B(const Vec *Qin, const Vec &etaf, Vec &b3, Vec &B3) const {
    const int N = p.order, nz = p.nz;
    b3.assign(n3, 0.0);
    B3.assign(n3, 0.0);
    for_columns(ncol, [&](int cb, int ce) {
    for (int c = cb; c < ce; ++c) {
        const size_t base = (size_t)c * nz * np3;
        for (int a = 0; a < np2; ++a) {
            // b - b_ref(z) = beta (S - S0) - alpha (T - T_ref(z)), T = HT / H, S = HS / H,
            // z = eta + sigma H
            const double e = etaf[(size_t)c * np2 + a], H = e + h[(size_t)c * np2 + a];
            const double iH = 1.0 / H;
            for (int ez = 0; ez < nz; ++ez)
                for (int k = 0; k < np; ++k) {
                    const size_t n = base + (size_t)ez * np3 + a + np2 * k;
                    const double sg = -1.0 + dsig * (ez + 0.5 * (b.nodes[k] + 1.0));
                    const double Tr = p.Tref_s + p.Tref_dz * (e + sg * H);
                    b3[n] = p.beta * (Qin[3][n] * iH - p.S0) - p.alpha * (Qin[2][n] * iH - Tr);
                }
            // I(sigma) = int_{-1}^{sigma} b, layer by layer (as the omega scan); B = I(0) - I
            double Ib = 0.0;
            std::vector<double> I((size_t)nz * np);
            for (int ez = 0; ez < nz; ++ez) {
                double J[16];
                for (int k = 0; k < np; ++k) {
                    double s = 0.0;
                    for (int m = 0; m < np; ++m)
                        s += b.S[k * np + m] * b3[base + (size_t)ez * np3 + a + np2 * m];
                    J[k] = 0.5 * dsig * s;
                }
                J[0] = 0.0;
                for (int k = 0; k < np; ++k) I[ez * np + k] = Ib + J[k];
                Ib += J[N];
            }
            for (int ez = 0; ez < nz; ++ez)
                for (int k = 0; k < np; ++k) {
                    double Bv = Ib - I[ez * np + k];
                    if (ez == nz - 1 && k == N) Bv = 0.0;
                    B3[base + (size_t)ez * np3 + a + np2 * k] = Bv;
                }
        }
    }
    });
}

void PhysModel::rhs3d(const Vec *Qin, const Vec &etaf, double tb, Vec *R, Vec *omega3,
                      Vec *deta2, const Vec *etab_in) const {
    const Vec &etab = etab_in ? *etab_in : etaf;
    const int N = p.order, nz = p.nz;
    const double *D = b.D.data();
    const double wend = b.weights[0];
    const double Lx = (2.0 / dx) / wend, Ly = (2.0 / dy) / wend, Ls = (2.0 / dsig) / wend;
    const double cx = 2.0 / dx, cy = 2.0 / dy, cs = 2.0 / dsig;
    const int ncn = nz * np3;
    if (omega3) omega3->assign(n3, 0.0);
    if (deta2) deta2->assign(n2, 0.0);
    for (int v = 0; v < 4; ++v) R[v].assign(n3, 0.0);
    const double etide = tide(tb);
    // baroclinic pressure: b and B at every node (neighbour columns' B is read at faces)
    const bool baroclinic = p.alpha != 0.0 || p.beta != 0.0;
    Vec b3, B3;
    if (baroclinic) baroclinic_B(Qin, etab, b3, B3);
    // water columns are independent given the inputs: split them over host threads (each
    // column is computed by one thread in the same order, so the result does not depend on
    // the thread count)
    for_columns(ncol, [&](int c0, int c1) {
    Vec om(ncn), del(ncn), Mf((size_t)(nz + 1) * np2);  // Mf: mass flux H omega through layer faces
    Vec Hc(np2), iHc(np2);
    for (int c = c0; c < c1; ++c) {
        const int ex = c % p.nx, ey = c / p.nx;
        const size_t base = (size_t)c * ncn;
        auto q = [&](int v, int ez, int i, int j, int k) -> double {
            return Qin[v][base + (size_t)ez * np3 + i + np * (j + np * k)];
        };
        for (int a = 0; a < np2; ++a) {
            Hc[a] = etaf[(size_t)c * np2 + a] + h[(size_t)c * np2 + a];
            iHc[a] = 1.0 / Hc[a];
        }
        // neighbour / ghost access for horizontal faces. side: 0 W,1 E,2 S,3 N
        // returns q+ (4), eta+, H+ for own node (ez,i,j,k) across side.
        auto outside = [&](int side, int ez, int i, int j, int k, double qp[4], double &etap,
                           double &Hp) {
            int nc = -1, ni = i, nj = j;
            if (side == 0 && ex > 0) { nc = c - 1; ni = N; }
            if (side == 1 && ex < p.nx - 1) { nc = c + 1; ni = 0; }
            if (side == 2 && ey > 0) { nc = c - p.nx; nj = N; }
            if (side == 3 && ey < p.ny - 1) { nc = c + p.nx; nj = 0; }
            const int a = i + np * j;
            if (nc >= 0) {
                const size_t nb = (size_t)nc * ncn + (size_t)ez * np3 + ni + np * (nj + np * k);
                for (int v = 0; v < 4; ++v) qp[v] = Qin[v][nb];
                etap = etaf[(size_t)nc * np2 + ni + np * nj];
                Hp = etap + h[(size_t)nc * np2 + ni + np * nj];
                return;
            }
            double qm[4];
            for (int v = 0; v < 4; ++v) qm[v] = q(v, ez, i, j, k);
            if (p.bc[side] == 1) {
                etap = etide;
                Hp = etap + h[(size_t)c * np2 + a];
                const double r = Hp * iHc[a];
                for (int v = 0; v < 4; ++v) qp[v] = qm[v] * r;
            } else {
                etap = etaf[(size_t)c * np2 + a];
                Hp = Hc[a];
                for (int v = 0; v < 4; ++v) qp[v] = qm[v];
                if (side <= 1) qp[0] = -qm[0]; else qp[1] = -qm[1];
            }
        };
        // ---- horizontal divergence of (Hu, Hv) with central face flux
        for (int ez = 0; ez < nz; ++ez)
            for (int k = 0; k < np; ++k)
                for (int j = 0; j < np; ++j)
                    for (int i = 0; i < np; ++i) {
                        double sx = 0.0, sy = 0.0;
                        for (int m = 0; m < np; ++m) {
                            sx += D[i * np + m] * q(0, ez, m, j, k);
                            sy += D[j * np + m] * q(1, ez, i, m, k);
                        }
                        double d = cx * sx + cy * sy;
                        const int sides[4] = {i == 0 ? 0 : -1, i == N ? 1 : -1, j == 0 ? 2 : -1, j == N ? 3 : -1};
                        for (int s : sides) {
                            if (s < 0) continue;
                            double qp[4], ep, Hp;
                            outside(s, ez, i, j, k, qp, ep, Hp);
                            const int comp = s <= 1 ? 0 : 1;
                            const double nrm = (s == 0 || s == 2) ? -1.0 : 1.0;
                            const double L = s <= 1 ? Lx : Ly;
                            const double fm = q(comp, ez, i, j, k) * nrm;
                            const double fs = 0.5 * (q(comp, ez, i, j, k) + qp[comp]) * nrm;
                            d += L * (fs - fm);
                        }
                        del[ez * np3 + i + np * (j + np * k)] = d;
                    }
        // ---- sigma velocity consistent with the discrete tracer divergence: per layer, bottom
        // up, H omega = y solves the strong-form continuity cs D y + Ls e_0 (y_0 - y*) = I - delta
        // with y* the mass flux through the layer's bottom face (0 at the bed) and I the
        // LGL-quadrature column integral of delta (so that the flux through the surface is 0).
        // Integrated with the LGL weights each layer gives y*(top) = y*(bottom) + dsig I -
        // (dsig/2) sum_k w_k delta_k, the prefix that defines the face mass fluxes.
        for (int a = 0; a < np2; ++a) {
            const double hds = 0.5 * dsig;
            double Iq = 0.0;
            std::vector<double> Ql(nz);
            for (int ez = 0; ez < nz; ++ez) {
                double qv = 0.0;
                for (int k = 0; k < np; ++k) qv += b.weights[k] * del[ez * np3 + a + np2 * k];
                Ql[ez] = hds * qv;
                Iq += Ql[ez];
            }
            double ystar = 0.0;
            for (int ez = 0; ez < nz; ++ez) {
                Mf[ez * np2 + a] = ystar;
                double g[16];
                for (int k = 0; k < np; ++k) g[k] = Iq - del[ez * np3 + a + np2 * k];
                for (int k = 0; k < np; ++k) {
                    double s = 0.0;
                    for (int m = 0; m < np; ++m) s += b.Ainv[k * np + m] * g[m];
                    const double y = hds * s + b.a0[k] * ystar;
                    om[ez * np3 + a + np2 * k] = y * iHc[a];
                }
                ystar += dsig * Iq - Ql[ez];
            }
            Mf[nz * np2 + a] = 0.0;  // no flux through the surface
            if (deta2) (*deta2)[(size_t)c * np2 + a] = -Iq;
        }
        if (omega3)
            for (int n = 0; n < ncn; ++n) (*omega3)[base + n] = om[n];
        // ---- right-hand side
        for (int ez = 0; ez < nz; ++ez)
            for (int k = 0; k < np; ++k)
                for (int j = 0; j < np; ++j)
                    for (int i = 0; i < np; ++i) {
                        const int a = i + np * j;
                        const int ln = ez * np3 + i + np * (j + np * k);
                        const double iH = iHc[a], Hh = Hc[a];
                        auto vel = [&](int ez2, int i2, int j2, int k2, int comp) {
                            return q(comp, ez2, i2, j2, k2) * iHc[i2 + np * j2];
                        };
                        auto omg = [&](int i2, int j2, int k2) { return om[ez * np3 + i2 + np * (j2 + np * k2)]; };
                        double r[4];
                        for (int v = 0; v < 4; ++v) {
                            double ax = 0.0, ay = 0.0, as = 0.0;
                            for (int m = 0; m < np; ++m) {
                                ax += D[i * np + m] * q(v, ez, m, j, k) * vel(ez, m, j, k, 0);
                                ay += D[j * np + m] * q(v, ez, i, m, k) * vel(ez, i, m, k, 1);
                                as += D[k * np + m] * q(v, ez, i, j, m) * omg(i, j, m);
                            }
                            r[v] = -(cx * ax + cy * ay + cs * as);
                        }
                        const double fa = f[(size_t)c * np2 + a];
                        double gex = 0.0, gey = 0.0;
                        for (int m = 0; m < np; ++m) {
                            gex += D[i * np + m] * etaf[(size_t)c * np2 + m + np * j];
                            gey += D[j * np + m] * etaf[(size_t)c * np2 + i + np * m];
                        }
                        r[0] += fa * q(1, ez, i, j, k) - p.g * Hh * cx * gex;
                        r[1] += -fa * q(0, ez, i, j, k) - p.g * Hh * cy * gey;
                        // baroclinic pressure gradient -(H/rho0) grad_z p' with p'/rho0 = g H B:
                        // -g H [d(H B)/dx|_sigma + b (d(eta)/dx + sigma dH/dx)], as z = eta + sigma H
                        // gives d(sigma)/dx|_z = -(d(eta)/dx + sigma dH/dx) / H and dp'/dsigma =
                        // -rho0 g H b (PressureGradientElement::baroclinic_gradient_standard,
                        // include/physics/pressure_gradient.hpp:251-292). The derivative of P = H B
                        // is the strong DG derivative with a central face value (below).
                        if (baroclinic) {
                            // flux form: H dp'/dx|_z = d(H p')/dx|_sigma - d(p' dz/dx|_sigma)/dsigma,
                            // p' = rho0 g P, P = Hb B, with the column depth Hb = etab + h of the
                            // pressure's own elevation; dz/dx|_sigma = d(etab)/dx + sigma dHb/dx
                            double dPx = 0.0, dPy = 0.0, dEx = 0.0, dEy = 0.0, dHx = 0.0, dHy = 0.0;
                            for (int m = 0; m < np; ++m) {
                                const size_t ax = (size_t)c * np2 + m + np * j, ay = (size_t)c * np2 + i + np * m;
                                const double Hx2 = etab[ax] + h[ax], Hy2 = etab[ay] + h[ay];
                                dPx += D[i * np + m] * Hx2 * Hx2 * B3[base + (size_t)ez * np3 + m + np * (j + np * k)];
                                dPy += D[j * np + m] * Hy2 * Hy2 * B3[base + (size_t)ez * np3 + i + np * (m + np * k)];
                                dEx += D[i * np + m] * etab[ax];
                                dEy += D[j * np + m] * etab[ay];
                                dHx += D[i * np + m] * Hx2;
                                dHy += D[j * np + m] * Hy2;
                            }
                            const double Hb = etab[(size_t)c * np2 + a] + h[(size_t)c * np2 + a];
                            double dSx = 0.0, dSy = 0.0;
                            for (int m = 0; m < np; ++m) {
                                const double sgm = -1.0 + dsig * (ez + 0.5 * (b.nodes[m] + 1.0));
                                const double Pm_ = Hb * B3[base + (size_t)ez * np3 + i + np * (j + np * m)];
                                dSx += D[k * np + m] * Pm_ * (cx * dEx + sgm * cx * dHx);
                                dSy += D[k * np + m] * Pm_ * (cy * dEy + sgm * cy * dHy);
                            }
                            r[0] -= p.g * (cx * dPx - cs * dSx);
                            r[1] -= p.g * (cy * dPy - cs * dSy);
                        }
                        if (p.nu_h > 0.0) {
                            for (int comp = 0; comp < 2; ++comp) {
                                double sxx = 0.0, syy = 0.0;
                                for (int m = 0; m < np; ++m) {
                                    double tx = 0.0, ty = 0.0;
                                    for (int l = 0; l < np; ++l) {
                                        tx += D[m * np + l] * vel(ez, l, j, k, comp);
                                        ty += D[m * np + l] * vel(ez, i, l, k, comp);
                                    }
                                    sxx += D[i * np + m] * tx;
                                    syy += D[j * np + m] * ty;
                                }
                                r[comp] += p.nu_h * Hh * (cx * cx * sxx + cy * cy * syy);
                            }
                        }
                        const double kap[4] = {p.nu_v, p.nu_v, p.kappa_v_T, p.kappa_v_S};
                        for (int v = 0; v < 4; ++v) {
                            if (!(kap[v] > 0.0)) continue;
                            double szz = 0.0;
                            for (int m = 0; m < np; ++m) {
                                double tz = 0.0;
                                for (int l = 0; l < np; ++l) tz += D[m * np + l] * q(v, ez, i, j, l) * iHc[a];
                                szz += D[k * np + m] * tz;
                            }
                            r[v] += kap[v] * iH * cs * cs * szz;
                        }
                        // horizontal faces: LF advective flux + eta jump for pressure
                        const int sides[4] = {i == 0 ? 0 : -1, i == N ? 1 : -1, j == 0 ? 2 : -1, j == N ? 3 : -1};
                        for (int s : sides) {
                            if (s < 0) continue;
                            double qp[4], ep, Hp;
                            outside(s, ez, i, j, k, qp, ep, Hp);
                            const double nx = s == 0 ? -1.0 : (s == 1 ? 1.0 : 0.0);
                            const double ny = s == 2 ? -1.0 : (s == 3 ? 1.0 : 0.0);
                            const double L = s <= 1 ? Lx : Ly;
                            const double unm = (q(0, ez, i, j, k) * nx + q(1, ez, i, j, k) * ny) * iH;
                            const double unp = (qp[0] * nx + qp[1] * ny) / Hp;
                            const double lam = std::max(std::abs(unm), std::abs(unp));
                            for (int v = 0; v < 4; ++v) {
                                const double qm = q(v, ez, i, j, k);
                                const double fs = 0.5 * (qm * unm + qp[v] * unp) - 0.5 * lam * (qp[v] - qm);
                                r[v] -= L * (fs - qm * unm);
                            }
                            const double em = etaf[(size_t)c * np2 + a];
                            const double pj = p.g * Hh * 0.5 * (ep - em);
                            r[0] -= L * pj * nx;
                            r[1] -= L * pj * ny;
                            if (baroclinic) {
                                // (H P)+ across the face: the neighbour's Hb^2 B; on a wall the
                                // mirror state (no jump); on the tidal side the exterior depth with
                                // this column's B (T, S copied across)
                                const double Hb = etab[(size_t)c * np2 + a] + h[(size_t)c * np2 + a];
                                const double Pm = Hb * Hb * B3[base + ln];
                                double Pp = Pm;
                                int nc = -1, ni = i, nj = j;
                                if (s == 0 && ex > 0) { nc = c - 1; ni = N; }
                                if (s == 1 && ex < p.nx - 1) { nc = c + 1; ni = 0; }
                                if (s == 2 && ey > 0) { nc = c - p.nx; nj = N; }
                                if (s == 3 && ey < p.ny - 1) { nc = c + p.nx; nj = 0; }
                                if (nc >= 0) {
                                    const size_t n2n = (size_t)nc * np2 + ni + np * nj;
                                    const double Hbn = etab[n2n] + h[n2n];
                                    Pp = Hbn * Hbn * B3[(size_t)nc * ncn + (size_t)ez * np3 + ni + np * (nj + np * k)];
                                } else if (p.bc[s] == 1) {
                                    Pp = Hp * Hp * B3[base + ln];
                                }
                                const double pb = p.g * 0.5 * (Pp - Pm);
                                r[0] -= L * pb * nx;
                                r[1] -= L * pb * ny;
                            }
                        }
                        // vertical faces: the layer face's mass flux M (upward) carries the
                        // upwind value; at the bed and the surface M = 0
                        if (k == 0 || k == N) {
                            const double nrm = k == 0 ? -1.0 : 1.0;
                            const double wm = om[ln] * nrm;
                            const double M = Mf[(k == 0 ? ez : ez + 1) * np2 + a];
                            const bool interior = (k == 0 && ez > 0) || (k == N && ez < nz - 1);
                            const int ez2 = k == 0 ? ez - 1 : ez + 1, k2 = k == 0 ? N : 0;
                            for (int v = 0; v < 4; ++v) {
                                const double qm = q(v, ez, i, j, k);
                                // upward flux M q_up / H, q_up from below when M > 0
                                double qup = qm;
                                if (interior && ((k == 0) == (M > 0.0))) qup = q(v, ez2, i, j, k2);
                                const double fs = nrm * M * qup * iH;
                                r[v] -= Ls * (fs - qm * wm);
                            }
                            if (!interior) {
                                if (k == 0) {
                                    const double uu = q(0, ez, i, j, k) * iH, vv = q(1, ez, i, j, k) * iH;
                                    const double sp = std::sqrt(uu * uu + vv * vv);
                                    r[0] -= Ls * p.cd * sp * uu;
                                    r[1] -= Ls * p.cd * sp * vv;
                                } else {
                                    r[0] += Ls * taux[(size_t)c * np2 + a] / p.rho0;
                                    r[1] += Ls * tauy[(size_t)c * np2 + a] / p.rho0;
                                }
                            }
                        }
                        for (int v = 0; v < 4; ++v) R[v][base + ln] = r[v];
                    }
    }
    });
}

void PhysModel::rhs2d(const Vec &e, const Vec &hu, const Vec &hv, const Vec *Fx, const Vec *Fy,
                      double time, Vec &ke, Vec &khu, Vec &khv) const {
    const int N = p.order;
    const double *D = b.D.data();
    const double wend = b.weights[0];
    const double Lx = (2.0 / dx) / wend, Ly = (2.0 / dy) / wend, cx = 2.0 / dx, cy = 2.0 / dy;
    ke.assign(n2, 0.0); khu.assign(n2, 0.0); khv.assign(n2, 0.0);
    const double etide = tide(time);
    for (int c = 0; c < ncol; ++c) {
        const int ex = c % p.nx, ey = c / p.nx;
        const size_t o = (size_t)c * np2;
        for (int j = 0; j < np; ++j)
            for (int i = 0; i < np; ++i) {
                const int a = i + np * j;
                const double H = e[o + a] + h[o + a];
                double dhu = 0, dhv = 0, auu = 0, auv = 0, avu = 0, avv = 0, gex = 0, gey = 0;
                for (int m = 0; m < np; ++m) {
                    const size_t px = o + m + np * j, py = o + i + np * m;
                    const double Hx = e[px] + h[px], Hy = e[py] + h[py];
                    dhu += D[i * np + m] * hu[px];
                    dhv += D[j * np + m] * hv[py];
                    auu += D[i * np + m] * hu[px] * hu[px] / Hx;
                    avu += D[i * np + m] * hv[px] * hu[px] / Hx;
                    auv += D[j * np + m] * hu[py] * hv[py] / Hy;
                    avv += D[j * np + m] * hv[py] * hv[py] / Hy;
                    gex += D[i * np + m] * e[px];
                    gey += D[j * np + m] * e[py];
                }
                double re = -(cx * dhu + cy * dhv);
                double ru = -(cx * auu + cy * auv) - p.g * H * cx * gex + f[o + a] * hv[o + a] + (Fx ? (*Fx)[o + a] : 0.0);
                double rv = -(cx * avu + cy * avv) - p.g * H * cy * gey - f[o + a] * hu[o + a] + (Fy ? (*Fy)[o + a] : 0.0);
                const int sides[4] = {i == 0 ? 0 : -1, i == N ? 1 : -1, j == 0 ? 2 : -1, j == N ? 3 : -1};
                for (int s : sides) {
                    if (s < 0) continue;
                    const double nx = s == 0 ? -1.0 : (s == 1 ? 1.0 : 0.0);
                    const double ny = s == 2 ? -1.0 : (s == 3 ? 1.0 : 0.0);
                    const double L = s <= 1 ? Lx : Ly;
                    int nc = -1, ni = i, nj = j;
                    if (s == 0 && ex > 0) { nc = c - 1; ni = N; }
                    if (s == 1 && ex < p.nx - 1) { nc = c + 1; ni = 0; }
                    if (s == 2 && ey > 0) { nc = c - p.nx; nj = N; }
                    if (s == 3 && ey < p.ny - 1) { nc = c + p.nx; nj = 0; }
                    double UL[3] = {H, hu[o + a], hv[o + a]}, UR[3];
                    if (nc >= 0) {
                        const size_t q = (size_t)nc * np2 + ni + np * nj;
                        UR[0] = e[q] + h[q]; UR[1] = hu[q]; UR[2] = hv[q];
                    } else if (p.bc[s] == 1) {
                        UR[0] = etide + h[o + a];
                        const double r = UR[0] / H;
                        UR[1] = UL[1] * r; UR[2] = UL[2] * r;
                    } else {
                        UR[0] = H; UR[1] = UL[1]; UR[2] = UL[2];
                        if (s <= 1) UR[1] = -UL[1]; else UR[2] = -UL[2];
                    }
                    double Fs[3], Fm[3];
                    sw_flux(p.flux2d, UL, UR, nx, ny, p.g, Fs);
                    sw_physical_flux(UL, nx, ny, p.g, Fm);
                    re -= L * (Fs[0] - Fm[0]);
                    ru -= L * (Fs[1] - Fm[1]);
                    rv -= L * (Fs[2] - Fm[2]);
                }
                ke[o + a] = re; khu[o + a] = ru; khv[o + a] = rv;
            }
    }
}

void PhysModel::split_step(double dt, int nsub) {
    if (nsub < 1) throw std::invalid_argument("nsub must be >= 1");
    Vec R[4], res[4];
    for (int v = 0; v < 4; ++v) res[v].assign(n3, 0.0);
    Vec dHU(n2, 0.0), dHV(n2, 0.0), tmp;
    // the stage elevation of the baroclinic pressure: advanced with the 3D stages by the
    // column divergence, so that T = HT / H and S = HS / H see the depth the 3D transport implies
    Vec etas = eta, rese(n2, 0.0), de;
    for (int s = 0; s < 5; ++s) {
        rhs3d(Q, eta, t, R, nullptr, &de, &etas);
        for (int v = 0; v < 4; ++v)
            for (long n = 0; n < n3; ++n) {
                res[v][n] = LSRK_A[s] * res[v][n] + dt * R[v][n];
                Q[v][n] += LSRK_B[s] * res[v][n];
            }
        for (long a2 = 0; a2 < n2; ++a2) {
            rese[a2] = LSRK_A[s] * rese[a2] + dt * de[a2];
            etas[a2] += LSRK_B[s] * rese[a2];
        }
        Vec inc(n3);
        for (long n = 0; n < n3; ++n) inc[n] = LSRK_B[s] * res[0][n];
        column_integral(inc, tmp);
        for (long a = 0; a < n2; ++a) dHU[a] += tmp[a];
        for (long n = 0; n < n3; ++n) inc[n] = LSRK_B[s] * res[1][n];
        column_integral(inc, tmp);
        for (long a = 0; a < n2; ++a) dHV[a] += tmp[a];
    }
    // slow forcing = 3D-integrated tendency minus the 2D operator at the start state
    Vec pe, pu, pv, Fx(n2), Fy(n2);
    rhs2d(eta, HU, HV, nullptr, nullptr, t, pe, pu, pv);
    for (long a = 0; a < n2; ++a) { Fx[a] = dHU[a] / dt - pu[a]; Fy[a] = dHV[a] / dt - pv[a]; }
    const double dtb = dt / nsub;
    Vec e = eta, u = HU, v = HV, k1e, k1u, k1v, k2e, k2u, k2v, es(n2), us(n2), vs(n2), esum(n2, 0.0);
    for (int m = 0; m < nsub; ++m) {
        const double tm = t + m * dtb;
        rhs2d(e, u, v, &Fx, &Fy, tm, k1e, k1u, k1v);
        for (long a = 0; a < n2; ++a) { es[a] = e[a] + dtb * k1e[a]; us[a] = u[a] + dtb * k1u[a]; vs[a] = v[a] + dtb * k1v[a]; }
        rhs2d(es, us, vs, &Fx, &Fy, tm + dtb, k2e, k2u, k2v);
        for (long a = 0; a < n2; ++a) {
            e[a] += 0.5 * dtb * (k1e[a] + k2e[a]);
            u[a] += 0.5 * dtb * (k1u[a] + k2u[a]);
            v[a] += 0.5 * dtb * (k1v[a] + k2v[a]);
            esum[a] += e[a];
        }
    }
    // transport correction: make the 3D depth integral match the barotropic transport
    for (int c = 0; c < ncol; ++c)
        for (int a = 0; a < np2; ++a) {
            const size_t i2 = (size_t)c * np2 + a;
            const double cu = u[i2] - (HU[i2] + dHU[i2]), cv = v[i2] - (HV[i2] + dHV[i2]);
            for (int ez = 0; ez < p.nz; ++ez)
                for (int k = 0; k < np; ++k) {
                    const size_t n = ((size_t)c * p.nz + ez) * np3 + a + np2 * k;
                    Q[0][n] += cu;
                    Q[1][n] += cv;
                }
        }
    for (long a = 0; a < n2; ++a) eta_avg[a] = esum[a] / nsub;
    // volume consistency of the tracers: the 3D stages moved HT and HS with the column
    // divergence of the 3D transport (depth etas + h); the barotropic step ended at eta + h.
    // Rescaling the columns' tracer contents by that depth ratio keeps T = HT / H (a uniform
    // tracer stays uniform); the tracer content changes by the 3D/2D transport mismatch.
    for (int c = 0; c < ncol; ++c)
        for (int a2 = 0; a2 < np2; ++a2) {
            const size_t i2 = (size_t)c * np2 + a2;
            const double rr = (e[i2] + h[i2]) / (etas[i2] + h[i2]);
            for (int ez = 0; ez < p.nz; ++ez)
                for (int k = 0; k < np; ++k) {
                    const size_t n = ((size_t)c * p.nz + ez) * np3 + a2 + np2 * k;
                    Q[2][n] *= rr;
                    Q[3][n] *= rr;
                }
        }
    eta = e; HU = u; HV = v;
    t += dt;
}

void PhysModel::rk_step(int scheme, double dt) {
    // non-split RK over the packed [Hu, Hv, HT, HS, eta] vector (SimulationDriver::pack_state
    // src/solver/simulation_driver.cpp:199 order differs; packing is internal here).
    Vec U((size_t)4 * n3 + n2);
    for (int v = 0; v < 4; ++v) std::copy(Q[v].begin(), Q[v].end(), U.begin() + (size_t)v * n3);
    std::copy(eta.begin(), eta.end(), U.begin() + (size_t)4 * n3);
    auto rhs = [&](double tt, const Vec &X, Vec &dX) {
        Vec Qi[4], R[4], e(X.begin() + (size_t)4 * n3, X.end()), de;
        for (int v = 0; v < 4; ++v) Qi[v].assign(X.begin() + (size_t)v * n3, X.begin() + (size_t)(v + 1) * n3);
        rhs3d(Qi, e, tt, R, nullptr, &de);
        dX.resize(X.size());
        for (int v = 0; v < 4; ++v) std::copy(R[v].begin(), R[v].end(), dX.begin() + (size_t)v * n3);
        std::copy(de.begin(), de.end(), dX.begin() + (size_t)4 * n3);
    };
    orc::rk_step(scheme, t, dt, U, rhs);
    for (int v = 0; v < 4; ++v) std::copy(U.begin() + (size_t)v * n3, U.begin() + (size_t)(v + 1) * n3, Q[v].begin());
    std::copy(U.begin() + (size_t)4 * n3, U.end(), eta.begin());
    column_integral(Q[0], HU);
    column_integral(Q[1], HV);
    t += dt;
}

// SimulationDriver::compute_diagnostics src/solver/simulation_driver.cpp:237, plus
// quadrature-weighted integrals.
void PhysModel::diagnostics(double out[10]) const {
    const double *w = b.weights.data();
    double massw = 0, massu = 0, en = 0, heat = 0, salt = 0, umax = 0;
    double emax = -1e300, emin = 1e300, Tmax = -1e300, Tmin = 1e300;
    for (int c = 0; c < ncol; ++c)
        for (int j = 0; j < np; ++j)
            for (int i = 0; i < np; ++i) {
                const size_t i2 = (size_t)c * np2 + i + np * j;
                const double H = eta[i2] + h[i2], wa = 0.25 * dx * dy * w[i] * w[j];
                massw += wa * H;
                massu += (double)p.nz * np * H;
                en += wa * 0.5 * p.g * eta[i2] * eta[i2];
                emax = std::max(emax, eta[i2]); emin = std::min(emin, eta[i2]);
                for (int ez = 0; ez < p.nz; ++ez)
                    for (int k = 0; k < np; ++k) {
                        const size_t n = ((size_t)c * p.nz + ez) * np3 + i + np * (j + np * k);
                        const double wv = wa * 0.5 * dsig * w[k];
                        const double hu = Q[0][n], hv = Q[1][n];
                        en += wv * 0.5 * (hu * hu + hv * hv) / H;
                        heat += wv * Q[2][n];
                        salt += wv * Q[3][n];
                        const double sp = std::sqrt(hu * hu + hv * hv) / H;
                        umax = std::max(umax, sp);
                        const double T = Q[2][n] / H;
                        Tmax = std::max(Tmax, T); Tmin = std::min(Tmin, T);
                    }
            }
    out[0] = massw; out[1] = massu; out[2] = en; out[3] = heat; out[4] = salt;
    out[5] = umax; out[6] = emax; out[7] = emin; out[8] = Tmax; out[9] = Tmin;
}

}  // namespace orc
