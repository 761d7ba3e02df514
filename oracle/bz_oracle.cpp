// ORACLE — test infrastructure only. Cubic Bezier smoother restatement (see bz_oracle.hpp).
#include "bz_oracle.hpp"
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace orc {

void CSR::matvec(const double *x, double *y) const {
    for (long r = 0; r < n; ++r) {
        double s = 0.0;
        for (long p = rp[r]; p < rp[r + 1]; ++p) s += v[p] * x[ci[p]];
        y[r] = s;
    }
}
double CSR::frob2() const {
    double s = 0.0;
    for (double a : v) s += a * a;
    return s;
}

// Bernstein polynomials of degree 3 and their derivatives
// (CubicBezierBasis2D::evaluate_bernstein_1d / _derivative_1d, cubic_bezier_basis_2d.cpp:42-125)
void bernstein3(double t, int deriv, double o[4]) {
    const double s = 1.0 - t;
    if (deriv == 0) {
        o[0] = s * s * s; o[1] = 3 * t * s * s; o[2] = 3 * t * t * s; o[3] = t * t * t;
    } else if (deriv == 1) {  // 3 [B_{i-1,2} - B_{i,2}]
        const double b0 = s * s, b1 = 2 * t * s, b2 = t * t;
        o[0] = -3 * b0; o[1] = 3 * (b0 - b1); o[2] = 3 * (b1 - b2); o[3] = 3 * b2;
    } else if (deriv == 2) {  // 6 [B_{i-2,1} - 2 B_{i-1,1} + B_{i,1}]
        const double b0 = s, b1 = t;
        o[0] = 6 * b0; o[1] = 6 * (b1 - 2 * b0); o[2] = 6 * (b0 - 2 * b1); o[3] = 6 * b1;
    } else {
        o[0] = o[1] = o[2] = o[3] = 0.0;
    }
}

// CGBezierSmootherBase::gauss_legendre_01 (cg_bezier_smoother_base.cpp:28-58); n >= 4 -> 4 points
void gauss01(int n, BVec &p, BVec &w) {
    if (n == 1) { p = {0.5}; w = {1.0}; return; }
    if (n == 2) { p = {0.5 - 0.5 / std::sqrt(3.0), 0.5 + 0.5 / std::sqrt(3.0)}; w = {0.5, 0.5}; return; }
    if (n == 3) {
        p = {0.5 - 0.5 * std::sqrt(0.6), 0.5, 0.5 + 0.5 * std::sqrt(0.6)};
        w = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
        return;
    }
    const double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    const double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    const double wa = (18.0 + std::sqrt(30.0)) / 72.0, wb = (18.0 - std::sqrt(30.0)) / 72.0;
    p = {0.5 * (1.0 - b), 0.5 * (1.0 - a), 0.5 * (1.0 + a), 0.5 * (1.0 + b)};
    w = {0.5 * wb, 0.5 * wa, 0.5 * wa, 0.5 * wb};
}

// CubicThinPlateHessian::scaled_hessian (cubic_thin_plate_hessian.cpp:131) with the
// energy quadrature of compute_gauss_quadrature (:18); only ngauss = 4 is used here.
void element_hessian(double dx, double dy, int ngauss, double Hout[256]) {
    if (ngauss != 4) throw std::invalid_argument("element_hessian: ngauss 4 only");
    BVec p, w;
    gauss01(4, p, w);  // same nodes/weights as the 4-point table of the Hessian class
    double Huu[256] = {0}, Hvv[256] = {0}, Huv_[256] = {0}, Hx[256] = {0};
    for (int qj = 0; qj < 4; ++qj)
        for (int qi = 0; qi < 4; ++qi) {
            const double W = w[qi] * w[qj];
            double B0u[4], B1u[4], B2u[4], B0v[4], B1v[4], B2v[4];
            bernstein3(p[qi], 0, B0u); bernstein3(p[qi], 1, B1u); bernstein3(p[qi], 2, B2u);
            bernstein3(p[qj], 0, B0v); bernstein3(p[qj], 1, B1v); bernstein3(p[qj], 2, B2v);
            double d2u[16], d2v[16], duv[16];
            for (int j = 0; j < 4; ++j)
                for (int i = 0; i < 4; ++i) {
                    d2u[i + 4 * j] = B2u[i] * B0v[j];
                    d2v[i + 4 * j] = B0u[i] * B2v[j];
                    duv[i + 4 * j] = B1u[i] * B1v[j];
                }
            for (int k = 0; k < 16; ++k)
                for (int l = 0; l < 16; ++l) {
                    Huu[k * 16 + l] += W * d2u[k] * d2u[l];
                    Hvv[k * 16 + l] += W * d2v[k] * d2v[l];
                    Hx[k * 16 + l] += W * d2u[k] * d2v[l];
                    Huv_[k * 16 + l] += W * duv[k] * duv[l];
                }
        }
    const double s1 = dy / (dx * dx * dx), s2 = dx / (dy * dy * dy), s3 = 1.0 / (dx * dy),
                 s4 = 2.0 / (dx * dy);
    double T[256];
    for (int k = 0; k < 16; ++k)
        for (int l = 0; l < 16; ++l)
            T[k * 16 + l] = s1 * Huu[k * 16 + l] + s2 * Hvv[k * 16 + l] +
                            s3 * (Hx[k * 16 + l] + Hx[l * 16 + k]) + s4 * Huv_[k * 16 + l];
    for (int k = 0; k < 16; ++k)
        for (int l = 0; l < 16; ++l) Hout[k * 16 + l] = 0.5 * (T[k * 16 + l] + T[l * 16 + k]);
}

// B_local of assemble_data_fitting_global (cg_bezier_smoother_base.cpp:308-366), relaxation off
void element_mass(double dx, double dy, int ngauss, double B[256]) {
    BVec p, w;
    gauss01(ngauss, p, w);
    std::memset(B, 0, sizeof(double) * 256);
    for (size_t qi = 0; qi < p.size(); ++qi)
        for (size_t qj = 0; qj < p.size(); ++qj) {
            const double W = w[qi] * w[qj] * dx * dy;
            double Bu[4], Bv[4], phi[16];
            bernstein3(p[qi], 0, Bu);
            bernstein3(p[qj], 0, Bv);
            for (int j = 0; j < 4; ++j)
                for (int i = 0; i < 4; ++i) phi[i + 4 * j] = Bu[i] * Bv[j];
            for (int i = 0; i < 16; ++i)
                for (int j = 0; j < 16; ++j) B[i * 16 + j] += W * phi[i] * phi[j];
        }
}

// CubicBezierBasis2D::compute_1d_extraction_matrix for [0, 1/2] and [1/2, 1] (:397)
void subdivision_1d(double S[2][16]) {
    auto binom = [](int n, int k) {
        double r = 1;
        for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
        return r;
    };
    std::memset(S, 0, sizeof(double) * 32);
    for (int k = 0; k <= 3; ++k) {
        for (int j = 0; j <= k; ++j) S[0][k * 4 + j] = binom(k, j) / std::pow(2.0, k);
        for (int j = k; j <= 3; ++j) S[1][k * 4 + j] = binom(3 - k, j - k) / std::pow(2.0, 3 - k);
    }
}

static void assemble(const BzSystem &S, const double *Ke, CSR &M) {
    // CSR with the 7x7 stencil pattern of the control-point grid
    const long nd = S.ndof;
    M.n = M.m = nd;
    M.rp.assign(nd + 1, 0);
    std::vector<std::vector<std::pair<long, double>>> rows(nd);
    for (int ey = 0; ey < S.g.ny; ++ey)
        for (int ex = 0; ex < S.g.nx; ++ex)
            for (int a = 0; a < 16; ++a) {
                const long I = S.dof(ex, ey, a);
                for (int b = 0; b < 16; ++b) {
                    const double val = Ke[a * 16 + b];
                    if (std::abs(val) > 1e-16) rows[I].push_back({S.dof(ex, ey, b), val});
                }
            }
    for (long r = 0; r < nd; ++r) {
        auto &R = rows[r];
        std::sort(R.begin(), R.end(), [](auto &x, auto &y) { return x.first < y.first; });
        std::vector<std::pair<long, double>> merged;
        for (auto &e : R) {
            if (!merged.empty() && merged.back().first == e.first) merged.back().second += e.second;
            else merged.push_back(e);
        }
        R.swap(merged);
        M.rp[r + 1] = M.rp[r] + (long)R.size();
    }
    M.ci.resize(M.rp[nd]);
    M.v.resize(M.rp[nd]);
    for (long r = 0; r < nd; ++r) {
        long p = M.rp[r];
        for (auto &e : rows[r]) { M.ci[p] = e.first; M.v[p] = e.second; ++p; }
    }
}

void bz_build(BzSystem &S, const BzGrid &g, const double *dgauss) {
    S.g = g;
    S.nxd = 3 * g.nx + 1;
    S.nyd = 3 * g.ny + 1;
    S.ndof = (long)S.nxd * S.nyd;
    S.dx = g.Lx / g.nx;
    S.dy = g.Ly / g.ny;
    element_hessian(S.dx, S.dy, g.ngauss_energy, S.He);
    element_mass(S.dx, S.dy, g.ngauss_data, S.Be);
    assemble(S, S.He, S.H);
    assemble(S, S.Be, S.BtWB);
    // BtWd and dTWd from data at the Gauss points
    BVec p, w;
    gauss01(g.ngauss_data, p, w);
    const int ng = (int)p.size();
    S.BtWd.assign(S.ndof, 0.0);
    S.dTWd = 0.0;
    for (int ey = 0; ey < g.ny; ++ey)
        for (int ex = 0; ex < g.nx; ++ex) {
            const double *de = dgauss + ((size_t)ey * g.nx + ex) * ng * ng;
            for (int qi = 0; qi < ng; ++qi)
                for (int qj = 0; qj < ng; ++qj) {
                    const double W = w[qi] * w[qj] * S.dx * S.dy;
                    const double d = de[qj * ng + qi];
                    S.dTWd += W * d * d;
                    double Bu[4], Bv[4];
                    bernstein3(p[qi], 0, Bu);
                    bernstein3(p[qj], 0, Bv);
                    for (int k = 0; k < 16; ++k)
                        S.BtWd[S.dof(ex, ey, k)] += W * Bu[k % 4] * Bv[k / 4] * d;
                }
        }
    // alpha = ||B^T W B||_F / ||H||_F (cg_bezier_smoother_base.cpp:387-389)
    const double nh = std::sqrt(S.H.frob2()), nb = std::sqrt(S.BtWB.frob2());
    S.alpha = nh > 1e-14 ? nb / nh : 0.0;
    // Q = alpha H + lambda B^T W B + lambda eps I (assemble_Q :396); same pattern
    S.Q = S.H;
    for (long r = 0; r < S.ndof; ++r)
        for (long q = S.Q.rp[r]; q < S.Q.rp[r + 1]; ++q) {
            double v = S.alpha * S.H.v[q];
            // BtWB has the same pattern except entries dropped below 1e-16
            for (long t = S.BtWB.rp[r]; t < S.BtWB.rp[r + 1]; ++t)
                if (S.BtWB.ci[t] == S.Q.ci[q]) { v += g.lambda * S.BtWB.v[t]; break; }
            if (S.Q.ci[q] == r) v += g.lambda * g.eps;
            S.Q.v[q] = v;
        }
    S.b.resize(S.ndof);
    for (long i = 0; i < S.ndof; ++i) S.b[i] = g.lambda * S.BtWd[i];
}

// C1 continuity of the normal derivative at edge_ngauss Gauss points of every interior edge
// (CGCubicBezierDofManager::build_edge_derivative_constraints + assemble_A_edge_free)
void bz_constraints(const BzSystem &S, int edge_ngauss, CSR &A) {
    BVec p, w;
    gauss01(edge_ngauss, p, w);
    std::vector<std::vector<std::pair<long, double>>> rows;
    auto add_row = [&](int e1x, int e1y, double u1, double v1, int e2x, int e2y, double u2,
                       double v2, int nu, int nv, double scale) {
        std::vector<std::pair<long, double>> r;
        double Bu[4], Bv[4];
        bernstein3(u1, nu, Bu); bernstein3(v1, nv, Bv);
        for (int k = 0; k < 16; ++k) {
            const double c = Bu[k % 4] * Bv[k / 4] / scale;
            if (std::abs(c) > 1e-14) r.push_back({S.dof(e1x, e1y, k), c});
        }
        bernstein3(u2, nu, Bu); bernstein3(v2, nv, Bv);
        for (int k = 0; k < 16; ++k) {
            const double c = Bu[k % 4] * Bv[k / 4] / scale;
            if (std::abs(c) > 1e-14) r.push_back({S.dof(e2x, e2y, k), -c});
        }
        rows.push_back(r);
    };
    for (int ey = 0; ey < S.g.ny; ++ey)
        for (int ex = 0; ex < S.g.nx; ++ex) {
            if (ex + 1 < S.g.nx)  // right edge of (ex,ey) = left edge of (ex+1,ey): z_u
                for (double t : p) add_row(ex, ey, 1.0, t, ex + 1, ey, 0.0, t, 1, 0, S.dx);
            if (ey + 1 < S.g.ny)  // top edge = bottom edge of (ex,ey+1): z_v
                for (double t : p) add_row(ex, ey, t, 1.0, ex, ey + 1, t, 0.0, 0, 1, S.dy);
        }
    A.n = (long)rows.size();
    A.m = S.ndof;
    A.rp.assign(A.n + 1, 0);
    for (long r = 0; r < A.n; ++r) A.rp[r + 1] = A.rp[r] + (long)rows[r].size();
    A.ci.resize(A.rp[A.n]);
    A.v.resize(A.rp[A.n]);
    for (long r = 0; r < A.n; ++r) {
        long q = A.rp[r];
        for (auto &e : rows[r]) { A.ci[q] = e.first; A.v[q] = e.second; ++q; }
    }
}

// objective_value = alpha * x^T H x + lambda * (x^T BtWB x - 2 x^T BtWd + dTWd)
double bz_objective(const BzSystem &S, const double *x, double parts[2]) {
    BVec y(S.ndof);
    S.H.matvec(x, y.data());
    double reg = 0.0;
    for (long i = 0; i < S.ndof; ++i) reg += x[i] * y[i];
    S.BtWB.matvec(x, y.data());
    double dat = S.dTWd;
    for (long i = 0; i < S.ndof; ++i) dat += x[i] * y[i] - 2.0 * x[i] * S.BtWd[i];
    if (parts) { parts[0] = reg; parts[1] = dat; }
    return S.alpha * reg + S.g.lambda * dat;
}

// ----------------------------------------------------------------------------- multigrid
static void invert(const double *A, int n, double *Ainv) {
    std::vector<double> M(A, A + n * n), I(n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(M[r * n + c]) > std::abs(M[piv * n + c])) piv = r;
        if (std::abs(M[piv * n + c]) < 1e-300) throw std::runtime_error("singular block");
        if (piv != c)
            for (int k = 0; k < n; ++k) { std::swap(M[c * n + k], M[piv * n + k]); std::swap(I[c * n + k], I[piv * n + k]); }
        const double d = 1.0 / M[c * n + c];
        for (int k = 0; k < n; ++k) { M[c * n + k] *= d; I[c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = M[r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) { M[r * n + k] -= f * M[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
        }
    }
    std::memcpy(Ainv, I.data(), sizeof(double) * n * n);
}

// 1D prolongation row of fine index f: 4 weights on coarse 3E..3E+3
static int p1_row(int f, int nc, const double S[2][16], double w[4]) {
    int E = f / 6;
    if (E > nc - 1) E = nc - 1;
    const int k = f - 6 * E;
    const double *row = k <= 3 ? &S[0][k * 4] : &S[1][(k - 3) * 4];
    for (int c = 0; c < 4; ++c) w[c] = row[c];
    return 3 * E;
}

static double level_ridge(const BzMG &M, int l, int ix, int iy) {
    return M.lam_eps * M.lv[l].rho[ix] * M.lv[l].rho[iy];
}

// (Q_l x) at control point (gi, gj)
static double row_apply(const BzMG &M, int l, const double *x, int gi, int gj) {
    const BzLevel &L = M.lv[l];
    double s = level_ridge(M, l, gi, gj) * x[gi + (long)L.nd * gj];
    for (int ex = (gi - 1) / 3 - 1; ex <= gi / 3; ++ex) {
        if (ex < 0 || ex >= L.n) continue;
        const int li = gi - 3 * ex;
        if (li < 0 || li > 3) continue;
        for (int ey = (gj - 1) / 3 - 1; ey <= gj / 3; ++ey) {
            if (ey < 0 || ey >= L.n) continue;
            const int lj = gj - 3 * ey;
            if (lj < 0 || lj > 3) continue;
            const int a = li + 4 * lj;
            for (int b = 0; b < 16; ++b)
                s += L.K[a * 16 + b] * x[(3 * ex + b % 4) + (long)L.nd * (3 * ey + b / 4)];
        }
    }
    return s;
}

void bz_level_apply(const BzMG &M, int l, const double *x, double *y) {
    const int nd = M.lv[l].nd;
    for (int gj = 0; gj < nd; ++gj)
        for (int gi = 0; gi < nd; ++gi) y[gi + (long)nd * gj] = row_apply(M, l, x, gi, gj);
}

static void element_block(const BzMG &M, int l, int ex, int ey, double *blk) {
    const BzLevel &L = M.lv[l];
    for (int a = 0; a < 16; ++a)
        for (int b = 0; b < 16; ++b) {
            const int gia = 3 * ex + a % 4, gja = 3 * ey + a / 4;
            const int gib = 3 * ex + b % 4, gjb = 3 * ey + b / 4;
            double s = (a == b) ? level_ridge(M, l, gia, gja) : 0.0;
            for (int e2x = ex - 1; e2x <= ex + 1; ++e2x)
                for (int e2y = ey - 1; e2y <= ey + 1; ++e2y) {
                    if (e2x < 0 || e2y < 0 || e2x >= L.n || e2y >= L.n) continue;
                    const int la = gia - 3 * e2x, ma = gja - 3 * e2y, lb = gib - 3 * e2x, mb = gjb - 3 * e2y;
                    if (la < 0 || la > 3 || ma < 0 || ma > 3 || lb < 0 || lb > 3 || mb < 0 || mb > 3) continue;
                    s += L.K[(la + 4 * ma) * 16 + (lb + 4 * mb)];
                }
            blk[a * 16 + b] = s;
        }
}

void bz_mg_setup(const BzSystem &S, BzMG &M, int coarsest_n) {
    if (S.g.nx != S.g.ny) throw std::invalid_argument("multigrid needs a square grid");
    int nlev = 1, n = S.g.nx;
    while (n > coarsest_n && n % 2 == 0) { n /= 2; ++nlev; }
    M.lv.assign(nlev, BzLevel());
    M.lam_eps = S.g.lambda * S.g.eps;
    double Sd[2][16];
    subdivision_1d(Sd);
    // finest
    BzLevel &F = M.lv[nlev - 1];
    F.n = S.g.nx;
    F.nd = 3 * F.n + 1;
    for (int i = 0; i < 256; ++i) F.K[i] = S.alpha * S.He[i] + S.g.lambda * S.Be[i];
    F.rho.assign(F.nd, 1.0);
    for (int l = nlev - 2; l >= 0; --l) {
        BzLevel &C = M.lv[l], &Fi = M.lv[l + 1];
        C.n = Fi.n / 2;
        C.nd = 3 * C.n + 1;
        // K_c = sum_children S_c^T K_f S_c
        std::memset(C.K, 0, sizeof(C.K));
        for (int cv = 0; cv < 2; ++cv)
            for (int cu = 0; cu < 2; ++cu) {
                double Sc[256];
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b)
                        Sc[a * 16 + b] = Sd[cu][(a % 4) * 4 + (b % 4)] * Sd[cv][(a / 4) * 4 + (b / 4)];
                double T[256] = {0};
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b) {
                        double s = 0;
                        for (int k = 0; k < 16; ++k) s += Fi.K[a * 16 + k] * Sc[k * 16 + b];
                        T[a * 16 + b] = s;
                    }
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b) {
                        double s = 0;
                        for (int k = 0; k < 16; ++k) s += Sc[k * 16 + a] * T[k * 16 + b];
                        C.K[a * 16 + b] += s;
                    }
            }
        // separable Galerkin ridge diagonal: rho_c(I) = sum_f P1[f][I]^2 rho_f(f)
        C.rho.assign(C.nd, 0.0);
        for (int f = 0; f < Fi.nd; ++f) {
            double w[4];
            const int c0 = p1_row(f, C.n, Sd, w);
            for (int c = 0; c < 4; ++c) C.rho[c0 + c] += w[c] * w[c] * Fi.rho[f];
        }
    }
    // element-block inverses per class for levels >= 1
    for (int l = 1; l < nlev; ++l) {
        BzLevel &L = M.lv[l];
        L.binv.assign(9 * 256, 0.0);
        for (int cy = 0; cy < 3; ++cy)
            for (int cx = 0; cx < 3; ++cx) {
                const int ex = cx == 0 ? 0 : (cx == 1 ? 1 : L.n - 1);
                const int ey = cy == 0 ? 0 : (cy == 1 ? 1 : L.n - 1);
                if ((cx == 1 && L.n < 3) || (cy == 1 && L.n < 3)) continue;
                double blk[256];
                element_block(M, l, ex, ey, blk);
                invert(blk, 16, &L.binv[(cx + 3 * cy) * 256]);
            }
    }
    // dense coarsest operator
    BzLevel &C = M.lv[0];
    const int nc = C.nd * C.nd;
    std::vector<double> A((size_t)nc * nc), e(nc, 0.0), y(nc);
    for (int j = 0; j < nc; ++j) {
        e[j] = 1.0;
        bz_level_apply(M, 0, e.data(), y.data());
        for (int i = 0; i < nc; ++i) A[(size_t)i * nc + j] = y[i];
        e[j] = 0.0;
    }
    M.coarse_inv.resize((size_t)nc * nc);
    invert(A.data(), nc, M.coarse_inv.data());
}

static int elem_class(int e, int n) { return e == 0 ? 0 : (e == n - 1 ? 2 : 1); }

// ColoredSchwarzMethod::apply (src/bathymetry/schwarz_method.cpp:125): per color, the
// residual of every element of the color is taken from the same x, then all block
// corrections of that color are applied.
static void smooth_color(const BzMG &M, int l, int color, double *x, const double *b) {
    const BzLevel &L = M.lv[l];
    const int px = color & 1, py = color >> 1;
    std::vector<double> rs;
    for (int ey = py; ey < L.n; ey += 2)
        for (int ex = px; ex < L.n; ex += 2)
            for (int a = 0; a < 16; ++a) {
                const int gi = 3 * ex + a % 4, gj = 3 * ey + a / 4;
                rs.push_back(b[gi + (long)L.nd * gj] - row_apply(M, l, x, gi, gj));
            }
    size_t q = 0;
    for (int ey = py; ey < L.n; ey += 2)
        for (int ex = px; ex < L.n; ex += 2) {
            const double *r = &rs[q];
            q += 16;
            const double *Bi = &L.binv[(elem_class(ex, L.n) + 3 * elem_class(ey, L.n)) * 256];
            for (int a = 0; a < 16; ++a) {
                double s2 = 0.0;
                for (int k = 0; k < 16; ++k) s2 += Bi[a * 16 + k] * r[k];
                x[(3 * ex + a % 4) + (long)L.nd * (3 * ey + a / 4)] += s2;
            }
        }
}

// ref = false: this build's SPD V-cycle (R = P^T, post-smoothing in reverse colour order).
// ref = true: BezierMultigridPreconditioner::v_cycle as written
// (src/bathymetry/bezier_multigrid_preconditioner.cpp:740-812): R = P^T with its rows scaled to
// sum to one where they do not already (:209-225, |sum - 1| > 1e-10), and the same smoother
// (colours 0..3) before and after the coarse correction.
static void vcycle(const BzMG &M, int l, double *x, const double *b, bool ref = false) {
    const BzLevel &L = M.lv[l];
    const long nd2 = (long)L.nd * L.nd;
    if (l == 0) {
        for (long i = 0; i < nd2; ++i) {
            double s = 0.0;
            for (long k = 0; k < nd2; ++k) s += M.coarse_inv[i * nd2 + k] * b[k];
            x[i] = s;
        }
        return;
    }
    for (int it = 0; it < M.pre; ++it)
        for (int c = 0; c < 4; ++c) smooth_color(M, l, c, x, b);
    std::vector<double> r(nd2), tmp;
    bz_level_apply(M, l, x, r.data());
    for (long i = 0; i < nd2; ++i) r[i] = b[i] - r[i];
    const BzLevel &C = M.lv[l - 1];
    double Sd[2][16];
    subdivision_1d(Sd);
    // restriction P^T r (separable): first along x then along y
    tmp.assign((size_t)C.nd * L.nd, 0.0);
    for (int fj = 0; fj < L.nd; ++fj)
        for (int fi = 0; fi < L.nd; ++fi) {
            double w[4];
            const int c0 = p1_row(fi, C.n, Sd, w);
            for (int c = 0; c < 4; ++c) tmp[(c0 + c) + (long)C.nd * fj] += w[c] * r[fi + (long)L.nd * fj];
        }
    std::vector<double> rc((size_t)C.nd * C.nd, 0.0), ec((size_t)C.nd * C.nd, 0.0);
    for (int fj = 0; fj < L.nd; ++fj) {
        double w[4];
        const int c0 = p1_row(fj, C.n, Sd, w);
        for (int ci = 0; ci < C.nd; ++ci)
            for (int c = 0; c < 4; ++c) rc[ci + (long)C.nd * (c0 + c)] += w[c] * tmp[ci + (long)C.nd * fj];
    }
    if (ref) {
        // row sums of R = P^T: separable, (restriction of ones along x) x (along y)
        std::vector<double> sx(C.nd, 0.0);
        for (int fi = 0; fi < L.nd; ++fi) {
            double w[4];
            const int c0 = p1_row(fi, C.n, Sd, w);
            for (int c = 0; c < 4; ++c) sx[c0 + c] += w[c];
        }
        for (int cj = 0; cj < C.nd; ++cj)
            for (int ci = 0; ci < C.nd; ++ci) {
                const double scale = sx[ci] * sx[cj];
                if (std::abs(scale) > 1e-14 && std::abs(scale - 1.0) > 1e-10)
                    rc[ci + (long)C.nd * cj] /= scale;
            }
    }
    vcycle(M, l - 1, ec.data(), rc.data(), ref);
    // prolongation x += P e_c
    for (int fj = 0; fj < L.nd; ++fj) {
        double wy[4];
        const int cy0 = p1_row(fj, C.n, Sd, wy);
        for (int fi = 0; fi < L.nd; ++fi) {
            double wx[4];
            const int cx0 = p1_row(fi, C.n, Sd, wx);
            double s = 0.0;
            for (int b2 = 0; b2 < 4; ++b2)
                for (int a2 = 0; a2 < 4; ++a2) s += wy[b2] * wx[a2] * ec[(cx0 + a2) + (long)C.nd * (cy0 + b2)];
            x[fi + (long)L.nd * fj] += s;
        }
    }
    for (int it = 0; it < M.post; ++it)
        for (int s2 = 0; s2 < 4; ++s2) smooth_color(M, l, ref ? s2 : 3 - s2, x, b);
}

// BezierMultigridPreconditioner::apply (src/bathymetry/bezier_multigrid_preconditioner.cpp:
// 690-735): x = 0, then V-cycles (reference semantics) until ||b - Q x|| < tol ||b|| or
// max_cycles; returns the cycles run.
int bz_mg_apply_ref(const BzMG &M, const double *b, double *x, double tol, int max_cycles) {
    const int l = (int)M.lv.size() - 1;
    const long nd2 = (long)M.lv[l].nd * M.lv[l].nd;
    std::fill(x, x + nd2, 0.0);
    double bb = 0.0;
    for (long i = 0; i < nd2; ++i) bb += b[i] * b[i];
    if (std::sqrt(bb) < 1e-30) return 0;
    const double tol_sq = tol * tol * bb;
    std::vector<double> qx(nd2);
    int cycle = 0;
    for (; cycle < max_cycles; ++cycle) {
        vcycle(M, l, x, b, true);
        bz_level_apply(M, l, x, qx.data());
        double rr = 0.0;
        for (long i = 0; i < nd2; ++i) rr += (b[i] - qx[i]) * (b[i] - qx[i]);
        if (rr < tol_sq) {
            ++cycle;
            break;
        }
    }
    return cycle;
}

void bz_mg_vcycle(const BzMG &M, const double *r, double *z) {
    const int l = (int)M.lv.size() - 1;
    const long nd2 = (long)M.lv[l].nd * M.lv[l].nd;
    std::fill(z, z + nd2, 0.0);
    vcycle(M, l, z, r);
}

int bz_pcg(const BzSystem &S, const BzMG *M, int precond, const double *b, double *x, double tol,
           int maxit, double *relres) {
    const long n = S.ndof;
    BVec r(n), z(n), p(n), q(n);
    S.Q.matvec(x, q.data());
    double bn = 0;
    for (long i = 0; i < n; ++i) { r[i] = b[i] - q[i]; bn += b[i] * b[i]; }
    bn = std::sqrt(bn);
    auto prec = [&](const BVec &in, BVec &out) {
        if (precond == 2) bz_mg_vcycle(*M, in.data(), out.data());
        else if (precond == 1) {
            for (long i = 0; i < n; ++i) {
                double d = 1.0;
                for (long k = S.Q.rp[i]; k < S.Q.rp[i + 1]; ++k)
                    if (S.Q.ci[k] == i) d = S.Q.v[k];
                out[i] = in[i] / d;
            }
        } else out = in;
    };
    prec(r, z);
    p = z;
    double rz = 0;
    for (long i = 0; i < n; ++i) rz += r[i] * z[i];
    int it = 0;
    double rn = 0;
    for (long i = 0; i < n; ++i) rn += r[i] * r[i];
    rn = std::sqrt(rn);
    if (bn == 0.0) { if (relres) *relres = 0.0; return 0; }
    while (it < maxit && rn / bn > tol) {
        S.Q.matvec(p.data(), q.data());
        double pq = 0;
        for (long i = 0; i < n; ++i) pq += p[i] * q[i];
        const double a = rz / pq;
        rn = 0;
        for (long i = 0; i < n; ++i) { x[i] += a * p[i]; r[i] -= a * q[i]; rn += r[i] * r[i]; }
        rn = std::sqrt(rn);
        ++it;
        if (rn / bn <= tol) break;
        prec(r, z);
        double rz2 = 0;
        for (long i = 0; i < n; ++i) rz2 += r[i] * z[i];
        const double beta = rz2 / rz;
        rz = rz2;
        for (long i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    if (relres) *relres = rn / bn;
    return it;
}

}  // namespace orc

// AdaptiveCGCubicBezierSmoother::compute_element_l2_error
// (src/bathymetry/adaptive_cg_cubic_bezier_smoother.cpp:100-138) and the normalized error of
// estimate_element_error (:142-150) for every element of a uniform nx x ny grid: the Gauss
// point (u, v) on [0, 1]^2 is mapped to x = xmin + u dx and evaluated through
// CGBezierSmootherBase::evaluate_in_element (src/bathymetry/cg_bezier_smoother_base.cpp:166:
// u = (x - xmin) / dx, clamped), with the cubic Bernstein basis and the element's control
// points (dof i + 4j). zdata: [ey][ex][qj][qi]. Returns 0, -1 on bad arguments.
extern "C" int orc_bz_element_errors(int nx, int ny, double x0, double y0, double Lx, double Ly, int ng,
                                     const double *x, const double *zdata, double *l2, double *nrm) {
    if (nx < 1 || ny < 1 || ng < 1) return -1;
    orc::Vec gx, gw;
    orc::gauss_legendre(ng, gx, gw);
    std::vector<double> gn(ng), gwt(ng);
    for (int i = 0; i < ng; ++i) {
        gn[i] = 0.5 * (gx[i] + 1.0);
        gwt[i] = 0.5 * gw[i];
    }
    const double dx = Lx / nx, dy = Ly / ny;
    const long stride = 3L * nx + 1;
    auto bern = [](double t, double b[4]) {
        const double s = 1.0 - t;
        b[0] = s * s * s; b[1] = 3.0 * t * s * s; b[2] = 3.0 * t * t * s; b[3] = t * t * t;
    };
    for (int ey = 0; ey < ny; ++ey)
        for (int ex = 0; ex < nx; ++ex) {
            const double xmin = x0 + ex * dx, ymin = y0 + ey * dy;
            double c[16];
            for (int j = 0; j < 4; ++j)
                for (int i = 0; i < 4; ++i) c[i + 4 * j] = x[(3L * ex + i) + stride * (3L * ey + j)];
            double err2 = 0.0;
            for (int j = 0; j < ng; ++j)
                for (int i = 0; i < ng; ++i) {
                    const double px = xmin + gn[i] * dx, py = ymin + gn[j] * dy;
                    double u = (px - xmin) / dx, v = (py - ymin) / dy;
                    u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
                    v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
                    double bu[4], bv[4];
                    bern(u, bu);
                    bern(v, bv);
                    double z = 0.0;
                    for (int b = 0; b < 4; ++b)
                        for (int a = 0; a < 4; ++a) z += c[a + 4 * b] * bu[a] * bv[b];
                    const long e = (long)ey * nx + ex;
                    const double diff = zdata[(e * ng + j) * ng + i] - z;
                    err2 += gwt[i] * gwt[j] * diff * diff;
                }
            const long e = (long)ey * nx + ex;
            l2[e] = std::sqrt(err2 * dx * dy);
            if (nrm) nrm[e] = l2[e] / std::sqrt(dx * dy);
        }
    return 0;
}
