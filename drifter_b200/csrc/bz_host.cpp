// Host-side setup of the GPU Bezier smoother (see bz_host.hpp).
//
// Element operators follow the reference's cubic Bezier smoother: thin-plate Hessian
// E = int (z_xx + z_yy)^2 + 2 z_xy^2 with the dx/dy scalings of
// CubicThinPlateHessian::scaled_hessian (src/bathymetry/cubic_thin_plate_hessian.cpp:131),
// data-fitting mass sum_q w_q B B^T on 4x4 Gauss points
// (src/bathymetry/cg_bezier_smoother_base.cpp:308), alpha = ||B^T W B||_F / ||H||_F (:387).
#include "bz_host.hpp"

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "common.cuh"

namespace drf {

static void bern(double t, int d, double o[4]) {
    const double s = 1.0 - t;
    if (d == 0) { o[0] = s * s * s; o[1] = 3 * t * s * s; o[2] = 3 * t * t * s; o[3] = t * t * t; }
    else if (d == 1) { o[0] = -3 * s * s; o[1] = 3 * s * s - 6 * t * s; o[2] = 6 * t * s - 3 * t * t; o[3] = 3 * t * t; }
    else { o[0] = 6 * s; o[1] = 6 * t - 12 * s; o[2] = 6 * s - 12 * t; o[3] = 6 * t; }
}

// 4-point Gauss-Legendre on [0, 1]
static void gl4(double p[4], double w[4]) {
    const double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    const double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
    const double wa = (18.0 + std::sqrt(30.0)) / 72.0, wb = (18.0 - std::sqrt(30.0)) / 72.0;
    p[0] = 0.5 * (1 - b); p[1] = 0.5 * (1 - a); p[2] = 0.5 * (1 + a); p[3] = 0.5 * (1 + b);
    w[0] = 0.5 * wb; w[1] = 0.5 * wa; w[2] = 0.5 * wa; w[3] = 0.5 * wb;
}

void bz_subdivision_1d(double S[2][16]) {
    // de Casteljau halves: left Q_k = sum_{j<=k} C(k,j) 2^-k P_j, right mirrored
    static const double L[16] = {1, 0, 0, 0, .5, .5, 0, 0, .25, .5, .25, 0, .125, .375, .375, .125};
    for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 4; ++j) {
            S[0][k * 4 + j] = L[k * 4 + j];
            S[1][k * 4 + j] = L[(3 - k) * 4 + (3 - j)];
        }
}

static void element_ops(double dx, double dy, double H[256], double B[256], double *Bq) {
    double p[4], w[4];
    gl4(p, w);
    double Huu[256] = {0}, Hvv[256] = {0}, Hx[256] = {0}, Hm[256] = {0};
    std::memset(B, 0, 256 * sizeof(double));
    for (int qj = 0; qj < 4; ++qj)
        for (int qi = 0; qi < 4; ++qi) {
            const double W = w[qi] * w[qj];
            double b0u[4], b1u[4], b2u[4], b0v[4], b1v[4], b2v[4];
            bern(p[qi], 0, b0u); bern(p[qi], 1, b1u); bern(p[qi], 2, b2u);
            bern(p[qj], 0, b0v); bern(p[qj], 1, b1v); bern(p[qj], 2, b2v);
            double uu[16], vv[16], uv[16], ph[16];
            for (int k = 0; k < 16; ++k) {
                const int i = k % 4, j = k / 4;
                uu[k] = b2u[i] * b0v[j]; vv[k] = b0u[i] * b2v[j]; uv[k] = b1u[i] * b1v[j];
                ph[k] = b0u[i] * b0v[j];
            }
            for (int k = 0; k < 16; ++k)
                for (int l = 0; l < 16; ++l) {
                    Huu[k * 16 + l] += W * uu[k] * uu[l];
                    Hvv[k * 16 + l] += W * vv[k] * vv[l];
                    Hx[k * 16 + l] += W * uu[k] * vv[l];
                    Hm[k * 16 + l] += W * uv[k] * uv[l];
                    B[k * 16 + l] += W * dx * dy * ph[k] * ph[l];
                }
            for (int k = 0; k < 16; ++k) Bq[k * 16 + (qi + 4 * qj)] = W * dx * dy * ph[k];
        }
    const double s1 = dy / (dx * dx * dx), s2 = dx / (dy * dy * dy), s3 = 1.0 / (dx * dy), s4 = 2.0 / (dx * dy);
    for (int k = 0; k < 16; ++k)
        for (int l = 0; l < 16; ++l) {
            const double a = s1 * Huu[k * 16 + l] + s2 * Hvv[k * 16 + l] + s3 * (Hx[k * 16 + l] + Hx[l * 16 + k]) + s4 * Hm[k * 16 + l];
            const double b = s1 * Huu[l * 16 + k] + s2 * Hvv[l * 16 + k] + s3 * (Hx[l * 16 + k] + Hx[k * 16 + l]) + s4 * Hm[l * 16 + k];
            H[k * 16 + l] = 0.5 * (a + b);
        }
}

// squared Frobenius norms of the assembled global matrices, row by row over the stencil
static void global_frob2(int n, const double *A, const double *B, double &fa, double &fb) {
    const int nd = 3 * n + 1;
    fa = fb = 0.0;
    for (int gj = 0; gj < nd; ++gj)
        for (int gi = 0; gi < nd; ++gi) {
            double ra[49] = {0}, rb[49] = {0};
            const int ex1 = std::min(gi / 3, n - 1), ey1 = std::min(gj / 3, n - 1);
            const int ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
            const int ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
            for (int ey = ey0; ey <= ey1; ++ey)
                for (int ex = ex0; ex <= ex1; ++ex) {
                    const int a = (gi - 3 * ex) + 4 * (gj - 3 * ey);
                    for (int b = 0; b < 16; ++b) {
                        const int oi = 3 * ex + b % 4 - gi + 3, oj = 3 * ey + b / 4 - gj + 3;
                        const double va = A[a * 16 + b], vb = B[a * 16 + b];
                        if (std::abs(va) > 1e-16) ra[oi + 7 * oj] += va;
                        if (std::abs(vb) > 1e-16) rb[oi + 7 * oj] += vb;
                    }
                }
            for (int k = 0; k < 49; ++k) { fa += ra[k] * ra[k]; fb += rb[k] * rb[k]; }
        }
}

void bz_fine_operator(const drf_bz_grid_desc &g, double K[256], double *alpha) {
    double He[256], Be[256], Bq[256];
    element_ops(g.Lx / g.nx, g.Ly / g.ny, He, Be, Bq);
    double fh, fb;
    global_frob2(g.nx, He, Be, fh, fb);
    const double a = fh > 0 ? std::sqrt(fb) / std::sqrt(fh) : 0.0;
    for (int i = 0; i < 256; ++i) K[i] = a * He[i] + g.lambda * Be[i];
    *alpha = a;
}

void bz_setup_fine(BzSetup &s, const drf_bz_grid_desc &g) {
    s.g = g;
    s.dx = g.Lx / g.nx;
    s.dy = g.Ly / g.ny;
    s.Bq.assign(256, 0.0);
    element_ops(s.dx, s.dy, s.He, s.Be, s.Bq.data());
    double fh, fb;
    global_frob2(g.nx, s.He, s.Be, fh, fb);
    s.alpha = fh > 0 ? std::sqrt(fb) / std::sqrt(fh) : 0.0;
    s.lam_eps = g.lambda * g.ridge_epsilon;
    s.levels.assign(1, BzLevelHost());
    BzLevelHost &F = s.levels[0];
    F.n = g.nx;
    F.nd = 3 * g.nx + 1;
    for (int i = 0; i < 256; ++i) F.K[i] = s.alpha * s.He[i] + g.lambda * s.Be[i];
    F.rho.assign(F.nd, 1.0);
}

static void invert(const double *A, int n, double *Ainv) {
    std::vector<double> M(A, A + (size_t)n * n), I((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) I[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(M[(size_t)r * n + c]) > std::abs(M[(size_t)piv * n + c])) piv = r;
        DRF_CHECK(std::abs(M[(size_t)piv * n + c]) > 1e-300, DRF_E_INVALID, "singular multigrid block");
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(M[(size_t)c * n + k], M[(size_t)piv * n + k]);
                std::swap(I[(size_t)c * n + k], I[(size_t)piv * n + k]);
            }
        const double d = 1.0 / M[(size_t)c * n + c];
        for (int k = 0; k < n; ++k) { M[(size_t)c * n + k] *= d; I[(size_t)c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = M[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                M[(size_t)r * n + k] -= f * M[(size_t)c * n + k];
                I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
            }
        }
    }
    std::memcpy(Ainv, I.data(), sizeof(double) * (size_t)n * n);
}

static int p1_row(int f, int nc, const double S[2][16], double w[4]) {
    int E = f / 6;
    if (E > nc - 1) E = nc - 1;
    const int k = f - 6 * E;
    const double *row = k <= 3 ? &S[0][k * 4] : &S[1][(k - 3) * 4];
    for (int c = 0; c < 4; ++c) w[c] = row[c];
    return 3 * E;
}

static double row_entry_block(const BzSetup &s, const BzLevelHost &L, int ex, int ey, int a, int b) {
    const int gia = 3 * ex + a % 4, gja = 3 * ey + a / 4, gib = 3 * ex + b % 4, gjb = 3 * ey + b / 4;
    double v = (a == b) ? s.lam_eps * L.rho[gia] * L.rho[gja] : 0.0;
    for (int e2y = ey - 1; e2y <= ey + 1; ++e2y)
        for (int e2x = ex - 1; e2x <= ex + 1; ++e2x) {
            if (e2x < 0 || e2y < 0 || e2x >= L.n || e2y >= L.n) continue;
            const int la = gia - 3 * e2x, ma = gja - 3 * e2y, lb = gib - 3 * e2x, mb = gjb - 3 * e2y;
            if (la < 0 || la > 3 || ma < 0 || ma > 3 || lb < 0 || lb > 3 || mb < 0 || mb > 3) continue;
            v += L.K[(la + 4 * ma) * 16 + (lb + 4 * mb)];
        }
    return v;
}

void bz_setup_levels(BzSetup &s, int coarsest_n, int pre, int post) {
    s.pre = pre;
    s.post = post;
    DRF_CHECK(s.g.nx == s.g.ny, DRF_E_UNSUPPORTED, "multigrid needs a square grid");
    int nlev = 1, n = s.g.nx;
    while (n > coarsest_n && n % 2 == 0) { n /= 2; ++nlev; }
    std::vector<BzLevelHost> lv(nlev);
    BzLevelHost &F = lv[nlev - 1];
    F.n = s.g.nx;
    F.nd = 3 * F.n + 1;
    for (int i = 0; i < 256; ++i) F.K[i] = s.alpha * s.He[i] + s.g.lambda * s.Be[i];
    F.rho.assign(F.nd, 1.0);
    double Sd[2][16];
    bz_subdivision_1d(Sd);
    for (int l = nlev - 2; l >= 0; --l) {
        BzLevelHost &C = lv[l];
        const BzLevelHost &Fi = lv[l + 1];
        C.n = Fi.n / 2;
        C.nd = 3 * C.n + 1;
        std::memset(C.K, 0, sizeof(C.K));
        for (int cv = 0; cv < 2; ++cv)
            for (int cu = 0; cu < 2; ++cu) {
                double Sc[256], T[256];
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b)
                        Sc[a * 16 + b] = Sd[cu][(a % 4) * 4 + (b % 4)] * Sd[cv][(a / 4) * 4 + (b / 4)];
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b) {
                        double t = 0;
                        for (int k = 0; k < 16; ++k) t += Fi.K[a * 16 + k] * Sc[k * 16 + b];
                        T[a * 16 + b] = t;
                    }
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b) {
                        double t = 0;
                        for (int k = 0; k < 16; ++k) t += Sc[k * 16 + a] * T[k * 16 + b];
                        C.K[a * 16 + b] += t;
                    }
            }
        C.rho.assign(C.nd, 0.0);
        for (int f = 0; f < Fi.nd; ++f) {
            double w[4];
            const int c0 = p1_row(f, C.n, Sd, w);
            for (int c = 0; c < 4; ++c) C.rho[c0 + c] += w[c] * w[c] * Fi.rho[f];
        }
    }
    for (int l = 1; l < nlev; ++l) {
        BzLevelHost &L = lv[l];
        L.binv.assign(9 * 256, 0.0);
        for (int cy = 0; cy < 3; ++cy)
            for (int cx = 0; cx < 3; ++cx) {
                if ((cx == 1 || cy == 1) && L.n < 3) continue;
                const int ex = cx == 0 ? 0 : (cx == 1 ? 1 : L.n - 1);
                const int ey = cy == 0 ? 0 : (cy == 1 ? 1 : L.n - 1);
                double blk[256];
                for (int a = 0; a < 16; ++a)
                    for (int b = 0; b < 16; ++b) blk[a * 16 + b] = row_entry_block(s, L, ex, ey, a, b);
                invert(blk, 16, &L.binv[(cx + 3 * cy) * 256]);
            }
    }
    // dense coarsest operator and its inverse
    const BzLevelHost &C = lv[0];
    const int nc = C.nd * C.nd;
    DRF_CHECK(nc <= 4096, DRF_E_UNSUPPORTED, "coarsest level too large for the dense solve");
    std::vector<double> A((size_t)nc * nc, 0.0);
    for (int gj = 0; gj < C.nd; ++gj)
        for (int gi = 0; gi < C.nd; ++gi) {
            const int I = gi + C.nd * gj;
            A[(size_t)I * nc + I] += s.lam_eps * C.rho[gi] * C.rho[gj];
        }
    for (int ey = 0; ey < C.n; ++ey)
        for (int ex = 0; ex < C.n; ++ex)
            for (int a = 0; a < 16; ++a)
                for (int b = 0; b < 16; ++b) {
                    const int I = (3 * ex + a % 4) + C.nd * (3 * ey + a / 4);
                    const int J = (3 * ex + b % 4) + C.nd * (3 * ey + b / 4);
                    A[(size_t)I * nc + J] += C.K[a * 16 + b];
                }
    s.coarse_inv.assign((size_t)nc * nc, 0.0);
    invert(A.data(), nc, s.coarse_inv.data());
    s.levels = std::move(lv);
}

}  // namespace drf
