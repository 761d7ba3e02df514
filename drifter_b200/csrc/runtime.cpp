// Host runtime of libdrifter_b200: error buffer, launch counter, LGL basis construction.
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace drf {

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

std::atomic<uint64_t> &launch_counter() {
    static std::atomic<uint64_t> c{0};
    return c;
}

std::atomic<uint64_t> &alloc_counter() {
    static std::atomic<uint64_t> c{0};
    return c;
}

int &capture_depth() {
    static thread_local int d = 0;
    return d;
}

bool all_finite(const double *x, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(x[i])) return false;
    return true;
}

static void legendre(int n, double x, double &L, double &dL) {
    if (n == 0) { L = 1.0; dL = 0.0; return; }
    if (n == 1) { L = x; dL = 1.0; return; }
    double a = 1.0, b = x, da = 0.0, db = 1.0;
    for (int k = 2; k <= n; ++k) {
        L = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / k;
        dL = da + (2.0 * k - 1.0) * b;
        a = b; b = L; da = db; db = dL;
    }
}

// LGL nodes are the roots of (1 - x^2) P_N'(x); interior ones found by Newton on
// P_{N+1} - P_{N-1} (proportional to (1 - x^2) P_N'), started from Chebyshev-Gauss-Lobatto
// points. Weights 2 / (N (N + 1) P_N(x)^2). Same node set as the reference's
// compute_gauss_lobatto_nodes (src/dg/basis_hexahedron.cpp:70).
HostBasis make_lgl_basis(int order) {
    DRF_CHECK(order >= 1 && order < MAXNP, DRF_E_UNSUPPORTED,
              "polynomial order must be in [1, " + std::to_string(MAXNP - 1) + "]");
    HostBasis b;
    b.order = order;
    const int N = order, np = N + 1;
    b.np = np;
    b.x.assign(np, 0.0);
    b.w.assign(np, 0.0);
    for (int i = 0; i < np; ++i) {
        double xi = -std::cos(M_PI * i / N);
        if (i > 0 && i < N) {
            for (int it = 0; it < 200; ++it) {
                double Lm, dLm, L0, dL0, Lp, dLp;
                legendre(N - 1, xi, Lm, dLm);
                legendre(N, xi, L0, dL0);
                legendre(N + 1, xi, Lp, dLp);
                const double step = (Lp - Lm) / (dLp - dLm);
                xi -= step;
                if (std::abs(step) < 1e-16) break;
            }
        }
        b.x[i] = xi;
    }
    b.x[0] = -1.0;
    b.x[N] = 1.0;
    for (int i = 0; i < np / 2; ++i) {  // enforce exact symmetry
        const double s = 0.5 * (b.x[N - i] - b.x[i]);
        b.x[i] = -s;
        b.x[N - i] = s;
    }
    if (np % 2 == 1) b.x[N / 2] = 0.0;
    for (int i = 0; i < np; ++i) {
        double L, dL;
        legendre(N, b.x[i], L, dL);
        b.w[i] = 2.0 / (N * (N + 1) * L * L);
    }
    // barycentric weights and derivative matrix
    std::vector<double> bw(np, 1.0);
    for (int j = 0; j < np; ++j) {
        for (int k = 0; k < np; ++k)
            if (k != j) bw[j] *= (b.x[j] - b.x[k]);
        bw[j] = 1.0 / bw[j];
    }
    b.D.assign(np * np, 0.0);
    for (int i = 0; i < np; ++i) {
        double s = 0.0;
        for (int j = 0; j < np; ++j)
            if (j != i) {
                b.D[i * np + j] = (bw[j] / bw[i]) / (b.x[i] - b.x[j]);
                s += b.D[i * np + j];
            }
        b.D[i * np + i] = -s;
    }
    b.D2.assign(np * np, 0.0);
    for (int i = 0; i < np; ++i)
        for (int l = 0; l < np; ++l) {
            double s = 0.0;
            for (int m = 0; m < np; ++m) s += b.D[i * np + m] * b.D[m * np + l];
            b.D2[i * np + l] = s;
        }
    // integration matrix via Gauss-Legendre quadrature with np+1 points (exact for degree N)
    const int nq = np + 1;
    std::vector<double> gx(nq), gw(nq);
    for (int i = 0; i < nq; ++i) {
        double xi = -std::cos(M_PI * (i + 0.75) / (nq + 0.5));
        for (int it = 0; it < 200; ++it) {
            double L, dL;
            legendre(nq, xi, L, dL);
            const double step = L / dL;
            xi -= step;
            if (std::abs(step) < 1e-16) break;
        }
        double L, dL;
        legendre(nq, xi, L, dL);
        gx[i] = xi;
        gw[i] = 2.0 / ((1.0 - xi * xi) * dL * dL);
    }
    b.S.assign(np * np, 0.0);
    for (int k = 1; k < np; ++k) {
        const double half = 0.5 * (b.x[k] + 1.0);
        for (int q = 0; q < nq; ++q) {
            const double t = -1.0 + half * (gx[q] + 1.0);
            // Lagrange basis values at t
            for (int m = 0; m < np; ++m) {
                double lm = 1.0;
                for (int j = 0; j < np; ++j)
                    if (j != m) lm *= (t - b.x[j]) / (b.x[m] - b.x[j]);
                b.S[k * np + m] += half * gw[q] * lm;
            }
        }
    }
    return b;
}

}  // namespace drf

extern "C" {

int drf_last_error(char *buf, size_t n) {
    if (!buf || n == 0) return DRF_E_INVALID;
    const std::string &s = drf::g_last_error;
    const size_t m = s.size() < n - 1 ? s.size() : n - 1;
    std::memcpy(buf, s.data(), m);
    buf[m] = '\0';
    return DRF_OK;
}

const char *drf_version(void) { return "drifter_b200 0.1 (sm_100a)"; }

uint64_t drf_kernel_launch_count(void) { return drf::launch_counter().load(); }

uint64_t drf_device_alloc_count(void) { return drf::alloc_counter().load(); }

}  // extern "C"
