// Cubic Bezier bathymetry smoother on the GPU (uniform grid): matrix-free operator
// Q = alpha H + lambda (B^T W B + eps I) with one constant 16x16 element stencil per level,
// right-hand side assembly from data at the Gauss points, geometric multigrid V-cycle
// (Bezier subdivision transfers, exact Galerkin element matrices, colored multiplicative
// Schwarz with 16x16 element-block inverses, dense coarsest solve) and FP64 PCG with
// device-resident scalars, replayed as CUDA graphs in chunks of iterations.
//
// Layout: control point (gi, gj) of a level with n elements per direction is stored at
// gi + (3n + 1) * gj; element (ex, ey) owns control points 3ex..3ex+3 x 3ey..3ey+3 and its
// local dof k = i + 4 j (the reference's cubic dof order, include/bathymetry/cubic_bezier_basis_2d.hpp).
#include <algorithm>
#include <cmath>
#include <string>
#include <cstring>
#include <memory>
#include <vector>

#include "bz_host.hpp"
#include "cnn.hpp"
#include "common.cuh"

namespace drf {
namespace {

constexpr int BS = 256;
inline unsigned nblk(int64_t n) { return (unsigned)((n + BS - 1) / BS); }

struct LevelDev {
    int n, nd;
    const double *K;     // 256, row-major
    const double *rho;   // nd
    const double *binv;  // 9 x 256
    double lam_eps;
};

__device__ __forceinline__ double ridge(const LevelDev &L, int gi, int gj) {
    return L.lam_eps * L.rho[gi] * L.rho[gj];
}

// (Q_l x) at control point (gi, gj): gather over the <= 2 x 2 elements containing it
__device__ __forceinline__ double row_apply(const LevelDev &L, const double *__restrict__ K,
                                            const double *__restrict__ x, int gi, int gj) {
    double s = ridge(L, gi, gj) * x[gi + (int64_t)L.nd * gj];
    const int ex1 = min(gi / 3, L.n - 1), ey1 = min(gj / 3, L.n - 1);
    const int ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
    const int ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
    for (int ey = ey0; ey <= ey1; ++ey)
        for (int ex = ex0; ex <= ex1; ++ex) {
            const int a = (gi - 3 * ex) + 4 * (gj - 3 * ey);
            const double *xr = x + (3 * ex) + (int64_t)L.nd * (3 * ey);
            const double *Kr = K + a * 16;
#pragma unroll
            for (int bj = 0; bj < 4; ++bj)
#pragma unroll
                for (int bi = 0; bi < 4; ++bi) s += Kr[bi + 4 * bj] * xr[bi + (int64_t)L.nd * bj];
        }
    return s;
}

// y = Q x (mode 0) or y = b - Q x (mode 1); optional per-block partial of x.y (mode 0)
__global__ void __launch_bounds__(BS) bz_apply_kernel(LevelDev L, const double *__restrict__ x,
                                                      const double *__restrict__ b, double *y,
                                                      int mode, double *part, const int *stop) {
    __shared__ double K[256];
    __shared__ double red[BS];
    if (stop && *stop) return;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) K[i] = L.K[i];
    __syncthreads();
    const int64_t nd2 = (int64_t)L.nd * L.nd;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double dot = 0.0;
    if (t < nd2) {
        const int gi = (int)(t % L.nd), gj = (int)(t / L.nd);
        const double v = row_apply(L, K, x, gi, gj);
        if (mode == 0) {
            y[t] = v;
            dot = x[t] * v;
        } else {
            y[t] = b[t] - v;
        }
    }
    if (part) {
        red[threadIdx.x] = dot;
        __syncthreads();
        for (int s = BS / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[blockIdx.x] = red[0];
    }
}

__device__ __forceinline__ int elem_class(int e, int n) { return e == 0 ? 0 : (e == n - 1 ? 2 : 1); }

// colored Schwarz, part 1: residual at the dofs of every element of one color
__global__ void __launch_bounds__(BS) bz_smooth_res_kernel(LevelDev L, int color,
                                                           const double *__restrict__ x,
                                                           const double *__restrict__ b, double *r) {
    __shared__ double K[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) K[i] = L.K[i];
    __syncthreads();
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2, ncy = (L.n - py + 1) / 2;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)ncx * ncy * 16) return;
    const int ce = (int)(t / 16), a = (int)(t % 16);
    const int ex = px + 2 * (ce % ncx), ey = py + 2 * (ce / ncx);
    const int gi = 3 * ex + a % 4, gj = 3 * ey + a / 4;
    const int64_t I = gi + (int64_t)L.nd * gj;
    r[I] = b[I] - row_apply(L, K, x, gi, gj);
}

// colored Schwarz, part 2: x_e += Binv_class(e) r_e for every element of one color
__global__ void __launch_bounds__(BS) bz_smooth_upd_kernel(LevelDev L, int color,
                                                           const double *__restrict__ r, double *x) {
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2, ncy = (L.n - py + 1) / 2;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)ncx * ncy * 16) return;
    const int ce = (int)(t / 16), a = (int)(t % 16);
    const int ex = px + 2 * (ce % ncx), ey = py + 2 * (ce / ncx);
    const double *Bi = L.binv + (elem_class(ex, L.n) + 3 * elem_class(ey, L.n)) * 256 + a * 16;
    const double *re = r + 3 * ex + (int64_t)L.nd * (3 * ey);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += Bi[k] * re[(k % 4) + (int64_t)L.nd * (k / 4)];
    x[(3 * ex + a % 4) + (int64_t)L.nd * (3 * ey + a / 4)] += s;
}

// 1D prolongation weights: fine index f -> 4 weights on coarse 3E..3E+3
__constant__ double cSub[2][16];

__device__ __forceinline__ int p1_row(int f, int nc, double w[4]) {
    int E = f / 6;
    if (E > nc - 1) E = nc - 1;
    const int k = f - 6 * E;
    const double *row = k <= 3 ? &cSub[0][k * 4] : &cSub[1][(k - 3) * 4];
#pragma unroll
    for (int c = 0; c < 4; ++c) w[c] = row[c];
    return 3 * E;
}

// weight of coarse index c in the row of fine index f (0 if none)
__device__ __forceinline__ double p1_weight(int f, int c, int nc) {
    double w[4];
    const int c0 = p1_row(f, nc, w);
    const int d = c - c0;
    return (d >= 0 && d <= 3) ? w[d] : 0.0;
}

// r_c = P^T r_f (separable sums over the <= 13 fine indices per direction)
__global__ void __launch_bounds__(BS) bz_restrict_kernel(int ncel, int ndc, int ndf,
                                                         const double *__restrict__ rf, double *rc,
                                                         double *xc_zero) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)ndc * ndc) return;
    const int ci = (int)(t % ndc), cj = (int)(t / ndc);
    const int Ex1 = min(ci / 3, ncel - 1), Ey1 = min(cj / 3, ncel - 1);
    const int Ex0 = (ci % 3 == 0 && ci > 0) ? ci / 3 - 1 : Ex1;
    const int Ey0 = (cj % 3 == 0 && cj > 0) ? cj / 3 - 1 : Ey1;
    const int fi0 = 6 * Ex0, fi1 = min(6 * Ex1 + 6, ndf - 1);
    const int fj0 = 6 * Ey0, fj1 = min(6 * Ey1 + 6, ndf - 1);
    double s = 0.0;
    for (int fj = fj0; fj <= fj1; ++fj) {
        const double wy = p1_weight(fj, cj, ncel);
        if (wy == 0.0) continue;
        double sx = 0.0;
        for (int fi = fi0; fi <= fi1; ++fi) {
            const double wx = p1_weight(fi, ci, ncel);
            if (wx != 0.0) sx += wx * rf[fi + (int64_t)ndf * fj];
        }
        s += wy * sx;
    }
    rc[t] = s;
    xc_zero[t] = 0.0;
}

// x_f += P e_c
__global__ void __launch_bounds__(BS) bz_prolong_kernel(int ncel, int ndc, int ndf,
                                                        const double *__restrict__ ec, double *xf) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)ndf * ndf) return;
    const int fi = (int)(t % ndf), fj = (int)(t / ndf);
    double wx[4], wy[4];
    const int cx0 = p1_row(fi, ncel, wx), cy0 = p1_row(fj, ncel, wy);
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int a = 0; a < 4; ++a) s += wy[b] * wx[a] * ec[(cx0 + a) + (int64_t)ndc * (cy0 + b)];
    xf[t] += s;
}

// coarsest level: x = C^-1 b (one block, dense)
__global__ void bz_coarse_kernel(int n2, const double *__restrict__ Cinv, const double *__restrict__ b,
                                 double *x) {
    extern __shared__ double sb[];
    for (int i = threadIdx.x; i < n2; i += blockDim.x) sb[i] = b[i];
    __syncthreads();
    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < n2; ++k) s += Cinv[(int64_t)i * n2 + k] * sb[k];
        x[i] = s;
    }
}

// right-hand side b = lambda B^T W d: Bq[la][q] = W_q B_la(q) precomputed
__global__ void __launch_bounds__(BS) bz_rhs_kernel(int n, int nd, const double *__restrict__ d,
                                                    const double *__restrict__ Bq, double lam,
                                                    double *b) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nd * nd) return;
    const int gi = (int)(t % nd), gj = (int)(t / nd);
    const int ex1 = min(gi / 3, n - 1), ey1 = min(gj / 3, n - 1);
    const int ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
    const int ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
    double s = 0.0;
    for (int ey = ey0; ey <= ey1; ++ey)
        for (int ex = ex0; ex <= ex1; ++ex) {
            const int a = (gi - 3 * ex) + 4 * (gj - 3 * ey);
            const double *de = d + ((int64_t)ey * n + ex) * 16;
#pragma unroll
            for (int q = 0; q < 16; ++q) s += Bq[a * 16 + q] * de[q];
        }
    b[t] = lam * s;
}

// ------------------------------------------------------------------ PCG with device scalars
// scalar slots
enum { S_RZ = 0, S_PQ, S_ALPHA, S_RR, S_BETA, S_BB, S_TOL2, S_RZNEW, S_NSLOT };
struct PcgCtl {
    double *sc;   // scalars
    int *stop;    // 1 once converged (later kernels of the chunk return immediately)
    int *iters;   // iterations done
    int *maxit;   // iteration limit
    double *part; // per-block partials
};

__global__ void reduce_kernel(const double *part, int nparts, double *out) {
    __shared__ double red[BS];
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += BS) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// partial dot products a.b (and optionally c.c) per block
__global__ void __launch_bounds__(BS) dot_kernel(int64_t n, const double *a, const double *b,
                                                 double *part, const int *stop) {
    __shared__ double red[BS];
    if (stop && *stop) return;
    double s = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS)
        s += a[t] * b[t];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// partial dot products a.b and a.c per block (part and part + gridDim.x)
__global__ void __launch_bounds__(BS) dot2_kernel(int64_t n, const double *a, const double *b,
                                                  const double *cvec, double *part, const int *stop) {
    __shared__ double red[2][BS];
    if (stop && *stop) return;
    double s = 0.0, s2 = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS) {
        s += a[t] * b[t];
        s2 += a[t] * cvec[t];
    }
    red[0][threadIdx.x] = s;
    red[1][threadIdx.x] = s2;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            red[0][threadIdx.x] += red[0][threadIdx.x + k];
            red[1][threadIdx.x] += red[1][threadIdx.x + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = red[0][0];
        part[gridDim.x + blockIdx.x] = red[1][0];
    }
}

// flexible CG (Notay's FCG(1)): rz = r.z, beta = -(z.q)/(p.q)
__global__ void beta_fcg_kernel(PcgCtl c, int nparts) {
    __shared__ double red[2][BS];
    if (*c.stop) return;
    double s = 0.0, s2 = 0.0;
    for (int i = threadIdx.x; i < nparts; i += BS) {
        s += c.part[i];
        s2 += c.part[nparts + i];
    }
    red[0][threadIdx.x] = s;
    red[1][threadIdx.x] = s2;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            red[0][threadIdx.x] += red[0][threadIdx.x + k];
            red[1][threadIdx.x] += red[1][threadIdx.x + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c.sc[S_RZ] = red[0][0];
        c.sc[S_BETA] = -red[1][0] / c.sc[S_PQ];
    }
}

__global__ void alpha_kernel(PcgCtl c, int nparts) {
    __shared__ double red[BS];
    if (*c.stop) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += BS) s += c.part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c.sc[S_PQ] = red[0];
        c.sc[S_ALPHA] = c.sc[S_RZ] / red[0];
    }
}

// x += alpha p ; r -= alpha q ; partial r.r
__global__ void __launch_bounds__(BS) xr_update_kernel(int64_t n, PcgCtl c, const double *p,
                                                       const double *q, double *x, double *r) {
    __shared__ double red[BS];
    if (*c.stop) return;
    const double a = c.sc[S_ALPHA];
    double s = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS) {
        x[t] += a * p[t];
        const double rn = r[t] - a * q[t];
        r[t] = rn;
        s += rn * rn;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) c.part[blockIdx.x] = red[0];
}

// rr = sum(part); convergence test; iteration count
__global__ void conv_kernel(PcgCtl c, int nparts) {
    __shared__ double red[BS];
    if (*c.stop) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += BS) s += c.part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c.sc[S_RR] = red[0];
        *c.iters += 1;
        if (!(red[0] > c.sc[S_TOL2] * c.sc[S_BB]) || *c.iters >= *c.maxit) *c.stop = 1;
    }
}

__global__ void beta_kernel(PcgCtl c, int nparts) {
    __shared__ double red[BS];
    if (*c.stop) return;
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += BS) s += c.part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = BS / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c.sc[S_BETA] = red[0] / c.sc[S_RZ];
        c.sc[S_RZ] = red[0];
    }
}

// p = z + beta p (beta = 0 and p = z when init)
__global__ void __launch_bounds__(BS) p_update_kernel(int64_t n, PcgCtl c, const double *z, double *p,
                                                      int init) {
    if (*c.stop) return;
    const double be = init ? 0.0 : c.sc[S_BETA];
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS)
        p[t] = z[t] + be * p[t];
}

// z = r / diag(Q)
__global__ void __launch_bounds__(BS) jacobi_kernel(LevelDev L, const double *r, double *z,
                                                    const int *stop) {
    if (stop && *stop) return;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)L.nd * L.nd) return;
    const int gi = (int)(t % L.nd), gj = (int)(t / L.nd);
    double d = ridge(L, gi, gj);
    const int ex1 = min(gi / 3, L.n - 1), ey1 = min(gj / 3, L.n - 1);
    const int ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
    const int ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
    for (int ey = ey0; ey <= ey1; ++ey)
        for (int ex = ex0; ex <= ex1; ++ex) {
            const int a = (gi - 3 * ex) + 4 * (gj - 3 * ey);
            d += L.K[a * 16 + a];
        }
    z[t] = r[t] / d;
}

__global__ void copy_kernel(int64_t n, const double *a, double *b, const int *stop) {
    if (stop && *stop) return;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) b[t] = a[t];
}

__global__ void zero_kernel(int64_t n, double *a, const int *stop) {
    if (stop && *stop) return;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) a[t] = 0.0;
}

__global__ void fill_kernel(int64_t n, double v, double *a) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) a[t] = v;
}

}  // namespace

// ---------------------------------------------------------------- allocation-free solve
// Scratch of drf_bz_jacobi_pcg_noalloc: a file-scope device array that every GPU loading this
// library holds until process exit (NOALLOC_BYTES). Layout in doubles: element operator (256),
// ridge factors (NOALLOC_MAX_ND), PCG vectors r, z, p, q (NOALLOC_MAX_DOF each), per-block
// partials (NOALLOC_PARTS), scalars (S_NSLOT, padded to 16) and three int control words.
constexpr int64_t NOALLOC_MAX_DOF = 1 << 18;  // 262,144 control points (170 x 170 elements)
constexpr int NOALLOC_MAX_ND = 512;
constexpr int NOALLOC_PARTS = 1040;           // >= nblk(NOALLOC_MAX_DOF) and >= 1024
constexpr int64_t NOALLOC_DOUBLES =
    256 + NOALLOC_MAX_ND + 4 * NOALLOC_MAX_DOF + NOALLOC_PARTS + 16 + 4;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

}  // namespace drf

using namespace drf;

struct drf_bz {
    BzSetup H;  // host-side setup (element matrices, levels, transfers)
    cudaStream_t stream = nullptr, own = nullptr;
    int64_t ndof = 0;
    DevBuf<double> dat, Bq, b, bs, x, r, z, p, q, scal, part, mgbuf, coarse;  // b: assembled rhs, bs: rhs of the current solve
    DevBuf<int> ctl;
    struct Lv {
        DevBuf<double> K, rho, binv, x, b, r;
        int n = 0, nd = 0;
    };
    std::vector<Lv> lv;
    bool mg_ready = false;
    drf_cnn *cnn = nullptr;
    double cnn_scale = 1.0;
    cudaGraphExec_t graph = nullptr;
    int graph_kind = -1, graph_chunk = 0;

    ~drf_bz() {
        if (graph) cudaGraphExecDestroy(graph);
        if (own) cudaStreamDestroy(own);
    }
    LevelDev levdev(int l) const {
        LevelDev L;
        L.n = lv[l].n; L.nd = lv[l].nd; L.K = lv[l].K.p; L.rho = lv[l].rho.p;
        L.binv = lv[l].binv.p; L.lam_eps = H.lam_eps;
        return L;
    }
    int finest() const { return (int)lv.size() - 1; }
    unsigned nparts() const { return 1024; }
    PcgCtl pctl() {
        PcgCtl c;
        c.sc = scal.p; c.stop = ctl.p; c.iters = ctl.p + 1; c.maxit = ctl.p + 2; c.part = part.p;
        return c;
    }

    // z = M r for the given preconditioner kind (enqueued on stream)
    void precondition(int kind, const double *rin, double *zout, const int *stop) {
        const int L = finest();
        const int64_t n = ndof;
        if (kind == 0) {
            copy_kernel<<<nblk(n), BS, 0, stream>>>(n, rin, zout, stop);
            DRF_LAUNCHED();
        } else if (kind == 1) {
            jacobi_kernel<<<nblk(n), BS, 0, stream>>>(levdev(L), rin, zout, stop);
            DRF_LAUNCHED();
        } else if (kind == 3) {
            // Jacobi base (positive definite: a descent direction for any residual) plus the
            // learned correction of the error it leaves
            jacobi_kernel<<<nblk(n), BS, 0, stream>>>(levdev(L), rin, zout, stop);
            DRF_LAUNCHED();
            cnn_precondition(cnn_net(cnn), stream, lv[L].n, rin, scal.p + S_RR, cnn_scale, zout, 1,
                             stop);
        } else {
            vcycle(rin, zout);
        }
    }

    void smooth(int l, double *xl, const double *bl, double *rl, bool forward) {
        const LevelDev L = levdev(l);
        for (int s = 0; s < 4; ++s) {
            const int color = forward ? s : 3 - s;
            const int px = color & 1, py = color >> 1;
            const int64_t work = (int64_t)((L.n - px + 1) / 2) * ((L.n - py + 1) / 2) * 16;
            bz_smooth_res_kernel<<<nblk(work), BS, 0, stream>>>(L, color, xl, bl, rl);
            DRF_LAUNCHED();
            bz_smooth_upd_kernel<<<nblk(work), BS, 0, stream>>>(L, color, rl, xl);
            DRF_LAUNCHED();
        }
    }

    // one V-cycle z = M r (z overwritten), finest level uses rin/zout directly
    void vcycle(const double *rin, double *zout) {
        const int Lf = finest();
        std::vector<double *> X(lv.size()), B(lv.size()), R(lv.size());
        for (int l = 0; l < Lf; ++l) { X[l] = lv[l].x.p; B[l] = lv[l].b.p; R[l] = lv[l].r.p; }
        X[Lf] = zout; B[Lf] = const_cast<double *>(rin); R[Lf] = lv[Lf].r.p;
        zero_kernel<<<nblk(ndof), BS, 0, stream>>>(ndof, zout, nullptr);
        DRF_LAUNCHED();
        for (int l = Lf; l >= 1; --l) {
            for (int it = 0; it < H.pre; ++it) smooth(l, X[l], B[l], R[l], true);
            const int64_t nd2 = (int64_t)lv[l].nd * lv[l].nd;
            bz_apply_kernel<<<nblk(nd2), BS, 0, stream>>>(levdev(l), X[l], B[l], R[l], 1, nullptr, nullptr);
            DRF_LAUNCHED();
            const int64_t ndc2 = (int64_t)lv[l - 1].nd * lv[l - 1].nd;
            bz_restrict_kernel<<<nblk(ndc2), BS, 0, stream>>>(lv[l - 1].n, lv[l - 1].nd, lv[l].nd,
                                                              R[l], B[l - 1], X[l - 1]);
            DRF_LAUNCHED();
        }
        const int nc2 = lv[0].nd * lv[0].nd;
        bz_coarse_kernel<<<1, 256, nc2 * sizeof(double), stream>>>(nc2, coarse.p, B[0], X[0]);
        DRF_LAUNCHED();
        for (int l = 1; l <= Lf; ++l) {
            const int64_t nd2 = (int64_t)lv[l].nd * lv[l].nd;
            bz_prolong_kernel<<<nblk(nd2), BS, 0, stream>>>(lv[l - 1].n, lv[l - 1].nd, lv[l].nd,
                                                            X[l - 1], X[l]);
            DRF_LAUNCHED();
            for (int it = 0; it < H.post; ++it) smooth(l, X[l], B[l], R[l], false);
        }
    }

    // one PCG iteration (assumes r, z, p, rz set)
    void pcg_iteration(int kind) {
        const int Lf = finest();
        const LevelDev L = levdev(Lf);
        PcgCtl c = pctl();
        const unsigned nb = nblk(ndof);
        // q = Q p with partial p.q
        bz_apply_kernel<<<nb, BS, 0, stream>>>(L, p.p, nullptr, q.p, 0, part.p, c.stop);
        DRF_LAUNCHED();
        alpha_kernel<<<1, BS, 0, stream>>>(c, (int)nb);
        DRF_LAUNCHED();
        xr_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, p.p, q.p, x.p, r.p);
        DRF_LAUNCHED();
        conv_kernel<<<1, BS, 0, stream>>>(c, (int)nparts());
        DRF_LAUNCHED();
        precondition(kind, r.p, z.p, c.stop);
        if (kind == 3) {
            dot2_kernel<<<nparts(), BS, 0, stream>>>(ndof, z.p, r.p, q.p, part.p, c.stop);
            DRF_LAUNCHED();
            beta_fcg_kernel<<<1, BS, 0, stream>>>(c, (int)nparts());
            DRF_LAUNCHED();
        } else {
            dot_kernel<<<nparts(), BS, 0, stream>>>(ndof, r.p, z.p, part.p, c.stop);
            DRF_LAUNCHED();
            beta_kernel<<<1, BS, 0, stream>>>(c, (int)nparts());
            DRF_LAUNCHED();
        }
        p_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, z.p, p.p, 0);
        DRF_LAUNCHED();
    }
};

namespace drf {
namespace {

void upload_sub() {
    static bool done[64] = {false};
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && done[dev]) return;
    double S[2][16];
    bz_subdivision_1d(S);
    DRF_CUDA(cudaMemcpyToSymbol(cSub, S, sizeof(S)));
    if (dev < 64) done[dev] = true;
}

template <class V>
void up(DevBuf<double> &d, const V &v) {
    d.alloc(v.size());
    DRF_CUDA(cudaMemcpy(d.p, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
}

void check_bz(drf_bz *h) { DRF_CHECK(h != nullptr, DRF_E_INVALID, "null smoother handle"); }

}  // namespace
}  // namespace drf

extern "C" {

int drf_bz_create(const drf_bz_grid_desc *g, const double *dgauss, drf_bz **out) {
    return guard([&] {
        DRF_CHECK(g && dgauss && out, DRF_E_INVALID, "null argument");
        *out = nullptr;
        DRF_CHECK(g->nx >= 1 && g->ny >= 1 && g->nx == g->ny, DRF_E_INVALID,
                  "the GPU smoother needs a square uniform grid (nx == ny >= 1)");
        DRF_CHECK(g->Lx > 0 && g->Ly > 0 && g->lambda > 0 && g->ridge_epsilon >= 0, DRF_E_INVALID,
                  "extent and lambda must be positive, ridge_epsilon >= 0");
        const size_t nd = (size_t)g->nx * g->ny * 16;
        DRF_CHECK(all_finite(dgauss, nd), DRF_E_NONFINITE, "non-finite bathymetry sample");
        auto h = std::make_unique<drf_bz>();
        bz_setup_fine(h->H, *g);
        DRF_CUDA(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
        h->stream = h->own;
        upload_sub();
        h->ndof = (int64_t)(3 * g->nx + 1) * (3 * g->ny + 1);
        // finest level only until drf_mg_setup
        h->lv.resize(1);
        auto &F = h->lv[0];
        F.n = g->nx;
        F.nd = 3 * g->nx + 1;
        up(F.K, std::vector<double>(h->H.levels.back().K, h->H.levels.back().K + 256));
        up(F.rho, h->H.levels.back().rho);
        F.binv.alloc(9 * 256);
        DRF_CUDA(cudaMemset(F.binv.p, 0, 9 * 256 * 8));
        h->dat.alloc(nd);
        DRF_CUDA(cudaMemcpy(h->dat.p, dgauss, nd * 8, cudaMemcpyHostToDevice));
        up(h->Bq, h->H.Bq);
        for (auto *v : {&h->b, &h->bs, &h->x, &h->r, &h->z, &h->p, &h->q}) v->alloc(h->ndof);
        h->scal.alloc(S_NSLOT);
        // per-block partials: the fused apply-dot writes one value per apply block
        h->part.alloc(std::max<size_t>(4096, (size_t)nblk(h->ndof) + 16));
        h->ctl.alloc(3);
        bz_rhs_kernel<<<nblk(h->ndof), BS, 0, h->stream>>>(F.n, F.nd, h->dat.p, h->Bq.p, g->lambda, h->b.p);
        DRF_LAUNCHED();
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        *out = h.release();
    });
}

int drf_bz_destroy(drf_bz *h) {
    return guard([&] {
        if (!h) return;
        if (h->stream) cudaStreamSynchronize(h->stream);
        delete h;
    });
}

int drf_bz_set_stream(drf_bz *h, void *s) {
    return guard([&] {
        check_bz(h);
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; h->graph_kind = -1; }
        h->stream = s ? (cudaStream_t)s : h->own;
    });
}

int drf_bz_info(drf_bz *h, int64_t *ndof, double *alpha, int *nlevels) {
    return guard([&] {
        check_bz(h);
        if (ndof) *ndof = h->ndof;
        if (alpha) *alpha = h->H.alpha;
        if (nlevels) *nlevels = (int)h->lv.size();
    });
}

int drf_bz_get_rhs(drf_bz *h, double *b) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(b, DRF_E_INVALID, "null output");
        DRF_CUDA(cudaMemcpyAsync(b, h->b.p, h->ndof * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_bz_apply_Q(drf_bz *h, const double *xh, double *yh) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(xh && yh, DRF_E_INVALID, "null argument");
        DRF_CUDA(cudaMemcpyAsync(h->z.p, xh, h->ndof * 8, cudaMemcpyHostToDevice, h->stream));
        bz_apply_kernel<<<nblk(h->ndof), BS, 0, h->stream>>>(h->levdev(h->finest()), h->z.p, nullptr,
                                                             h->q.p, 0, nullptr, nullptr);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpyAsync(yh, h->q.p, h->ndof * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_mg_setup(drf_bz *h, int coarsest_n, int pre, int post) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(coarsest_n >= 1 && pre >= 0 && post >= 0, DRF_E_INVALID, "bad multigrid config");
        bz_setup_levels(h->H, coarsest_n, pre, post);
        const int nl = (int)h->H.levels.size();
        std::vector<drf_bz::Lv> lv(nl);
        for (int l = 0; l < nl; ++l) {
            const BzLevelHost &Lh = h->H.levels[l];
            lv[l].n = Lh.n;
            lv[l].nd = Lh.nd;
            up(lv[l].K, std::vector<double>(Lh.K, Lh.K + 256));
            up(lv[l].rho, Lh.rho);
            std::vector<double> bi = Lh.binv;
            if (bi.empty()) bi.assign(9 * 256, 0.0);
            up(lv[l].binv, bi);
            if (l < nl - 1) {
                const size_t n2 = (size_t)Lh.nd * Lh.nd;
                lv[l].x.alloc(n2); lv[l].b.alloc(n2); lv[l].r.alloc(n2);
            } else {
                lv[l].r.alloc((size_t)Lh.nd * Lh.nd);
            }
        }
        h->lv = std::move(lv);
        up(h->coarse, h->H.coarse_inv);
        const int nc2 = h->lv[0].nd * h->lv[0].nd;
        DRF_CHECK((size_t)nc2 * 8 <= 48 * 1024, DRF_E_UNSUPPORTED, "coarsest level too large");
        h->mg_ready = true;
        if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; h->graph_kind = -1; }
    });
}

int drf_bz_set_cnn(drf_bz *h, drf_cnn *net, double out_scale) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(net, DRF_E_INVALID, "null network");
        DRF_CHECK(std::isfinite(out_scale) && out_scale > 0, DRF_E_INVALID, "out_scale must be > 0");
        h->cnn = net;
        h->cnn_scale = out_scale;
        cnn_prepare(cnn_net(net), h->lv[h->finest()].n);
        if (h->graph && h->graph_kind == 3) {
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
            h->graph_kind = -1;
        }
    });
}

int drf_bz_precondition(drf_bz *h, int kind, const double *rh, double *zh) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(rh && zh, DRF_E_INVALID, "null argument");
        DRF_CHECK(kind >= 0 && kind <= 3, DRF_E_INVALID, "unknown preconditioner kind");
        DRF_CHECK(kind != 2 || h->mg_ready, DRF_E_INVALID, "multigrid preconditioner not set up");
        DRF_CHECK(kind != 3 || h->cnn, DRF_E_INVALID, "no learned preconditioner attached");
        DRF_CUDA(cudaMemcpyAsync(h->r.p, rh, h->ndof * 8, cudaMemcpyHostToDevice, h->stream));
        dot_kernel<<<h->nparts(), BS, 0, h->stream>>>(h->ndof, h->r.p, h->r.p, h->part.p, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, h->stream>>>(h->part.p, (int)h->nparts(), h->scal.p + S_RR);
        DRF_LAUNCHED();
        h->precondition(kind, h->r.p, h->z.p, nullptr);
        DRF_CUDA(cudaMemcpyAsync(zh, h->z.p, h->ndof * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_mg_apply(drf_bz *h, const double *rh, double *zh) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(h->mg_ready, DRF_E_INVALID, "drf_mg_setup has not been called");
        DRF_CHECK(rh && zh, DRF_E_INVALID, "null argument");
        DRF_CUDA(cudaMemcpyAsync(h->r.p, rh, h->ndof * 8, cudaMemcpyHostToDevice, h->stream));
        h->vcycle(h->r.p, h->z.p);
        DRF_CUDA(cudaMemcpyAsync(zh, h->z.p, h->ndof * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_pcg_solve(drf_bz *h, const double *bh, double *xh, double tol, int maxit, int kind,
                  int *iters, double *relres, double *ms) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(xh && tol > 0 && maxit >= 0, DRF_E_INVALID, "bad arguments");
        DRF_CHECK(kind >= 0 && kind <= 3, DRF_E_INVALID, "unknown preconditioner kind");
        DRF_CHECK(kind != 2 || h->mg_ready, DRF_E_INVALID, "multigrid preconditioner not set up");
        DRF_CHECK(kind != 3 || h->cnn, DRF_E_INVALID, "no learned preconditioner attached (drf_bz_set_cnn)");
        const int64_t n = h->ndof;
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        if (bh) DRF_CUDA(cudaMemcpyAsync(h->bs.p, bh, n * 8, cudaMemcpyHostToDevice, h->stream));
        else DRF_CUDA(cudaMemcpyAsync(h->bs.p, h->b.p, n * 8, cudaMemcpyDeviceToDevice, h->stream));
        DRF_CUDA(cudaMemcpyAsync(h->x.p, xh, n * 8, cudaMemcpyHostToDevice, h->stream));
        DRF_CUDA(cudaEventRecord(e0, h->stream));
        PcgCtl c = h->pctl();
        const int ctl0[3] = {0, 0, maxit};
        DRF_CUDA(cudaMemcpyAsync(h->ctl.p, ctl0, sizeof(ctl0), cudaMemcpyHostToDevice, h->stream));
        const double tol2 = tol * tol;
        DRF_CUDA(cudaMemcpyAsync(h->scal.p + S_TOL2, &tol2, 8, cudaMemcpyHostToDevice, h->stream));
        // r = b - Q x ; bb = b.b ; z = M r ; rz = r.z ; p = z
        const LevelDev L = h->levdev(h->finest());
        bz_apply_kernel<<<nblk(n), BS, 0, h->stream>>>(L, h->x.p, h->bs.p, h->r.p, 1, nullptr, nullptr);
        DRF_LAUNCHED();
        dot_kernel<<<h->nparts(), BS, 0, h->stream>>>(n, h->bs.p, h->bs.p, h->part.p, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, h->stream>>>(h->part.p, (int)h->nparts(), h->scal.p + S_BB);
        DRF_LAUNCHED();
        // converged at start (r = 0) handled through the convergence kernel on r.r
        dot_kernel<<<h->nparts(), BS, 0, h->stream>>>(n, h->r.p, h->r.p, h->part.p, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, h->stream>>>(h->part.p, (int)h->nparts(), h->scal.p + S_RR);
        DRF_LAUNCHED();
        h->precondition(kind, h->r.p, h->z.p, nullptr);
        dot_kernel<<<h->nparts(), BS, 0, h->stream>>>(n, h->r.p, h->z.p, h->part.p, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, h->stream>>>(h->part.p, (int)h->nparts(), h->scal.p + S_RZ);
        DRF_LAUNCHED();
        p_update_kernel<<<h->nparts(), BS, 0, h->stream>>>(n, c, h->z.p, h->p.p, 1);
        DRF_LAUNCHED();
        double sc[S_NSLOT];
        DRF_CUDA(cudaMemcpyAsync(sc, h->scal.p, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        int done = 0, it = 0;
        if (!(sc[S_RR] > tol2 * sc[S_BB])) done = 1;
        // iterations in graph-captured chunks; converged iterations return early on the device
        const int chunk = 8;
        if (!done && maxit > 0) {
            if (!h->graph || h->graph_kind != kind || h->graph_chunk != chunk) {
                if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
                cudaGraph_t g = nullptr;
                DRF_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    for (int k = 0; k < chunk; ++k) h->pcg_iteration(kind);
                } catch (...) {
                    cudaStreamEndCapture(h->stream, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                DRF_CUDA(cudaStreamEndCapture(h->stream, &g));
                cudaError_t e = cudaGraphInstantiate(&h->graph, g, 0);
                cudaGraphDestroy(g);
                DRF_CUDA(e);
                h->graph_kind = kind;
                h->graph_chunk = chunk;
            }
            int ctl[2] = {0, 0};
            while (true) {
                DRF_CUDA(cudaGraphLaunch(h->graph, h->stream));
                launch_counter().fetch_add(1);
                DRF_CUDA(cudaMemcpyAsync(ctl, h->ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, h->stream));
                DRF_CUDA(cudaStreamSynchronize(h->stream));
                if (ctl[0] || ctl[1] >= maxit) break;
            }
            it = ctl[1];
        }
        DRF_CUDA(cudaEventRecord(e1, h->stream));
        DRF_CUDA(cudaMemcpyAsync(sc, h->scal.p, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaMemcpyAsync(xh, h->x.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        float t = 0.f;
        DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (iters) *iters = it;
        if (relres) *relres = sc[S_BB] > 0 ? std::sqrt(sc[S_RR] / sc[S_BB]) : 0.0;
        if (ms) *ms = t;
        DRF_CHECK(std::isfinite(sc[S_RR]), DRF_E_NONFINITE, "PCG diverged (non-finite residual)");
    });
}

// Callers that cannot allocate device memory (a host application that hands this library
// only the buffers it already owns, code running under an allocator that forbids
// cudaMalloc/cudaFree, or a stream being used by another runtime that must not see
// device-wide synchronising allocation calls) solve Q x = b with Jacobi-preconditioned CG
// here. All scratch is the file-scope array g_noalloc_scratch; the caller passes the device
// right-hand side and the device solution buffer (initial guess in, solution out).
int drf_bz_jacobi_pcg_noalloc(const drf_bz_grid_desc *g, const double *d_b, double *d_x,
                              double tol, int maxit, void *stream, int *iters, double *relres) {
    return guard([&] {
        DRF_CHECK(g && d_b && d_x && iters && relres, DRF_E_INVALID, "null argument");
        DRF_CHECK(g->nx >= 1 && g->nx == g->ny, DRF_E_INVALID, "square grid (nx == ny >= 1) required");
        DRF_CHECK(g->Lx > 0 && g->Ly > 0 && g->lambda > 0 && g->ridge_epsilon >= 0, DRF_E_INVALID,
                  "extent and lambda must be positive, ridge_epsilon >= 0");
        DRF_CHECK(tol > 0 && maxit >= 0, DRF_E_INVALID, "tol must be > 0 and maxit >= 0");
        const int nd = 3 * g->nx + 1;
        const int64_t n = (int64_t)nd * nd;
        DRF_CHECK(nd <= NOALLOC_MAX_ND && n <= NOALLOC_MAX_DOF, DRF_E_UNSUPPORTED,
                  "grid too large for the allocation-free solve: at most " +
                      std::to_string(NOALLOC_MAX_DOF) + " control points (nx <= 170)");
        // device address of the scratch array, looked up once per device with it current
        static double *base[64] = {nullptr};
        int dev = 0;
        DRF_CUDA(cudaGetDevice(&dev));
        DRF_CHECK(dev >= 0 && dev < 64, DRF_E_UNSUPPORTED, "device ordinal out of range");
        if (!base[dev]) {
            void *ptr = nullptr;
            DRF_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
            base[dev] = static_cast<double *>(ptr);
        }
        double *K = base[dev], *rho = K + 256, *r = rho + NOALLOC_MAX_ND;
        double *z = r + NOALLOC_MAX_DOF, *p = z + NOALLOC_MAX_DOF, *q = p + NOALLOC_MAX_DOF;
        double *part = q + NOALLOC_MAX_DOF, *scal = part + NOALLOC_PARTS;
        int *ctl = reinterpret_cast<int *>(scal + 16);
        cudaStream_t st = (cudaStream_t)stream;
        upload_sub();
        double Kh[256], alpha = 0.0;
        bz_fine_operator(*g, Kh, &alpha);
        // every value the solve reads is written here first (the array keeps the last call's data)
        DRF_CUDA(cudaMemcpyAsync(K, Kh, sizeof(Kh), cudaMemcpyHostToDevice, st));
        fill_kernel<<<nblk(nd), BS, 0, st>>>(nd, 1.0, rho);
        DRF_LAUNCHED();
        const int ctl0[3] = {0, 0, maxit};
        DRF_CUDA(cudaMemcpyAsync(ctl, ctl0, sizeof(ctl0), cudaMemcpyHostToDevice, st));
        const double tol2 = tol * tol;
        DRF_CUDA(cudaMemcpyAsync(scal + S_TOL2, &tol2, sizeof(double), cudaMemcpyHostToDevice, st));
        LevelDev L;
        L.n = g->nx; L.nd = nd; L.K = K; L.rho = rho; L.binv = nullptr;
        L.lam_eps = g->lambda * g->ridge_epsilon;
        PcgCtl c;
        c.sc = scal; c.stop = ctl; c.iters = ctl + 1; c.maxit = ctl + 2; c.part = part;
        const unsigned nb = nblk(n), np = 1024;
        bz_apply_kernel<<<nb, BS, 0, st>>>(L, d_x, d_b, r, 1, nullptr, nullptr);
        DRF_LAUNCHED();
        dot_kernel<<<np, BS, 0, st>>>(n, d_b, d_b, part, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, st>>>(part, (int)np, scal + S_BB);
        DRF_LAUNCHED();
        dot_kernel<<<np, BS, 0, st>>>(n, r, r, part, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, st>>>(part, (int)np, scal + S_RR);
        DRF_LAUNCHED();
        jacobi_kernel<<<nb, BS, 0, st>>>(L, r, z, nullptr);
        DRF_LAUNCHED();
        dot_kernel<<<np, BS, 0, st>>>(n, r, z, part, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, st>>>(part, (int)np, scal + S_RZ);
        DRF_LAUNCHED();
        p_update_kernel<<<np, BS, 0, st>>>(n, c, z, p, 1);
        DRF_LAUNCHED();
        double sc[S_NSLOT];
        DRF_CUDA(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
        DRF_CUDA(cudaStreamSynchronize(st));
        int cl[3] = {0, 0, maxit};
        if (sc[S_RR] > tol2 * sc[S_BB] && maxit > 0) {
            while (true) {
                bz_apply_kernel<<<nb, BS, 0, st>>>(L, p, nullptr, q, 0, part, ctl);
                DRF_LAUNCHED();
                alpha_kernel<<<1, BS, 0, st>>>(c, (int)nb);
                DRF_LAUNCHED();
                xr_update_kernel<<<np, BS, 0, st>>>(n, c, p, q, d_x, r);
                DRF_LAUNCHED();
                conv_kernel<<<1, BS, 0, st>>>(c, (int)np);
                DRF_LAUNCHED();
                jacobi_kernel<<<nb, BS, 0, st>>>(L, r, z, ctl);
                DRF_LAUNCHED();
                dot_kernel<<<np, BS, 0, st>>>(n, r, z, part, ctl);
                DRF_LAUNCHED();
                beta_kernel<<<1, BS, 0, st>>>(c, (int)np);
                DRF_LAUNCHED();
                p_update_kernel<<<np, BS, 0, st>>>(n, c, z, p, 0);
                DRF_LAUNCHED();
                DRF_CUDA(cudaMemcpyAsync(cl, ctl, sizeof(cl), cudaMemcpyDeviceToHost, st));
                DRF_CUDA(cudaStreamSynchronize(st));
                if (cl[0] || cl[1] >= maxit) break;
            }
            DRF_CUDA(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
            DRF_CUDA(cudaStreamSynchronize(st));
        }
        *iters = cl[1];
        *relres = sc[S_BB] > 0 ? std::sqrt(sc[S_RR] / sc[S_BB]) : 0.0;
        DRF_CHECK(std::isfinite(sc[S_RR]), DRF_E_NONFINITE, "PCG diverged (non-finite residual)");
    });
}

}  // extern "C"
