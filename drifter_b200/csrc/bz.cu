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
#include <cstdlib>
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
// color steps with at least this many elements use one thread per element, smaller ones one
// thread per dof
constexpr int64_t ELEM_THREAD_MIN_ELEMS = 65536;
inline unsigned nblk(int64_t n) { return (unsigned)((n + BS - 1) / BS); }

// asynchronous 8-byte global -> shared copy (zero fill when !valid; src must still be a
// valid address then, it is not read); every copy of a thread completes at cp_async_wait_all
__device__ __forceinline__ void cp_async8(double *smem_dst, const double *gsrc, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

struct LevelDev {
    int n, nd;
    const double *K;     // 256, transposed: K[k * 16 + a] = K_ak (lanes of one row read one bank each)
    const double *rho;   // nd
    const double *binv;  // 9 x 256, each block transposed like K
    double lam_eps;
};

__device__ __forceinline__ double ridge(const LevelDev &L, int gi, int gj) {
    return L.lam_eps * L.rho[gi] * L.rho[gj];
}

// (Q_l x) at control point (gi, gj): gather over the <= 2 x 2 elements containing it
__device__ __forceinline__ double row_apply(const LevelDev &L, const double *K, const double *x,
                                            int gi, int gj) {
    double s = ridge(L, gi, gj) * x[gi + (int64_t)L.nd * gj];
    const int ex1 = min(gi / 3, L.n - 1), ey1 = min(gj / 3, L.n - 1);
    const int ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
    const int ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
    for (int ey = ey0; ey <= ey1; ++ey)
        for (int ex = ex0; ex <= ex1; ++ex) {
            const int a = (gi - 3 * ex) + 4 * (gj - 3 * ey);
            const double *xr = x + (3 * ex) + (int64_t)L.nd * (3 * ey);
            const double *Kc = K + a;
#pragma unroll
            for (int bj = 0; bj < 4; ++bj)
#pragma unroll
                for (int bi = 0; bi < 4; ++bi) s += Kc[16 * (bi + 4 * bj)] * xr[bi + (int64_t)L.nd * bj];
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

// ---------------------------------------------------------------- operator apply, tiled
// y = Q x (mode 0, with the block's partial of x.y in part[block]) or y = b - Q x (mode 1).
// One thread per element computes the dofs the element owns (local ai, aj < 3; ai = 3 / aj = 3
// too on the last element column / row of the grid) as its contributions plus those of the
// elements left, below and diagonally below-left of it; x is staged in shared memory over the
// tile and a one-element margin below and left, K (transposed) beside it, and the owned dofs
// are written row by row from a shared staging tile.
template <int TI, int TJ>
struct ApplyTile {
    static constexpr int WX = 3 * TI + 4, WY = 3 * TJ + 4;  // x: 3 TI bx - 3 .. 3 TI (bx + 1)
    static constexpr int OX = 3 * TI + 1, OY = 3 * TJ + 1;  // owned dofs (+ the grid's last)
};

template <int TI, int TJ>
__global__ void __launch_bounds__(TI *TJ) bz_apply_tile_kernel(LevelDev L, const double *__restrict__ x,
                                                               const double *__restrict__ b,
                                                               double *__restrict__ y, int mode,
                                                               double *__restrict__ part,
                                                               const int *__restrict__ stop) {
    using T = ApplyTile<TI, TJ>;
    __shared__ __align__(16) double Ks[256];
    __shared__ double xt[T::WY * T::WX];
    __shared__ double ys[T::OY * T::OX];
    __shared__ double red[TI * TJ / 32];
    if (stop && *stop) return;
    for (int i = threadIdx.x; i < 256; i += TI * TJ) cp_async8(Ks + i, L.K + i, true);
    const int X0 = 3 * TI * (int)blockIdx.x - 3, Y0 = 3 * TJ * (int)blockIdx.y - 3;
    for (int idx = threadIdx.x; idx < T::WX * T::WY; idx += TI * TJ) {
        const int u = idx % T::WX, v = idx / T::WX;
        const int gi = X0 + u, gj = Y0 + v;
        const bool in = gi >= 0 && gi < L.nd && gj >= 0 && gj < L.nd;
        cp_async8(xt + idx, in ? x + gi + (int64_t)L.nd * gj : x, in);
    }
    cp_async_wait_all();
    __syncthreads();
    const int ti = threadIdx.x % TI, tj = threadIdx.x / TI;
    const int ex = TI * blockIdx.x + ti, ey = TJ * blockIdx.y + tj;
    if (ex < L.n && ey < L.n) {
        // x of element (ex - dx, ey - dy), dx, dy in {0, 1}: tile origin (3 ti + 3 - 3 dx, 3 tj + 3 - 3 dy)
        const double *x0 = xt + (3 * tj + 3) * T::WX + 3 * ti + 3;
        double s[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) s[a] = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const double xk = x0[(k / 4) * T::WX + k % 4];
            const double *Kk = Ks + 16 * k;
#pragma unroll
            for (int aj = 0; aj < 3; ++aj)
#pragma unroll
                for (int ai = 0; ai < 3; ++ai) s[ai + 3 * aj] += Kk[ai + 4 * aj] * xk;
        }
        const bool hx = ex > 0, hy = ey > 0;
        if (hx) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const double xk = x0[(k / 4) * T::WX + k % 4 - 3];
#pragma unroll
                for (int aj = 0; aj < 3; ++aj) s[3 * aj] += Ks[16 * k + 3 + 4 * aj] * xk;
            }
        }
        if (hy) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const double xk = x0[(k / 4 - 3) * T::WX + k % 4];
#pragma unroll
                for (int ai = 0; ai < 3; ++ai) s[ai] += Ks[16 * k + ai + 12] * xk;
            }
        }
        if (hx && hy) {
#pragma unroll
            for (int k = 0; k < 16; ++k) s[0] += Ks[16 * k + 15] * x0[(k / 4 - 3) * T::WX + k % 4 - 3];
        }
        double *y0 = ys + (3 * tj) * T::OX + 3 * ti;
#pragma unroll
        for (int aj = 0; aj < 3; ++aj)
#pragma unroll
            for (int ai = 0; ai < 3; ++ai) y0[aj * T::OX + ai] = s[ai + 3 * aj];
        // the grid's last column / row of dofs: this element and the one below / left of it
        if (ex == L.n - 1) {
            double t[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const double xk = x0[(k / 4) * T::WX + k % 4];
#pragma unroll
                for (int aj = 0; aj < 4; ++aj) t[aj] += Ks[16 * k + 3 + 4 * aj] * xk;
            }
            if (hy)
                for (int k = 0; k < 16; ++k) t[0] += Ks[16 * k + 15] * x0[(k / 4 - 3) * T::WX + k % 4];
#pragma unroll
            for (int aj = 0; aj < 3; ++aj) y0[aj * T::OX + 3] = t[aj];
            if (ey == L.n - 1) y0[3 * T::OX + 3] = t[3];
        }
        if (ey == L.n - 1) {
            double t[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const double xk = x0[(k / 4) * T::WX + k % 4];
#pragma unroll
                for (int ai = 0; ai < 3; ++ai) t[ai] += Ks[16 * k + ai + 12] * xk;
            }
            if (hx)
                for (int k = 0; k < 16; ++k) t[0] += Ks[16 * k + 15] * x0[(k / 4) * T::WX + k % 4 - 3];
#pragma unroll
            for (int ai = 0; ai < 3; ++ai) y0[3 * T::OX + ai] = t[ai];
        }
    }
    __syncthreads();
    double dot = 0.0;
    for (int idx = threadIdx.x; idx < T::OX * T::OY; idx += TI * TJ) {
        const int u = idx % T::OX, v = idx / T::OX;
        const int gi = 3 * TI * blockIdx.x + u, gj = 3 * TJ * blockIdx.y + v;
        if (gi >= L.nd || gj >= L.nd) continue;
        if ((u == 3 * TI && gi != L.nd - 1) || (v == 3 * TJ && gj != L.nd - 1)) continue;
        const double xv = xt[(v + 3) * T::WX + u + 3];
        const double q = ys[idx] + L.lam_eps * L.rho[gi] * L.rho[gj] * xv;
        const int64_t I = gi + (int64_t)L.nd * gj;
        if (mode == 0) {
            y[I] = q;
            dot += xv * q;
        } else {
            y[I] = b[I] - q;
        }
    }
    if (part) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = dot;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < TI * TJ / 32; ++w) t += red[w];
            part[blockIdx.x + gridDim.x * blockIdx.y] = t;
        }
    }
}

__device__ __forceinline__ int elem_class(int e, int n) { return e == 0 ? 0 : (e == n - 1 ? 2 : 1); }

// ---------------------------------------------------------------- per-dof bodies
// Shared by the grid-wide kernels (one work item per thread) and the single-CTA coarse V-cycle
// (work items strided over the block). x, b, r may be written earlier in the same launch by
// other threads of the block, so none of them is declared __restrict__ here.

// colored Schwarz residual at dof a of the ce-th element of one color
__device__ __forceinline__ void schwarz_res_item(const LevelDev &L, const double *K, int color,
                                                 const double *x, const double *b, double *r,
                                                 int64_t t) {
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2;
    const int ce = (int)(t / 16), a = (int)(t % 16);
    const int ex = px + 2 * (ce % ncx), ey = py + 2 * (ce / ncx);
    const int gi = 3 * ex + a % 4, gj = 3 * ey + a / 4;
    const int64_t I = gi + (int64_t)L.nd * gj;
    r[I] = b[I] - row_apply(L, K, x, gi, gj);
}

// x_e += Binv_class(e) r_e at dof a of the ce-th element of one color
__device__ __forceinline__ void schwarz_upd_item(const LevelDev &L, int color, const double *r,
                                                 double *x, int64_t t) {
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2;
    const int ce = (int)(t / 16), a = (int)(t % 16);
    const int ex = px + 2 * (ce % ncx), ey = py + 2 * (ce / ncx);
    const double *Bi = L.binv + (elem_class(ex, L.n) + 3 * elem_class(ey, L.n)) * 256 + a;
    const double *re = r + 3 * ex + (int64_t)L.nd * (3 * ey);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += Bi[16 * k] * re[(k % 4) + (int64_t)L.nd * (k / 4)];
    x[(3 * ex + a % 4) + (int64_t)L.nd * (3 * ey + a / 4)] += s;
}

// 1D transfer between a level of nc elements and its refinement, as tables built on the host
// from the Bezier subdivision (the uniform grid is square, one table serves both directions):
// prolongation row of fine index f: coarse fc0[f] .. fc0[f] + 3 with weights fw[4 f ..];
// restriction row of coarse index c (the transpose): fine cf0[c] .. cf0[c] + 7 with weights
// cw[8 c ..], zero where f does not touch c. Lanes of neighbouring indices read neighbouring
// table entries (no divergent constant-memory reads).
struct TransferDev {
    const int *fc0, *cf0;
    const double *fw, *cw;
    // row sums of the 1D restriction (non-null: R's rows scaled to sum to one where
    // |sum - 1| > 1e-10, as BezierMultigridPreconditioner::setup builds R,
    // src/bathymetry/bezier_multigrid_preconditioner.cpp:209-225)
    const double *rs;
};

// r_c = P^T r_f at coarse dof t (fine rows ascending, columns ascending within a row)
__device__ __forceinline__ void restrict_item(const TransferDev &T, int ndc, int ndf, const double *rf,
                                              double *rc, double *xc_zero, int64_t t) {
    const int ci = (int)(t % ndc), cj = (int)(t / ndc);
    const int fi0 = T.cf0[ci], fj0 = T.cf0[cj];
    const double *wx = T.cw + 8 * ci, *wy = T.cw + 8 * cj;
    double w[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) w[p] = wx[p];
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const double wq = wy[q];
        if (wq == 0.0) continue;
        const double *row = rf + fi0 + (int64_t)ndf * (fj0 + q);
        double sx = 0.0;
#pragma unroll
        for (int p = 0; p < 8; ++p)
            if (w[p] != 0.0) sx += w[p] * row[p];
        s += wq * sx;
    }
    if (T.rs) {
        const double scale = T.rs[ci] * T.rs[cj];
        if (fabs(scale) > 1e-14 && fabs(scale - 1.0) > 1e-10) s /= scale;
    }
    rc[t] = s;
    xc_zero[t] = 0.0;
}

// x_f += P e_c at fine dof t
__device__ __forceinline__ void prolong_item(const TransferDev &T, int ndc, int ndf, const double *ec,
                                             double *xf, int64_t t) {
    const int fi = (int)(t % ndf), fj = (int)(t / ndf);
    const int cx0 = T.fc0[fi], cy0 = T.fc0[fj];
    double wx[4], wy[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        wx[a] = T.fw[4 * fi + a];
        wy[a] = T.fw[4 * fj + a];
    }
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int a = 0; a < 4; ++a) s += wy[b] * wx[a] * ec[(cx0 + a) + (int64_t)ndc * (cy0 + b)];
    xf[t] += s;
}

__global__ void __launch_bounds__(BS) bz_restrict_kernel(TransferDev T, int ndc, int ndf,
                                                         const double *__restrict__ rf, double *rc,
                                                         double *xc_zero) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < (int64_t)ndc * ndc) restrict_item(T, ndc, ndf, rf, rc, xc_zero, t);
}

__global__ void __launch_bounds__(BS) bz_prolong_kernel(TransferDev T, int ndc, int ndf,
                                                        const double *__restrict__ ec, double *xf) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < (int64_t)ndf * ndf) prolong_item(T, ndc, ndf, ec, xf, t);
}

// ---------------------------------------------------------------- fine-level Schwarz sweep
// One color step of the multiplicative Schwarz smoother on a level with many elements, split
// in two launches so that every residual of the color is formed before any update (Jacobi
// within a color, as the per-dof form):
//   bz_color_solve_kernel: one thread per element e of the color; z_e = Binv_class(e)(b - Q x)_e
//     from x staged in shared memory (the 3x3-element neighbourhood of every element of the
//     tile), K and the interior block inverse staged beside it (warp-wide broadcast reads);
//   bz_color_update_kernel: x_e += z_e.
// Shared tile: columns 3(px + 2 TI bx) - 3 .. + 6 TI + 3 and the same in y; column u is stored
// at u + u / 6, so that lanes six columns apart (neighbouring elements of one color) hit
// distinct bank pairs.
template <int TI, int TJ>
struct SchwarzTile {
    static constexpr int WX = 6 * TI + 4, WY = 6 * TJ + 4;
    static constexpr int WXP = WX + WX / 6 + 1;
    static constexpr int ZS = 17;  // padded row of the per-element staging
    static constexpr size_t smem_bytes() { return (size_t)(512 + WY * WXP) * sizeof(double); }
    static_assert(TI * TJ * ZS <= WX * WY, "staging must fit in the tile");
};

template <int TI, int TJ>
__global__ void __launch_bounds__(TI *TJ) bz_color_solve_kernel(LevelDev L, int color,
                                                                const double *__restrict__ x,
                                                                const double *__restrict__ b,
                                                                double *__restrict__ zc) {
    using T = SchwarzTile<TI, TJ>;
    extern __shared__ __align__(16) double smem[];
    double *Ks = smem, *Bs = smem + 256, *tile = smem + 512;
    for (int i = threadIdx.x; i < 256; i += TI * TJ) {
        cp_async8(Ks + i, L.K + i, true);
        cp_async8(Bs + i, L.binv + 4 * 256 + i, true);
    }
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2, ncy = (L.n - py + 1) / 2;
    const int X0 = 3 * (px + 2 * TI * (int)blockIdx.x) - 3;
    const int Y0 = 3 * (py + 2 * TJ * (int)blockIdx.y) - 3;
    for (int idx = threadIdx.x; idx < T::WX * T::WY; idx += TI * TJ) {
        const int u = idx % T::WX, v = idx / T::WX;
        const int gi = X0 + u, gj = Y0 + v;
        const bool in = gi >= 0 && gi < L.nd && gj >= 0 && gj < L.nd;
        cp_async8(tile + v * T::WXP + u + u / 6, in ? x + gi + (int64_t)L.nd * gj : x, in);
    }
    const int ti = threadIdx.x % TI, tj = threadIdx.x / TI;
    const int i = blockIdx.x * TI + ti, j = blockIdx.y * TJ + tj;
    const bool valid = i < ncx && j < ncy;
    const int ex = px + 2 * i, ey = py + 2 * j;
    // this element's right-hand side, in flight while the tile arrives
    double bv[16];
#pragma unroll
    for (int a = 0; a < 16; ++a)
        bv[a] = valid ? b[(3 * ex + a % 4) + (int64_t)L.nd * (3 * ey + a / 4)] : 0.0;
    cp_async_wait_all();
    __syncthreads();
    // element origin at tile column 6 ti + 3, row 6 tj + 3; local column c >= 0 from 6 ti lies
    // at 7 ti + c + c / 6
    const double *tl = tile + (6 * tj) * T::WXP + 7 * ti;
    double s[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) s[a] = 0.0;
    if (valid) {
        double rx[4], ry[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            rx[q] = L.rho[3 * ex + q];
            ry[q] = L.rho[3 * ey + q];
        }
#pragma unroll
        for (int a = 0; a < 16; ++a) {
            const int c = 3 + a % 4, rr = 3 + a / 4;
            s[a] = L.lam_eps * rx[a % 4] * ry[a / 4] * tl[rr * T::WXP + c + c / 6];
        }
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (ex + dx < 0 || ex + dx >= L.n || ey + dy < 0 || ey + dy >= L.n) continue;
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const int c = 3 + 3 * dx + k % 4, rr = 3 + 3 * dy + k / 4;
                    const double xk = tl[rr * T::WXP + c + c / 6];
                    const double *Kk = Ks + 16 * k;
                    // rows of the neighbour that are dofs of this element
#pragma unroll
                    for (int aj2 = 0; aj2 < 4; ++aj2)
#pragma unroll
                        for (int ai2 = 0; ai2 < 4; ++ai2) {
                            const int ai = ai2 + 3 * dx, aj = aj2 + 3 * dy;
                            if (ai < 0 || ai > 3 || aj < 0 || aj > 3) continue;
                            s[ai + 4 * aj] += Kk[ai2 + 4 * aj2] * xk;
                        }
                }
            }
    }
    __syncthreads();  // tile reads done: the tile now stages per-element vectors
    double *zs = tile;
    if (valid) {
        double r[16], z[16];
#pragma unroll
        for (int a = 0; a < 16; ++a) {
            r[a] = bv[a] - s[a];
            z[a] = 0.0;
        }
        const int cls = elem_class(ex, L.n) + 3 * elem_class(ey, L.n);
        const double *Bi = cls == 4 ? Bs : L.binv + cls * 256;
#pragma unroll
        for (int k = 0; k < 16; ++k)
#pragma unroll
            for (int a = 0; a < 16; ++a) z[a] += Bi[k * 16 + a] * r[k];
#pragma unroll
        for (int a = 0; a < 16; ++a) zs[threadIdx.x * T::ZS + a] = z[a];
    }
    __syncthreads();
    // z of element (i, j) of the color at zc[(i + ncx j) * 16 + a]
    for (int idx = threadIdx.x; idx < TI * TJ * 16; idx += TI * TJ) {
        const int el = idx / 16, a = idx % 16;
        const int ii = blockIdx.x * TI + el % TI, jj = blockIdx.y * TJ + el / TI;
        if (ii < ncx && jj < ncy) zc[((int64_t)ii + (int64_t)ncx * jj) * 16 + a] = zs[el * T::ZS + a];
    }
}

// The same color step with one thread per dof of an element (16 lanes per element): each lane
// forms the residual of its row from the shared x tile (gathering over the one, two or four
// elements that contain the dof), the element's residual is exchanged through shared memory and
// each lane forms one row of Binv_class(e) r_e. Shorter per-thread work than the element-per-
// thread form; the tile is (6 TI + 4) x (6 TJ + 4) control points, unpadded.
template <int TI, int TJ>
struct SchwarzDofTile {
    static constexpr int WX = 6 * TI + 4, WY = 6 * TJ + 4, NT = TI * TJ * 16;
    static constexpr size_t smem_bytes() { return (size_t)(256 + WX * WY + TI * TJ * 17) * sizeof(double); }
};

template <int TI, int TJ>
__global__ void __launch_bounds__(TI *TJ * 16) bz_color_solve_dof_kernel(LevelDev L, int color,
                                                                         const double *__restrict__ x,
                                                                         const double *__restrict__ b,
                                                                         double *__restrict__ zc) {
    using T = SchwarzDofTile<TI, TJ>;
    extern __shared__ __align__(16) double smem[];
    double *Ks = smem, *xt = smem + 256, *rs = smem + 256 + T::WX * T::WY;
    for (int i = threadIdx.x; i < 256; i += T::NT) cp_async8(Ks + i, L.K + i, true);
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2, ncy = (L.n - py + 1) / 2;
    const int X0 = 3 * (px + 2 * TI * (int)blockIdx.x) - 3;
    const int Y0 = 3 * (py + 2 * TJ * (int)blockIdx.y) - 3;
    for (int idx = threadIdx.x; idx < T::WX * T::WY; idx += T::NT) {
        const int u = idx % T::WX, v = idx / T::WX;
        const int gi = X0 + u, gj = Y0 + v;
        const bool in = gi >= 0 && gi < L.nd && gj >= 0 && gj < L.nd;
        cp_async8(xt + idx, in ? x + gi + (int64_t)L.nd * gj : x, in);
    }
    const int el = threadIdx.x / 16, a = threadIdx.x % 16;
    const int ti = el % TI, tj = el / TI;
    const int i = blockIdx.x * TI + ti, j = blockIdx.y * TJ + tj;
    const bool valid = i < ncx && j < ncy;
    const int ex = px + 2 * i, ey = py + 2 * j;
    const int ai = a % 4, aj = a / 4;
    const int gi = 3 * ex + ai, gj = 3 * ey + aj;
    const double bv = valid ? b[gi + (int64_t)L.nd * gj] : 0.0;
    const double ridge = valid ? L.lam_eps * L.rho[gi] * L.rho[gj] : 0.0;
    cp_async_wait_all();
    __syncthreads();
    if (valid) {
        // element origin at tile (6 ti + 3, 6 tj + 3); the dof at (+ai, +aj)
        const int u = 6 * ti + 3 + ai, v = 6 * tj + 3 + aj;
        double s = ridge * xt[v * T::WX + u];
        const int dx0 = (ai == 0 && ex > 0) ? -1 : 0, dx1 = (ai == 3 && ex < L.n - 1) ? 1 : 0;
        const int dy0 = (aj == 0 && ey > 0) ? -1 : 0, dy1 = (aj == 3 && ey < L.n - 1) ? 1 : 0;
        for (int dy = dy0; dy <= dy1; ++dy)
            for (int dx = dx0; dx <= dx1; ++dx) {
                const int ar = (ai - 3 * dx) + 4 * (aj - 3 * dy);  // the dof's row in that element
                const double *xe = xt + (6 * tj + 3 + 3 * dy) * T::WX + 6 * ti + 3 + 3 * dx;
#pragma unroll
                for (int k = 0; k < 16; ++k) s += Ks[16 * k + ar] * xe[(k / 4) * T::WX + k % 4];
            }
        rs[el * 17 + a] = bv - s;
    }
    __syncthreads();
    if (valid) {
        const int cls = elem_class(ex, L.n) + 3 * elem_class(ey, L.n);
        const double *Bi = L.binv + cls * 256 + a;
        const double *re = rs + el * 17;
        double z = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) z += Bi[16 * k] * re[k];
        zc[((int64_t)i + (int64_t)ncx * j) * 16 + a] = z;
    }
}

__global__ void __launch_bounds__(BS) bz_color_update_kernel(LevelDev L, int color,
                                                             const double *__restrict__ zc,
                                                             double *__restrict__ x) {
    const int px = color & 1, py = color >> 1;
    const int ncx = (L.n - px + 1) / 2, ncy = (L.n - py + 1) / 2;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)ncx * ncy * 16) return;
    const int ce = (int)(t / 16), a = (int)(t % 16);
    const int ex = px + 2 * (ce % ncx), ey = py + 2 * (ce / ncx);
    x[(3 * ex + a % 4) + (int64_t)L.nd * (3 * ey + a / 4)] += zc[t];
}

// ---------------------------------------------------------------- coarse V-cycle, one CTA
// Levels 0..top of the hierarchy (the coarsest few, n <= COARSE_CTA_MAX_N elements per
// direction) in one launch, their x, b, r resident in shared memory: smoothing, residual,
// restriction, the dense coarsest solve and prolongation, phase after phase with block-wide
// barriers. Operators, ridge factors, block inverses and transfer tables are read-only and
// come through L1. b of level top is read from global memory at the start and x of level top
// written back at the end.
constexpr int COARSE_MAX_LEVELS = 8;
constexpr int COARSE_THREADS = 1024;
constexpr int COARSE_CTA_MAX_N = 16;
constexpr size_t COARSE_SMEM_MAX = 200 * 1024;

struct CoarseStack {
    int top, pre, post, nc2;
    int post_forward;  // post-smoothing in the pre-smoothing's colour order (reference V-cycle)
    LevelDev L[COARSE_MAX_LEVELS];
    TransferDev T[COARSE_MAX_LEVELS];  // T[l]: between levels l - 1 and l
    int off[COARSE_MAX_LEVELS];        // shared offset (doubles) of x_l; b_l, r_l follow
    const double *bin;                 // b of level top
    double *xout;                      // x of level top
    const double *xinit;               // initial x of level top (null: zero)
    const double *Cinv;
};

// shared doubles of the coarse stack for levels 0..top: K staging + x, b, r per level
inline size_t coarse_smem_doubles(const std::vector<int> &nd, int top) {
    size_t t = 256;
    for (int l = 0; l <= top; ++l) t += 3 * (size_t)nd[l] * nd[l];
    return t;
}

__device__ void coarse_smooth(const LevelDev &L, const double *K, double *x, const double *b,
                              double *r, bool forward) {
    for (int s = 0; s < 4; ++s) {
        const int color = forward ? s : 3 - s;
        const int px = color & 1, py = color >> 1;
        const int64_t work = (int64_t)((L.n - px + 1) / 2) * ((L.n - py + 1) / 2) * 16;
        for (int64_t t = threadIdx.x; t < work; t += blockDim.x) schwarz_res_item(L, K, color, x, b, r, t);
        __syncthreads();
        for (int64_t t = threadIdx.x; t < work; t += blockDim.x) schwarz_upd_item(L, color, r, x, t);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(COARSE_THREADS) bz_coarse_vcycle_kernel(CoarseStack S) {
    extern __shared__ __align__(16) double sm[];
    double *K = sm;
    auto X = [&](int l) { return sm + S.off[l]; };
    auto B = [&](int l) { return sm + S.off[l] + S.L[l].nd * S.L[l].nd; };
    auto R = [&](int l) { return sm + S.off[l] + 2 * S.L[l].nd * S.L[l].nd; };
    {
        const int n2 = S.L[S.top].nd * S.L[S.top].nd;
        double *xt = X(S.top), *bt = B(S.top);
        for (int i = threadIdx.x; i < n2; i += blockDim.x) {
            bt[i] = S.bin[i];
            xt[i] = S.xinit ? S.xinit[i] : 0.0;
        }
        __syncthreads();
    }
    for (int l = S.top; l >= 1; --l) {
        const LevelDev &L = S.L[l];
        for (int i = threadIdx.x; i < 256; i += blockDim.x) K[i] = L.K[i];
        __syncthreads();
        for (int it = 0; it < S.pre; ++it) coarse_smooth(L, K, X(l), B(l), R(l), true);
        const int nd2 = L.nd * L.nd;
        double *xl = X(l), *bl = B(l), *rl = R(l);
        for (int t = threadIdx.x; t < nd2; t += blockDim.x)
            rl[t] = bl[t] - row_apply(L, K, xl, t % L.nd, t / L.nd);
        __syncthreads();
        const LevelDev &C = S.L[l - 1];
        const int ndc2 = C.nd * C.nd;
        for (int t = threadIdx.x; t < ndc2; t += blockDim.x) restrict_item(S.T[l], C.nd, L.nd, rl, B(l - 1), X(l - 1), t);
        __syncthreads();
    }
    {
        const double *b0 = B(0);
        double *x0 = X(0);
        for (int i = threadIdx.x; i < S.nc2; i += blockDim.x) {
            double s = 0.0;
            for (int k = 0; k < S.nc2; ++k) s += S.Cinv[(int64_t)i * S.nc2 + k] * b0[k];
            x0[i] = s;
        }
        __syncthreads();
    }
    for (int l = 1; l <= S.top; ++l) {
        const LevelDev &L = S.L[l];
        const LevelDev &C = S.L[l - 1];
        for (int i = threadIdx.x; i < 256; i += blockDim.x) K[i] = L.K[i];
        const int nd2 = L.nd * L.nd;
        for (int t = threadIdx.x; t < nd2; t += blockDim.x) prolong_item(S.T[l], C.nd, L.nd, X(l - 1), X(l), t);
        __syncthreads();
        for (int it = 0; it < S.post; ++it) coarse_smooth(L, K, X(l), B(l), R(l), S.post_forward != 0);
    }
    {
        const int n2 = S.L[S.top].nd * S.L[S.top].nd;
        const double *xt = X(S.top);
        for (int i = threadIdx.x; i < n2; i += blockDim.x) S.xout[i] = xt[i];
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
enum { S_RZ = 0, S_PQ, S_ALPHA, S_RR, S_BETA, S_BB, S_TOL2, S_RZNEW, S_TMP, S_NSLOT };
// BezierMultigridPreconditioner's defaults for its apply (vcycle_tolerance, max_vcycles,
// include/bathymetry/bezier_multigrid_preconditioner.hpp:127-130)
constexpr double MG_REF_TOL = 1e-6;
constexpr int MG_REF_MAX_CYCLES = 100;
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
__global__ void __launch_bounds__(BS) xr_update_kernel(int64_t n, PcgCtl c, const double *__restrict__ p,
                                                       const double *__restrict__ q, double *__restrict__ x,
                                                       double *__restrict__ r) {
    __shared__ double red[BS];
    if (*c.stop) return;
    const double a = c.sc[S_ALPHA];
    double s = 0.0;
#pragma unroll 4
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
// x += alpha p, r -= alpha q and the Jacobi step z = r / d in one pass, with per-block partials
// of r.r (part) and r.z (part + gridDim.x). Same grid-stride loop and block reduction as
// xr_update_kernel followed by jacobi_diag_kernel and dot_kernel: the iterates are unchanged.
__global__ void __launch_bounds__(BS) xr_jacobi_kernel(int64_t n, PcgCtl c, const double *__restrict__ p,
                                                       const double *__restrict__ q, const double *__restrict__ d,
                                                       double *__restrict__ x, double *__restrict__ r,
                                                       double *__restrict__ z) {
    __shared__ double red[2][BS];
    if (*c.stop) return;
    const double a = c.sc[S_ALPHA];
    double s = 0.0, s2 = 0.0;
    // distinct arrays (restrict): the loads of later elements need not wait for earlier stores
#pragma unroll 4
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS) {
        x[t] += a * p[t];
        const double rn = r[t] - a * q[t];
        r[t] = rn;
        s += rn * rn;
        const double zn = rn / d[t];
        z[t] = zn;
        s2 += rn * zn;
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
        c.part[blockIdx.x] = red[0][0];
        c.part[gridDim.x + blockIdx.x] = red[1][0];
    }
}
// conv_kernel and beta_kernel in one CTA: r.r from part[0, nparts) (convergence, iteration
// count), r.z from part[zoff, zoff + nparts) (beta; zoff = 0 when z = r); beta is left as it was
// once the iteration converged, as beta_kernel returns early then
__global__ void conv_beta_kernel(PcgCtl c, int nparts, int zoff) {
    __shared__ double red[2][BS];
    if (*c.stop) return;
    double s = 0.0, s2 = 0.0;
    for (int i = threadIdx.x; i < nparts; i += BS) {
        s += c.part[i];
        s2 += c.part[zoff + i];
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
        c.sc[S_RR] = red[0][0];
        *c.iters += 1;
        if (!(red[0][0] > c.sc[S_TOL2] * c.sc[S_BB]) || *c.iters >= *c.maxit) {
            *c.stop = 1;
        } else {
            c.sc[S_BETA] = red[1][0] / c.sc[S_RZ];
            c.sc[S_RZ] = red[1][0];
        }
    }
}
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
__global__ void __launch_bounds__(BS) p_update_kernel(int64_t n, PcgCtl c, const double *__restrict__ z,
                                                      double *__restrict__ p, int init) {
    if (*c.stop) return;
    const double be = init ? 0.0 : c.sc[S_BETA];
#pragma unroll 4
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

// the finest level's diagonal of Q (as jacobi_kernel forms it), stored once per handle
__global__ void __launch_bounds__(BS) diag_kernel(LevelDev L, double *d) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)L.nd * L.nd) return;
    const int gi = (int)(t % L.nd), gj = (int)(t / L.nd);
    double v = ridge(L, gi, gj);
    const int ex1 = min(gi / 3, L.n - 1), ey1 = min(gj / 3, L.n - 1);
    const int ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
    const int ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
    for (int ey = ey0; ey <= ey1; ++ey)
        for (int ex = ex0; ex <= ex1; ++ex) {
            const int a = (gi - 3 * ex) + 4 * (gj - 3 * ey);
            v += L.K[a * 16 + a];
        }
    d[t] = v;
}

// z = r / d with the stored diagonal (the same division as jacobi_kernel)
__global__ void __launch_bounds__(BS) jacobi_diag_kernel(int64_t n, const double *d, const double *r, double *z,
                                                         const int *stop) {
    if (stop && *stop) return;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) z[t] = r[t] / d[t];
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

// ---------------------------------------------------------------- C1 edge constraints
// Row (edge, q) of A: continuity of the normal derivative at Gauss point t_q of an interior
// edge, the derivative of each element at the shared edge taken from its Bernstein form and
// scaled by 1 / h: (3 / h) sum_j B_j(t_q) (2 x_line - x_line-1 - x_line+1) over the 4 control
// points along the edge (CGCubicBezierDofManager::build_edge_derivative_constraints,
// src/bathymetry/cg_cubic_bezier_dof_manager.cpp:319; coefficients / scale as in
// assemble_A_edge_free, src/bathymetry/cg_cubic_bezier_bathymetry_smoother.cpp:798).
// Row order: edges between (ex, ey) and (ex + 1, ey) first, ((ey (n - 1) + ex) ng + q), then
// edges between (ex, ey) and (ex, ey + 1), n (n - 1) ng + ((ey n + ex) ng + q).
constexpr int CONS_MAX_NG = 8;
struct ConsDev {
    int n, nd, ng;
    double sx, sy;                 // 3 / dx, 3 / dy
    double Bw[CONS_MAX_NG][4];     // B_j(t_q)
};

__global__ void __launch_bounds__(BS) bz_cons_apply_kernel(ConsDev C, const double *__restrict__ x,
                                                           double *__restrict__ y) {
    const int64_t nv = (int64_t)C.n * (C.n - 1) * C.ng;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 2 * nv) return;
    double s = 0.0;
    if (t < nv) {
        const int q = (int)(t % C.ng), e = (int)(t / C.ng);
        const int ex = e % (C.n - 1), ey = e / (C.n - 1);
        const double *g = x + (3 * ex + 2) + (int64_t)C.nd * (3 * ey);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double *r = g + (int64_t)C.nd * j;
            s += C.Bw[q][j] * (2.0 * r[1] - r[0] - r[2]);
        }
        y[t] = C.sx * s;
    } else {
        const int64_t u = t - nv;
        const int q = (int)(u % C.ng), e = (int)(u / C.ng);
        const int ex = e % C.n, ey = e / C.n;
        const double *g = x + 3 * ex + (int64_t)C.nd * (3 * ey + 2);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            s += C.Bw[q][i] * (2.0 * g[i + C.nd] - g[i] - g[i + 2 * (int64_t)C.nd]);
        y[t] = C.sy * s;
    }
}

// out = A^T lam (base == nullptr) or out = base - A^T lam, gathered per control point
__global__ void __launch_bounds__(BS) bz_cons_applyT_kernel(ConsDev C, const double *__restrict__ lam,
                                                            const double *__restrict__ base,
                                                            double *__restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)C.nd * C.nd) return;
    const int gi = (int)(t % C.nd), gj = (int)(t / C.nd);
    const int64_t nv = (int64_t)C.n * (C.n - 1) * C.ng;
    // the edge line (interior) whose 3-point stencil covers index g, and the stencil weight
    auto line = [&](int g, int &w) {
        const int r = g % 3;
        int e;
        if (r == 2) { e = (g - 2) / 3; w = -1; }
        else if (r == 0) { e = g / 3 - 1; w = 2; }
        else { e = g >= 4 ? (g - 4) / 3 : -1; w = -1; }
        return (e >= 0 && e <= C.n - 2) ? e : -1;
    };
    double s = 0.0;
    int w;
    const int lx = line(gi, w);
    if (lx >= 0) {
        const int ey1 = min(gj / 3, C.n - 1), ey0 = (gj % 3 == 0 && gj > 0) ? gj / 3 - 1 : ey1;
        double a = 0.0;
        for (int ey = ey0; ey <= ey1; ++ey) {
            const int j = gj - 3 * ey;
            const double *l = lam + ((int64_t)ey * (C.n - 1) + lx) * C.ng;
            for (int q = 0; q < C.ng; ++q) a += C.Bw[q][j] * l[q];
        }
        s += C.sx * w * a;
    }
    const int ly = line(gj, w);
    if (ly >= 0) {
        const int ex1 = min(gi / 3, C.n - 1), ex0 = (gi % 3 == 0 && gi > 0) ? gi / 3 - 1 : ex1;
        double a = 0.0;
        for (int ex = ex0; ex <= ex1; ++ex) {
            const int i = gi - 3 * ex;
            const double *l = lam + nv + ((int64_t)ly * C.n + ex) * C.ng;
            for (int q = 0; q < C.ng; ++q) a += C.Bw[q][i] * l[q];
        }
        s += C.sy * w * a;
    }
    out[t] = base ? base[t] - s : s;
}

// lam += a p ; r -= a q
__global__ void __launch_bounds__(BS) cg_update_kernel(int64_t n, double a, const double *__restrict__ p,
                                                       const double *__restrict__ q, double *lam, double *r) {
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS) {
        lam[t] += a * p[t];
        r[t] -= a * q[t];
    }
}

// p = r + beta p
__global__ void __launch_bounds__(BS) xpay_kernel(int64_t n, double beta, const double *__restrict__ r,
                                                  double *p) {
    for (int64_t t = blockIdx.x * (int64_t)BS + threadIdx.x; t < n; t += (int64_t)gridDim.x * BS)
        p[t] = r[t] + beta * p[t];
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

namespace drf {
namespace {
// AdaptiveCGCubicBezierSmoother::compute_element_l2_error
// (src/bathymetry/adaptive_cg_cubic_bezier_smoother.cpp:100) for every element at once: one
// warp per element evaluates the bicubic Bezier patch (Bernstein basis, the element's 16
// control points, dof i + 4j) at the ng x ng Gauss-Legendre points of [0, 1]^2, squares the
// misfit to the data sampled there, and reduces sqrt(sum w_i w_j diff^2 * dx dy).
__global__ void __launch_bounds__(256) bz_elem_error_kernel(int nx, int ny, int ng, const double *__restrict__ x,
                                                            const double *__restrict__ zd,
                                                            const double *__restrict__ gq, double area,
                                                            double *__restrict__ l2, double *__restrict__ nrm) {
    const int64_t e = (int64_t)blockIdx.x * 8 + threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (e >= (int64_t)nx * ny) return;
    const int ex = (int)(e % nx), ey = (int)(e / nx), stride = 3 * nx + 1;
    double c[16];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) c[i + 4 * j] = x[(size_t)(3 * ex + i) + (size_t)stride * (3 * ey + j)];
    const int ng2 = ng * ng;
    double acc = 0.0;
    for (int q = lane; q < ng2; q += 32) {
        const int qi = q % ng, qj = q / ng;
        const double u = gq[qi], v = gq[qj], w = gq[ng + qi] * gq[ng + qj];
        const double u1 = 1.0 - u, v1 = 1.0 - v;
        const double bu[4] = {u1 * u1 * u1, 3.0 * u * u1 * u1, 3.0 * u * u * u1, u * u * u};
        const double bv[4] = {v1 * v1 * v1, 3.0 * v * v1 * v1, 3.0 * v * v * v1, v * v * v};
        double z = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double r = 0.0;
#pragma unroll
            for (int i = 0; i < 4; ++i) r += c[i + 4 * j] * bu[i];
            z += r * bv[j];
        }
        const double diff = zd[e * ng2 + q] - z;
        acc += w * diff * diff;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        const double err = sqrt(acc * area);
        l2[e] = err;
        if (nrm) nrm[e] = err / sqrt(area);
    }
}
}  // namespace
}  // namespace drf

struct drf_bz {
    BzSetup H;  // host-side setup (element matrices, levels, transfers)
    cudaStream_t stream = nullptr, own = nullptr;
    int64_t ndof = 0;
    DevBuf<double> dat, Bq, b, bs, x, r, z, p, q, scal, part, mgbuf, coarse;  // b: assembled rhs, bs: rhs of the current solve
    DevBuf<double> diag;  // finest diagonal of Q for the Jacobi steps (formed at first use)
    DevBuf<int> ctl;
    struct Lv {
        DevBuf<double> K, rho, binv, x, b, r;
        DevBuf<int> fc0, cf0;     // transfer tables from the next coarser level (TransferDev)
        DevBuf<double> fw, cw, rs;
        int n = 0, nd = 0;
    };
    std::vector<Lv> lv;
    bool mg_ready = false;
    // color steps with at least this many elements use the element-per-thread Schwarz kernel
    // (environment DRF_BZ_ELEM_SMOOTHER_MIN overrides, read at drf_mg_setup)
    int64_t elem_min = ELEM_THREAD_MIN_ELEMS;
    drf_cnn *cnn = nullptr;
    double cnn_scale = 1.0;
    cudaGraphExec_t graph = nullptr;
    int graph_kind = -1, graph_chunk = 0;
    uint64_t graph_kernels = 0;  // kernel nodes of the chunk graph
    double cnn_ms[4][2] = {};     // the attached network's conv autotuning: ms per form per layer
    int cnn_form[4] = {};         // and the chosen form (0 mma.sync, 1 tcgen05)

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
    // the finest diagonal of Q, formed once per operator (outside any graph capture)
    void form_diag() {
        if (diag.n < (size_t)ndof) diag.alloc(ndof);
        diag_kernel<<<nblk(ndof), BS, 0, stream>>>(levdev(finest()), diag.p);
        DRF_LAUNCHED();
    }
    // transfer tables between level l - 1 and level l
    // ref: the reference's row-normalised restriction
    TransferDev tdev(int l, bool ref = false) const {
        TransferDev T;
        T.fc0 = lv[l].fc0.p; T.cf0 = lv[l].cf0.p; T.fw = lv[l].fw.p; T.cw = lv[l].cw.p;
        T.rs = ref ? lv[l].rs.p : nullptr;
        return T;
    }
    unsigned nparts() const { return 1024; }
    PcgCtl pctl() {
        PcgCtl c;
        c.sc = scal.p; c.stop = ctl.p; c.iters = ctl.p + 1; c.maxit = ctl.p + 2; c.part = part.p;
        return c;
    }

    // y = Q x (mode 0, per-tile partials of x.y in pt) or y = b - Q x (mode 1) on level l;
    // returns the number of partials written
    int apply(int l, const double *xin, const double *bin, double *yout, int mode, double *pt,
              const int *stop) {
        constexpr int TI = 32, TJ = 8;
        const LevelDev L = levdev(l);
        const dim3 grid((unsigned)((L.n + TI - 1) / TI), (unsigned)((L.n + TJ - 1) / TJ));
        bz_apply_tile_kernel<TI, TJ><<<grid, TI * TJ, 0, stream>>>(L, xin, bin, yout, mode, pt, stop);
        DRF_LAUNCHED();
        return (int)(grid.x * grid.y);
    }

    // z = M r for the given preconditioner kind (enqueued on stream)
    void precondition(int kind, const double *rin, double *zout, const int *stop) {
        const int L = finest();
        const int64_t n = ndof;
        if (kind == 0) {
            copy_kernel<<<nblk(n), BS, 0, stream>>>(n, rin, zout, stop);
            DRF_LAUNCHED();
        } else if (kind == 1) {
            jacobi_diag_kernel<<<nblk(n), BS, 0, stream>>>(n, diag.p, rin, zout, stop);
            DRF_LAUNCHED();
        } else if (kind == 3) {
            // Jacobi base (positive definite: a descent direction for any residual) plus the
            // learned correction of the error it leaves, formed in the network's output pass
            cnn_precondition(cnn_net(cnn), stream, lv[L].n, rin, scal.p + S_RR, cnn_scale, zout, 1,
                             stop, diag.p);
        } else if (kind == 4) {
            // the reference's apply: V-cycles to its default tolerance (host-driven; never in a graph)
            mg_apply_reference(rin, zout, MG_REF_TOL, MG_REF_MAX_CYCLES, nullptr);
        } else {
            vcycle(rin, zout);
        }
    }

    // one flexible-CG iteration with the reference multigrid apply (kind 4), host-driven:
    // returns false once converged (or at maxit)
    bool pcg_iteration_reference() {
        const int Lf = finest();
        PcgCtl c = pctl();
        const int na = apply(Lf, p.p, nullptr, q.p, 0, part.p, c.stop);
        alpha_kernel<<<1, BS, 0, stream>>>(c, na);
        DRF_LAUNCHED();
        xr_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, p.p, q.p, x.p, r.p);
        DRF_LAUNCHED();
        conv_kernel<<<1, BS, 0, stream>>>(c, (int)nparts());
        DRF_LAUNCHED();
        int cl[3] = {0, 0, 0};
        DRF_CUDA(cudaMemcpyAsync(cl, ctl.p, sizeof(cl), cudaMemcpyDeviceToHost, stream));
        DRF_CUDA(cudaStreamSynchronize(stream));
        if (cl[0] || cl[1] >= cl[2]) return false;
        mg_apply_reference(r.p, z.p, MG_REF_TOL, MG_REF_MAX_CYCLES, nullptr);
        // flexible CG: z.r and z.q partials side by side for beta = -(z.q)/(p.q)
        dot_kernel<<<nparts(), BS, 0, stream>>>(ndof, z.p, r.p, part.p, nullptr);
        DRF_LAUNCHED();
        dot_kernel<<<nparts(), BS, 0, stream>>>(ndof, z.p, q.p, part.p + nparts(), nullptr);
        DRF_LAUNCHED();
        beta_fcg_kernel<<<1, BS, 0, stream>>>(c, (int)nparts());
        DRF_LAUNCHED();
        p_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, z.p, p.p, 0);
        DRF_LAUNCHED();
        return true;
    }

    // one color step of the Schwarz smoother on a grid-wide level: z of every element of the
    // color into the level's residual buffer (free while smoothing), then x += z
    template <int TI, int TJ>
    void color_solve(int l, int color, int ncx, int ncy, const double *xl, const double *bl, double *zc) {
        const dim3 grid((unsigned)((ncx + TI - 1) / TI), (unsigned)((ncy + TJ - 1) / TJ));
        bz_color_solve_kernel<TI, TJ><<<grid, TI * TJ, SchwarzTile<TI, TJ>::smem_bytes(), stream>>>(
            levdev(l), color, xl, bl, zc);
        DRF_LAUNCHED();
    }

    template <int TI, int TJ>
    void color_solve_dof(int l, int color, int ncx, int ncy, const double *xl, const double *bl, double *zc) {
        const dim3 grid((unsigned)((ncx + TI - 1) / TI), (unsigned)((ncy + TJ - 1) / TJ));
        bz_color_solve_dof_kernel<TI, TJ><<<grid, TI * TJ * 16, SchwarzDofTile<TI, TJ>::smem_bytes(), stream>>>(
            levdev(l), color, xl, bl, zc);
        DRF_LAUNCHED();
    }

    void smooth(int l, double *xl, const double *bl, double *rl, bool forward) {
        const LevelDev L = levdev(l);
        for (int s = 0; s < 4; ++s) {
            const int color = forward ? s : 3 - s;
            const int px = color & 1, py = color >> 1;
            const int ncx = (L.n - px + 1) / 2, ncy = (L.n - py + 1) / 2;
            const int64_t nce = (int64_t)ncx * ncy;
            if (nce >= elem_min)
                color_solve<16, 4>(l, color, ncx, ncy, xl, bl, rl);
            else
                color_solve_dof<8, 2>(l, color, ncx, ncy, xl, bl, rl);
            bz_color_update_kernel<<<nblk(nce * 16), BS, 0, stream>>>(L, color, rl, xl);
            DRF_LAUNCHED();
        }
    }

    // highest level run by the single-CTA coarse V-cycle (level 0 at least)
    int coarse_top() const {
        std::vector<int> nd(lv.size());
        for (size_t l = 0; l < lv.size(); ++l) nd[l] = lv[l].nd;
        int top = 0;
        while (top + 1 < (int)lv.size() && top + 1 < COARSE_MAX_LEVELS && lv[top + 1].n <= COARSE_CTA_MAX_N &&
               coarse_smem_doubles(nd, top + 1) * sizeof(double) <= COARSE_SMEM_MAX)
            ++top;
        return top;
    }

    // one V-cycle z = M r, finest level uses rin/zout directly. This build's form (ref false):
    // z overwritten, R = P^T, post-smoothing in reverse colour order, an SPD preconditioner.
    // ref true: BezierMultigridPreconditioner::v_cycle as written
    // (src/bathymetry/bezier_multigrid_preconditioner.cpp:740-812), improving the z it is given:
    // row-normalised R, the same colour order before and after the coarse correction.
    void vcycle(const double *rin, double *zout, bool ref = false) {
        const int Lf = finest();
        std::vector<double *> X(lv.size()), B(lv.size()), R(lv.size());
        for (int l = 0; l < Lf; ++l) { X[l] = lv[l].x.p; B[l] = lv[l].b.p; R[l] = lv[l].r.p; }
        X[Lf] = zout; B[Lf] = const_cast<double *>(rin); R[Lf] = lv[Lf].r.p;
        if (!ref) {
            zero_kernel<<<nblk(ndof), BS, 0, stream>>>(ndof, zout, nullptr);
            DRF_LAUNCHED();
        }
        const int top = coarse_top();
        for (int l = Lf; l > top; --l) {
            for (int it = 0; it < H.pre; ++it) smooth(l, X[l], B[l], R[l], true);
            const int64_t nd2 = (int64_t)lv[l].nd * lv[l].nd;
            apply(l, X[l], B[l], R[l], 1, nullptr, nullptr);
            const int64_t ndc2 = (int64_t)lv[l - 1].nd * lv[l - 1].nd;
            bz_restrict_kernel<<<nblk(ndc2), BS, 0, stream>>>(tdev(l, ref), lv[l - 1].nd, lv[l].nd, R[l],
                                                              B[l - 1], X[l - 1]);
            DRF_LAUNCHED();
        }
        CoarseStack S;
        std::memset(&S, 0, sizeof(S));
        S.top = top; S.pre = H.pre; S.post = H.post;
        S.post_forward = ref ? 1 : 0;
        S.nc2 = lv[0].nd * lv[0].nd;
        S.Cinv = coarse.p;
        S.bin = B[top];
        S.xout = X[top];
        // the reference cycle improves the finest level's guess; coarser levels start from zero
        S.xinit = (ref && top == Lf) ? X[top] : nullptr;
        int off = 256;
        for (int l = 0; l <= top; ++l) {
            S.L[l] = levdev(l);
            if (l > 0) S.T[l] = tdev(l, ref);
            S.off[l] = off;
            off += 3 * lv[l].nd * lv[l].nd;
        }
        bz_coarse_vcycle_kernel<<<1, COARSE_THREADS, (size_t)off * sizeof(double), stream>>>(S);
        DRF_LAUNCHED();
        for (int l = top + 1; l <= Lf; ++l) {
            const int64_t nd2 = (int64_t)lv[l].nd * lv[l].nd;
            bz_prolong_kernel<<<nblk(nd2), BS, 0, stream>>>(tdev(l), lv[l - 1].nd, lv[l].nd, X[l - 1],
                                                            X[l]);
            DRF_LAUNCHED();
            for (int it = 0; it < H.post; ++it) smooth(l, X[l], B[l], R[l], ref);
        }
    }

    // ||v||^2 on the device, read back (synchronises the stream)
    double norm2(const double *v) {
        dot_kernel<<<nparts(), BS, 0, stream>>>(ndof, v, v, part.p, nullptr);
        DRF_LAUNCHED();
        reduce_kernel<<<1, BS, 0, stream>>>(part.p, (int)nparts(), scal.p + S_TMP);
        DRF_LAUNCHED();
        double v2 = 0.0;
        DRF_CUDA(cudaMemcpyAsync(&v2, scal.p + S_TMP, 8, cudaMemcpyDeviceToHost, stream));
        DRF_CUDA(cudaStreamSynchronize(stream));
        return v2;
    }

    // BezierMultigridPreconditioner::apply (src/bathymetry/bezier_multigrid_preconditioner.cpp:
    // 690-735): z = 0, then reference V-cycles until ||r - Q z|| < tol ||r|| or max_cycles (the
    // residual is checked on the host after each cycle). rin must not alias the level buffers.
    int mg_apply_reference(const double *rin, double *zout, double tol, int max_cycles, double *relres) {
        const int Lf = finest();
        zero_kernel<<<nblk(ndof), BS, 0, stream>>>(ndof, zout, nullptr);
        DRF_LAUNCHED();
        const double bb = norm2(rin);
        if (relres) *relres = 0.0;
        if (std::sqrt(bb) < 1e-30) return 0;
        const double tol_sq = tol * tol * bb;
        int cycle = 0;
        double rr = bb;
        for (; cycle < max_cycles; ++cycle) {
            vcycle(rin, zout, true);
            apply(Lf, zout, rin, lv[Lf].r.p, 1, nullptr, nullptr);
            rr = norm2(lv[Lf].r.p);
            if (rr < tol_sq) {
                ++cycle;
                break;
            }
        }
        if (relres) *relres = std::sqrt(rr / bb);
        return cycle;
    }

    // one PCG iteration (assumes r, z, p, rz set)
    void pcg_iteration(int kind) {
        const int Lf = finest();
        PcgCtl c = pctl();
        // q = Q p with partial p.q
        const int na = apply(Lf, p.p, nullptr, q.p, 0, part.p, c.stop);
        alpha_kernel<<<1, BS, 0, stream>>>(c, na);
        DRF_LAUNCHED();
        if (kind == 0 || kind == 1) {
            // z = r (none) or r / d (Jacobi) formed in the x, r update pass; the convergence
            // check and beta in one CTA
            if (kind == 1) xr_jacobi_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, p.p, q.p, diag.p, x.p, r.p, z.p);
            else xr_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, p.p, q.p, x.p, r.p);
            DRF_LAUNCHED();
            conv_beta_kernel<<<1, BS, 0, stream>>>(c, (int)nparts(), kind == 1 ? (int)nparts() : 0);
            DRF_LAUNCHED();
            p_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, kind == 1 ? z.p : r.p, p.p, 0);
            DRF_LAUNCHED();
            return;
        }
        xr_update_kernel<<<nparts(), BS, 0, stream>>>(ndof, c, p.p, q.p, x.p, r.p);
        DRF_LAUNCHED();
        conv_kernel<<<1, BS, 0, stream>>>(c, (int)nparts());
        DRF_LAUNCHED();
        if (kind == 3) {
            // z = r / d + the network's correction, with the partials of z.r and z.q (flexible
            // CG) from the same pass
            const int nb = cnn_precondition(cnn_net(cnn), stream, lv[Lf].n, r.p, scal.p + S_RR, cnn_scale, z.p, 1,
                                            c.stop, diag.p, q.p, part.p);
            beta_fcg_kernel<<<1, BS, 0, stream>>>(c, nb);
            DRF_LAUNCHED();
        } else {
            precondition(kind, r.p, z.p, c.stop);
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

// dynamic shared memory above the default 48 KB for the Schwarz tile kernels (per device, set
// outside any stream capture)
template <int TI, int TJ>
void allow_smem() {
    DRF_CUDA(cudaFuncSetAttribute(bz_color_solve_kernel<TI, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)SchwarzTile<TI, TJ>::smem_bytes()));
}

// 1D transfer tables between nc and 2 nc elements (layout of TransferDev): prolongation rows
// from the Bezier subdivision, fine index f in coarse element min(f / 6, nc - 1); restriction
// rows are their transpose
void transfer_tables(int nc, std::vector<int> &fc0, std::vector<double> &fw, std::vector<int> &cf0,
                     std::vector<double> &cw) {
    double S[2][16];
    bz_subdivision_1d(S);
    const int ndc = 3 * nc + 1, ndf = 6 * nc + 1;
    fc0.assign(ndf, 0);
    fw.assign((size_t)4 * ndf, 0.0);
    std::vector<int> lo(ndc, ndf), hi(ndc, -1);
    for (int f = 0; f < ndf; ++f) {
        const int E = std::min(f / 6, nc - 1), k = f - 6 * E;
        const double *row = k <= 3 ? &S[0][k * 4] : &S[1][(k - 3) * 4];
        fc0[f] = 3 * E;
        for (int a = 0; a < 4; ++a) {
            fw[4 * f + a] = row[a];
            if (row[a] != 0.0) {
                lo[3 * E + a] = std::min(lo[3 * E + a], f);
                hi[3 * E + a] = std::max(hi[3 * E + a], f);
            }
        }
    }
    cf0.assign(ndc, 0);
    cw.assign((size_t)8 * ndc, 0.0);
    for (int c = 0; c < ndc; ++c) {
        DRF_CHECK(hi[c] >= lo[c] && hi[c] - lo[c] < 8, DRF_E_INVALID, "restriction row wider than 8");
        cf0[c] = lo[c];
    }
    for (int f = 0; f < ndf; ++f)
        for (int a = 0; a < 4; ++a)
            if (fw[4 * f + a] != 0.0) {
                const int c = fc0[f] + a;
                cw[8 * c + (f - cf0[c])] = fw[4 * f + a];
            }
}

// count 16x16 blocks, each transposed (the device layout of K and of the block inverses)
std::vector<double> transposed16(const double *A, int count) {
    std::vector<double> T((size_t)count * 256);
    for (int c = 0; c < count; ++c)
        for (int a = 0; a < 16; ++a)
            for (int k = 0; k < 16; ++k) T[c * 256 + k * 16 + a] = A[c * 256 + a * 16 + k];
    return T;
}

template <class T, class V>
void up(DevBuf<T> &d, const V &v) {
    d.alloc(v.size());
    DRF_CUDA(cudaMemcpy(d.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}

void check_bz(drf_bz *h) { DRF_CHECK(h != nullptr, DRF_E_INVALID, "null smoother handle"); }

}  // namespace
}  // namespace drf

namespace drf {
namespace {

// PCG on Q x = bs from the x already on the device (bs, x set by the caller); returns the
// iterations done. Scalars (rr, bb) are left in scal.
int pcg_run(drf_bz *h, int kind, double tol, int maxit) {
    const int64_t n = h->ndof;
    PcgCtl c = h->pctl();
    const int ctl0[3] = {0, 0, maxit};
    DRF_CUDA(cudaMemcpyAsync(h->ctl.p, ctl0, sizeof(ctl0), cudaMemcpyHostToDevice, h->stream));
    const double tol2 = tol * tol;
    DRF_CUDA(cudaMemcpyAsync(h->scal.p + S_TOL2, &tol2, 8, cudaMemcpyHostToDevice, h->stream));
    // r = b - Q x ; bb = b.b ; z = M r ; rz = r.z ; p = z
    h->apply(h->finest(), h->x.p, h->bs.p, h->r.p, 1, nullptr, nullptr);
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
    if (kind == 4) {  // the reference multigrid apply is a host loop: no graph
        if (!done && maxit > 0)
            while (h->pcg_iteration_reference()) {
            }
        int cl[2] = {0, 0};
        DRF_CUDA(cudaMemcpyAsync(cl, h->ctl.p, sizeof(cl), cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        return cl[1];
    }
    // iterations in graph-captured chunks; converged iterations return early on the device
    const int chunk = 8;
    if (!done && maxit > 0) {
        if (!h->graph || h->graph_kind != kind || h->graph_chunk != chunk) {
            if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
            h->graph = capture_graph(h->stream, [&] {
                for (int k = 0; k < chunk; ++k) h->pcg_iteration(kind);
            }, &h->graph_kernels);
            h->graph_kind = kind;
            h->graph_chunk = chunk;
        }
        int ctl[2] = {0, 0};
        while (true) {
            DRF_CUDA(cudaGraphLaunch(h->graph, h->stream));
            launch_counter().fetch_add(h->graph_kernels);
            DRF_CUDA(cudaMemcpyAsync(ctl, h->ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, h->stream));
            DRF_CUDA(cudaStreamSynchronize(h->stream));
            if (ctl[0] || ctl[1] >= maxit) break;
        }
        it = ctl[1];
    }
    return it;
}

// n-point Gauss-Legendre nodes on [0, 1], ascending (Newton on P_n from cosine guesses)
void gauss01(int n, double *t) {
    for (int i = 0; i < n; ++i) {
        double x = std::cos(3.14159265358979323846 * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            const double dp = n * (x * p1 - p0) / (x * x - 1.0);
            const double d = p1 / dp;
            x -= d;
            if (std::abs(d) < 1e-16) break;
        }
        t[n - 1 - i] = 0.5 * (x + 1.0);
    }
}

ConsDev make_cons(const drf_bz *h, int ng) {
    DRF_CHECK(ng >= 1 && ng <= CONS_MAX_NG, DRF_E_INVALID, "edge_ngauss must be in 1..8");
    DRF_CHECK(h->H.g.nx == h->H.g.ny && h->H.g.nx >= 2, DRF_E_UNSUPPORTED,
              "edge constraints need a square grid of at least 2 x 2 elements");
    ConsDev C;
    std::memset(&C, 0, sizeof(C));
    C.n = h->H.g.nx;
    C.nd = 3 * C.n + 1;
    C.ng = ng;
    C.sx = 3.0 / h->H.dx;
    C.sy = 3.0 / h->H.dy;
    double t[CONS_MAX_NG];
    gauss01(ng, t);
    for (int q = 0; q < ng; ++q) {
        const double u = t[q], v = 1.0 - u;
        C.Bw[q][0] = v * v * v;
        C.Bw[q][1] = 3.0 * u * v * v;
        C.Bw[q][2] = 3.0 * u * u * v;
        C.Bw[q][3] = u * u * u;
    }
    return C;
}

inline int64_t cons_rows(const ConsDev &C) { return 2 * (int64_t)C.n * (C.n - 1) * C.ng; }

// a.b over n entries on the device, returned to the host (synchronous)
double dev_dot(drf_bz *h, int64_t n, const double *a, const double *b, double *slot) {
    dot_kernel<<<h->nparts(), BS, 0, h->stream>>>(n, a, b, h->part.p, nullptr);
    DRF_LAUNCHED();
    reduce_kernel<<<1, BS, 0, h->stream>>>(h->part.p, (int)h->nparts(), slot);
    DRF_LAUNCHED();
    double v = 0.0;
    DRF_CUDA(cudaMemcpyAsync(&v, slot, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    DRF_CUDA(cudaStreamSynchronize(h->stream));
    return v;
}

}  // namespace
}  // namespace drf

namespace drf {
namespace {
// Gauss-Legendre nodes and weights on [0, 1] (Newton on the Legendre recurrence): gq[0..n) the
// nodes in increasing order, gq[n..2n) the weights
std::vector<double> gauss_legendre_01_newton(int ngauss) {
    std::vector<double> gq(2 * ngauss);
    for (int i = 0; i < ngauss; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (ngauss + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= ngauss; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (ngauss == 1) { p1 = z; p0 = 1.0; }
            dp = ngauss * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::abs(dz) < 1e-16) break;
        }
        gq[ngauss - 1 - i] = 0.5 * (z + 1.0);
        gq[ngauss + ngauss - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
    return gq;
}

// The data-fitting rule of CGBezierSmootherBase::gauss_legendre_01
// (src/bathymetry/cg_bezier_smoother_base.cpp:28-58): the closed forms of the 1- to 4-point
// Gauss-Legendre rules on [0, 1] (the reference gives the 4-point rule for every n >= 4).
void gauss_legendre_01_closed(int n, double pts[4], double wts[4]) {
    if (n == 1) {
        pts[0] = 0.5;
        wts[0] = 1.0;
    } else if (n == 2) {
        pts[0] = 0.5 - 0.5 / std::sqrt(3.0);
        pts[1] = 0.5 + 0.5 / std::sqrt(3.0);
        wts[0] = wts[1] = 0.5;
    } else if (n == 3) {
        pts[0] = 0.5 - 0.5 * std::sqrt(0.6);
        pts[1] = 0.5;
        pts[2] = 0.5 + 0.5 * std::sqrt(0.6);
        wts[0] = wts[2] = 5.0 / 18.0;
        wts[1] = 8.0 / 18.0;
    } else {
        const double a = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
        const double b = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
        pts[0] = 0.5 * (1.0 - b);
        pts[1] = 0.5 * (1.0 - a);
        pts[2] = 0.5 * (1.0 + a);
        pts[3] = 0.5 * (1.0 + b);
        const double wa = (18.0 + std::sqrt(30.0)) / 72.0, wb = (18.0 - std::sqrt(30.0)) / 72.0;
        wts[0] = wts[3] = 0.5 * wb;
        wts[1] = wts[2] = 0.5 * wa;
    }
}

// ------------------------------------------------------------ element lists of quadtree meshes
// CubicBezierBasis2D::evaluate_bernstein_1d's recurrence (src/bathymetry/cubic_bezier_basis_2d.cpp:42),
// each product and sum rounded on its own (no fused multiply-add)
__device__ __forceinline__ void bern3_rn(double t, double B[4]) {
    const double s = __dadd_rn(1.0, -t);
    double p[4] = {1.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int deg = 1; deg <= 3; ++deg) {
        double c[4];
        c[0] = __dmul_rn(s, p[0]);
#pragma unroll
        for (int i = 1; i < deg; ++i) c[i] = __dadd_rn(__dmul_rn(t, p[i - 1]), __dmul_rn(s, p[i]));
        c[deg] = __dmul_rn(t, p[deg - 1]);
#pragma unroll
        for (int i = 0; i <= deg; ++i) p[i] = c[i];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) B[i] = p[i];
}

// compute_element_l2_error on an element list: one thread per element, the points in the
// reference's order (v outer, u inner), each mapped to physical coordinates and back as
// evaluate(x, y) does, the sums rounded term by term
__global__ void __launch_bounds__(256) bz_mesh_error_kernel(int64_t n, int ng, const double *__restrict__ bounds,
                                                            const double *__restrict__ coeffs,
                                                            const double *__restrict__ zd,
                                                            const double *__restrict__ gq, double *__restrict__ l2,
                                                            double *__restrict__ nrm) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double x0 = bounds[4 * e], y0 = bounds[4 * e + 1];
    const double dx = bounds[4 * e + 2] - x0, dy = bounds[4 * e + 3] - y0;
    double c[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) c[a] = coeffs[16 * e + a];
    double err2 = 0.0;
    for (int j = 0; j < ng; ++j)
        for (int i = 0; i < ng; ++i) {
            const double px = __dadd_rn(x0, __dmul_rn(gq[i], dx)), py = __dadd_rn(y0, __dmul_rn(gq[j], dy));
            const double u = fmin(1.0, fmax(0.0, __ddiv_rn(px - x0, dx)));
            const double v = fmin(1.0, fmax(0.0, __ddiv_rn(py - y0, dy)));
            double bu[4], bv[4];
            bern3_rn(u, bu);
            bern3_rn(v, bv);
            double z = 0.0;
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int a = 0; a < 4; ++a) z = __dadd_rn(z, __dmul_rn(__dmul_rn(c[a + 4 * b], bu[a]), bv[b]));
            const double w = __dmul_rn(gq[ng + i], gq[ng + j]);
            const double diff = zd[(e * ng + j) * ng + i] - z;
            err2 = __dadd_rn(err2, __dmul_rn(__dmul_rn(w, diff), diff));
        }
    const double err = sqrt(__dmul_rn(__dmul_rn(err2, dx), dy));
    l2[e] = err;
    if (nrm) nrm[e] = __ddiv_rn(err, sqrt(__dmul_rn(dx, dy)));
}

// the element part of assemble_data_fitting_global on an element list: one CTA per element, the
// 16 basis values of each quadrature point in shared memory, one thread per entry of the
// 16 x 16 block; points in the reference's order (qi outer, qj inner), each term rounded as
// weight * B_i * B_j
__global__ void __launch_bounds__(256) bz_mesh_fit_kernel(int64_t n, int ng, const double *__restrict__ bounds,
                                                          const double *__restrict__ zd,
                                                          const double *__restrict__ relax, const double *g01,
                                                          double *__restrict__ K, double *__restrict__ r,
                                                          double *__restrict__ dd) {
    __shared__ double sB[16][16], sw[16], sd[16];
    const int64_t e = blockIdx.x;
    const int t = threadIdx.x, nq = ng * ng;
    const double x0 = bounds[4 * e], y0 = bounds[4 * e + 1];
    const double jac = __dmul_rn(bounds[4 * e + 2] - x0, bounds[4 * e + 3] - y0);
    if (t < 16 * nq) {
        const int q = t / 16, a = t % 16, qi = q / ng, qj = q % ng;
        double bu[4], bv[4];
        bern3_rn(g01[qi], bu);
        bern3_rn(g01[qj], bv);
        sB[q][a] = __dmul_rn(bu[a % 4], bv[a / 4]);
        if (a == 0) {
            const int64_t idx = (e * ng + qj) * ng + qi;
            const double rel = relax ? relax[idx] : 1.0;
            sw[q] = __dmul_rn(__dmul_rn(__dmul_rn(g01[4 + qi], g01[4 + qj]), jac), rel);
            sd[q] = zd[idx];
        }
    }
    __syncthreads();
    const int a = t / 16, b = t % 16;
    double acc = 0.0;
    for (int q = 0; q < nq; ++q) acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(sw[q], sB[q][a]), sB[q][b]));
    K[256 * e + t] = acc;
    if (t < 16) {
        double ra = 0.0;
        for (int q = 0; q < nq; ++q) ra = __dadd_rn(ra, __dmul_rn(__dmul_rn(sw[q], sB[q][t]), sd[q]));
        r[16 * e + t] = ra;
    }
    if (t == 0) {
        double s = 0.0;
        for (int q = 0; q < nq; ++q) s = __dadd_rn(s, __dmul_rn(__dmul_rn(sw[q], sd[q]), sd[q]));
        dd[e] = s;
    }
}

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
        h->ndof = (int64_t)(3 * g->nx + 1) * (3 * g->ny + 1);
        // finest level only until drf_mg_setup
        h->lv.resize(1);
        auto &F = h->lv[0];
        F.n = g->nx;
        F.nd = 3 * g->nx + 1;
        up(F.K, transposed16(h->H.levels.back().K, 1));
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
        h->form_diag();
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
        h->apply(h->finest(), h->z.p, nullptr, h->q.p, 0, nullptr, nullptr);
        DRF_CUDA(cudaMemcpyAsync(yh, h->q.p, h->ndof * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_bz_element_errors(drf_bz *h, const double *xh, const double *zdata, int ngauss, double *l2,
                          double *normalized) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(xh && zdata && l2, DRF_E_INVALID, "null argument");
        DRF_CHECK(ngauss >= 1 && ngauss <= 16, DRF_E_INVALID, "ngauss must be 1..16");
        const drf_bz_grid_desc &g = h->H.g;
        const int64_t ne = (int64_t)g.nx * g.ny, npt = ne * ngauss * ngauss;
        DRF_CHECK(all_finite(zdata, (size_t)npt), DRF_E_NONFINITE, "non-finite data");
        const std::vector<double> gq = gauss_legendre_01_newton(ngauss);
        DevBuf<double> dz((size_t)npt), dgq(gq.size()), dl2(ne), dnrm(normalized ? ne : 1);
        DRF_CUDA(cudaMemcpyAsync(h->z.p, xh, h->ndof * 8, cudaMemcpyHostToDevice, h->stream));
        DRF_CUDA(cudaMemcpyAsync(dz.p, zdata, npt * 8, cudaMemcpyHostToDevice, h->stream));
        DRF_CUDA(cudaMemcpyAsync(dgq.p, gq.data(), gq.size() * 8, cudaMemcpyHostToDevice, h->stream));
        bz_elem_error_kernel<<<(unsigned)((ne + 7) / 8), 256, 0, h->stream>>>(
            g.nx, g.ny, ngauss, h->z.p, dz.p, dgq.p, h->H.dx * h->H.dy, dl2.p, normalized ? dnrm.p : nullptr);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpyAsync(l2, dl2.p, ne * 8, cudaMemcpyDeviceToHost, h->stream));
        if (normalized) DRF_CUDA(cudaMemcpyAsync(normalized, dnrm.p, ne * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_bz_mesh_element_errors(int64_t n_elem, const double *bounds, const double *coeffs, const double *zdata,
                               int ngauss, double *l2, double *normalized) {
    return guard([&] {
        DRF_CHECK(n_elem >= 0, DRF_E_INVALID, "negative element count");
        if (n_elem == 0) return;
        DRF_CHECK(bounds && coeffs && zdata && l2, DRF_E_INVALID, "null argument");
        DRF_CHECK(ngauss >= 1 && ngauss <= 16, DRF_E_INVALID, "ngauss must be 1..16");
        const int64_t npt = n_elem * ngauss * ngauss;
        DRF_CHECK(all_finite(bounds, (size_t)(4 * n_elem)) && all_finite(coeffs, (size_t)(16 * n_elem)) &&
                      all_finite(zdata, (size_t)npt),
                  DRF_E_NONFINITE, "non-finite input");
        for (int64_t e = 0; e < n_elem; ++e)
            DRF_CHECK(bounds[4 * e + 2] > bounds[4 * e] && bounds[4 * e + 3] > bounds[4 * e + 1], DRF_E_INVALID,
                      "element bounds must have xmax > xmin and ymax > ymin");
        const std::vector<double> gq = gauss_legendre_01_newton(ngauss);
        DevBuf<double> db(4 * n_elem), dc(16 * n_elem), dz(npt), dg(gq.size()), dl(n_elem), dn(normalized ? n_elem : 1);
        DRF_CUDA(cudaMemcpy(db.p, bounds, 32 * n_elem, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(dc.p, coeffs, 128 * n_elem, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(dz.p, zdata, 8 * npt, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(dg.p, gq.data(), 8 * gq.size(), cudaMemcpyHostToDevice));
        bz_mesh_error_kernel<<<(unsigned)((n_elem + 255) / 256), 256>>>(n_elem, ngauss, db.p, dc.p, dz.p, dg.p, dl.p,
                                                                       normalized ? dn.p : nullptr);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpy(l2, dl.p, 8 * n_elem, cudaMemcpyDeviceToHost));
        if (normalized) DRF_CUDA(cudaMemcpy(normalized, dn.p, 8 * n_elem, cudaMemcpyDeviceToHost));
    });
}

int drf_bz_mesh_data_fitting(int64_t n_elem, const double *bounds, const double *zdata, const double *relax,
                             int ngauss, double *BtWB, double *BtWd, double *dTWd) {
    return guard([&] {
        DRF_CHECK(n_elem >= 0, DRF_E_INVALID, "negative element count");
        if (n_elem == 0) return;
        DRF_CHECK(bounds && zdata && BtWB && BtWd && dTWd, DRF_E_INVALID, "null argument");
        DRF_CHECK(ngauss >= 1 && ngauss <= 4, DRF_E_INVALID,
                  "ngauss must be 1..4 (the data-fitting rule has 4 points at most)");
        const int64_t npt = n_elem * ngauss * ngauss;
        DRF_CHECK(all_finite(bounds, (size_t)(4 * n_elem)) && all_finite(zdata, (size_t)npt) &&
                      (!relax || all_finite(relax, (size_t)npt)),
                  DRF_E_NONFINITE, "non-finite input");
        double g01[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        gauss_legendre_01_closed(ngauss, g01, g01 + 4);
        DevBuf<double> db(4 * n_elem), dz(npt), drl(relax ? npt : 1), dg(8), dK(256 * n_elem), dr(16 * n_elem),
            dd(n_elem);
        DRF_CUDA(cudaMemcpy(db.p, bounds, 32 * n_elem, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(dz.p, zdata, 8 * npt, cudaMemcpyHostToDevice));
        if (relax) DRF_CUDA(cudaMemcpy(drl.p, relax, 8 * npt, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(dg.p, g01, sizeof(g01), cudaMemcpyHostToDevice));
        bz_mesh_fit_kernel<<<(unsigned)n_elem, 256>>>(n_elem, ngauss, db.p, dz.p, relax ? drl.p : nullptr, dg.p, dK.p,
                                                     dr.p, dd.p);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpy(BtWB, dK.p, 8 * 256 * n_elem, cudaMemcpyDeviceToHost));
        DRF_CUDA(cudaMemcpy(BtWd, dr.p, 8 * 16 * n_elem, cudaMemcpyDeviceToHost));
        DRF_CUDA(cudaMemcpy(dTWd, dd.p, 8 * n_elem, cudaMemcpyDeviceToHost));
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
            const std::vector<double> kt = transposed16(Lh.K, 1);
            up(lv[l].K, kt);
            up(lv[l].rho, Lh.rho);
            std::vector<double> bi =
                Lh.binv.empty() ? std::vector<double>(9 * 256, 0.0) : transposed16(Lh.binv.data(), 9);
            up(lv[l].binv, bi);
            if (l > 0) {
                std::vector<int> fc0, cf0;
                std::vector<double> fw, cw;
                transfer_tables(h->H.levels[l - 1].n, fc0, fw, cf0, cw);
                up(lv[l].fc0, fc0); up(lv[l].fw, fw); up(lv[l].cf0, cf0); up(lv[l].cw, cw);
                std::vector<double> rs(cf0.size(), 0.0);
                for (size_t c = 0; c < rs.size(); ++c)
                    for (int k = 0; k < 8; ++k) rs[c] += cw[8 * c + k];
                up(lv[l].rs, rs);
            }
            if (l < nl - 1) {
                const size_t n2 = (size_t)Lh.nd * Lh.nd;
                lv[l].x.alloc(n2); lv[l].b.alloc(n2); lv[l].r.alloc(n2);
            } else {
                lv[l].r.alloc((size_t)Lh.nd * Lh.nd);
            }
        }
        h->lv = std::move(lv);
        up(h->coarse, h->H.coarse_inv);
        DRF_CHECK(coarse_smem_doubles({h->lv[0].nd}, 0) * sizeof(double) <= COARSE_SMEM_MAX, DRF_E_UNSUPPORTED,
                  "coarsest level too large");
        DRF_CUDA(cudaFuncSetAttribute(bz_coarse_vcycle_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)COARSE_SMEM_MAX));
        allow_smem<16, 4>();
        const char *em = std::getenv("DRF_BZ_ELEM_SMOOTHER_MIN");
        h->elem_min = em ? std::max<int64_t>(0, std::atoll(em)) : ELEM_THREAD_MIN_ELEMS;
        h->mg_ready = true;
        h->form_diag();
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
        // the conv form of every layer at this grid's size, timed now (before any capture)
        cnn_tune(cnn_net(net), h->lv[h->finest()].n, h->cnn_ms, h->cnn_form);
        if (h->graph && h->graph_kind == 3) {
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
            h->graph_kind = -1;
        }
    });
}

int drf_bz_cnn_tuning(drf_bz *h, int *form4, double *ms8) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(h->cnn, DRF_E_INVALID, "no learned preconditioner attached");
        for (int l = 0; l < 4; ++l) {
            if (form4) form4[l] = h->cnn_form[l];
            if (ms8) { ms8[2 * l] = h->cnn_ms[l][0]; ms8[2 * l + 1] = h->cnn_ms[l][1]; }
        }
    });
}

int drf_bz_precondition(drf_bz *h, int kind, const double *rh, double *zh) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(rh && zh, DRF_E_INVALID, "null argument");
        DRF_CHECK(kind >= 0 && kind <= 4, DRF_E_INVALID, "unknown preconditioner kind");
        DRF_CHECK((kind != 2 && kind != 4) || h->mg_ready, DRF_E_INVALID, "multigrid preconditioner not set up");
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

int drf_mg_apply_reference(drf_bz *h, const double *rh, double *zh, double tol, int max_vcycles,
                           int *cycles, double *relres) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(h->mg_ready, DRF_E_INVALID, "drf_mg_setup has not been called");
        DRF_CHECK(rh && zh, DRF_E_INVALID, "null argument");
        DRF_CHECK(tol > 0 && max_vcycles >= 0, DRF_E_INVALID, "tol must be > 0 and max_vcycles >= 0");
        DRF_CUDA(cudaMemcpyAsync(h->r.p, rh, h->ndof * 8, cudaMemcpyHostToDevice, h->stream));
        double rel = 0.0;
        const int c = h->mg_apply_reference(h->r.p, h->z.p, tol, max_vcycles, &rel);
        DRF_CUDA(cudaMemcpyAsync(zh, h->z.p, h->ndof * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        if (cycles) *cycles = c;
        if (relres) *relres = rel;
    });
}

int drf_bz_constraints_apply(drf_bz *h, int edge_ngauss, const double *xh, double *yh) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(xh && yh, DRF_E_INVALID, "null argument");
        const ConsDev C = make_cons(h, edge_ngauss);
        const int64_t m = cons_rows(C);
        DevBuf<double> y(m);
        DRF_CUDA(cudaMemcpyAsync(h->z.p, xh, h->ndof * 8, cudaMemcpyHostToDevice, h->stream));
        bz_cons_apply_kernel<<<nblk(m), BS, 0, h->stream>>>(C, h->z.p, y.p);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpyAsync(yh, y.p, m * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_bz_constrained_solve(drf_bz *h, int edge_ngauss, int inner_kind, double tol, int maxit,
                             double inner_tol, double *xh, int *outer_iters, double *relres, double *ms) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(xh && tol > 0 && maxit >= 0 && inner_tol > 0, DRF_E_INVALID, "bad arguments");
        DRF_CHECK(inner_kind >= 0 && inner_kind <= 3, DRF_E_INVALID, "unknown preconditioner kind");
        DRF_CHECK(inner_kind != 2 || h->mg_ready, DRF_E_INVALID, "multigrid preconditioner not set up");
        DRF_CHECK(inner_kind != 3 || h->cnn, DRF_E_INVALID, "no learned preconditioner attached");
        const ConsDev C = make_cons(h, edge_ngauss);
        const int64_t m = cons_rows(C), n = h->ndof;
        DevBuf<double> lam(m), rs(m), ps(m), qs(m), slot(1);
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        DRF_CUDA(cudaEventRecord(e0, h->stream));
        // x = Q^-1 bs from x = 0 (the apply_Qinv seam)
        auto qinv = [&] {
            zero_kernel<<<nblk(n), BS, 0, h->stream>>>(n, h->x.p, nullptr);
            DRF_LAUNCHED();
            pcg_run(h, inner_kind, inner_tol, 100000);
        };
        const unsigned gm = nblk(m), gn = nblk(n);
        // rhs = A Q^-1 b ; lambda = 0 ; r = rhs ; p = r
        DRF_CUDA(cudaMemcpyAsync(h->bs.p, h->b.p, n * 8, cudaMemcpyDeviceToDevice, h->stream));
        qinv();
        bz_cons_apply_kernel<<<gm, BS, 0, h->stream>>>(C, h->x.p, rs.p);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemsetAsync(lam.p, 0, m * 8, h->stream));
        DRF_CUDA(cudaMemcpyAsync(ps.p, rs.p, m * 8, cudaMemcpyDeviceToDevice, h->stream));
        const double rz_init = dev_dot(h, m, rs.p, rs.p, slot.p);
        double rz = rz_init;
        int it = 0;
        if (rz_init > 1e-30) {
            while (it < maxit) {
                bz_cons_applyT_kernel<<<gn, BS, 0, h->stream>>>(C, ps.p, nullptr, h->bs.p);
                DRF_LAUNCHED();
                qinv();
                bz_cons_apply_kernel<<<gm, BS, 0, h->stream>>>(C, h->x.p, qs.p);
                DRF_LAUNCHED();
                const double pSp = dev_dot(h, m, ps.p, qs.p, slot.p);
                if (!(std::abs(pSp) >= 1e-30)) break;
                cg_update_kernel<<<1024, BS, 0, h->stream>>>(m, rz / pSp, ps.p, qs.p, lam.p, rs.p);
                DRF_LAUNCHED();
                const double rz_new = dev_dot(h, m, rs.p, rs.p, slot.p);
                ++it;
                if (rz_new / rz_init < tol * tol) {
                    rz = rz_new;
                    break;
                }
                xpay_kernel<<<1024, BS, 0, h->stream>>>(m, rz_new / rz, rs.p, ps.p);
                DRF_LAUNCHED();
                rz = rz_new;
            }
        }
        // x = Q^-1 (b - A^T lambda)
        bz_cons_applyT_kernel<<<gn, BS, 0, h->stream>>>(C, lam.p, h->b.p, h->bs.p);
        DRF_LAUNCHED();
        qinv();
        DRF_CUDA(cudaEventRecord(e1, h->stream));
        DRF_CUDA(cudaMemcpyAsync(xh, h->x.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        float t = 0.f;
        DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (outer_iters) *outer_iters = it;
        if (relres) *relres = rz_init > 0 ? std::sqrt(rz / rz_init) : 0.0;
        if (ms) *ms = t;
        DRF_CHECK(std::isfinite(rz), DRF_E_NONFINITE, "Schur CG diverged (non-finite residual)");
    });
}

int drf_pcg_solve(drf_bz *h, const double *bh, double *xh, double tol, int maxit, int kind,
                  int *iters, double *relres, double *ms) {
    return guard([&] {
        check_bz(h);
        DRF_CHECK(xh && tol > 0 && maxit >= 0, DRF_E_INVALID, "bad arguments");
        DRF_CHECK(kind >= 0 && kind <= 4, DRF_E_INVALID, "unknown preconditioner kind");
        DRF_CHECK((kind != 2 && kind != 4) || h->mg_ready, DRF_E_INVALID, "multigrid preconditioner not set up");
        DRF_CHECK(kind != 3 || h->cnn, DRF_E_INVALID, "no learned preconditioner attached (drf_bz_set_cnn)");
        const int64_t n = h->ndof;
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        if (bh) DRF_CUDA(cudaMemcpyAsync(h->bs.p, bh, n * 8, cudaMemcpyHostToDevice, h->stream));
        else DRF_CUDA(cudaMemcpyAsync(h->bs.p, h->b.p, n * 8, cudaMemcpyDeviceToDevice, h->stream));
        DRF_CUDA(cudaMemcpyAsync(h->x.p, xh, n * 8, cudaMemcpyHostToDevice, h->stream));
        DRF_CUDA(cudaEventRecord(e0, h->stream));
        const int it = pcg_run(h, kind, tol, maxit);
        DRF_CUDA(cudaEventRecord(e1, h->stream));
        double sc[S_NSLOT];
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
        if (kind == 3) cnn_check(cnn_net(h->cnn), h->stream);
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
        // device address of the scratch array in the current device's context, looked up on
        // every call (cheap, allocates nothing, and stays right if the context was re-created)
        void *sym = nullptr;
        DRF_CUDA(cudaGetSymbolAddress(&sym, g_noalloc_scratch));
        double *K = static_cast<double *>(sym), *rho = K + 256, *r = rho + NOALLOC_MAX_ND;
        double *z = r + NOALLOC_MAX_DOF, *p = z + NOALLOC_MAX_DOF, *q = p + NOALLOC_MAX_DOF;
        double *part = q + NOALLOC_MAX_DOF, *scal = part + NOALLOC_PARTS;
        int *ctl = reinterpret_cast<int *>(scal + 16);
        cudaStream_t st = (cudaStream_t)stream;
        double Kr[256], Kh[256], alpha = 0.0;
        bz_fine_operator(*g, Kr, &alpha);
        for (int a = 0; a < 16; ++a)
            for (int k = 0; k < 16; ++k) Kh[k * 16 + a] = Kr[a * 16 + k];
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
            // iterations are queued 8 at a time between reads of the control word: after
            // convergence (or at maxit) every kernel returns early on it, so the extra ones
            // change nothing
            constexpr int chunk = 8;
            while (true) {
                for (int k = 0; k < chunk; ++k) {
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
                }
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
