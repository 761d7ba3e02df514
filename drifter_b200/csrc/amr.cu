// DG3DIntegration::compute_rhs (src/dg/operators_3d.cpp:228-282) on a directionally refined
// (AMR) hexahedral mesh, for the scalar conservation law u_t + div(a u) = 0 with a constant
// velocity a, plus a low-storage RK45 step replayed as one CUDA graph.
//
// Semantics, as the reference computes them (reference coordinates: identity Jacobian):
//   R_e = M^-1 ( -sum_q w_q grad(phi)(x_q) . a u(x_q)          volume_integral (:81), N-point
//                                                              Gauss-Legendre per direction
//                + conforming / boundary face lifts            mode 1 only (TODO in the reference)
//                + mortar lifts of the non-conforming faces )  compute_interface_flux_nonconforming (:345)
// and the step integrates du/dt = -R (R is the weak divergence of a u: volume -grad(phi), faces +F).
//
// Kernel design. The volume term is a tensor product: with B (N x (N+1)) the LGL basis at the
// Gauss-Legendre points, B' its derivative and W the weights, the quadrature equals
//   -(a_x K x M x M + a_y M x K x M + a_z M x M x K) u,  K = B'^T W B,  M = B^T W B,
// applied sum-factorized (six small passes over an element's (N+1)^3 nodes in shared memory).
// One thread per node, several elements per CTA; each node then adds the flux of every face
// it lies on (faces 0..5 in order, own outward normal, the neighbour's face node read from
// global memory), so the result needs no atomics. The mortar kernels (mortar.cu) add the
// non-conforming lifts in interface order; the mass inverse is fused into the output or the
// LSRK update.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "amr_layout.hpp"
#include "common.cuh"
#include "mortar_internal.hpp"

namespace drf {
namespace {

struct AmrBasis {
    double K[MAXNP * MAXNP], M[MAXNP * MAXNP], w[MAXNP];
};
__constant__ AmrBasis cAmr[MAXNP + 1];  // per node count

const double AMR_LSRK_A[5] = {0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257};
const double AMR_LSRK_B[5] = {0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488,
                              0.1530572479681};

struct AmrArgs {
    const double *U;
    double *R;              // weak right-hand side (before the mass inverse)
    const int64_t *nbe;     // [elem][6] conforming neighbour element (or -1)
    const int8_t *nbk;      // [elem][6] 0 none, 1 conforming, 2 boundary
    const int8_t *nbf;      // [elem][6] neighbour face
    int64_t n_elem;
    double ax, ay, az;
    int flux;               // 0 central, 1 upwind, 2 Lax-Friedrichs
    // the LSRK stage form (amr_rhs_kernel<NP, true>): the mortar lifts added in the lift
    // kernel's order, then the mass inverse and res = A res + dt (-M^-1 R), Uout = U + B res
    const double *contrib;  // staged mortar lifts (null: no interfaces)
    const int64_t *lptr;    // lift entries of touched element u: lent[lptr[u] .. lptr[u + 1])
    const int *lent;        // (interface, slot, face)
    const int *e2u;         // touched-element index of each element, -1 if none
    int slots;
    double *res, *Uout;
    double A, B, dt;
    int first;
};

// One node's LSRK45 stage from its weak right-hand side R (before the mass inverse, the
// diagonal LGL mass w_i w_j w_k): res = A res + dt (-M^-1 R), u += B res.
__device__ __forceinline__ void amr_lsrk_node(double R, double wi, double wj, double wk, double &res, double &u,
                                              double A, double B, double dt, int first) {
    const double rhs = R * (1.0 / (wi * wj * wk));
    const double rn = (first ? 0.0 : A * res) + dt * (-rhs);
    res = rn;
    u = u + B * rn;
}

__device__ __forceinline__ double amr_flux(int kind, double uL, double uR, double vn) {
    if (kind == 0) return 0.5 * (vn * uL + vn * uR);
    if (kind == 1) return vn * (vn >= 0 ? uL : uR);
    return 0.5 * (vn * uL + vn * uR) - 0.5 * fabs(vn) * (uR - uL);
}

// volume node of face node (it, jt) of face f: normal index at the boundary, tangents in axis order
template <int NP>
__device__ __forceinline__ int face_node(int f, int it, int jt) {
    const int axis = f / 2, b = (f % 2) ? NP - 1 : 0;
    if (axis == 0) return b + NP * (it + NP * jt);
    if (axis == 1) return it + NP * (b + NP * jt);
    return it + NP * (jt + NP * b);
}

template <int NP>
constexpr int amr_epb() {  // elements per CTA: about 256 threads
    return (256 / (NP * NP * NP)) < 1 ? 1 : 256 / (NP * NP * NP);
}

// R = volume term + conforming/boundary face lifts, one thread per node. The element's face
// table and its conforming neighbours' face traces are loaded at the start (each thread takes
// face-node slots n, n + NP^3, ...) so those global loads overlap the volume passes. STAGE:
// the node's mortar lifts are added and the LSRK stage applied (U read, Uout written).
template <int NP, bool STAGE = false>
__global__ void __launch_bounds__(amr_epb<NP>() * NP * NP * NP) amr_rhs_kernel(AmrArgs a) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP, EPB = amr_epb<NP>(), NFS = 6 * NP2;
    constexpr int SLOTS = (NFS + NP3 - 1) / NP3;  // face-node slots per thread
    __shared__ double sU[EPB * NP3], sP[EPB * NP3], sQ[EPB * NP3], s1[EPB * NP3], s2[EPB * NP3];
    __shared__ double sN[EPB * NFS];                // neighbour face traces [elem][face][node]
    __shared__ int sNbe[EPB * 6];
    __shared__ int8_t sK[EPB * 6], sNf[EPB * 6];
    // the 1D operators in shared memory: lanes index them by their own node (a constant-memory
    // read with different addresses across a warp is serialised)
    __shared__ AmrBasis Bs;
    for (int t = threadIdx.x; t < NP2; t += blockDim.x) {
        Bs.K[t] = cAmr[NP].K[t];
        Bs.M[t] = cAmr[NP].M[t];
        if (t < NP) Bs.w[t] = cAmr[NP].w[t];
    }
    const int le = threadIdx.x / NP3, n = threadIdx.x % NP3;
    const int i = n % NP, j = (n / NP) % NP, k = n / NP2;
    const int64_t e = (int64_t)blockIdx.x * EPB + le;
    const bool valid = e < a.n_elem;
    double *U = sU + le * NP3, *P = sP + le * NP3, *Q = sQ + le * NP3, *T1 = s1 + le * NP3, *T2 = s2 + le * NP3;
    const double u = valid ? a.U[e * NP3 + n] : 0.0;
    if (n < 6) {
        sK[le * 6 + n] = valid ? a.nbk[e * 6 + n] : (int8_t)0;
        sNbe[le * 6 + n] = valid ? (int)a.nbe[e * 6 + n] : -1;
        sNf[le * 6 + n] = valid ? a.nbf[e * 6 + n] : (int8_t)0;
    }
    U[n] = u;
    __syncthreads();
    // neighbour face traces: loads issued now, stored to shared memory after the volume passes
    double nv[SLOTS];
#pragma unroll
    for (int sl = 0; sl < SLOTS; ++sl) {
        const int slot = n + sl * NP3;
        nv[sl] = 0.0;
        if (slot < NFS) {
            const int f = slot / NP2, fn = slot % NP2;
            if (sK[le * 6 + f] == 1)
                nv[sl] = a.U[(int64_t)sNbe[le * 6 + f] * NP3 + face_node<NP>(sNf[le * 6 + f], fn % NP, fn / NP)];
        }
    }
    // z: P = (I x I x M) u, Q = (I x I x K) u
    double p = 0.0, q = 0.0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const double um = U[i + NP * (j + NP * m)];
        p += Bs.M[k * NP + m] * um;
        q += Bs.K[k * NP + m] * um;
    }
    P[n] = p;
    Q[n] = q;
    __syncthreads();
    // y: T1 = (I x M x I) P, T2 = (I x K x I) P, U <- (I x M x I) Q
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const int nm = i + NP * (m + NP * k);
        t1 += Bs.M[j * NP + m] * P[nm];
        t2 += Bs.K[j * NP + m] * P[nm];
        t3 += Bs.M[j * NP + m] * Q[nm];
    }
    __syncthreads();  // every thread has read U (its own node) and P, Q
    T1[n] = t1;
    T2[n] = t2;
    U[n] = t3;
#pragma unroll
    for (int sl = 0; sl < SLOTS; ++sl)
        if (n + sl * NP3 < NFS) sN[le * NFS + n + sl * NP3] = nv[sl];
    __syncthreads();
    // x: r = -(a_x (K x I x I) T1 + a_y (M x I x I) T2 + a_z (M x I x I) T3)
    double vx = 0.0, vy = 0.0, vz = 0.0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const int nm = m + NP * (j + NP * k);
        vx += Bs.K[i * NP + m] * T1[nm];
        vy += Bs.M[i * NP + m] * T2[nm];
        vz += Bs.M[i * NP + m] * U[nm];
    }
    if (!valid) return;
    double r = -(a.ax * vx + a.ay * vy + a.az * vz);
    // faces this node lies on, in face order
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int axis = f / 2;
        const int idx = axis == 0 ? i : (axis == 1 ? j : k);
        if (idx != ((f % 2) ? NP - 1 : 0)) continue;
        const int kd = sK[le * 6 + f];
        if (kd == 0) continue;
        const int it = axis == 0 ? j : i, jt = axis == 2 ? j : k;
        const double vn = ((f % 2) ? 1.0 : -1.0) * (axis == 0 ? a.ax : (axis == 1 ? a.ay : a.az));
        const double uR = kd == 1 ? sN[le * NFS + f * NP2 + it + NP * jt] : u;
        r += Bs.w[it] * Bs.w[jt] * amr_flux(a.flux, u, uR, vn);
    }
    if constexpr (STAGE) {
        // mortar lifts of the interfaces touching this element, in the lift kernel's order
        const int ut = a.e2u ? a.e2u[e] : -1;
        if (ut >= 0)
            for (int64_t q = a.lptr[ut]; q < a.lptr[ut + 1]; ++q) {
                const int iface = a.lent[3 * q], slot = a.lent[3 * q + 1], f = a.lent[3 * q + 2];
                const int axis = f >> 1, b = (f & 1) ? NP - 1 : 0;
                const int on = axis == 0 ? i : (axis == 1 ? j : k);
                if (on != b) continue;
                const int it = axis == 0 ? j : i, jt = axis == 2 ? j : k;
                r += a.contrib[((size_t)iface * a.slots + slot) * NP2 + it + NP * jt];
            }
        const size_t t = (size_t)e * NP3 + n;
        double rs = a.first ? 0.0 : a.res[t], uo = u;
        amr_lsrk_node(r, Bs.w[i], Bs.w[j], Bs.w[k], rs, uo, a.A, a.B, a.dt, a.first);
        a.res[t] = rs;
        a.Uout[t] = uo;
    } else {
        a.R[e * NP3 + n] = r;
    }
}

// out = M^-1 R (the right-hand side the caller sees)
template <int NP>
__global__ void amr_massinv_kernel(int64_t n, const double *R, double *out) {
    constexpr int NP3 = NP * NP * NP;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int nn = (int)(t % NP3), i = nn % NP, j = (nn / NP) % NP, k = nn / (NP * NP);
    const AmrBasis &Bs = cAmr[NP];
    out[t] = R[t] * (1.0 / (Bs.w[i] * Bs.w[j] * Bs.w[k]));
}

template <class F>
void amr_dispatch(int np, F &&f) {
    switch (np) {
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    default: throw Error(DRF_E_UNSUPPORTED, "AMR: order must be 1..5");
    }
}

// ------------------------------------------------------------------ AMR refinement
// GradientErrorEstimator::estimate_element and compute_directional_mask
// (src/amr/refinement.cpp:70-160), one warp per element: the element's nodal values are staged
// in shared memory, the range (max - min) over all of them and along every node line of each
// axis reduced across the warp. Comparisons only, so the results are exact; value = range x
// h (the element's characteristic length, supplied), and each block's largest value goes to
// bmax for the normalisation.
constexpr int AMR_EST_WARPS = 8;
template <int NP>
__global__ void __launch_bounds__(32 * AMR_EST_WARPS)
    amr_estimate_kernel(int64_t n_elem, const double *__restrict__ U, const double *__restrict__ hchar, double sf,
                        double *__restrict__ value, int *__restrict__ mask, double *__restrict__ bmax) {
    constexpr int ND = NP * NP * NP, NL = NP * NP;
    __shared__ double s[AMR_EST_WARPS][ND];
    __shared__ double wv[AMR_EST_WARPS];
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int64_t e = (int64_t)blockIdx.x * AMR_EST_WARPS + w;
    double v = 0.0;
    if (e < n_elem) {
        const double *u = U + e * ND;
        double mx = -INFINITY, mn = INFINITY;
        for (int q = lane; q < ND; q += 32) {
            const double x = u[q];
            s[w][q] = x;
            mx = fmax(mx, x);
            mn = fmin(mn, x);
        }
        __syncwarp();
        double var[3] = {0.0, 0.0, 0.0};
        for (int l = lane; l < NL; l += 32) {
            const int a = l % NP, b = l / NP;
            // node lines along x (j = a, k = b), y (i = a, k = b) and z (i = a, j = b)
            const int base[3] = {NP * (a + NP * b), a + NL * b, a + NP * b};
            const int step[3] = {1, NP, NL};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double lo = s[w][base[d]], hi = lo;
#pragma unroll
                for (int m = 1; m < NP; ++m) {
                    const double x = s[w][base[d] + step[d] * m];
                    lo = fmin(lo, x);
                    hi = fmax(hi, x);
                }
                var[d] = fmax(var[d], hi - lo);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
#pragma unroll
            for (int d = 0; d < 3; ++d) var[d] = fmax(var[d], __shfl_xor_sync(0xffffffffu, var[d], o));
        }
        v = (mx - mn) * hchar[e];
        if (lane == 0) {
            const double mv = fmax(fmax(var[0], var[1]), var[2]);
            int m = 0;
            if (mv >= 1e-14) {
                const double thr = sf * mv;
                for (int d = 0; d < 3; ++d)
                    if (var[d] > thr) m |= 1 << d;
            }
            value[e] = v;
            mask[e] = m;
        }
    }
    if (lane == 0) wv[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int k = 0; k < AMR_EST_WARPS; ++k) b = fmax(b, wv[k]);
        bmax[blockIdx.x] = b;
    }
}
// the largest block maximum (one CTA), then the normalisation and the flags (estimate, :56-67)
__global__ void amr_max_kernel(const double *__restrict__ part, int64_t n, double *out) {
    __shared__ double s[1024];
    double m = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, part[i]);
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}
__global__ void amr_flags_kernel(int64_t n_elem, const double *__restrict__ vmax, double rt, double ct,
                                 double *__restrict__ value, int *__restrict__ flags) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    const double m = *vmax;
    int f = 0;
    if (m > 1e-14) {
        const double v = value[e] / m;
        value[e] = v;
        f = (v > rt ? 1 : 0) | (v < ct ? 2 : 0);
    }
    flags[e] = f;
}

// The solution carried to new per-column levels: every new node takes, per axis, the old cell
// on its side and its coordinate there (SolutionProjection::project_to_children on a refined
// axis, project_from_children on a coarsened one, src/amr/refinement.cpp:217-343; k levels at a
// time in general), and the old cell's interpolant at that point (interpolate_3d, :345: the
// Lagrange product formula, then the sum in dof order with separate roundings).
struct AmrTransferArgs {
    const double *Uo;
    double *Un;
    const int *col_of;          // column of each new element
    const int *lvo, *lvn;       // old / new levels [3 c + d]
    const int64_t *offo, *offn; // old / new first element of each column
    double xn[MAXNP];           // LGL nodes
    // Lagrange rows of the one-level cases, [case][node][m]: 0 unchanged, 1 / 2 refined into the
    // lower / upper half, 3 coarsened (the node's side); other level changes are formed per node
    const double *rows;
    int64_t n_new;
};
// old sub-cell and its coordinate of node coordinate x in new sub-cell s, along one axis
__device__ __forceinline__ void amr_old_cell(int s, int ln, int lo, double x, int &so, double &xo) {
    if (ln == lo) {
        so = s;
        xo = x;
    } else if (ln > lo) {  // refined k levels: sub-cell r of old cell s >> k
        const int k = ln - lo, r = s & ((1 << k) - 1);
        const double cl = -1.0 + 2.0 * r / (1 << k), ch = cl + 2.0 / (1 << k);
        so = s >> k;
        xo = cl + 0.5 * (x + 1.0) * (ch - cl);
    } else {  // coarsened k levels: the old cell on the node's side (0 goes to the upper one)
        const int k = lo - ln;
        const int ch = k == 1 ? (x >= 0 ? 1 : 0) : min((1 << k) - 1, (int)floor((x + 1.0) * (1 << (k - 1))));
        const double cl = -1.0 + 2.0 * ch / (1 << k), chi = cl + 2.0 / (1 << k);
        so = (s << k) + ch;
        xo = fmin(1.0, fmax(-1.0, 2.0 * (x - cl) / (chi - cl) - 1.0));
    }
}
template <int NP>
__global__ void __launch_bounds__(256) amr_transfer_kernel(AmrTransferArgs a) {
    constexpr int ND = NP * NP * NP, NL = NP * NP;
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.n_new * ND) return;
    const int64_t e = g / ND;
    const int n = (int)(g % ND);
    const int m3[3] = {n % NP, (n / NP) % NP, n / NL};
    const int c = a.col_of[e];
    const int *ln = a.lvn + 3 * c, *lo = a.lvo + 3 * c;
    const int64_t loc = e - a.offn[c];
    const int nxn = 1 << ln[0], nyn = 1 << ln[1];
    const int s3[3] = {(int)(loc % nxn), (int)((loc / nxn) % nyn), (int)(loc / ((int64_t)nxn * nyn))};
    int so[3];
    double L[3][NP];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double xo;
        amr_old_cell(s3[d], ln[d], lo[d], a.xn[m3[d]], so[d], xo);
        const int dl = ln[d] - lo[d];
        if (dl >= -1 && dl <= 1) {
            const int cs = dl == 0 ? 0 : (dl > 0 ? 1 + (s3[d] & 1) : 3);
#pragma unroll
            for (int i = 0; i < NP; ++i) L[d][i] = a.rows[(cs * NP + m3[d]) * NP + i];
        } else {
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                double v = 1.0;
#pragma unroll
                for (int j = 0; j < NP; ++j)
                    if (j != i) v = __dmul_rn(v, __ddiv_rn(xo - a.xn[j], a.xn[i] - a.xn[j]));
                L[d][i] = v;
            }
        }
    }
    const int nxo = 1 << lo[0], nyo = 1 << lo[1];
    const int64_t eo = a.offo[c] + so[0] + (int64_t)nxo * (so[1] + (int64_t)nyo * so[2]);
    const double *u = a.Uo + eo * ND;
    double r = 0.0;
    for (int k = 0; k < NP; ++k)
        for (int j = 0; j < NP; ++j)
#pragma unroll
            for (int i = 0; i < NP; ++i)
                r = __dadd_rn(r, __dmul_rn(__dmul_rn(__dmul_rn(u[i + NP * (j + NP * k)], L[0][i]), L[1][j]), L[2][k]));
    a.Un[g] = r;
}

}  // namespace
}  // namespace drf

using namespace drf;

struct drf_amr {
    int order = 0, np = 0, nd = 0;
    int64_t n_elem = 0, n_conf = 0, n_bnd = 0, n_if = 0;
    cudaStream_t stream = nullptr, own = nullptr;
    DevBuf<int64_t> nbe;
    DevBuf<int8_t> nbk, nbf;
    // device state (two buffers: an LSRK stage reads one and writes the other; cur holds the
    // state between steps), weak rhs, LSRK register, caller-visible rhs
    DevBuf<double> U, R, res, out;
    int cur = 0;
    drf_mortar *mortar = nullptr;
    DevBuf<int> e2u;  // touched-element index of each element for the stage kernel's lifts
    // step graphs for each starting buffer (a step's five stages flip it)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_kernels = 0;  // kernel nodes of a step graph
    int g_mode = -1, g_flux = -1;
    double g_a[3] = {0, 0, 0}, g_dt = 0.0;

    double *state() { return U.p + (size_t)cur * n_elem * nd; }
    double *buf(int b) { return U.p + (size_t)b * n_elem * nd; }
    ~drf_amr() {
        for (auto &g : graph)
            if (g) cudaGraphExecDestroy(g);
        if (mortar) drf_mortar_destroy(mortar);
        if (own) cudaStreamDestroy(own);
    }
    void drop_graph() {
        for (auto &g : graph)
            if (g) cudaGraphExecDestroy(g);
        graph[0] = graph[1] = nullptr;
        g_mode = -1;
    }
    // R = weak right-hand side of U (volume + faces of the mode + mortar lifts)
    void enqueue_rhs(int mode, int flux, const double a[3]) {
        AmrArgs A{};
        A.U = state(); A.R = R.p; A.nbe = nbe.p; A.nbf = nbf.p; A.n_elem = n_elem;
        A.ax = a[0]; A.ay = a[1]; A.az = a[2]; A.flux = flux;
        // mode 0 reads an all-zero face table: the reference's TODO branches
        A.nbk = mode == 1 ? nbk.p : nbk.p + (size_t)6 * n_elem;
        amr_dispatch(np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            constexpr int EPB = amr_epb<NP>();
            amr_rhs_kernel<NP><<<(unsigned)((n_elem + EPB - 1) / EPB), EPB * NP * NP * NP, 0, stream>>>(A);
            DRF_LAUNCHED();
        });
        if (mortar) {
            const int rc = drf_mortar_apply_device(mortar, flux, a, state(), R.p);
            DRF_CHECK(rc == DRF_OK, rc, "mortar apply failed");
        }
    }
    // one LSRK45 step from buffer b0: per stage the mortar face kernel, then the stage kernel
    // (volume, faces, mortar lifts, mass inverse and update) from one buffer into the other
    void enqueue_step(int mode, int flux, const double a[3], double dt, int b0) {
        const MortarLifts L = mortar ? mortar_lifts(mortar) : MortarLifts{};
        for (int s = 0; s < 5; ++s) {
            const int src = (b0 + s) % 2;
            if (mortar) mortar_stage_faces(mortar, flux, a, buf(src));
            AmrArgs A{};
            A.U = buf(src); A.Uout = buf(1 - src); A.res = res.p;
            A.nbe = nbe.p; A.nbf = nbf.p; A.n_elem = n_elem;
            A.nbk = mode == 1 ? nbk.p : nbk.p + (size_t)6 * n_elem;
            A.ax = a[0]; A.ay = a[1]; A.az = a[2]; A.flux = flux;
            A.contrib = mortar ? L.contrib : nullptr; A.lptr = L.ptr; A.lent = L.ent;
            A.e2u = mortar ? e2u.p : nullptr; A.slots = L.slots;
            A.A = AMR_LSRK_A[s]; A.B = AMR_LSRK_B[s]; A.dt = dt; A.first = s == 0;
            amr_dispatch(np, [&](auto npc) {
                constexpr int NP = decltype(npc)::value;
                constexpr int EPB = amr_epb<NP>();
                amr_rhs_kernel<NP, true>
                    <<<(unsigned)((n_elem + EPB - 1) / EPB), EPB * NP * NP * NP, 0, stream>>>(A);
                DRF_LAUNCHED();
            });
        }
    }
};

namespace {

void amr_check(drf_amr *h) { DRF_CHECK(h != nullptr, DRF_E_INVALID, "null AMR handle"); }

void amr_check_args(int mode, int flux, const double *a) {
    DRF_CHECK(mode == 0 || mode == 1, DRF_E_INVALID, "mode must be 0 (reference) or 1 (complete)");
    DRF_CHECK(flux >= 0 && flux <= 2, DRF_E_INVALID, "flux kind must be 0 (central), 1 (upwind) or 2 (LF)");
    DRF_CHECK(a && std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]), DRF_E_INVALID,
              "advection velocity must be finite");
}

// Gauss-Legendre nodes and weights (n points) by Newton on the Legendre recurrence
void gl_rule(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) p1 = z, p0 = 1.0;
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::abs(dz) < 1e-16) break;
        }
        x[n - 1 - i] = z;  // ascending
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// K = B'^T W B and M = B^T W B of the reference's volume quadrature (N Gauss-Legendre points)
void upload_amr_basis(int order) {
    static std::mutex mu;
    static bool done[64][MAXNP + 1] = {};
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    const HostBasis b = make_lgl_basis(order);
    const int np = b.np, nq = order;
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && done[dev][np]) return;
    std::vector<double> gx, gw;
    gl_rule(nq, gx, gw);
    // barycentric Lagrange interpolation of the LGL basis at the GL points
    std::vector<double> bw(np, 1.0), B((size_t)nq * np, 0.0), Bd((size_t)nq * np, 0.0);
    for (int j = 0; j < np; ++j)
        for (int k = 0; k < np; ++k)
            if (k != j) bw[j] /= (b.x[j] - b.x[k]);
    for (int q = 0; q < nq; ++q) {
        double den = 0.0;
        for (int j = 0; j < np; ++j) den += bw[j] / (gx[q] - b.x[j]);
        for (int j = 0; j < np; ++j) B[q * np + j] = bw[j] / (gx[q] - b.x[j]) / den;
    }
    for (int q = 0; q < nq; ++q)  // phi_m'(x_q) = sum_i phi_i(x_q) D[i][m]
        for (int m = 0; m < np; ++m)
            for (int i = 0; i < np; ++i) Bd[q * np + m] += B[q * np + i] * b.D[i * np + m];
    AmrBasis ab;
    std::memset(&ab, 0, sizeof(ab));
    for (int i = 0; i < np; ++i) {
        ab.w[i] = b.w[i];
        for (int m = 0; m < np; ++m) {
            double k = 0.0, mm = 0.0;
            for (int q = 0; q < nq; ++q) {
                k += Bd[q * np + i] * gw[q] * B[q * np + m];
                mm += B[q * np + i] * gw[q] * B[q * np + m];
            }
            ab.K[i * np + m] = k;
            ab.M[i * np + m] = mm;
        }
    }
    DRF_CUDA(cudaMemcpyToSymbol(cAmr, &ab, sizeof(ab), (size_t)np * sizeof(AmrBasis)));
    if (dev < 64) done[dev][np] = true;
}

}  // namespace

extern "C" {

int drf_amr_create(int order, int64_t n_elem, int64_t n_conf, const int64_t *conf, int64_t n_bnd,
                   const int64_t *bnd, int64_t n_if, const int *type, const int64_t *coarse_elem,
                   const int *coarse_face, const int64_t *fine_elem, const int *fine_face, drf_amr **out) {
    return guard([&] {
        DRF_CHECK(out, DRF_E_INVALID, "null output");
        *out = nullptr;
        DRF_CHECK(order >= 1 && order < MAXNP, DRF_E_UNSUPPORTED, "AMR: order must be 1..5");
        DRF_CHECK(n_elem >= 1 && n_conf >= 0 && n_bnd >= 0 && n_if >= 0, DRF_E_INVALID, "bad sizes");
        DRF_CHECK(n_elem < ((int64_t)1 << 31), DRF_E_UNSUPPORTED, "AMR: at most 2^31 - 1 elements");
        DRF_CHECK((n_conf == 0 || conf) && (n_bnd == 0 || bnd), DRF_E_INVALID, "null face list");
        auto h = std::make_unique<drf_amr>();
        h->order = order;
        h->np = order + 1;
        h->nd = h->np * h->np * h->np;
        h->n_elem = n_elem;
        h->n_conf = n_conf;
        h->n_bnd = n_bnd;
        h->n_if = n_if;
        // face table: the second half stays zero (the reference-semantics launches read it)
        std::vector<int64_t> nbe((size_t)6 * n_elem, -1);
        std::vector<int8_t> nbk((size_t)12 * n_elem, 0), nbf((size_t)6 * n_elem, 0);
        auto set = [&](int64_t e, int64_t f, int8_t kd, int64_t e2, int64_t f2) {
            DRF_CHECK(e >= 0 && e < n_elem && f >= 0 && f < 6, DRF_E_INVALID, "face list entry out of range");
            DRF_CHECK(nbk[e * 6 + f] == 0, DRF_E_INVALID, "face listed twice");
            nbk[e * 6 + f] = kd;
            nbe[e * 6 + f] = e2;
            nbf[e * 6 + f] = (int8_t)f2;
        };
        for (int64_t i = 0; i < n_conf; ++i) {
            const int64_t *c = conf + 4 * i;
            DRF_CHECK(c[2] >= 0 && c[2] < n_elem && c[3] >= 0 && c[3] < 6 && c[1] / 2 == c[3] / 2 &&
                          c[1] != c[3],
                      DRF_E_INVALID, "conforming pair must join opposite faces of one axis");
            set(c[0], c[1], 1, c[2], c[3]);
            set(c[2], c[3], 1, c[0], c[1]);
        }
        for (int64_t i = 0; i < n_bnd; ++i) set(bnd[2 * i], bnd[2 * i + 1], 2, -1, 0);
        upload_amr_basis(order);
        DRF_CUDA(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
        h->stream = h->own;
        h->nbe.alloc(nbe.size());
        h->nbk.alloc(nbk.size());
        h->nbf.alloc(nbf.size());
        DRF_CUDA(cudaMemcpy(h->nbe.p, nbe.data(), nbe.size() * 8, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(h->nbk.p, nbk.data(), nbk.size(), cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(h->nbf.p, nbf.data(), nbf.size(), cudaMemcpyHostToDevice));
        const size_t n = (size_t)n_elem * h->nd;
        h->U.alloc(2 * n);
        h->R.alloc(n);
        h->res.alloc(n);
        h->out.alloc(n);
        DRF_CUDA(cudaMemset(h->U.p, 0, 2 * n * 8));
        DRF_CUDA(cudaMemset(h->res.p, 0, n * 8));
        if (n_if > 0) {
            const int rc = drf_mortar_create(order, n_if, type, coarse_elem, coarse_face, fine_elem, fine_face,
                                             n_elem, &h->mortar);
            DRF_CHECK(rc == DRF_OK, rc, "mortar interfaces rejected");
            DRF_CHECK(drf_mortar_set_stream(h->mortar, h->stream) == DRF_OK, DRF_E_CUDA, "mortar stream");
            // each element's index in the mortar space's touched-element list (-1: none)
            const MortarLifts L = mortar_lifts(h->mortar);
            std::vector<int64_t> touched((size_t)std::max<int64_t>(L.n_touched, 1));
            if (L.n_touched > 0)
                DRF_CUDA(cudaMemcpy(touched.data(), L.touched, L.n_touched * 8, cudaMemcpyDeviceToHost));
            std::vector<int> e2u((size_t)n_elem, -1);
            for (int64_t u = 0; u < L.n_touched; ++u) e2u[touched[u]] = (int)u;
            h->e2u.alloc(n_elem);
            DRF_CUDA(cudaMemcpy(h->e2u.p, e2u.data(), n_elem * 4, cudaMemcpyHostToDevice));
        }
        *out = h.release();
    });
}

int drf_amr_destroy(drf_amr *h) {
    return guard([&] {
        if (!h) return;
        if (h->stream) cudaStreamSynchronize(h->stream);
        delete h;
    });
}

int drf_amr_set_stream(drf_amr *h, void *s) {
    return guard([&] {
        amr_check(h);
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        h->drop_graph();
        h->stream = s ? (cudaStream_t)s : h->own;
        if (h->mortar) DRF_CHECK(drf_mortar_set_stream(h->mortar, h->stream) == DRF_OK, DRF_E_CUDA, "mortar stream");
    });
}

int drf_amr_upload(drf_amr *h, const double *U) {
    return guard([&] {
        amr_check(h);
        DRF_CHECK(U, DRF_E_INVALID, "null argument");
        const size_t n = (size_t)h->n_elem * h->nd;
        DRF_CHECK(all_finite(U, n), DRF_E_NONFINITE, "non-finite state");
        DRF_CUDA(cudaMemcpyAsync(h->state(), U, n * 8, cudaMemcpyHostToDevice, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_amr_download(drf_amr *h, double *U) {
    return guard([&] {
        amr_check(h);
        DRF_CHECK(U, DRF_E_INVALID, "null argument");
        const size_t n = (size_t)h->n_elem * h->nd;
        DRF_CUDA(cudaMemcpyAsync(U, h->state(), n * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        DRF_CHECK(all_finite(U, n), DRF_E_NONFINITE, "non-finite state (the run blew up)");
    });
}

int drf_amr_compute_rhs(drf_amr *h, int mode, int flux_kind, const double *a, const double *U, double *rhs) {
    return guard([&] {
        amr_check(h);
        amr_check_args(mode, flux_kind, a);
        DRF_CHECK(rhs, DRF_E_INVALID, "null output");
        const int64_t n = h->n_elem * h->nd;
        if (U) {
            DRF_CHECK(all_finite(U, (size_t)n), DRF_E_NONFINITE, "non-finite state");
            DRF_CUDA(cudaMemcpyAsync(h->state(), U, n * 8, cudaMemcpyHostToDevice, h->stream));
        }
        h->enqueue_rhs(mode, flux_kind, a);
        amr_dispatch(h->np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            amr_massinv_kernel<NP><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(n, h->R.p, h->out.p);
            DRF_LAUNCHED();
        });
        DRF_CUDA(cudaMemcpyAsync(rhs, h->out.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_amr_step(drf_amr *h, int mode, int flux_kind, const double *a, double dt, int nsteps) {
    return guard([&] {
        amr_check(h);
        amr_check_args(mode, flux_kind, a);
        DRF_CHECK(dt > 0.0 && std::isfinite(dt), DRF_E_INVALID, "dt must be positive");
        DRF_CHECK(nsteps >= 0, DRF_E_INVALID, "nsteps must be >= 0");
        if (!h->graph[0] || h->g_mode != mode || h->g_flux != flux_kind || h->g_dt != dt ||
            std::memcmp(h->g_a, a, sizeof(h->g_a)) != 0) {
            h->drop_graph();
            for (int b = 0; b < 2; ++b)
                h->graph[b] = capture_graph(h->stream, [&] { h->enqueue_step(mode, flux_kind, a, dt, b); },
                                            &h->graph_kernels);
            h->g_mode = mode;
            h->g_flux = flux_kind;
            h->g_dt = dt;
            std::memcpy(h->g_a, a, sizeof(h->g_a));
        }
        for (int s = 0; s < nsteps; ++s) {
            DRF_CUDA(cudaGraphLaunch(h->graph[h->cur], h->stream));
            launch_counter().fetch_add(h->graph_kernels);
            h->cur = 1 - h->cur;  // five stages leave the state in the other buffer
        }
    });
}

int drf_amr_sync(drf_amr *h) {
    return guard([&] {
        amr_check(h);
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int drf_amr_time_rhs(drf_amr *h, int mode, int flux_kind, const double *a, int nrep, double *ms,
                     double *alg_bytes) {
    return guard([&] {
        amr_check(h);
        amr_check_args(mode, flux_kind, a);
        DRF_CHECK(nrep >= 1 && ms, DRF_E_INVALID, "bad arguments");
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        h->enqueue_rhs(mode, flux_kind, a);  // warm-up
        DRF_CUDA(cudaEventRecord(e0, h->stream));
        for (int r = 0; r < nrep; ++r) h->enqueue_rhs(mode, flux_kind, a);
        DRF_CUDA(cudaEventRecord(e1, h->stream));
        DRF_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = (double)t / nrep;
        // algorithmic bytes of one right-hand side: u read and R written once per node, the
        // neighbours' face traces of the conforming faces (mode 1) and the mortars' face traces
        // read once, and the mortar lifts read-modify-written on the touched face nodes.
        const double npf = (double)h->np * h->np;
        const double faces = (mode == 1 ? 2.0 * h->n_conf : 0.0) + 3.0 * h->n_if;
        if (alg_bytes) *alg_bytes = 16.0 * h->n_elem * h->nd + 8.0 * faces * npf + 16.0 * 3.0 * h->n_if * npf;
    });
}

// GradientErrorEstimator::estimate (src/amr/refinement.cpp:44-68) of the resident state.
int drf_amr_estimate(drf_amr *h, const double *hchar, double refine_threshold, double coarsen_threshold,
                     double smoothness_factor, double *value, int32_t *mask, int32_t *flags) {
    return guard([&] {
        amr_check(h);
        DRF_CHECK(hchar && value && mask && flags, DRF_E_INVALID, "null argument");
        const int64_t ne = h->n_elem;
        if (ne == 0) return;
        DRF_CHECK(all_finite(hchar, (size_t)ne), DRF_E_NONFINITE, "non-finite element length");
        const int64_t nb = (ne + AMR_EST_WARPS - 1) / AMR_EST_WARPS;
        DevBuf<double> dh(ne), dv(ne), part(nb + 1);
        DevBuf<int> dm(ne), df(ne);
        DRF_CUDA(cudaMemcpyAsync(dh.p, hchar, ne * 8, cudaMemcpyHostToDevice, h->stream));
        amr_dispatch(h->np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            amr_estimate_kernel<NP><<<(unsigned)nb, 32 * AMR_EST_WARPS, 0, h->stream>>>(
                ne, h->state(), dh.p, smoothness_factor, dv.p, dm.p, part.p);
        });
        DRF_LAUNCHED();
        amr_max_kernel<<<1, 1024, 0, h->stream>>>(part.p, nb, part.p + nb);
        DRF_LAUNCHED();
        amr_flags_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, h->stream>>>(ne, part.p + nb, refine_threshold,
                                                                               coarsen_threshold, dv.p, df.p);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpyAsync(value, dv.p, ne * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaMemcpyAsync(mask, dm.p, ne * 4, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaMemcpyAsync(flags, df.p, ne * 4, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

// The resident state of `from` (levels old_*) carried into `to` (levels new_*), both of one
// order over the same nx x ny base columns.
int drf_amr_transfer(drf_amr *from, drf_amr *to, int nx, int ny, const int *old_lx, const int *old_ly,
                     const int *old_lz, const int *new_lx, const int *new_ly, const int *new_lz) {
    return guard([&] {
        amr_check(from);
        amr_check(to);
        DRF_CHECK(from != to, DRF_E_INVALID, "transfer needs two meshes");
        DRF_CHECK(nx >= 1 && ny >= 1 && old_lx && old_ly && old_lz && new_lx && new_ly && new_lz, DRF_E_INVALID,
                  "bad arguments");
        DRF_CHECK(from->order == to->order, DRF_E_INVALID, "meshes of different orders");
        const int ncol = nx * ny;
        std::vector<int> lvo(3 * ncol), lvn(3 * ncol);
        for (int c = 0; c < ncol; ++c) {
            const int o[3] = {old_lx[c], old_ly[c], old_lz[c]}, n[3] = {new_lx[c], new_ly[c], new_lz[c]};
            for (int d = 0; d < 3; ++d) {
                DRF_CHECK(o[d] >= 0 && o[d] <= 10 && n[d] >= 0 && n[d] <= 10, DRF_E_INVALID,
                          "refinement level out of range (0..10)");
                lvo[3 * c + d] = o[d];
                lvn[3 * c + d] = n[d];
            }
        }
        const std::vector<int64_t> offo = amr_column_offsets(ncol, lvo.data()), offn = amr_column_offsets(ncol, lvn.data());
        DRF_CHECK(offo[ncol] == from->n_elem && offn[ncol] == to->n_elem, DRF_E_INVALID,
                  "element counts do not match the levels");
        const int64_t nn = to->n_elem;
        std::vector<int> col(nn);
        for (int c = 0; c < ncol; ++c) {
            const int64_t cells = (int64_t)1 << (lvn[3 * c] + lvn[3 * c + 1] + lvn[3 * c + 2]);
            for (int64_t e = offn[c]; e < offn[c] + cells; ++e) col[e] = c;
        }
        const HostBasis b = make_lgl_basis(from->order);
        // the one-level rows, with the kernel's own formulas for the old-cell coordinate and
        // interpolate_3d's product formula
        const int np = b.np;
        std::vector<double> rows((size_t)4 * np * np);
        for (int cs = 0; cs < 4; ++cs)
            for (int m = 0; m < np; ++m) {
                const double x = b.x[m];
                double xo = x;
                if (cs == 1 || cs == 2) {
                    const double cl = -1.0 + 2.0 * (cs - 1) / 2, ch = cl + 2.0 / 2;
                    xo = cl + 0.5 * (x + 1.0) * (ch - cl);
                } else if (cs == 3) {
                    const int c1 = x >= 0 ? 1 : 0;
                    const double cl = -1.0 + 2.0 * c1 / 2, chi = cl + 2.0 / 2;
                    xo = std::min(1.0, std::max(-1.0, 2.0 * (x - cl) / (chi - cl) - 1.0));
                }
                for (int i = 0; i < np; ++i) {
                    double v = 1.0;
                    for (int j = 0; j < np; ++j)
                        if (j != i) v *= (xo - b.x[j]) / (b.x[i] - b.x[j]);
                    rows[((size_t)cs * np + m) * np + i] = v;
                }
            }
        DevBuf<double> drows(rows.size());
        DevBuf<int> dcol(nn), dlvo(3 * ncol), dlvn(3 * ncol);
        DevBuf<int64_t> doffo(ncol + 1), doffn(ncol + 1);
        DRF_CUDA(cudaStreamSynchronize(from->stream));
        cudaStream_t st = to->stream;
        DRF_CUDA(cudaMemcpyAsync(dcol.p, col.data(), nn * 4, cudaMemcpyHostToDevice, st));
        DRF_CUDA(cudaMemcpyAsync(dlvo.p, lvo.data(), lvo.size() * 4, cudaMemcpyHostToDevice, st));
        DRF_CUDA(cudaMemcpyAsync(dlvn.p, lvn.data(), lvn.size() * 4, cudaMemcpyHostToDevice, st));
        DRF_CUDA(cudaMemcpyAsync(doffo.p, offo.data(), offo.size() * 8, cudaMemcpyHostToDevice, st));
        DRF_CUDA(cudaMemcpyAsync(doffn.p, offn.data(), offn.size() * 8, cudaMemcpyHostToDevice, st));
        DRF_CUDA(cudaMemcpyAsync(drows.p, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice, st));
        AmrTransferArgs A{};
        A.Uo = from->state(); A.Un = to->state(); A.col_of = dcol.p; A.lvo = dlvo.p; A.lvn = dlvn.p;
        A.offo = doffo.p; A.offn = doffn.p; A.rows = drows.p; A.n_new = nn;
        for (int i = 0; i < b.np; ++i) A.xn[i] = b.x[i];
        const int64_t nthr = nn * from->nd;
        amr_dispatch(from->np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            amr_transfer_kernel<NP><<<(unsigned)((nthr + 255) / 256), 256, 0, st>>>(A);
        });
        DRF_LAUNCHED();
        DRF_CUDA(cudaStreamSynchronize(st));
    });
}

}  // extern "C"
