// Coupled DG model on the GPU: sum-factorized strong-form DGSEM right-hand side of the
// sigma-coordinate primitive equations with face fluxes and full-column omega, fused with
// the LSRK45 stage update; FP64 barotropic (2D) subcycles with the reference's shallow-water
// fluxes; one CUDA graph per baroclinic step.
//
// Layout in HBM (SoA, one array per variable):
//   3D: q[v][((c * nz + ez) * np^3) + i + np*(j + np*k)], c = ex + nx*ey  (a water column is
//       one contiguous block of nz*np^3 nodes per variable)
//   2D: x[c * np^2 + i + np*j]
// Kernel map (one baroclinic step, graph-captured):
//   dg3d_stage x5 (one CTA per water column: load column -> horizontal divergence ->
//   omega column scan in shared memory -> RHS -> LSRK update -> FP64 column increments)
//   baro_force, (baro_pred, baro_corr) x nsub, baro_finish; the transport correction the
//   barotropic step leaves is folded into the next step's first stage.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <map>
#include <tuple>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "flux.cuh"

namespace drf {
namespace {

// Basis tables per node count NP (orders 1..MAXNP-1 each keep their own entry, so models of
// different orders can live in one process).
__constant__ DevBasis cBs[MAXNP + 1];

template <typename T, int NP>
struct BT;
template <int NP>
struct BT<double, NP> {
    __device__ static double D(int i) { return cBs[NP].D[i]; }
    __device__ static double D2(int i) { return cBs[NP].D2[i]; }
    __device__ static double S(int i) { return cBs[NP].S[i]; }
    __device__ static double w(int i) { return cBs[NP].w[i]; }
    __device__ static double x(int i) { return cBs[NP].x[i]; }
    __device__ static double Ai(int i) { return cBs[NP].Ai[i]; }
    __device__ static double a0(int i) { return cBs[NP].a0[i]; }
};
template <int NP>
struct BT<float, NP> {
    __device__ static float D(int i) { return cBs[NP].Df[i]; }
    __device__ static float D2(int i) { return cBs[NP].D2f[i]; }
    __device__ static float S(int i) { return cBs[NP].Sf[i]; }
    __device__ static float w(int i) { return cBs[NP].wf[i]; }
    __device__ static float x(int i) { return cBs[NP].xf[i]; }
    __device__ static float Ai(int i) { return cBs[NP].Aif[i]; }
    __device__ static float a0(int i) { return cBs[NP].a0f[i]; }
};

struct Geo {
    int nx, ny, nz, flux2d;
    int bc[4];
    double cx, cy, cs, Lx, Ly, Ls, dsig;
    double g, rho0, nu_h, nu_v, kT, kS, cd;
    double tide_amp, tide_w;
    // linear equation of state of the baroclinic pressure gradient; eos = 0 switches it off
    double alpha, beta, T0, S0;
    double Tref_s, Tref_dz;  // reference stratification T_ref(z) = Tref_s + Tref_dz z
    int eos;
};

__device__ __forceinline__ double tide_at(const Geo &G, double t) {
    return G.tide_amp * sin(G.tide_w * t);
}

template <typename T>
struct StageArgs {
    const T *qin[4];
    T *qout[4];
    T *res[4];
    const double *eta, *h, *f, *taux, *tauy, *tdev;
    const double *corrU, *corrV;  // pending transport correction added to Hu, Hv on load (or null)
    // pending volume correction of the tracers (with corrU): HT, HS scaled by 1 + corrR
    const double *corrR;
    // stage elevation of the baroclinic pressure (the step's eta at its first stage), and in an
    // LSRK stage its update: etab_out = etab + B (A rese + dt deta), rese the 2D register
    const double *etab;
    double *etab_out, *rese;
    double toff;
    double *dHU3, *dHV3;
    T *omega_out;
    double *deta_out;
    T A, B, dt;
    int mode;   // 0: LSRK stage update, 1: write the right-hand side into res[]
    int first;  // 1: A = 0 stage (res not read, column increments overwritten)
    int bulk;   // 1: column blocks are 16-byte aligned -> staged with cp.async.bulk
    // with bulk staging: the column pf columns ahead (the one a CTA launched about one wave of
    // resident CTAs later takes) is prefetched into L2 at this column's start; 0 = none
    int pf;
    int *err;   // device status word (DRF_E_TIMEOUT when a bounded wait gives up)
    Geo G;
};

// ---- TMA bulk copy (global -> shared) completed on an mbarrier, with bounded waits
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    uint64_t g;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(src));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(g), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Bulk prefetch of global memory into L2 (no completion to wait for); 16-byte aligned source,
// size a multiple of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
    uint64_t g;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(src));
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g), "r"(bytes) : "memory");
}
// Prefetch of the 128-byte line holding a global address into L2 (no completion to wait for).
__device__ __forceinline__ void line_prefetch_l2(const void *p) {
    uint64_t g;
    asm volatile("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(p));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(g));
}
// Spins on the barrier's phase with an iteration limit; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase) {
    const uint32_t a = smem_addr(bar);
    for (long it = 0; it < (1L << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Threads per stage CTA at most (pencils are strided over the block); two CTAs of this size
// share an SM (the register budget the kernel is compiled for: 65536 / (2 * 448) = 73).
constexpr int STAGE_MAX_THREADS = 448;

// Two prognostic variables of one node processed together ((Hu, Hv) and (HT, HS) share every
// 1D operator entry and every face speed). FP32 pairs use Blackwell's packed FP32x2
// instructions (one instruction for both lanes, IEEE single rounding per lane, as the scalar
// form); FP64 pairs are two scalar operations.
template <typename T>
struct P2 {
    T x, y;
};
template <typename T>
__device__ __forceinline__ P2<T> bc(T s) { return {s, s}; }

__device__ __forceinline__ P2<float> p2fma(P2<float> a, P2<float> b, P2<float> c) {
    P2<float> r;
    asm("{ .reg .b64 ra, rb, rc, rd; mov.b64 ra, {%2, %3}; mov.b64 rb, {%4, %5}; mov.b64 rc, {%6, %7};"
        " fma.rn.f32x2 rd, ra, rb, rc; mov.b64 {%0, %1}, rd; }"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
__device__ __forceinline__ P2<float> p2mul(P2<float> a, P2<float> b) {
    P2<float> r;
    asm("{ .reg .b64 ra, rb, rd; mov.b64 ra, {%2, %3}; mov.b64 rb, {%4, %5};"
        " mul.rn.f32x2 rd, ra, rb; mov.b64 {%0, %1}, rd; }"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ P2<float> p2add(P2<float> a, P2<float> b) {
    P2<float> r;
    asm("{ .reg .b64 ra, rb, rd; mov.b64 ra, {%2, %3}; mov.b64 rb, {%4, %5};"
        " add.rn.f32x2 rd, ra, rb; mov.b64 {%0, %1}, rd; }"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ P2<float> p2sub(P2<float> a, P2<float> b) {
    P2<float> r;
    asm("{ .reg .b64 ra, rb, rd; mov.b64 ra, {%2, %3}; mov.b64 rb, {%4, %5};"
        " sub.rn.f32x2 rd, ra, rb; mov.b64 {%0, %1}, rd; }"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
// k * x + c with a scalar k (an operator entry from constant memory): two scalar FMAs, which
// take the constant as an operand (a packed FMA would first need it duplicated in registers)
template <typename T>
__device__ __forceinline__ P2<T> p2fma_k(T k, P2<T> x, P2<T> c) {
    return {fma(k, x.x, c.x), fma(k, x.y, c.y)};
}
__device__ __forceinline__ P2<double> p2fma(P2<double> a, P2<double> b, P2<double> c) {
    return {fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)};
}
__device__ __forceinline__ P2<double> p2mul(P2<double> a, P2<double> b) { return {a.x * b.x, a.y * b.y}; }
__device__ __forceinline__ P2<double> p2add(P2<double> a, P2<double> b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ P2<double> p2sub(P2<double> a, P2<double> b) { return {a.x - b.x, a.y - b.y}; }

// Shared-memory plan of the stage kernel for one water column (ncn = nz*(N+1)^3 nodes):
//   three mbarriers (32 B), the FP64 column increments of the earlier stages [2][(N+1)^2],
//   sQ[4][ncn] state, sRes[4][ncn] LSRK 2N register, sR[4][ncn] right-hand side, sD[ncn]
//   horizontal divergence, per layer x 2D-node increments, the
//   column's 2D fields (1/H, H, eta), its pressure-gradient rows, 1 + sigma per z node and the
//   baroclinic pressure's 2D rows (its stage elevation, depth, 1 / depth and the slopes of
//   both), and per layer x 2D-node quadrature totals of the divergence.
// The baroclinic pressure P = H B at the column's nodes and across its four sides is formed
// before the horizontal passes in the register slots of HT and HS (whose register is staged
// after those passes), and its layer totals in sD; for N + 1 <= 3 the side values (and for
// N = 1 the layer totals) do not fit there and take a tail of their own.
template <int NP>
struct StageTail {
    static constexpr bool pn_in_res = 4 * NP * NP <= NP * NP * NP;  // sides' P in sRes[3]
    static constexpr bool tb_in_d = NP + 4 <= NP * NP;             // layer totals in sD
    static constexpr size_t elems(int nz) {
        return (pn_in_res ? 0 : (size_t)4 * nz * NP * NP) + (tb_in_d ? 0 : (size_t)nz * NP * (NP + 4));
    }
};
// Per side and face node, the neighbouring column's 2D values a face flux needs (its elevation
// e, depth H = e + h, pending corrections of Hu, Hv and the tracers, and the baroclinic
// pressure's depth Hb = etab + h, stage elevation etab and 1 / Hb), staged once per column
// instead of loaded by every pencil end and face line.
constexpr int STAGE_NF = 8;
inline size_t stage_tail_elems(int nz, int np) {
    switch (np) {
    case 2: return StageTail<2>::elems(nz);
    case 3: return StageTail<3>::elems(nz);
    case 4: return StageTail<4>::elems(nz);
    case 5: return StageTail<5>::elems(nz);
    default: return StageTail<6>::elems(nz);
    }
}
inline size_t stage_smem_bytes(int nz, int np, size_t tsz) {
    const int np2 = np * np, ncn = nz * np2 * np;
    return 32 + (size_t)4 * np2 * 8 +
           ((size_t)13 * ncn + (size_t)3 * nz * np2 + 12 * np2 + (size_t)nz * np + stage_tail_elems(nz, np) +
            (size_t)4 * np * STAGE_NF + (size_t)6 * np2) *
               tsz;
}

// One CTA per water column; work is organised in pencils (lines of N+1 nodes) so every
// thread applies the 1D operators to registers, with the operator entries read as
// warp-uniform constants: x pencils (j,k,layer), y pencils (i,k,layer), z pencils (i,j,layer).
//
// Layer-half thread mapping of the stage kernel instances with a compile-time, even layer count
// (pencils per half HP, threads per half HT, a whole number of warps; 2 HT threads a CTA).
template <int NP, int NZ>
struct StageHalves {
    static constexpr bool on = NZ > 0 && NZ % 2 == 0;
    static constexpr int HP = on ? NZ * NP * NP / 2 : 0;
    static constexpr int HT = on ? ((HP + 31) / 32) * 32 : 0;
};

// Where a column's data live: a single model's arrays (zero offsets, clock 0), or an ensemble
// member's slices of the pooled arrays (element offsets of its 3D and 2D arrays, its clock, its
// bulk-copy alignment and its baroclinic step).
struct ColView {
    int64_t off3, off2;
    int tidx, bulk;
    double dt;
};

// stage_column is the work of one CTA on column c. `ph` is the phase parity the column's
// mbarrier waits expect and `init` says whether this CTA still has to initialise the two
// mbarriers (the first column a CTA processes). Returns false when a bounded wait gave up
// (the status word is set); the CTA must then stop.
// NZ > 0 compiles the column for that layer count (its sizes and shared-memory offsets become
// constants); NZ = 0 takes the layer count from the arguments.
template <typename T, int NP, int NZ = 0>
__device__ __forceinline__ bool stage_column(const StageArgs<T> &a, const Geo &G, const ColView &cv, int c,
                                             uint32_t ph, bool init) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP, N = NP - 1;
    using B = BT<T, NP>;
    const int nz = NZ > 0 ? NZ : G.nz, ncn = nz * NP3, npen = nz * NP2;
    const int ex = c % G.nx, ey = c / G.nx;
    // Pencils to threads. With the layer count a compile-time even number, the layers' two
    // halves go to two groups of whole warps (StageHalves), each with one pencil per thread,
    // and the horizontal passes synchronise each half alone (named barriers 1 and 2): a
    // pass of a layer reads only that layer. Otherwise thread t takes pencils t, t + blockDim.
    using SH = StageHalves<NP, NZ>;
    const int hf = SH::on ? (int)threadIdx.x / SH::HT : 0;
    const int my_p = SH::on ? hf * SH::HP + (int)threadIdx.x % SH::HT : (int)threadIdx.x;
    const bool my_valid = SH::on ? (hf < 2 && (int)threadIdx.x % SH::HT < SH::HP) : (int)threadIdx.x < npen;
    const int p_first = my_valid ? my_p : npen;
    auto p_next = [&](int p) { return SH::on ? npen : p + (int)blockDim.x; };
    auto half_sync = [&] {
        if constexpr (SH::on) asm volatile("bar.sync %0, %1;" ::"r"(1 + hf), "r"(SH::HT) : "memory");
        else __syncthreads();
    };
    const size_t base = (size_t)cv.off3 + (size_t)c * ncn, c2 = (size_t)cv.off2 + (size_t)c * NP2;
    const T dtc = (T)cv.dt;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // mbarriers: state, register of (Hu, Hv), register of (HT, HS)
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    double *sOld = reinterpret_cast<double *>(smem_raw + 32);  // [2][NP2] column increments so far
    double *sRe = sOld + 2 * NP2, *sEtb = sRe + NP2;  // the bed's 2D register and stage elevation
    T *sQ = reinterpret_cast<T *>(smem_raw + 32 + 4 * NP2 * sizeof(double));  // [4][ncn]
    T *sRes = sQ + 4 * ncn;                        // [4][ncn]
    T *sR = sRes + 4 * ncn;                        // [4][ncn]
    T *sD = sR + 4 * ncn;                          // [ncn] divergence -> layer integrals
    T *sL1 = sD + ncn;                             // [nz][NP2] column increments (Hu)
    T *sL2 = sL1 + nz * NP2;                       // [nz][NP2] column increments (Hv)
    T *sIH = sL2 + nz * NP2, *sHt = sIH + NP2, *sEt = sHt + NP2;
    T *sPx = sEt + NP2, *sPy = sPx + NP2;          // g H d(eta)/dx, g H d(eta)/dy per 2D node
    T *sS1 = sPy + NP2;                            // [nz][NP] 1 + sigma at the column's z nodes
    // the baroclinic pressure's 2D rows (stage elevation etab): etab, Hb = etab + h, 1 / Hb,
    // g d(etab)/dx, g d(etab)/dy, g dHb/dx, g dHb/dy
    T *sEb = sS1 + nz * NP, *sHb = sEb + NP2, *sIHb = sHb + NP2;
    T *sGEx = sIHb + NP2, *sGEy = sGEx + NP2, *sGHx = sGEy + NP2, *sGHy = sGHx + NP2;
    T *sQl = sGHy + NP2;  // [nz][NP2] layer quadrature totals of the horizontal divergence
    T *tail = sQl + nz * NP2;
    // baroclinic pressure P = H B (B = int_sigma^0 b, b the density anomaly / rho0): at the
    // column's nodes, across its sides [side][face node][layer][k], and the layer totals of b
    // [layer][2D node] and [side][face node][layer]; alive from the pre-pass to the y pass
    using Tl = StageTail<NP>;
    T *sP = sRes + 2 * ncn;
    T *sPn = Tl::pn_in_res ? sRes + 3 * ncn : tail;
    T *sTb = Tl::tb_in_d ? sD : tail + (Tl::pn_in_res ? 0 : 4 * nz * NP2);
    T *sTbn = sTb + nz * NP2;
    // the neighbours' 2D face values [side][face node][STAGE_NF]
    T *sNF = tail + Tl::elems(nz);
    // the z pass's 2D fields per 2D node: Coriolis, surface stress / rho0 (x, y); and the pending
    // transport correction of the column (Hu, Hv, tracers)
    T *sFc = sNF + 4 * NP * STAGE_NF, *sTx = sFc + NP2, *sTy = sTx + NP2;
    T *sCu = sTy + NP2, *sCv = sCu + NP2, *sCr = sCv + NP2;
    __shared__ int s_ok, s_ok2;

    const bool need_res = a.mode == 0 && !a.first;
    // with the baroclinic pressure on, the register of (HT, HS) is staged after the horizontal
    // passes (its shared memory holds P until then)
    const bool late = need_res && G.eos;

    // ---- stage the column: state by TMA bulk copies when aligned (the 2N register follows after
    // the first barrier). They are issued first: any global load thread 0 made before them
    // would hold them back by its latency.
    if (cv.bulk) {
        if (threadIdx.x == 0) {
            if (init) {
                mbar_init(&bars[0], 1);
                mbar_init(&bars[1], 1);
                mbar_init(&bars[2], 1);
            } else {
                // shared memory of the previous column was read and written by this CTA's
                // threads: order those accesses before the bulk copies overwrite it
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            const uint32_t bytes = (uint32_t)(ncn * sizeof(T));
            mbar_expect_tx(&bars[0], 4 * bytes);
#pragma unroll
            for (int v = 0; v < 4; ++v) bulk_g2s(sQ + v * ncn, a.qin[v] + base, bytes, &bars[0]);
        }
    }
    // tidal elevation: evaluated once per CTA, and only by a column on a tidal side
    __shared__ T s_etide;
    if (threadIdx.x == 0) {
        s_ok2 = 1;
        const bool tidal = (ex == 0 && G.bc[0] == DRF_BC_TIDE) || (ex == G.nx - 1 && G.bc[1] == DRF_BC_TIDE) ||
                           (ey == 0 && G.bc[2] == DRF_BC_TIDE) || (ey == G.ny - 1 && G.bc[3] == DRF_BC_TIDE);
        s_etide = tidal ? (T)tide_at(G, a.tdev[cv.tidx] + a.toff) : T(0);
    }
    T etide = 0;  // read after the first barrier
    const T cx = (T)G.cx, cy = (T)G.cy, cs = (T)G.cs;
    const T Lx = (T)G.Lx, Ly = (T)G.Ly, Ls = (T)G.Ls;
    const T g = (T)G.g;
    // the column a CTA launched about pf columns later takes, into L2: its state and register
    // blocks (bulk prefetches, threads 32-39) and the lines of its 2D blocks (threads 40-87:
    // four probes per block of NP2 doubles, the first and last at its ends and less than 128
    // bytes apart, so every 128-byte line of the block holds one)
    if (a.pf > 0 && threadIdx.x >= 32 && threadIdx.x < 88 && c + a.pf < G.nx * G.ny) {
        const int l = threadIdx.x - 32;
        if (l < 8) {
            if (cv.bulk) {
                const size_t pb = (size_t)(c + a.pf) * ncn;
                const uint32_t bytes = (uint32_t)(ncn * sizeof(T));
                if (l < 4) bulk_prefetch_l2(a.qin[l] + pb, bytes);
                else if (need_res) bulk_prefetch_l2(a.res[l - 4] + pb, bytes);
            }
        } else {
            const int k = (l - 8) / 4, pr = (l - 8) % 4;
            const double *arr = nullptr;
            switch (k) {
            case 0: arr = a.eta; break;
            case 1: arr = a.h; break;
            case 2: arr = a.f; break;
            case 3: arr = a.dHU3; break;
            case 4: arr = a.dHV3; break;
            case 5: arr = a.taux; break;
            case 6: arr = a.tauy; break;
            case 7: arr = a.etab; break;
            case 8: arr = a.rese; break;
            case 9: arr = a.corrU; break;
            case 10: arr = a.corrV; break;
            default: arr = a.corrR; break;
            }
            if (arr) line_prefetch_l2(arr + (size_t)cv.off2 + (size_t)(c + a.pf) * NP2 + pr * (NP2 - 1) / 3);
        }
    }
    // the column increments of the earlier stages, read while the column is being staged: loaded
    // here and stored after the column's 2D loads below, so the first warp waits for one global
    // round trip instead of two
    const bool old = a.mode == 0 && !a.first;
    double old0 = 0.0, old1 = 0.0;
    if (old && (int)threadIdx.x < NP2) {
        old0 = a.dHU3[c2 + threadIdx.x];
        old1 = a.dHV3[c2 + threadIdx.x];
    }
    if (!cv.bulk) {
        for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
#pragma unroll
            for (int v = 0; v < 4; ++v) sQ[v * ncn + n] = a.qin[v][base + n];
            if (need_res)
                for (int v = 0; v < (late ? 2 : 4); ++v) sRes[v * ncn + n] = a.res[v][base + n];
        }
    }
    for (int t = threadIdx.x; t < NP2; t += blockDim.x) {
        const double *ec = a.eta + c2;
        const double e = ec[t];
        const double H = e + a.h[c2 + t];
        sEt[t] = (T)e;
        sHt[t] = (T)H;
        sIH[t] = (T)(1.0 / H);
        // the column's pressure-gradient rows g H d(eta)/dx, g H d(eta)/dy (shared by its layers)
        const int i = t % NP, j = t / NP;
        T gex = 0, gey = 0;
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            gex += B::D(i * NP + m) * (T)ec[m + NP * j];
            gey += B::D(j * NP + m) * (T)ec[i + NP * m];
        }
        sPx[t] = g * (T)H * cx * gex;
        sPy[t] = g * (T)H * cy * gey;
        if (G.eos) {
            // the baroclinic pressure's column: depth Hb = etab + h and g dz/dx|_sigma =
            // g d(etab)/dx + sigma g dHb/dx (element-local derivatives)
            const double *bc = a.etab + c2, *hc = a.h + c2;
            T gex2 = 0, gey2 = 0, ghx = 0, ghy = 0;
#pragma unroll
            for (int m = 0; m < NP; ++m) {
                const T ex_ = (T)bc[m + NP * j], ey_ = (T)bc[i + NP * m];
                gex2 += B::D(i * NP + m) * ex_;
                gey2 += B::D(j * NP + m) * ey_;
                ghx += B::D(i * NP + m) * (ex_ + (T)hc[m + NP * j]);
                ghy += B::D(j * NP + m) * (ey_ + (T)hc[i + NP * m]);
            }
            const double Hb = bc[t] + hc[t];
            sEb[t] = (T)bc[t];
            sHb[t] = (T)Hb;
            sIHb[t] = (T)(1.0 / Hb);
            sGEx[t] = g * cx * gex2;
            sGEy[t] = g * cy * gey2;
            sGHx[t] = g * cx * ghx;
            sGHy[t] = g * cy * ghy;
        }
    }
    if (old) {
        if ((int)threadIdx.x < NP2) {
            sOld[threadIdx.x] = old0;
            sOld[NP2 + threadIdx.x] = old1;
        }
        for (int t = threadIdx.x + blockDim.x; t < NP2; t += blockDim.x) {
            sOld[t] = a.dHU3[c2 + t];
            sOld[NP2 + t] = a.dHV3[c2 + t];
        }
    }
    for (int t = threadIdx.x; t < nz * NP; t += blockDim.x) {
        const int ez = t / NP, k = t % NP;
        sS1[t] = (ez == nz - 1 && k == N) ? T(1) : (T)(G.dsig * (ez + 0.5 * ((double)B::x(k) + 1.0)));
    }
    // the neighbours' 2D face values, side sd, face node tt (threads from 96 on where the CTA
    // has them, clear of the first warps' 2D loads and prefetches)
    {
        const int so = (int)blockDim.x >= 96 + 4 * NP ? 96 : 0;
        for (int t = (int)threadIdx.x - so; t >= 0 && t < 4 * NP; t += blockDim.x) {
            const int sd = t / NP, tt = t % NP;
            int nc = -1, ni = tt, nj = tt;
            if (sd == 0 && ex > 0) { nc = c - 1; ni = N; }
            if (sd == 1 && ex < G.nx - 1) { nc = c + 1; ni = 0; }
            if (sd == 2 && ey > 0) { nc = c - G.nx; nj = N; }
            if (sd == 3 && ey < G.ny - 1) { nc = c + G.nx; nj = 0; }
            if (nc < 0) continue;
            const size_t n2 = ((size_t)cv.off2 + (size_t)nc * NP2) + ni + NP * nj;
            T *f = sNF + t * STAGE_NF;
            const double e = a.eta[n2], hn = a.h[n2];
            f[0] = (T)e;
            f[1] = (T)(e + hn);
            if (a.corrU) {
                f[2] = (T)a.corrU[n2];
                f[3] = (T)a.corrV[n2];
                f[4] = (T)a.corrR[n2];
            }
            if (G.eos) {
                const double eb = a.etab[n2], Hd = eb + hn;
                f[5] = (T)Hd;
                f[6] = (T)eb;
                f[7] = (T)(1.0 / Hd);
            }
        }
    }
    // the z pass's 2D fields and the column's pending correction, staged now so that no pass
    // after the column load waits for a global load (threads from 128 on where the CTA has them)
    {
        const int so = (int)blockDim.x >= 128 + NP2 ? 128 : 0;
        for (int t = (int)threadIdx.x - so; t >= 0 && t < NP2; t += blockDim.x) {
            sFc[t] = (T)a.f[c2 + t];
            sTx[t] = (T)(a.taux[c2 + t] / G.rho0);
            sTy[t] = (T)(a.tauy[c2 + t] / G.rho0);
            if (a.mode == 0) {
                sRe[t] = a.first ? 0.0 : a.rese[c2 + t];
                sEtb[t] = a.etab[c2 + t];
            }
            if (a.corrU) {
                sCu[t] = (T)a.corrU[c2 + t];
                sCv[t] = (T)a.corrV[c2 + t];
                sCr[t] = (T)a.corrR[c2 + t];
            }
        }
    }
    // state across horizontal side s at own node (ez,i,j,k): q+ (4), eta+, H+
    struct Side {
        T q[4], e, H;
    };
    // the neighbouring column's state across side s (global loads); false on a basin side
    auto fetch_side = [&](int s, int ez, int i, int j, int k, Side &o) -> bool {
        int nc = -1, ni = i, nj = j;
        if (s == 0 && ex > 0) { nc = c - 1; ni = N; }
        if (s == 1 && ex < G.nx - 1) { nc = c + 1; ni = 0; }
        if (s == 2 && ey > 0) { nc = c - G.nx; nj = N; }
        if (s == 3 && ey < G.ny - 1) { nc = c + G.nx; nj = 0; }
        if (nc < 0) return false;
        const size_t nb = ((size_t)cv.off3 + (size_t)nc * ncn) + (size_t)ez * NP3 + ni + NP * (nj + NP * k);
#pragma unroll
        for (int v = 0; v < 4; ++v) o.q[v] = a.qin[v][nb];
        return true;
    };
    // completes a fetched side at face node tt from the staged 2D face values (after the first
    // barrier): the neighbour's pending transport correction, its elevation and depth
    auto finish_side = [&](int s, int tt, Side &o) {
        const T *f = sNF + (s * NP + tt) * STAGE_NF;
        if (a.corrU) {
            o.q[0] += f[2];
            o.q[1] += f[3];
            const T dr = f[4];
            o.q[2] = fma(o.q[2], dr, o.q[2]);
            o.q[3] = fma(o.q[3], dr, o.q[3]);
        }
        o.e = f[0];
        o.H = f[1];
    };
    // the exterior state on a basin side (wall mirror or tidal elevation) at own node n
    auto basin_side = [&](int s, int i, int j, int n, Side &o) {
        const int an = i + NP * j;
        const int bcs = s == 0 ? G.bc[0] : (s == 1 ? G.bc[1] : (s == 2 ? G.bc[2] : G.bc[3]));
        if (bcs == DRF_BC_TIDE) {
            o.e = etide;
            o.H = etide + (T)a.h[c2 + an];
            const T r = o.H * sIH[an];
#pragma unroll
            for (int v = 0; v < 4; ++v) o.q[v] = sQ[v * ncn + n] * r;
        } else {
            o.e = sEt[an];
            o.H = sHt[an];
#pragma unroll
            for (int v = 0; v < 4; ++v) o.q[v] = sQ[v * ncn + n];
            if (s <= 1) o.q[0] = -o.q[0]; else o.q[1] = -o.q[1];
        }
    };
    // the neighbour faces of this thread's first x pencil are loaded while the column's bulk
    // copies are in flight (the x pass then starts without a global-load wait)
    Side fx0, fxN;
    bool hx0 = false, hxN = false;
    if (my_valid) {
        const int p = my_p, ez = p / NP2, j = p % NP, k = (p / NP) % NP;
        hx0 = fetch_side(0, ez, 0, j, k, fx0);
        hxN = fetch_side(1, ez, N, j, k, fxN);
    }
    // with the baroclinic pressure on: the tracers along this thread's first neighbour face line
    // of the pre-pass below (item npen + fl0 of its strided loop), loaded now like the x faces;
    // FP32 instances with a compile-time layer count only (the others have no registers to spare)
    constexpr bool PRE = NZ > 0 && sizeof(T) == 4;
    const int nfl = 4 * NP * nz;  // neighbour face lines: (side, face node, layer)
    int fl0 = -1;
    T flT[NP], flS[NP];
    if (PRE && G.eos) {
        const int x = (int)threadIdx.x, bd = (int)blockDim.x;
        const int i0 = x >= npen ? x : x + bd * ((npen - x + bd - 1) / bd);
        const int f = i0 - npen, sd = f / (NP * nz), tt = (f / nz) % NP, ez = f % nz;
        int nc = -1, ni = tt, nj = tt;
        if (sd == 0 && ex > 0) { nc = c - 1; ni = N; }
        if (sd == 1 && ex < G.nx - 1) { nc = c + 1; ni = 0; }
        if (sd == 2 && ey > 0) { nc = c - G.nx; nj = N; }
        if (sd == 3 && ey < G.ny - 1) { nc = c + G.nx; nj = 0; }
        if (f < nfl && nc >= 0) {
            fl0 = f;
            const size_t nb = ((size_t)cv.off3 + (size_t)nc * ncn) + (size_t)ez * NP3 + ni + NP * nj;
#pragma unroll
            for (int m = 0; m < NP; ++m) {
                flT[m] = a.qin[2][nb + NP2 * m];
                flS[m] = a.qin[3][nb + NP2 * m];
            }
        }
    }
    if (threadIdx.x == 0) s_ok = cv.bulk ? (int)mbar_wait(&bars[0], ph) : 1;
    __syncthreads();
    if (!s_ok) {
        if (threadIdx.x == 0) atomicExch(a.err, DRF_E_TIMEOUT);
        return false;
    }
    etide = s_etide;
    // the register in two halves, each completing one phase of its own barrier; issued once the
    // state is in, so the state's copies do not share the memory system with them (the register
    // is first read in the z pass)
    if (cv.bulk && need_res && threadIdx.x == 0) {
        const uint32_t bytes = (uint32_t)(ncn * sizeof(T));
        mbar_expect_tx(&bars[1], 2 * bytes);
        for (int v = 0; v < 2; ++v) bulk_g2s(sRes + v * ncn, a.res[v] + base, bytes, &bars[1]);
        if (!late) {
            mbar_expect_tx(&bars[2], 2 * bytes);
            for (int v = 2; v < 4; ++v) bulk_g2s(sRes + v * ncn, a.res[v] + base, bytes, &bars[2]);
        }
    }
    if (a.corrU) {  // pending transport correction of the previous step
        for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
            const int an = n % NP2;
            sQ[n] += sCu[an];
            sQ[ncn + n] += sCv[an];
            const T dr = sCr[an];
            sQ[2 * ncn + n] = fma(sQ[2 * ncn + n], dr, sQ[2 * ncn + n]);
            sQ[3 * ncn + n] = fma(sQ[3 * ncn + n], dr, sQ[3 * ncn + n]);
        }
        __syncthreads();
    }

    // ---- baroclinic pressure (linear equation of state). The density anomaly against the
    // reference stratification, b = beta (S - S0) - alpha (T - T_ref(z)) (T = HT / H, S = HS / H
    // formed as deviations to keep their digits, z = eta + sigma H), at every node;
    // B(sigma) = int_sigma^0 b is the sum of the totals of the layers from this one up minus the
    // layer integral J_k = (dsig/2) sum_m S[k][m] b_m, and P = H B (p' = rho0 g P). The same is
    // formed along the neighbouring columns' face lines (their P is the face value P+). The
    // force on (Hu, Hv) is taken in flux form, -g [d(H P)/dx|_sigma - d(P dz/dx|_sigma)/dsigma]
    // with dz/dx|_sigma = d(eta)/dx + sigma dH/dx: its sigma part is formed here along the
    // column's z lines and starts the right-hand side of Hu and Hv; the horizontal passes add
    // the x and y parts.
    if (G.eos) {
        const T al = (T)G.alpha, be = (T)G.beta, S0 = (T)G.S0;
        const T Trs = (T)G.Tref_s, Trz = (T)G.Tref_dz;
        const T hd2 = (T)(0.5 * G.dsig);
        // the neighbouring column across side sd and the face node (ni, nj) of face line tt
        auto face_line = [&](int sd, int tt, int &ni, int &nj) -> int {
            int nc = -1;
            ni = tt; nj = tt;
            if (sd == 0 && ex > 0) { nc = c - 1; ni = N; }
            if (sd == 1 && ex < G.nx - 1) { nc = c + 1; ni = 0; }
            if (sd == 2 && ey > 0) { nc = c - G.nx; nj = N; }
            if (sd == 3 && ey < G.ny - 1) { nc = c + G.nx; nj = 0; }
            return nc;
        };
        // phase 1: layer integrals J_k into sP / sPn, layer totals into sTb / sTbn
        for (int t = threadIdx.x; t < npen + nfl; t += blockDim.x) {
            T bv[NP];
            T *dst, *tot;
            int dstep;
            if (t < npen) {
                const int ez = t / NP2, an = t % NP2, e0 = ez * NP3 + an;
                const T iH = sIHb[an], H = sHb[an], et = sEb[an];
#pragma unroll
                for (int m = 0; m < NP; ++m) {
                    const int n = e0 + NP2 * m;
                    const T Tr = fma(Trz, fma(sS1[ez * NP + m] - T(1), H, et), Trs);
                    bv[m] = fma(be, fma(sQ[3 * ncn + n], iH, -S0), -al * fma(sQ[2 * ncn + n], iH, -Tr));
                }
                dst = sP + e0;
                dstep = NP2;
                tot = sTb + ez * NP2 + an;
            } else {
                const int f = t - npen, sd = f / (NP * nz), tt = (f / nz) % NP, ez = f % nz;
                int ni, nj;
                const int nc = face_line(sd, tt, ni, nj);
                if (nc < 0) continue;
                const T *nf = sNF + (sd * NP + tt) * STAGE_NF;
                const T Hn = nf[5], etn = nf[6], iHn = nf[7];
                // the neighbour's pending tracer volume correction, with the arithmetic of the
                // neighbour's own load (or of the correction applied to the state)
                const T dr = a.corrU ? nf[4] : T(0);
                const size_t nb = ((size_t)cv.off3 + (size_t)nc * ncn) + (size_t)ez * NP3 + ni + NP * nj;
                const bool pre = PRE && f == fl0;  // loaded before the first barrier
#pragma unroll
                for (int m = 0; m < NP; ++m) {
                    const T Tr = fma(Trz, fma(sS1[ez * NP + m] - T(1), Hn, etn), Trs);
                    const T hs = pre ? flS[m] : a.qin[3][nb + NP2 * m], ht = pre ? flT[m] : a.qin[2][nb + NP2 * m];
                    bv[m] = fma(be, fma(fma(hs, dr, hs), iHn, -S0), -al * fma(fma(ht, dr, ht), iHn, -Tr));
                }
                dst = sPn + ((sd * NP + tt) * nz + ez) * NP;
                dstep = 1;
                tot = sTbn + (sd * NP + tt) * nz + ez;
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                T sk = 0;
#pragma unroll
                for (int m = 0; m < NP; ++m) sk += B::S(k * NP + m) * bv[m];
                const T J = k == 0 ? T(0) : hd2 * sk;
                dst[dstep * k] = J;
                if (k == N) *tot = J;
            }
        }
        __syncthreads();
        // phase 2: P = H (sum of the layer totals from this layer up - J_k), in place; the
        // column's z lines also form the sigma part of the force, g d(P dz/dx)/dsigma
        for (int t = threadIdx.x; t < npen + nfl; t += blockDim.x) {
            if (t < npen) {
                const int ez = t / NP2, an = t % NP2, e0 = ez * NP3 + an;
                T Tab = 0;
                for (int e = nz - 1; e >= ez; --e) Tab += sTb[e * NP2 + an];
                const T H = sHb[an];
                const T px = sGEx[an], py = sGEy[an], hx = sGHx[an], hy = sGHy[an];
                T Pk[NP], zx[NP], zy[NP];
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    Pk[k] = H * (Tab - sP[e0 + NP2 * k]);
                    sP[e0 + NP2 * k] = Pk[k];
                    // g dz/dx|_sigma = g d(etab)/dx + sigma g dHb/dx
                    const T sg = sS1[ez * NP + k] - T(1);
                    zx[k] = fma(sg, hx, px);
                    zy[k] = fma(sg, hy, py);
                }
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    T sx = 0, sy = 0;
#pragma unroll
                    for (int m = 0; m < NP; ++m) {
                        sx += B::D(k * NP + m) * (Pk[m] * zx[m]);
                        sy += B::D(k * NP + m) * (Pk[m] * zy[m]);
                    }
                    sR[e0 + NP2 * k] = cs * sx;
                    sR[ncn + e0 + NP2 * k] = cs * sy;
                }
            } else {
                const int f = t - npen, sd = f / (NP * nz), tt = (f / nz) % NP, ez = f % nz;
                int ni, nj;
                const int nc = face_line(sd, tt, ni, nj);
                if (nc < 0) continue;
                (void)ni;
                (void)nj;
                const T Hn = sNF[(sd * NP + tt) * STAGE_NF + 5];
                const T *tl = sTbn + (sd * NP + tt) * nz;
                T Tab = 0;
                for (int e = nz - 1; e >= ez; --e) Tab += tl[e];
                T *pl = sPn + ((sd * NP + tt) * nz + ez) * NP;
#pragma unroll
                for (int k = 0; k < NP; ++k) pl[k] = Hn * (Tab - pl[k]);
            }
        }
        __syncthreads();
    }

    // ---- horizontal passes. Each pencil (a line of N+1 nodes) gives its direction's part of
    // (1) the horizontal divergence of (Hu, Hv) with a central face flux, which feeds omega, and
    // (2) the right-hand side: advection, pressure, horizontal diffusion and the LF face terms,
    // with the variables processed in pairs (Hu, Hv), (HT, HS). Both face neighbours are
    // fetched up front so their latencies overlap.
    const T nh = (T)G.nu_h;
    const bool hdiff = G.nu_h > 0.0;
    // one horizontal pencil: axis 0 (x, sides 0/1) or 1 (y, sides 2/3), a compile-time
    // constant of each instance; nodes e0 + st*m
    auto hpass = [&](auto AX, int e0, int st, int iy, int jx, const Side &o0, const Side &oN, T Pp0,
                     T PpN) {
        constexpr int axis = decltype(AX)::value;
        const T cd = axis == 0 ? cx : cy, Ld = axis == 0 ? Lx : Ly;
        const T ep0 = o0.e, epN = oN.e, Hp0 = o0.H, HpN = oN.H;
        // the neighbours' momentum normal to this pencil's faces and the two variable pairs
        const T qn0 = axis == 0 ? o0.q[0] : o0.q[1], qnN = axis == 0 ? oN.q[0] : oN.q[1];
        const P2<T> p0a = {o0.q[0], o0.q[1]}, p0b = {o0.q[2], o0.q[3]};
        const P2<T> pNa = {oN.q[0], oN.q[1]}, pNb = {oN.q[2], oN.q[3]};
        // 2D node of pencil node m: x pencil (m, iy), y pencil (jx, m)
        auto an2 = [&](int m) { return axis == 0 ? m + NP * iy : jx + NP * m; };
        P2<T> q01[NP];
        T ih[NP], un[NP];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            q01[m] = {sQ[e0 + st * m], sQ[ncn + e0 + st * m]};
            ih[m] = sIH[an2(m)];
            un[m] = (axis == 0 ? q01[m].x : q01[m].y) * ih[m];  // velocity along the pencil
        }
        // (1) divergence part, central face flux on the normal momentum
        {
            const T qa = qn0, qb = qnN;
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                const T q0 = axis == 0 ? q01[0].x : q01[0].y, qN = axis == 0 ? q01[N].x : q01[N].y;
                T s = 0;
#pragma unroll
                for (int m = 0; m < NP; ++m) s += B::D(i * NP + m) * (axis == 0 ? q01[m].x : q01[m].y);
                T d = cd * s;
                if (i == 0) d += Ld * (T(0.5) * (q0 + qa) * T(-1) - q0 * T(-1));
                if (i == N) d += Ld * (T(0.5) * (qN + qb) - qN);
                if (axis == 0) sD[e0 + st * i] = d;
                else sD[e0 + st * i] += d;
            }
        }
        // (3) baroclinic pressure: -g d(H P)/dx|_sigma with the central face value, added to the
        // momentum component of this direction (the pre-pass left the sigma part there, and the
        // x pass's momentum pair adds to it)
        if (G.eos) {
            T HP[NP];  // H P along the pencil
#pragma unroll
            for (int m = 0; m < NP; ++m) HP[m] = sHb[an2(m)] * sP[e0 + st * m];
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                T dP = 0;
#pragma unroll
                for (int m = 0; m < NP; ++m) dP += B::D(i * NP + m) * HP[m];
                T fp = cd * dP;
                if (i == 0) fp -= Ld * (T(0.5) * (Pp0 - HP[0]));
                if (i == N) fp += Ld * (T(0.5) * (PpN - HP[N]));
                sR[(axis == 0 ? 0 : ncn) + e0 + st * i] -= g * fp;
            }
        }
        // normal velocities and LF speeds at both ends
        const T unm0 = -un[0], unp0 = -qn0 / Hp0;
        const T lam0 = fmax(fabs(unm0), fabs(unp0));
        const T unmN = un[N], unpN = qnN / HpN;
        const T lamN = fmax(fabs(unmN), fabs(unpN));
        // (2) right-hand side, one variable pair at a time
#pragma unroll 1
        for (int pr = 0; pr < 2; ++pr) {
            P2<T> q[NP], f[NP], vel[NP];
#pragma unroll
            for (int m = 0; m < NP; ++m) {
                q[m] = {sQ[2 * pr * ncn + e0 + st * m], sQ[(2 * pr + 1) * ncn + e0 + st * m]};
                f[m] = p2mul(q[m], bc(un[m]));
                vel[m] = p2mul(q[m], bc(ih[m]));  // (u, v) for the diffusion of (Hu, Hv)
            }
            const P2<T> qp0v = pr == 0 ? p0a : p0b;
            const P2<T> qpNv = pr == 0 ? pNa : pNb;
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                P2<T> s = bc(T(0));
#pragma unroll
                for (int m = 0; m < NP; ++m) s = p2fma_k(B::D(i * NP + m), f[m], s);
                P2<T> r = p2mul(bc(-cd), s);
                const int a2 = an2(i);
                const T Hh = sHt[a2];
                if (pr == 0) {
                    if (axis == 0) r.x -= sPx[a2];
                    else r.y -= sPy[a2];
                    if (hdiff) {
                        P2<T> dd = bc(T(0));
#pragma unroll
                        for (int m = 0; m < NP; ++m) dd = p2fma_k(B::D2(i * NP + m), vel[m], dd);
                        r = p2fma(bc(nh * Hh), p2mul(bc(cd * cd), dd), r);
                    }
                }
                if (i == 0 || i == N) {
                    const P2<T> qm = q[i], qpv = i == 0 ? qp0v : qpNv;
                    const T unm = i == 0 ? unm0 : unmN, unp = i == 0 ? unp0 : unpN;
                    const T lam = i == 0 ? lam0 : lamN;
                    const P2<T> fs = p2sub(p2mul(bc(T(0.5)), p2add(p2mul(qm, bc(unm)), p2mul(qpv, bc(unp)))),
                                           p2mul(bc(T(0.5) * lam), p2sub(qpv, qm)));
                    r = p2fma(bc(-Ld), p2sub(fs, p2mul(qm, bc(unm))), r);
                    if (pr == 0) {
                        const T nn = i == 0 ? T(-1) : T(1);
                        const T ep = i == 0 ? ep0 : epN;
                        const T pf = Ld * (g * Hh * T(0.5) * (ep - sEt[a2])) * nn;
                        if (axis == 0) r.x -= pf;
                        else r.y -= pf;
                    }
                }
                const int n = e0 + st * i, v0 = 2 * pr;
                if (axis == 0 && !(pr == 0 && G.eos)) {
                    sR[v0 * ncn + n] = r.x;
                    sR[(v0 + 1) * ncn + n] = r.y;
                } else {
                    sR[v0 * ncn + n] += r.x;
                    sR[(v0 + 1) * ncn + n] += r.y;
                }
            }
        }
    };
    // H+ P+ across side sd at the pencil end node nEnd (2D node anEnd): the neighbour's face
    // line, else the mirror value on a wall, else the exterior depth squared times this
    // column's B
    auto pplus = [&](bool has, int sd, int tt, int ez, int k, int nEnd, int anEnd, const Side &o) -> T {
        if (!G.eos) return T(0);
        if (has) return sNF[(sd * NP + tt) * STAGE_NF + 5] * sPn[((sd * NP + tt) * nz + ez) * NP + k];
        const T HPm = sHb[anEnd] * sP[nEnd];
        const int bcs = sd == 0 ? G.bc[0] : (sd == 1 ? G.bc[1] : (sd == 2 ? G.bc[2] : G.bc[3]));
        if (bcs != DRF_BC_TIDE) return HPm;
        const T r = o.H * sIHb[anEnd];
        return r * r * HPm;
    };
    // x pencils (j, k, layer); the first one's neighbour faces were prefetched
    auto xpencil = [&](int p, Side &o0, Side &oN, bool h0, bool hN) {
        const int ez = p / NP2, j = p % NP, k = (p / NP) % NP;
        const int e0 = ez * NP3 + NP * (j + NP * k);
        if (!h0) basin_side(0, 0, j, e0, o0);
        else finish_side(0, j, o0);
        if (!hN) basin_side(1, N, j, e0 + N, oN);
        else finish_side(1, j, oN);
        const T Pp0 = pplus(h0, 0, j, ez, k, e0, NP * j, o0);
        const T PpN = pplus(hN, 1, j, ez, k, e0 + N, N + NP * j, oN);
        hpass(std::integral_constant<int, 0>{}, e0, 1, j, 0, o0, oN, Pp0, PpN);
    };
    if (my_valid) xpencil(my_p, fx0, fxN, hx0, hxN);
    for (int p = SH::on ? npen : (int)threadIdx.x + (int)blockDim.x; p < npen; p += blockDim.x) {
        const int ez = p / NP2, j = p % NP, k = (p / NP) % NP;
        Side o0, oN;
        const bool h0 = fetch_side(0, ez, 0, j, k, o0), hN = fetch_side(1, ez, N, j, k, oN);
        xpencil(p, o0, oN, h0, hN);
    }
    // the first y pencil's neighbour faces are loaded across the barrier
    Side fy0, fyN;
    bool hy0 = false, hyN = false;
    if (my_valid) {
        const int p = my_p, ez = p / NP2, i = p % NP, k = (p / NP) % NP;
        hy0 = fetch_side(2, ez, i, 0, k, fy0);
        hyN = fetch_side(3, ez, i, N, k, fyN);
    }
    half_sync();
    // y pencils (i, k, layer)
    auto ypencil = [&](int p, Side &o0, Side &oN, bool h0, bool hN) {
        const int ez = p / NP2, i = p % NP, k = (p / NP) % NP;
        const int e0 = ez * NP3 + i + NP2 * k;
        if (!h0) basin_side(2, i, 0, e0, o0);
        else finish_side(2, i, o0);
        if (!hN) basin_side(3, i, N, e0 + NP * N, oN);
        else finish_side(3, i, oN);
        const T Pp0 = pplus(h0, 2, i, ez, k, e0, i, o0);
        const T PpN = pplus(hN, 3, i, ez, k, e0 + NP * N, i + NP * N, oN);
        hpass(std::integral_constant<int, 1>{}, e0, NP, 0, i, o0, oN, Pp0, PpN);
    };
    if (my_valid) ypencil(my_p, fy0, fyN, hy0, hyN);
    for (int p = SH::on ? npen : (int)threadIdx.x + (int)blockDim.x; p < npen; p += blockDim.x) {
        const int ez = p / NP2, i = p % NP, k = (p / NP) % NP;
        Side o0, oN;
        const bool h0 = fetch_side(2, ez, i, 0, k, o0), hN = fetch_side(3, ez, i, N, k, oN);
        ypencil(p, o0, oN, h0, hN);
    }
    // the late register half overwrites P, read by every layer's passes: a full barrier then
    if (late) __syncthreads();
    else half_sync();
    // the register of (HT, HS) now that P is no longer read from its shared memory
    if (late) {
        if (cv.bulk) {
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const uint32_t bytes = (uint32_t)(ncn * sizeof(T));
                mbar_expect_tx(&bars[2], 2 * bytes);
                for (int v = 2; v < 4; ++v) bulk_g2s(sRes + v * ncn, a.res[v] + base, bytes, &bars[2]);
            }
        } else {
            for (int n = threadIdx.x; n < ncn; n += blockDim.x)
                for (int v = 2; v < 4; ++v) sRes[v * ncn + n] = a.res[v][base + n];
        }
    }
    // ---- layer quadrature totals of the horizontal divergence, Q = (dsig/2) sum_k w_k delta_k
    const T hds = (T)(0.5 * G.dsig);
    for (int p = p_first; p < npen; p = p_next(p)) {
        const int ez = p / NP2, an = p % NP2;
        const int e0 = ez * NP3 + an;
        T sq = 0;
#pragma unroll
        for (int m = 0; m < NP; ++m) sq += B::w(m) * sD[e0 + NP2 * m];
        sQl[ez * NP2 + an] = hds * sq;
    }
    __syncthreads();

    // ---- z pencils: advection d/dsigma, Coriolis, vertical diffusion, sigma faces, surface
    // and bed stresses, then the LSRK update and the FP64 column increments. Each thread
    // waits for the register halves itself: (Hu, Hv) here, (HT, HS) before its first (HT, HS)
    // pair; a wait that gives up clears s_ok2, checked at the barrier after the pass.
    if (cv.bulk && need_res && !mbar_wait(&bars[1], ph)) s_ok2 = 0;
    bool w2 = !(cv.bulk && need_res);
    for (int p = p_first; p < npen; p = p_next(p)) {
        const int ez = p / NP2, an = p % NP2;
        const int e0 = ez * NP3 + an;
        const T iH = sIH[an], fa = sFc[an];
        const bool bed = ez == 0, top = ez == nz - 1;
        // the sigma velocity consistent with the discrete divergence: per layer, bottom up,
        // H omega = y solves cs D y + Ls e_0 (y_0 - M0) = I - delta (the strong-form continuity
        // with the mass flux M0 through the layer's bottom face lifted in), I the column's
        // quadrature total of delta; with the LGL weights each layer passes on M1 = M0 + dsig I
        // - Q(layer), and the flux through the surface is 0 by the choice of I
        // Iq the column total, Pq the total of the layers below this one:
        // M0 = sum over those layers of (dsig Iq - Q(layer)) = ez dsig Iq - Pq
        T Iq = 0, Pq = 0;
#pragma unroll 4
        for (int e = 0; e < nz; ++e) {
            const T v = sQl[e * NP2 + an];
            Iq += v;
            if (e < ez) Pq += v;
        }
        const T dsg = (T)G.dsig;
        T M0 = fma((T)ez * dsg, Iq, -Pq);
        const T M1 = top ? T(0) : M0 + (dsg * Iq - sQl[ez * NP2 + an]);
        if (bed) M0 = 0;
        if (a.mode == 1 && a.deta_out && bed) a.deta_out[c2 + an] = -(double)Iq;
        if (a.mode == 0 && bed) {  // the stage elevation, advanced like the 3D state
            const size_t i2 = c2 + an;
            const double re = (a.first ? 0.0 : (double)a.A * sRe[an]) - (double)dtc * (double)Iq;
            a.rese[i2] = re;
            a.etab_out[i2] = sEtb[an] + (double)a.B * re;
        }
        T om[NP];
        {
            T gq[NP];
#pragma unroll
            for (int m = 0; m < NP; ++m) gq[m] = Iq - sD[e0 + NP2 * m];
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                T sy = 0;
#pragma unroll
                for (int m = 0; m < NP; ++m) sy += B::Ai(k * NP + m) * gq[m];
                om[k] = fma(hds, sy, B::a0(k) * M0) * iH;
                if (a.mode == 1 && a.omega_out) a.omega_out[base + e0 + NP2 * k] = om[k];
            }
        }
        // bed stress (only the bottom layer's k = 0 node) and surface stress
        T fbx = 0, fby = 0;
        if (bed) {
            const T uu = sQ[e0] * iH, vv = sQ[ncn + e0] * iH;
            const T sp = sqrt(uu * uu + vv * vv);
            fbx = -Ls * (T)G.cd * sp * uu;
            fby = -Ls * (T)G.cd * sp * vv;
        }
        T fsx = 0, fsy = 0;
        if (top) {
            fsx = Ls * sTx[an];
            fsy = Ls * sTy[an];
        }
        const T w0 = om[0] * T(-1), wN = om[N];
        const int nb0 = (ez - 1) * NP3 + an + NP2 * N, nbN = (ez + 1) * NP3 + an;
        // face fluxes n M q_up / H: the mass flux carries the upwind value (from below when it
        // is upward)
        const bool up0 = !bed && M0 > T(0), dn1 = !top && M1 < T(0);
        const T f0 = -M0 * iH, f1 = M1 * iH;
        P2<T> inc = bc(T(0));
        // vertical diffusion kappa / H d2(q / H)/dsigma2 with the 1/H of q / H taken out of the sum
        const T ihc = iH * cs * cs * iH;
#pragma unroll 1
        for (int pr = 0; pr < 2; ++pr) {
            if (pr == 1 && !w2) {
                if (!mbar_wait(&bars[2], ph)) s_ok2 = 0;
                w2 = true;
            }
            const int v0 = 2 * pr, v1 = v0 + 1;
            // the pair's output arrays, selected without indexing the parameter arrays
            T *const res0 = pr == 0 ? a.res[0] : a.res[2], *const res1 = pr == 0 ? a.res[1] : a.res[3];
            T *const out0 = pr == 0 ? a.qout[0] : a.qout[2], *const out1 = pr == 0 ? a.qout[1] : a.qout[3];
            // vertical diffusivities of the pair (a zero one contributes exactly nothing)
            const T k0 = pr == 0 ? (T)G.nu_v : (T)G.kT, k1 = pr == 0 ? (T)G.nu_v : (T)G.kS;
            const P2<T> kc = {k0 > T(0) ? k0 * ihc : T(0), k1 > T(0) ? k1 * ihc : T(0)};
            P2<T> q[NP], fo[NP];
#pragma unroll
            for (int m = 0; m < NP; ++m) {
                q[m] = {sQ[v0 * ncn + e0 + NP2 * m], sQ[v1 * ncn + e0 + NP2 * m]};
                fo[m] = p2mul(q[m], bc(om[m]));
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const int n = e0 + NP2 * k;
                P2<T> s = bc(T(0)), z2 = bc(T(0));
#pragma unroll
                for (int m = 0; m < NP; ++m) {
                    s = p2fma_k(B::D(k * NP + m), fo[m], s);
                    z2 = p2fma_k(B::D2(k * NP + m), q[m], z2);
                }
                P2<T> r = p2fma(bc(-cs), s, P2<T>{sR[v0 * ncn + n], sR[v1 * ncn + n]});
                r = p2fma(kc, z2, r);
                if (pr == 0) {  // Coriolis
                    r.x += fa * q[k].y;
                    r.y += -fa * q[k].x;
                }
                if (k == 0) {
                    const P2<T> qup = up0 ? P2<T>{sQ[v0 * ncn + nb0], sQ[v1 * ncn + nb0]} : q[0];
                    r = p2fma(bc(-Ls), p2sub(p2mul(qup, bc(f0)), p2mul(q[0], bc(w0))), r);
                    if (bed && pr == 0) {
                        r.x += fbx;
                        r.y += fby;
                    }
                }
                if (k == N) {
                    const P2<T> qup = dn1 ? P2<T>{sQ[v0 * ncn + nbN], sQ[v1 * ncn + nbN]} : q[N];
                    r = p2fma(bc(-Ls), p2sub(p2mul(qup, bc(f1)), p2mul(q[N], bc(wN))), r);
                    if (top && pr == 0) {
                        r.x += fsx;
                        r.y += fsy;
                    }
                }
                const size_t gi = base + n;
                if (a.mode == 1) {
                    res0[gi] = r.x;
                    res1[gi] = r.y;
                } else {
                    const P2<T> r0 = a.first ? bc(T(0))
                                             : p2mul(bc(a.A), P2<T>{sRes[v0 * ncn + n], sRes[v1 * ncn + n]});
                    const P2<T> rn = p2fma(bc(dtc), r, r0);
                    res0[gi] = rn.x;
                    res1[gi] = rn.y;
                    const P2<T> qn = p2fma(bc(a.B), rn, q[k]);
                    out0[gi] = qn.x;
                    out1[gi] = qn.y;
                    if (pr == 0) inc = p2fma(bc(B::w(k)), p2mul(bc(a.B), rn), inc);
                }
            }
        }
        if (a.mode == 0) {
            sL1[ez * NP2 + an] = inc.x;
            sL2[ez * NP2 + an] = inc.y;
        }
    }
    if (cv.bulk && need_res) {
        __syncthreads();
        if (!s_ok2) {
            if (threadIdx.x == 0) atomicExch(a.err, DRF_E_TIMEOUT);
            return false;
        }
    }
    if (a.mode == 0) {
        if (!(cv.bulk && need_res)) __syncthreads();  // (else the barrier above)
        // one thread per (2D node, component): FP64 sum over the layers in four partial sums
        for (int t = threadIdx.x; t < 2 * NP2; t += blockDim.x) {
            const int v = t / NP2, an = t % NP2;
            const T *L = (v == 0 ? sL1 : sL2) + an;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            int ez = 0;
            for (; ez + 4 <= nz; ez += 4) {
                s0 += (double)L[ez * NP2];
                s1 += (double)L[(ez + 1) * NP2];
                s2 += (double)L[(ez + 2) * NP2];
                s3 += (double)L[(ez + 3) * NP2];
            }
            for (; ez < nz; ++ez) s0 += (double)L[ez * NP2];
            const double sum = (s0 + s1) + (s2 + s3);
            const size_t i2 = c2 + an;
            double *out = v == 0 ? a.dHU3 : a.dHV3;
            out[i2] = (a.first ? 0.0 : sOld[t]) + 0.5 * G.dsig * sum;
        }
    }
    return true;
}

// One model: one CTA per water column.
template <typename T, int NP, int NZ>
__global__ void __launch_bounds__(STAGE_MAX_THREADS, sizeof(T) == 4 ? 2 : 1) dg3d_stage_kernel(StageArgs<T> a) {
    stage_column<T, NP, NZ>(a, a.G, ColView{0, 0, 0, a.bulk, (double)a.dt}, blockIdx.x, 0u, true);
}
// Layer counts the single-model stage kernel is compiled for (others run the NZ = 0 form):
// 4 (config C1) and 16 (C2) at orders 3 and 4.
template <typename T, int NP, class F>
void dispatch_stage_nz(int nz, F &&f) {
    if constexpr (NP == 4 || NP == 5) {
        if (nz == 4) return f(dg3d_stage_kernel<T, NP, 4>);
        if (nz == 16) return f(dg3d_stage_kernel<T, NP, 16>);
    }
    f(dg3d_stage_kernel<T, NP, 0>);
}

// ------------------------------------------------------------------------- barotropic (FP64)
// One CTA per tile of BARO_CPB water columns (one thread per 2D node): the column's state is
// staged in shared memory with 1/H computed once per node; element-local derivatives read the
// tile, face fluxes read the neighbouring column's face node from global memory.
constexpr int BARO_CPB = 8;  // tile of the ensemble launches and the default of a single model
// Columns per CTA the autotuner tries for a single model's barotropic kernels.
constexpr int BARO_TILES[4] = {2, 4, 8, 16};

struct BaroArgs {
    const double *e, *hu, *hv, *h, *f, *Fx, *Fy, *tdev;
    double toff;
    Geo G;
    int64_t ncol;
};

// F*(U-, U+) - F(U-) for the Lax-Friedrichs flux (sw_flux_lf minus sw_phys_flux of U-) with
// the interior side's 1/h and sqrt(g h) supplied: one division and one square root per face
// (the exterior side's). Same formulas, reciprocals in place of divisions.
__device__ __forceinline__ void lf_minus_phys(const double UL[3], double ihL, double cL, const double UR[3],
                                              double nx, double ny, double g, double d[3]) {
    const double hLc = UL[0] < 1e-10 ? 1e-10 : UL[0], hRc = UR[0] < 1e-10 ? 1e-10 : UR[0];
    const double iL = UL[0] < 1e-10 ? 1e10 : ihL, iR = 1.0 / hRc;
    const double cLc = UL[0] < 1e-10 ? sqrt(g * hLc) : cL, cR = sqrt(g * hRc);
    const double uL = UL[1] * iL, vL = UL[2] * iL, uR = UR[1] * iR, vR = UR[2] * iR;
    const double FxL[3] = {UL[1], UL[1] * uL + 0.5 * g * hLc * hLc, UL[1] * vL};
    const double FyL[3] = {UL[2], UL[2] * uL, UL[2] * vL + 0.5 * g * hLc * hLc};
    const double FxR[3] = {UR[1], UR[1] * uR + 0.5 * g * hRc * hRc, UR[1] * vR};
    const double FyR[3] = {UR[2], UR[2] * uR, UR[2] * vR + 0.5 * g * hRc * hRc};
    const double unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
    const double lam = fmax(fabs(unL) + cLc, fabs(unR) + cR);
    const double Fm[3] = {hLc * unL, hLc * uL * unL + 0.5 * g * hLc * hLc * nx,
                          hLc * vL * unL + 0.5 * g * hLc * hLc * ny};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double FnL = FxL[q] * nx + FyL[q] * ny, FnR = FxR[q] * nx + FyR[q] * ny;
        d[q] = (0.5 * (FnL + FnR) - 0.5 * lam * (UR[q] - UL[q])) - Fm[q];
    }
}

// Register budget of the subcycle kernels: 800 resident threads per SM (80 registers) for up to
// 5 x 5 nodes per column, 576 (112 registers) for 6 x 6, whatever the tile.
constexpr int baro_min_blocks(int threads, int np) {
    return (np <= 5 ? 800 : 576) / threads < 1 ? 1 : (np <= 5 ? 800 : 576) / threads;
}
#define BARO_BOUNDS __launch_bounds__(CPB * NP * NP, baro_min_blocks(CPB * NP * NP, NP))

// One tile of CPB columns: the barotropic right-hand side Phi(U) at this thread's 2D node.
// FK is the face flux (the model's flux2d).
//  * Volume terms: each node stores its state, h, 1/H and its momentum-flux products
//    (hu u, hu v, hv v) in shared memory once; the derivative sums read them.
//  * Face terms: the 4(N+1) face nodes of an element side by side are work items spread over
//    the element's threads (one flux per thread for N >= 3), not evaluated by the face nodes
//    themselves, so no warp runs the flux twice (x then y) under divergence. Each item writes
//    F*(U-, U+) - F(U-) to shared memory; a node subtracts its x face's, then its y face's.
//  * Every global load (own state, the face items' neighbour values) is issued before the
//    first tile barrier; the tidal elevation is evaluated only by items on a tidal side.
template <int NP, int FK, int CPB>
__device__ __forceinline__ bool baro_tile_phi(const BaroArgs &a, int64_t tile, double toff, double &re, double &ru,
                                              double &rv, int64_t &t) {
    constexpr int NP2 = NP * NP, N = NP - 1, NF = 4 * NP;
    constexpr int NI = (NF + NP2 - 1) / NP2;  // face items per thread
    __shared__ double sE[CPB * NP2], sU[CPB * NP2], sV[CPB * NP2], sB[CPB * NP2], sI[CPB * NP2];
    __shared__ double sUU[CPB * NP2], sUV[CPB * NP2], sVV[CPB * NP2], sD[NP2];
    __shared__ double sF[CPB * NF * 3];  // per element and face item: d = F* - F(U-)
    const Geo &G = a.G;
    const int lc = threadIdx.x / NP2, an = threadIdx.x % NP2, i = an % NP, j = an / NP;
    const int64_t c = tile * CPB + lc;
    const bool valid = c < a.ncol;
    if (threadIdx.x < NP2) sD[threadIdx.x] = cBs[NP].D[threadIdx.x];
    t = c * NP2 + an;
    const int ex = (int)(c % G.nx), ey = (int)(c / G.nx);
    double e = 0.0, hb = 0.0, hu0 = 0.0, hv0 = 0.0, fc = 0.0, fx = 0.0, fy = 0.0;
    if (valid) {
        e = a.e[t]; hb = a.h[t]; hu0 = a.hu[t]; hv0 = a.hv[t]; fc = a.f[t];
        if (a.Fx) { fx = a.Fx[t]; fy = a.Fy[t]; }
    }
    // this thread's face items: side s = it / NP (0 -x, 1 +x, 2 -y, 3 +y), position k = it % NP;
    // the neighbour's e, h, hu, hv across the face (q < 0 on a basin side)
    int64_t qn[NI];
    double nb[NI][4];
#pragma unroll
    for (int r = 0; r < NI; ++r) {
        const int it = an + r * NP2;
        qn[r] = -1;
        nb[r][0] = nb[r][1] = nb[r][2] = nb[r][3] = 0.0;
        if (!valid || it >= NF) continue;
        const int s = it / NP, k = it % NP;
        if (s == 0 && ex > 0) qn[r] = (c - 1) * NP2 + N + NP * k;
        if (s == 1 && ex < G.nx - 1) qn[r] = (c + 1) * NP2 + NP * k;
        if (s == 2 && ey > 0) qn[r] = (c - G.nx) * NP2 + k + NP * N;
        if (s == 3 && ey < G.ny - 1) qn[r] = (c + G.nx) * NP2 + k;
        if (qn[r] >= 0) {
            nb[r][0] = a.e[qn[r]]; nb[r][1] = a.h[qn[r]]; nb[r][2] = a.hu[qn[r]]; nb[r][3] = a.hv[qn[r]];
        }
    }
    const double H = valid ? e + hb : 1.0;
    const double iH = 1.0 / H;
    if (valid) {
        const int n = threadIdx.x;
        const double u = hu0 * iH, v = hv0 * iH;
        sE[n] = e; sU[n] = hu0; sV[n] = hv0; sB[n] = hb; sI[n] = iH;
        sUU[n] = hu0 * u; sUV[n] = hv0 * u; sVV[n] = hv0 * v;
    }
    __syncthreads();
    // face items: the flux difference at face node (fi, fj) of this element
#pragma unroll
    for (int r = 0; r < NI; ++r) {
        const int it = an + r * NP2;
        if (!valid || it >= NF) continue;
        const int s = it / NP, k = it % NP;
        const int fi = s == 0 ? 0 : (s == 1 ? N : k), fj = s <= 1 ? k : (s == 2 ? 0 : N);
        const int ln = lc * NP2 + fi + NP * fj;
        const double HL = sE[ln] + sB[ln];  // the node's own H, recomputed exactly
        const double UL[3] = {HL, sU[ln], sV[ln]};
        const double nx = s == 0 ? -1.0 : (s == 1 ? 1.0 : 0.0);
        const double ny = s == 2 ? -1.0 : (s == 3 ? 1.0 : 0.0);
        double UR[3];
        if (qn[r] >= 0) {
            UR[0] = nb[r][0] + nb[r][1]; UR[1] = nb[r][2]; UR[2] = nb[r][3];
        } else if ((s == 0 ? G.bc[0] : (s == 1 ? G.bc[1] : (s == 2 ? G.bc[2] : G.bc[3]))) == DRF_BC_TIDE) {
            UR[0] = tide_at(G, a.tdev[0] + toff) + sB[ln];
            const double rr = UR[0] / HL;
            UR[1] = UL[1] * rr; UR[2] = UL[2] * rr;
        } else {
            UR[0] = HL; UR[1] = UL[1]; UR[2] = UL[2];
            if (s <= 1) UR[1] = -UL[1]; else UR[2] = -UL[2];
        }
        double d[3];
        if (FK == DRF_FLUX_LF) {
            lf_minus_phys(UL, sI[ln], sqrt(G.g * (HL < 1e-10 ? 1e-10 : HL)), UR, nx, ny, G.g, d);
        } else {
            double Fs[3], Fm[3];
            sw_flux(FK, UL, UR, nx, ny, G.g, Fs);
            sw_phys_flux(UL, nx, ny, G.g, Fm);
            d[0] = Fs[0] - Fm[0]; d[1] = Fs[1] - Fm[1]; d[2] = Fs[2] - Fm[2];
        }
        double *o = sF + (lc * NF + it) * 3;
        o[0] = d[0]; o[1] = d[1]; o[2] = d[2];
    }
    const int b0 = lc * NP2;
    double dhu = 0, dhv = 0, auu = 0, auv = 0, avu = 0, avv = 0, gex = 0, gey = 0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const int px = b0 + m + NP * j, py = b0 + i + NP * m;
        const double dxm = sD[i * NP + m], dym = sD[j * NP + m];
        dhu += dxm * sU[px];
        dhv += dym * sV[py];
        auu += dxm * sUU[px];
        avu += dxm * sUV[px];
        auv += dym * sUV[py];
        avv += dym * sVV[py];
        gex += dxm * sE[px];
        gey += dym * sE[py];
    }
    __syncthreads();  // the face items are in sF
    if (!valid) return false;
    re = -(G.cx * dhu + G.cy * dhv);
    ru = -(G.cx * auu + G.cy * auv) - G.g * H * G.cx * gex + fc * hv0 + fx;
    rv = -(G.cx * avu + G.cy * avv) - G.g * H * G.cy * gey - fc * hu0 + fy;
    // x face first, then y face (a corner node has both)
    if (i == 0 || i == N) {
        const double *d = sF + (lc * NF + (i == 0 ? 0 : NP) + j) * 3;
        re -= G.Lx * d[0]; ru -= G.Lx * d[1]; rv -= G.Lx * d[2];
    }
    if (j == 0 || j == N) {
        const double *d = sF + (lc * NF + (j == 0 ? 2 * NP : 3 * NP) + i) * 3;
        re -= G.Ly * d[0]; ru -= G.Ly * d[1]; rv -= G.Ly * d[2];
    }
    return true;
}

template <int NP, int FK, int CPB>
__global__ void baro_rhs_kernel(BaroArgs a, double *ke, double *ku, double *kv) {
    double re, ru, rv;
    int64_t t;
    if (!baro_tile_phi<NP, FK, CPB>(a, blockIdx.x, a.toff, re, ru, rv, t)) return;
    ke[t] = re; ku[t] = ru; kv[t] = rv;
}

// F = (3D-integrated increment)/dt - Phi(U^n); keeps HU^n, HV^n for the transport correction.
template <int NP, int FK, int CPB>
__device__ __forceinline__ void baro_force_body(const BaroArgs &a, int64_t tile, double toff, double dt, const double *dHU3,
                                                const double *dHV3, double *Fx, double *Fy, double *HUo,
                                                double *HVo) {
    double re, ru, rv;
    int64_t t;
    if (!baro_tile_phi<NP, FK, CPB>(a, tile, toff, re, ru, rv, t)) return;
    Fx[t] = dHU3[t] / dt - ru;
    Fy[t] = dHV3[t] / dt - rv;
    HUo[t] = a.hu[t];
    HVo[t] = a.hv[t];
}
template <int NP, int FK, int CPB>
__global__ void baro_force_kernel(BaroArgs a, double dt, const double *dHU3, const double *dHV3,
                                  double *Fx, double *Fy, double *HUo, double *HVo) {
    baro_force_body<NP, FK, CPB>(a, blockIdx.x, a.toff, dt, dHU3, dHV3, Fx, Fy, HUo, HVo);
}

// Heun predictor: k1 = Phi(U^m), U* = U^m + dtb k1
template <int NP, int FK, int CPB>
__device__ __forceinline__ void baro_pred_body(const BaroArgs &a, int64_t tile, double toff, double dtb, double *k1e,
                                               double *k1u, double *k1v, double *es, double *us, double *vs) {
    double re, ru, rv;
    int64_t t;
    if (!baro_tile_phi<NP, FK, CPB>(a, tile, toff, re, ru, rv, t)) return;
    k1e[t] = re; k1u[t] = ru; k1v[t] = rv;
    es[t] = a.e[t] + dtb * re;
    us[t] = a.hu[t] + dtb * ru;
    vs[t] = a.hv[t] + dtb * rv;
}
template <int NP, int FK, int CPB>
__global__ void BARO_BOUNDS baro_pred_kernel(BaroArgs a, double dtb, double *k1e, double *k1u, double *k1v,
                                 double *es, double *us, double *vs) {
    baro_pred_body<NP, FK, CPB>(a, blockIdx.x, a.toff, dtb, k1e, k1u, k1v, es, us, vs);
}

// Heun corrector: U^{m+1} = U^m + dtb/2 (k1 + Phi(U*)); accumulates eta for its time mean
template <int NP, int FK, int CPB>
__device__ __forceinline__ void baro_corr_body(const BaroArgs &a, int64_t tile, double toff, double dtb, const double *k1e,
                                               const double *k1u, const double *k1v, double *e, double *hu,
                                               double *hv, double *esum, int first) {
    double re, ru, rv;
    int64_t t;
    if (!baro_tile_phi<NP, FK, CPB>(a, tile, toff, re, ru, rv, t)) return;
    const double hd = 0.5 * dtb;
    const double en = e[t] + hd * (k1e[t] + re);
    e[t] = en;
    hu[t] = hu[t] + hd * (k1u[t] + ru);
    hv[t] = hv[t] + hd * (k1v[t] + rv);
    esum[t] = (first ? 0.0 : esum[t]) + en;
}
template <int NP, int FK, int CPB>
__global__ void BARO_BOUNDS baro_corr_kernel(BaroArgs a, double dtb, const double *k1e, const double *k1u,
                                 const double *k1v, double *e, double *hu, double *hv,
                                 double *esum, int first) {
    baro_corr_body<NP, FK, CPB>(a, blockIdx.x, a.toff, dtb, k1e, k1u, k1v, e, hu, hv, esum, first);
}

// the tracer volume correction: the 3D stages moved HT, HS with the column divergence of the
// 3D transport (stage elevation etbf at the step's end), the barotropic step ended at eta;
// scaling the columns' tracers by (eta + h) / (etbf + h) = 1 + corrR keeps T = HT / H
__device__ __forceinline__ double tracer_volume_correction(double eta, double etbf, double h) {
    return (eta - etbf) / (etbf + h);
}

__global__ void baro_finish_kernel(int64_t n2, int nsub, double dt, const double *esum,
                                   double *eta_avg, const double *HU, const double *HV,
                                   const double *HUo, const double *HVo, const double *dHU3,
                                   const double *dHV3, double *corrU, double *corrV, double *tdev,
                                   const double *eta, const double *etbf, const double *h,
                                   double *corrR) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t == 0) tdev[0] = tdev[0] + dt;
    if (t >= n2) return;
    eta_avg[t] = esum[t] / nsub;
    corrU[t] = HU[t] - (HUo[t] + dHU3[t]);
    corrV[t] = HV[t] - (HVo[t] + dHV3[t]);
    corrR[t] = tracer_volume_correction(eta[t], etbf[t], h[t]);
}

// Memory-only counterpart of the stage kernel: the same CTA shape and dynamic shared memory
// (so the same CTAs per SM), the column's state and LSRK register staged by the same bulk
// copies, and the 8 arrays written back in the z-pencil pattern of the LSRK update, with no
// arithmetic in between. Its bandwidth is the ceiling this access structure can reach.
template <typename T, int NP>
__global__ void __launch_bounds__(STAGE_MAX_THREADS, sizeof(T) == 4 ? 2 : 1) dg3d_copy_kernel(StageArgs<T> a) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP;
    const int nz = a.G.nz, ncn = nz * NP3, npen = nz * NP2;
    const size_t base = (size_t)blockIdx.x * ncn;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    T *sQ = reinterpret_cast<T *>(smem_raw + 16 + 2 * NP2 * sizeof(double));
    __shared__ int s_ok;
    const uint32_t bytes = (uint32_t)(ncn * sizeof(T));
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_expect_tx(&bars[0], 8 * bytes);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            bulk_g2s(sQ + v * ncn, a.qin[v] + base, bytes, &bars[0]);
            bulk_g2s(sQ + (4 + v) * ncn, a.res[v] + base, bytes, &bars[0]);
        }
        s_ok = (int)mbar_wait(&bars[0], 0);
    }
    __syncthreads();
    if (!s_ok) {
        if (threadIdx.x == 0) atomicExch(a.err, DRF_E_TIMEOUT);
        return;
    }
    for (int p = threadIdx.x; p < npen; p += blockDim.x) {
        const int e0 = (p / NP2) * NP3 + p % NP2;
#pragma unroll
        for (int v = 0; v < 4; ++v)
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const int n = e0 + NP2 * k;
                a.qout[v][base + n] = sQ[v * ncn + n];
                a.res[v][base + n] = sQ[(4 + v) * ncn + n];
            }
    }
}

// ------------------------------------------------------------------------- ensembles
// An ensemble keeps every array of its members in pools laid out array-major: member m's slice
// of a 3D array starts at element off3, of a 2D array at off2, and its model time is tdev[m].
// The launches below are built from the pool bases (member 0's pointers) and shift them per
// CTA to the member the CTA works on.
struct EnsMember {
    int64_t off3, off2;
    Geo G;
    double dt;  // baroclinic step of this member
    int ncol, bulk;
};

// Stage launch over the members of one layer count: one CTA per work item (member, column),
// the CTA size and shared memory those columns need (one such launch per layer count, tallest
// first). The member's geometry is staged in shared memory; its arrays are addressed through the
// column view (element offsets into the pools).
template <typename T, int NP>
__global__ void __launch_bounds__(STAGE_MAX_THREADS, sizeof(T) == 4 ? 2 : 1)
    dg3d_stage_ens_kernel(StageArgs<T> a, const EnsMember *mem, const int2 *items, int nitems) {
    __shared__ Geo sG;
    if ((int)blockIdx.x >= nitems) return;
    const int2 wi = items[blockIdx.x];
    const EnsMember &m = mem[wi.x];
    if (threadIdx.x == 0) sG = m.G;
    __syncthreads();
    stage_column<T, NP>(a, sG, ColView{m.off3, m.off2, wi.x, m.bulk, m.dt}, wi.y, 0u, true);
}

__device__ __forceinline__ void shift_baro(BaroArgs &a, const EnsMember &m, int idx) {
    a.e += m.off2; a.hu += m.off2; a.hv += m.off2; a.h += m.off2; a.f += m.off2;
    if (a.Fx) { a.Fx += m.off2; a.Fy += m.off2; }
    a.tdev += idx;
    a.G = m.G;
    a.ncol = m.ncol;
}

// Barotropic launches of an ensemble: block b is tile tiles[b].y of member tiles[b].x. The
// substep's time offset is sub * (dt_m / nsub) as in the single-model step.
struct BaroEns {
    const EnsMember *mem;
    const int2 *tiles;
    int nsub, sub;
};

template <int NP, int FK>
__global__ void baro_force_ens_kernel(BaroArgs a, BaroEns E, const double *dHU3, const double *dHV3,
                                      double *Fx, double *Fy, double *HUo, double *HVo) {
    const int2 w = E.tiles[blockIdx.x];
    const EnsMember &m = E.mem[w.x];
    shift_baro(a, m, w.x);
    a.toff = 0.0;
    const int64_t o = m.off2;
    baro_force_body<NP, FK, BARO_CPB>(a, w.y, a.toff, m.dt, dHU3 + o, dHV3 + o, Fx + o, Fy + o, HUo + o, HVo + o);
}
template <int NP, int FK, int CPB = BARO_CPB>
__global__ void BARO_BOUNDS baro_pred_ens_kernel(BaroArgs a, BaroEns E, double *k1e, double *k1u,
                                                 double *k1v, double *es, double *us, double *vs) {
    const int2 w = E.tiles[blockIdx.x];
    const EnsMember &m = E.mem[w.x];
    shift_baro(a, m, w.x);
    const double dtb = m.dt / E.nsub;
    a.toff = __dmul_rn((double)E.sub, dtb);
    const int64_t o = m.off2;
    baro_pred_body<NP, FK, BARO_CPB>(a, w.y, a.toff, dtb, k1e + o, k1u + o, k1v + o, es + o, us + o, vs + o);
}
template <int NP, int FK, int CPB = BARO_CPB>
__global__ void BARO_BOUNDS baro_corr_ens_kernel(BaroArgs a, BaroEns E, const double *k1e, const double *k1u,
                                                 const double *k1v, double *e, double *hu, double *hv,
                                                 double *esum) {
    const int2 w = E.tiles[blockIdx.x];
    const EnsMember &m = E.mem[w.x];
    shift_baro(a, m, w.x);
    const double dtb = m.dt / E.nsub;
    a.toff = __dadd_rn(__dmul_rn((double)E.sub, dtb), dtb);  // unfused, as the host computes it
    const int64_t o = m.off2;
    baro_corr_body<NP, FK, BARO_CPB>(a, w.y, a.toff, dtb, k1e + o, k1u + o, k1v + o, e + o, hu + o, hv + o, esum + o,
                           E.sub == 0);
}

// baro_finish_kernel over the pooled 2D arrays; each member's clock advances by its own dt.
__global__ void baro_finish_ens_kernel(int64_t n2, int nsub, const EnsMember *mem, int nmem,
                                       const double *esum, double *eta_avg, const double *HU,
                                       const double *HV, const double *HUo, const double *HVo,
                                       const double *dHU3, const double *dHV3, double *corrU,
                                       double *corrV, double *tdev, const double *eta,
                                       const double *etbf, const double *h, double *corrR) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < nmem) tdev[t] = tdev[t] + mem[t].dt;
    if (t >= n2) return;
    eta_avg[t] = esum[t] / nsub;
    corrU[t] = HU[t] - (HUo[t] + dHU3[t]);
    corrV[t] = HV[t] - (HVo[t] + dHV3[t]);
    corrR[t] = tracer_volume_correction(eta[t], etbf[t], h[t]);
}

// ------------------------------------------------------- persistent barotropic step (FP64)
// All barotropic work of one baroclinic step in ONE cooperative launch: the slow-forcing pass,
// nsub Heun subcycles (predictor and corrector passes over every tile) and the finish pass.
// Tiles go to CTAs as b, b + gridDim.x, ... in every pass, so each thread meets the same
// nodes in every pass and only the face neighbours cross CTAs; a grid barrier separates the
// passes that read neighbours written by the pass before. Every node sees the arithmetic of
// the per-pass kernels above, in the same order, so both forms give identical results.
struct SubcycleArgs {
    double dt, dtb;            // one model: baroclinic step and substep
    int nsub, ntiles;
    const EnsMember *mem;      // ensemble: member table and the (member, tile) list
    const int2 *tiles;
    int nmem;
    const double *dHU3, *dHV3;
    double *Fx, *Fy, *HUo, *HVo, *k1e, *k1u, *k1v, *es, *us, *vs;
    double *eta, *HU, *HV, *esum, *eta_avg, *corrU, *corrV;
    const double *etbf;        // stage elevation at the end of the 3D stages
    double *corrR;             // tracer volume correction
    double *tdev;              // the model's clock (an ensemble: member 0's, the others follow)
    unsigned *sync;            // [0] barrier arrivals, [1] CTAs finished, [2] abort; zero at launch
    int *err;
    // failure-detection check: the CTA of this index withholds its arrival at the first grid
    // barrier, so every CTA's bounded wait there gives up (-1: none, the normal case)
    int hold;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of a cooperative launch (all CTAs resident): the n-th barrier completes
// when n * gridDim.x arrivals are counted. The wait is bounded; a CTA that gives up, or that
// sees another CTA's abort word, sets the abort word and the status word and returns false.
// `arrive` false withholds this CTA's arrival (the failure-detection check only).
__device__ __forceinline__ bool grid_barrier(unsigned *sync, unsigned target, int *err, bool arrive = true) {
    __shared__ int s_go;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (arrive) atomicAdd(&sync[0], 1u);
        int go = 1;
        for (long it = 0; ld_acquire_gpu(&sync[0]) < target; ++it) {
            if (it > (1L << 21) || ld_acquire_gpu(&sync[2]) != 0u) {
                go = 0;
                break;
            }
            __nanosleep(32);
        }
        if (!go) {
            atomicExch(&sync[2], 1u);
            atomicExch(err, DRF_E_TIMEOUT);
        }
        __threadfence();
        s_go = go;
    }
    __syncthreads();
    return s_go != 0;
}

// Pass item w: fn(args, tile, 2D offset, step, substep) with the pass's arguments as they are
// (one model) or shifted to the item's member (an ensemble).
template <bool ENS, class F>
__device__ __forceinline__ void sub_item(const SubcycleArgs &s, const BaroArgs &base, int w, F &&fn) {
    if constexpr (ENS) {
        const int2 t = s.tiles[w];
        const EnsMember &m = s.mem[t.x];
        BaroArgs a = base;
        shift_baro(a, m, t.x);
        fn(a, (int64_t)t.y, m.off2, m.dt, m.dt / s.nsub);
    } else {
        fn(base, (int64_t)w, (int64_t)0, s.dt, s.dtb);
    }
}

// af, ap, ac: the forcing, predictor and corrector passes' arguments (state pointers).
template <int NP, int FK, int CPB, bool ENS>
__global__ void BARO_BOUNDS baro_subcycles_kernel(const __grid_constant__ BaroArgs af,
                                                  const __grid_constant__ BaroArgs ap,
                                                  const __grid_constant__ BaroArgs ac,
                                                  const __grid_constant__ SubcycleArgs s) {
    constexpr int NP2 = NP * NP;
    unsigned nbar = 0;
    // slow forcing F = dHU3/dt - Phi(U^n); the first predictor reads only this thread's F
    for (int w = blockIdx.x; w < s.ntiles; w += gridDim.x) {
        __syncthreads();  // the tile's shared memory is reused
        sub_item<ENS>(s, af, w, [&](const BaroArgs &a, int64_t tile, int64_t o, double dt, double) {
            baro_force_body<NP, FK, CPB>(a, tile, 0.0, dt, s.dHU3 + o, s.dHV3 + o, s.Fx + o, s.Fy + o, s.HUo + o,
                                         s.HVo + o);
        });
    }
    for (int m = 0; m < s.nsub; ++m) {
        for (int w = blockIdx.x; w < s.ntiles; w += gridDim.x) {
            __syncthreads();
            sub_item<ENS>(s, ap, w, [&](const BaroArgs &a, int64_t tile, int64_t o, double, double dtb) {
                baro_pred_body<NP, FK, CPB>(a, tile, __dmul_rn((double)m, dtb), dtb, s.k1e + o, s.k1u + o,
                                            s.k1v + o, s.es + o, s.us + o, s.vs + o);
            });
        }
        const bool arrive = !(nbar == 0 && (int)blockIdx.x == s.hold);
        if (!grid_barrier(s.sync, ++nbar * gridDim.x, s.err, arrive)) return;
        for (int w = blockIdx.x; w < s.ntiles; w += gridDim.x) {
            __syncthreads();
            sub_item<ENS>(s, ac, w, [&](const BaroArgs &a, int64_t tile, int64_t o, double, double dtb) {
                // the substep's end time, unfused as the host computes it
                baro_corr_body<NP, FK, CPB>(a, tile, __dadd_rn(__dmul_rn((double)m, dtb), dtb), dtb, s.k1e + o,
                                            s.k1u + o, s.k1v + o, s.eta + o, s.HU + o, s.HV + o, s.esum + o,
                                            m == 0);
            });
        }
        if (m + 1 < s.nsub && !grid_barrier(s.sync, ++nbar * gridDim.x, s.err)) return;
    }
    // finish: eta's time mean and the transport correction at this thread's own nodes
    for (int w = blockIdx.x; w < s.ntiles; w += gridDim.x) {
        sub_item<ENS>(s, af, w, [&](const BaroArgs &a, int64_t tile, int64_t o, double, double) {
            const int64_t c = tile * CPB + threadIdx.x / NP2;
            if (c >= a.ncol) return;
            const int64_t t = o + c * NP2 + threadIdx.x % NP2;
            s.eta_avg[t] = s.esum[t] / s.nsub;
            s.corrU[t] = s.HU[t] - (s.HUo[t] + s.dHU3[t]);
            s.corrV[t] = s.HV[t] - (s.HVo[t] + s.dHV3[t]);
            s.corrR[t] = tracer_volume_correction(s.eta[t], s.etbf[t], a.h[t - o]);
        });
    }
    // the clock(s) advance once every CTA is past its last read of them
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&s.sync[1], 1u) == gridDim.x - 1) {
            __threadfence();
            if constexpr (ENS) {
                for (int i = 0; i < s.nmem; ++i) s.tdev[i] = s.tdev[i] + s.mem[i].dt;
            } else {
                s.tdev[0] = s.tdev[0] + s.dt;
            }
        }
    }
}

// Launches baro_subcycles_kernel cooperatively, with as many CTAs as can be resident (at most
// one per tile), after zeroing its barrier words on the same stream.
template <int NP, int FK, int CPB, bool ENS>
void launch_subcycles(const BaroArgs &af, const BaroArgs &ap, const BaroArgs &ac, const SubcycleArgs &s,
                      cudaStream_t st) {
    auto fn = baro_subcycles_kernel<NP, FK, CPB, ENS>;
    const int threads = CPB * NP * NP;
    int dev = 0, nsm = 0, per_sm = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    DRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DRF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
    DRF_CHECK(per_sm >= 1, DRF_E_UNSUPPORTED, "the barotropic kernel cannot be resident");
    const int64_t cap = (int64_t)per_sm * nsm;
    const unsigned grid = (unsigned)(s.ntiles < cap ? s.ntiles : cap);
    DRF_CUDA(cudaMemsetAsync(s.sync, 0, 3 * sizeof(unsigned), st));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    DRF_CUDA(cudaLaunchKernelEx(&cfg, fn, af, ap, ac, s));
    DRF_LAUNCHED();
}

template <typename T, int NP>
__global__ void correct3d_kernel(int64_t n3, int nz, T *Hu, T *Hv, T *HT, T *HS, const double *cu,
                                 const double *cv, const double *cr) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const int64_t c = t / ((int64_t)nz * NP3);
    const int an = (int)((t % NP3) % NP2);
    const int64_t i2 = c * NP2 + an;
    Hu[t] = Hu[t] + (T)cu[i2];
    Hv[t] = Hv[t] + (T)cv[i2];
    const T dr = (T)cr[i2];
    HT[t] = fma(HT[t], dr, HT[t]);
    HS[t] = fma(HS[t], dr, HS[t]);
}

// FP64 copy of a 3D field (the output snapshot)
template <typename T>
__global__ void widen_kernel(int64_t n, const T *__restrict__ src, double *__restrict__ dst) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) dst[t] = (double)src[t];
}

// depth integral per 2D node of a 3D field (FP64 accumulation)
template <typename T, int NP>
__global__ void column_integral_kernel(int64_t n2, int nz, double dsig, const T *q, double *out) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n2) return;
    const int64_t c = t / NP2;
    const int an = (int)(t % NP2);
    double s = 0.0;
    for (int ez = 0; ez < nz; ++ez)
#pragma unroll
        for (int k = 0; k < NP; ++k)
            s += 0.5 * dsig * cBs[NP].w[k] * (double)q[(c * nz + ez) * NP3 + an + NP2 * k];
    out[t] = s;
}

// out = sum_i coef[i] * in[i] (up to 7 inputs), for the generic RK schemes
template <typename T>
struct Comb {
    const T *in[7];
    double coef[7];
    int nin;
    T *out;
};
template <typename T>
__global__ void combine_kernel(int64_t n, Comb<T> cb) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    double s = 0.0;
    for (int i = 0; i < cb.nin; ++i) s += cb.coef[i] * (double)cb.in[i][t];
    cb.out[t] = (T)s;
}

// diagnostics: per-block partials (fixed order -> deterministic)
// block sum / max / min of v[q] over the block, through warp shuffles (blockDim.x = 256)
template <int Q>
__device__ __forceinline__ void block_reduce(double (&v)[Q], const int (&op)[Q], double (*red)[8]) {
    const int lane = threadIdx.x % 32, w = threadIdx.x / 32;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = op[q] == 0 ? v[q] + x : (op[q] == 1 ? fmax(v[q], x) : fmin(v[q], x));
        }
        if (lane == 0) red[q][w] = v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            double a = red[q][0];
            for (int i = 1; i < 8; ++i) a = op[q] == 0 ? a + red[q][i] : (op[q] == 1 ? fmax(a, red[q][i]) : fmin(a, red[q][i]));
            v[q] = a;
        }
}

// 3D diagnostics, one block per column at a time (grid-stride over columns), 256 threads. A
// pending transport correction (corrU, corrV non-null) is added on the fly with the same
// arithmetic as folding it into the state, which is left untouched.
template <typename T, int NP>
__global__ void __launch_bounds__(256) diag3d_kernel(int ncol, int nz, const T *Hu, const T *Hv, const T *HT,
                                                     const T *HS, const double *eta, const double *h,
                                                     const double *corrU, const double *corrV,
                                                     const double *corrR, double wvol, double *part) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP;
    __shared__ double red[6][8];
    const int ncn = nz * NP3;
    double v[6] = {0.0, 0.0, 0.0, 0.0, -1e300, 1e300};  // energy, heat, salt, max speed, max T, min T
    for (int c = blockIdx.x; c < ncol; c += gridDim.x) {
        const size_t base = (size_t)c * ncn;
        for (int ln = threadIdx.x; ln < ncn; ln += blockDim.x) {
            const int an = ln % NP2, i = an % NP, j = an / NP, k = (ln % NP3) / NP2;
            const size_t i2 = (size_t)c * NP2 + an, t = base + ln;
            const double H = eta[i2] + h[i2];
            const double wv = wvol * cBs[NP].w[i] * cBs[NP].w[j] * cBs[NP].w[k];
            T huT = Hu[t], hvT = Hv[t], htT = HT[t], hsT = HS[t];
            if (corrU) {
                huT = huT + (T)corrU[i2];
                hvT = hvT + (T)corrV[i2];
                const T dr = (T)corrR[i2];
                htT = fma(htT, dr, htT);
                hsT = fma(hsT, dr, hsT);
            }
            const double hu = huT, hv = hvT, ht = htT;
            v[0] += wv * 0.5 * (hu * hu + hv * hv) / H;
            v[1] += wv * ht;
            v[2] += wv * (double)hsT;
            v[3] = fmax(v[3], sqrt(hu * hu + hv * hv) / H);
            v[4] = fmax(v[4], ht / H);
            v[5] = fmin(v[5], ht / H);
        }
    }
    const int op[6] = {0, 0, 0, 1, 1, 2};
    block_reduce<6>(v, op, red);
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) part[blockIdx.x * 6 + q] = v[q];
}

template <int NP>
__global__ void diag2d_kernel(int64_t n2, int nz, const double *eta, const double *h, double warea,
                              double g, double *part) {
    constexpr int NP2 = NP * NP;
    __shared__ double red[5][256];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double mw = 0, mu = 0, pe = 0, emax = -1e300, emin = 1e300;
    if (t < n2) {
        const int an = (int)(t % NP2), i = an % NP, j = an / NP;
        const double H = eta[t] + h[t], wa = warea * cBs[NP].w[i] * cBs[NP].w[j];
        mw = wa * H;
        mu = (double)nz * NP * H;
        pe = wa * 0.5 * g * eta[t] * eta[t];
        emax = emin = eta[t];
    }
    red[0][threadIdx.x] = mw; red[1][threadIdx.x] = mu; red[2][threadIdx.x] = pe;
    red[3][threadIdx.x] = emax; red[4][threadIdx.x] = emin;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
            red[3][threadIdx.x] = fmax(red[3][threadIdx.x], red[3][threadIdx.x + s]);
            red[4][threadIdx.x] = fmin(red[4][threadIdx.x], red[4][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 5; ++q) part[blockIdx.x * 5 + q] = red[q][0];
}

// second pass: one block folds the per-block partials (fixed order -> deterministic)
__global__ void diag_final_kernel(const double *p3, unsigned nb3, const double *p2, unsigned nb2,
                                  double *out) {
    __shared__ double red[11][256];
    double v[11] = {0, 0, 0, 0, -1e300, 1e300, 0, 0, 0, -1e300, 1e300};
    for (unsigned b = threadIdx.x; b < nb3; b += blockDim.x) {
        v[0] += p3[b * 6]; v[1] += p3[b * 6 + 1]; v[2] += p3[b * 6 + 2];
        v[3] = fmax(v[3], p3[b * 6 + 3]); v[4] = fmax(v[4], p3[b * 6 + 4]);
        v[5] = fmin(v[5], p3[b * 6 + 5]);
    }
    for (unsigned b = threadIdx.x; b < nb2; b += blockDim.x) {
        v[6] += p2[b * 5]; v[7] += p2[b * 5 + 1]; v[8] += p2[b * 5 + 2];
        v[9] = fmax(v[9], p2[b * 5 + 3]); v[10] = fmin(v[10], p2[b * 5 + 4]);
    }
    for (int q = 0; q < 11; ++q) red[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 11; ++q) {
                const double a = red[q][threadIdx.x], b = red[q][threadIdx.x + s];
                red[q][threadIdx.x] = (q == 3 || q == 4 || q == 9) ? fmax(a, b)
                                      : (q == 5 || q == 10)        ? fmin(a, b)
                                                                   : a + b;
            }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // {mass_w, mass_u, energy, heat, salt, max_speed, max_eta, min_eta, max_T, min_T}
        out[0] = red[6][0]; out[1] = red[7][0]; out[2] = red[0][0] + red[8][0];
        out[3] = red[1][0]; out[4] = red[2][0]; out[5] = red[3][0];
        out[6] = red[9][0]; out[7] = red[10][0]; out[8] = red[4][0]; out[9] = red[5][0];
    }
}

template <class F>
void dispatch_np(int np, F &&f) {
    switch (np) {
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    default: throw Error(DRF_E_UNSUPPORTED, "unsupported number of nodes per direction");
    }
}

// the 2D face flux as a compile-time constant of the barotropic kernels
template <class F>
void dispatch_flux(int kind, F &&f) {
    if (kind == DRF_FLUX_HLLC) f(std::integral_constant<int, DRF_FLUX_HLLC>{});
    else if (kind == DRF_FLUX_ROE) f(std::integral_constant<int, DRF_FLUX_ROE>{});
    else f(std::integral_constant<int, DRF_FLUX_LF>{});
}

const double LSRK_A[5] = {0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257};
const double LSRK_B[5] = {0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488,
                          0.1530572479681};
const double LSRK_C[5] = {0.0, 0.1496590219993, 0.3704009573644, 0.6222557631345, 0.9582821306748};

inline unsigned blocks_for(int64_t n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

// the barotropic tile (columns per CTA) as a compile-time constant
template <class F>
void dispatch_cpb(int cpb, F &&f) {
    switch (cpb) {
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    default: f(std::integral_constant<int, 8>{}); break;
    }
}

}  // namespace
}  // namespace drf

using namespace drf;

struct drf_dg {
    drf_mesh_desc mesh{};
    drf_dg_params prm{};
    HostBasis basis;
    Geo G{};
    int np = 0, np2 = 0, np3 = 0, ncol = 0;
    int64_t n3 = 0, n2 = 0;
    bool mixed = false;
    size_t tsz = 8;  // bytes per 3D value
    cudaStream_t stream = nullptr, own = nullptr;
    DevBuf<unsigned char> q3;  // [2 ping-pong][4 vars] + [4 res] + [4 tmp] of n3 values each
    DevBuf<double> d2;         // 2D FP64 arrays
    DevBuf<int> errbuf;        // device status word written by bounded waits
    int *err = nullptr;        // the status word in use (errbuf, or the ensemble's)
    DevBuf<unsigned> syncbuf;  // grid-barrier words of the persistent barotropic launch
    // barotropic step as one persistent launch (false: one launch per pass); fixed when the
    // step graphs are built, from DRIFTER_B200_BARO_PERSISTENT (1 selects the persistent form)
    bool baro_persist = false;
    // failure-detection check of the persistent barotropic launch: the CTA that withholds its
    // first grid-barrier arrival (-1 none); fixed when the step graphs are built, from
    // DRIFTER_B200_DEBUG_HOLD_ARRIVAL
    int debug_hold = -1;
    // 3D arrays: q3p + (array * n3s + node) * tsz; n3s = n3 for a model that owns its memory,
    // the pool length for an ensemble member (a view into the ensemble's pools)
    unsigned char *q3p = nullptr;
    int64_t n3s = 0;
    bool view = false;
    DevBuf<double> diag;       // diagnostics partials
    double *h = nullptr, *f = nullptr, *taux = nullptr, *tauy = nullptr, *eta = nullptr,
           *HU = nullptr, *HV = nullptr, *eta_avg = nullptr, *esum = nullptr, *Fx = nullptr,
           *Fy = nullptr, *HUo = nullptr, *HVo = nullptr, *k1[3] = {}, *us[3] = {}, *dHU3 = nullptr,
           *dHV3 = nullptr, *tdev = nullptr, *scratch2 = nullptr, *corrU = nullptr,
           *corrV = nullptr, *etb[2] = {}, *rese = nullptr, *corrR = nullptr;
    int cur = 0;
    bool pending = false;  // a transport correction in corrU/corrV is not yet in q(cur)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_kernels[2] = {0, 0};  // kernel nodes of each step graph
    double graph_dt = 0.0;
    // barotropic tile chosen by the autotuner (0 = not tuned yet) and the candidates' times
    int baro_cpb = 0;
    double baro_ms[4] = {0.0, 0.0, 0.0, 0.0};
    int graph_nsub = 0;
    size_t smem = 0;
    // L2 prefetch distance of the stage launch in columns, 0 for none: stage_hw half waves of
    // stage_pf_unit resident stage CTAs. Tuned at the first step (0, 1 or 2 half waves, each
    // timed: stage_ms) unless DRIFTER_B200_STAGE_PREFETCH=<half waves> fixes it
    // (DRIFTER_B200_TUNE=0: 1)
    int stage_pf = 0, stage_pf_unit = 0, stage_hw = -1;
    double stage_ms[3] = {0.0, 0.0, 0.0};
    // asynchronous output staging: FP64 snapshot buffers (4 3D fields, 4 2D fields and the
    // time), a copy stream and its events; allocated at the first drf_dg_output_stage
    DevBuf<double> out3, out2;
    cudaStream_t ostream = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_copied = nullptr;
    bool out_pending = false;

    void *q(int buf, int v) { return q3p + ((size_t)buf * 4 + v) * n3s * tsz; }
    void *res(int v) { return q3p + ((size_t)8 + v) * n3s * tsz; }
    void *tmp(int v) { return q3p + ((size_t)12 + v) * n3s * tsz; }

    // 2D arrays per model (28 named arrays, then the model time)
    static constexpr int N2ARRAYS = 29;
    // Points the model at its device memory: 16 3D arrays of stride3 values from q3base and
    // 28 2D arrays of stride2 values from d2base; tdev_ is its clock and err_ its status word.
    void bind(unsigned char *q3base, int64_t stride3, double *d2base, int64_t stride2, double *tdev_,
              int *err_) {
        q3p = q3base;
        n3s = stride3;
        double *p = d2base;
        auto take = [&]() { double *r = p; p += stride2; return r; };
        h = take(); f = take(); taux = take(); tauy = take(); eta = take();
        HU = take(); HV = take(); eta_avg = take(); esum = take(); Fx = take();
        Fy = take(); HUo = take(); HVo = take();
        for (int i = 0; i < 3; ++i) k1[i] = take();
        for (int i = 0; i < 3; ++i) us[i] = take();
        dHU3 = take(); dHV3 = take(); scratch2 = take();
        corrU = take(); corrV = take();
        etb[0] = take(); etb[1] = take(); rese = take(); corrR = take();
        tdev = tdev_;
        err = err_;
    }
    void setup(const drf_mesh_desc *mesh, const drf_dg_params *params, const double *h_,
               const double *f_, const double *taux_, const double *tauy_);
    void tune_baro();
    void tune_stage();

    void drop_graphs() {
        for (auto &g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        graph_nsub = 0;
    }
    ~drf_dg() {
        drop_graphs();
        if (ostream) {
            cudaStreamSynchronize(ostream);
            cudaStreamDestroy(ostream);
        }
        if (ev_snap) cudaEventDestroy(ev_snap);
        if (ev_copied) cudaEventDestroy(ev_copied);
        if (own) cudaStreamDestroy(own);
    }

    // threads of the single-model stage CTA: the layer-half mapping of the instances compiled
    // for a layer count (dispatch_stage_nz), else one thread per pencil up to the maximum
    int stage_threads() const {
        const int npen = G.nz * np2;
        if ((np == 4 || np == 5) && (G.nz == 4 || G.nz == 16)) return 2 * (((npen / 2) + 31) / 32) * 32;
        return stage_threads_generic();
    }
    int stage_threads_generic() const {
        const int npen = G.nz * np2;
        int bs = ((npen + 31) / 32) * 32;
        return bs < 64 ? 64 : (bs > STAGE_MAX_THREADS ? STAGE_MAX_THREADS : bs);
    }

    template <typename T, int NP>
    void launch_stage(int in, int out, int s, double dt, int mode, void *const *rout,
                      T *omega_out, double *deta_out, const double *eta_use, double toff,
                      bool with_corr = false) {
        const StageArgs<T> a = stage_args<T>(in, out, s, dt, mode, rout, omega_out, deta_out, eta_use, toff,
                                             with_corr);
        dispatch_stage_nz<T, NP>(G.nz, [&](auto kern) { kern<<<ncol, stage_threads(), smem, stream>>>(a); });
        DRF_LAUNCHED();
    }
    template <typename T>
    StageArgs<T> stage_args(int in, int out, int s, double dt, int mode, void *const *rout,
                            T *omega_out, double *deta_out, const double *eta_use, double toff,
                            bool with_corr) {
        StageArgs<T> a{};
        for (int v = 0; v < 4; ++v) {
            a.qin[v] = (const T *)q(in, v);
            a.qout[v] = (T *)q(out, v);
            a.res[v] = mode == 1 ? (T *)rout[v] : (T *)res(v);
        }
        a.eta = eta_use; a.h = h; a.f = f; a.taux = taux; a.tauy = tauy; a.tdev = tdev;
        // the baroclinic pressure's stage elevation: the step's eta at its first stage, then
        // ping-pong buffers advanced by the stages (an RHS-only launch reads eta_use)
        a.etab = (mode == 1 || s == 0) ? eta_use : etb[(s - 1) % 2];
        a.etab_out = mode == 1 ? nullptr : etb[s % 2];
        a.rese = mode == 1 ? nullptr : rese;
        a.toff = toff;
        a.dHU3 = dHU3; a.dHV3 = dHV3;
        a.omega_out = omega_out; a.deta_out = deta_out;
        a.A = (T)LSRK_A[s]; a.B = (T)LSRK_B[s]; a.dt = (T)dt;
        a.mode = mode; a.first = (s == 0);
        a.corrU = with_corr ? corrU : nullptr;
        a.corrV = with_corr ? corrV : nullptr;
        a.corrR = with_corr ? corrR : nullptr;
        a.bulk = ((size_t)G.nz * np3 * sizeof(T)) % 16 == 0;
        a.pf = stage_pf;
        a.err = err;
        a.G = G;
        return a;
    }

    // folds a pending transport correction into the current state buffer
    template <typename T, int NP>
    void materialize_t() {
        if (!pending) return;
        correct3d_kernel<T, NP><<<blocks_for(n3), 256, 0, stream>>>(
            n3, G.nz, (T *)q(cur, 0), (T *)q(cur, 1), (T *)q(cur, 2), (T *)q(cur, 3), corrU, corrV, corrR);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemsetAsync(corrU, 0, n2 * 8, stream));
        DRF_CUDA(cudaMemsetAsync(corrV, 0, n2 * 8, stream));
        DRF_CUDA(cudaMemsetAsync(corrR, 0, n2 * 8, stream));
        pending = false;
    }
    void materialize() {
        with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            this->template materialize_t<T, NP>();
        });
    }

    template <int NP>
    BaroArgs baro(const double *e, const double *u, const double *v, bool forced, double toff) {
        BaroArgs b{};
        b.e = e; b.hu = u; b.hv = v; b.h = h; b.f = f;
        b.Fx = forced ? Fx : nullptr; b.Fy = forced ? Fy : nullptr;
        b.tdev = tdev; b.toff = toff; b.G = G; b.ncol = ncol;
        return b;
    }

    // arguments of the persistent barotropic launch over this model's arrays
    SubcycleArgs subcycle_args(double dt, int nsub, int ntiles) {
        SubcycleArgs s{};
        s.dt = dt; s.dtb = dt / nsub; s.nsub = nsub; s.ntiles = ntiles;
        s.dHU3 = dHU3; s.dHV3 = dHV3;
        s.Fx = Fx; s.Fy = Fy; s.HUo = HUo; s.HVo = HVo;
        s.k1e = k1[0]; s.k1u = k1[1]; s.k1v = k1[2];
        s.es = us[0]; s.us = us[1]; s.vs = us[2];
        s.eta = eta; s.HU = HU; s.HV = HV; s.esum = esum; s.eta_avg = eta_avg;
        s.corrU = corrU; s.corrV = corrV;
        s.etbf = etb[0]; s.corrR = corrR;
        s.tdev = tdev;
        s.sync = syncbuf.p;
        s.err = err;
        s.hold = debug_hold;
        return s;
    }

    template <typename T, int NP>
    void enqueue_step(int in, double dt, int nsub) {
        const int out = 1 - in;
        int src = in;
        for (int s = 0; s < 5; ++s) {
            const int dst = (s % 2 == 0) ? out : in;
            // stage 0 folds in the transport correction left by the previous step
            launch_stage<T, NP>(src, dst, s, dt, 0, nullptr, nullptr, nullptr, eta, 0.0, s == 0);
            src = dst;
        }
        // after 5 stages the state is in `out`; the barotropic tile is the tuned one
        if (baro_persist) {
            dispatch_cpb(baro_cpb, [&](auto cpbc) {
                constexpr int CPB = decltype(cpbc)::value;
                dispatch_flux(G.flux2d, [&](auto fk) {
                    constexpr int FK = decltype(fk)::value;
                    launch_subcycles<NP, FK, CPB, false>(
                        baro<NP>(eta, HU, HV, false, 0.0), baro<NP>(eta, HU, HV, true, 0.0),
                        baro<NP>(us[0], us[1], us[2], true, 0.0),
                        subcycle_args(dt, nsub, (int)((ncol + CPB - 1) / CPB)), stream);
                });
            });
            return;
        }
        dispatch_cpb(baro_cpb, [&](auto cpbc) {
            constexpr int CPB = decltype(cpbc)::value;
            const unsigned nbt = (unsigned)((ncol + CPB - 1) / CPB);
            const int bt = CPB * NP * NP;
            dispatch_flux(G.flux2d, [&](auto fk) {
                constexpr int FK = decltype(fk)::value;
                baro_force_kernel<NP, FK, CPB><<<nbt, bt, 0, stream>>>(baro<NP>(eta, HU, HV, false, 0.0), dt,
                                                                       dHU3, dHV3, Fx, Fy, HUo, HVo);
                DRF_LAUNCHED();
                const double dtb = dt / nsub;
                for (int m = 0; m < nsub; ++m) {
                    baro_pred_kernel<NP, FK, CPB><<<nbt, bt, 0, stream>>>(
                        baro<NP>(eta, HU, HV, true, m * dtb), dtb, k1[0], k1[1], k1[2], us[0], us[1], us[2]);
                    DRF_LAUNCHED();
                    baro_corr_kernel<NP, FK, CPB><<<nbt, bt, 0, stream>>>(
                        baro<NP>(us[0], us[1], us[2], true, m * dtb + dtb), dtb, k1[0], k1[1], k1[2], eta,
                        HU, HV, esum, m == 0);
                    DRF_LAUNCHED();
                }
            });
        });
        baro_finish_kernel<<<blocks_for(n2), 256, 0, stream>>>(n2, nsub, dt, esum, eta_avg, HU, HV,
                                                               HUo, HVo, dHU3, dHV3, corrU, corrV,
                                                               tdev, eta, etb[0], h, corrR);
        DRF_LAUNCHED();
    }

    template <class F>
    void with_types(F &&fn) {
        dispatch_np(np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            if (mixed) fn(float{}, npc);
            else fn(double{}, npc);
            (void)NP;
        });
    }
};

namespace drf {
namespace {

// Raises a kernel's dynamic shared-memory limit to what the device allows next to the kernel's
// static shared memory.
void allow_max_dynamic_smem(const void *fn, int optin_max) {
    cudaFuncAttributes fa{};
    DRF_CUDA(cudaFuncGetAttributes(&fa, fn));
    DRF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin_max - (int)fa.sharedSizeBytes));
}

void upload_phys_basis(const HostBasis &b) {
    static std::mutex mu;
    static bool done[64][MAXNP + 1] = {};
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    DRF_CHECK(b.np >= 2 && b.np <= MAXNP, DRF_E_UNSUPPORTED, "polynomial order out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && done[dev][b.np]) return;
    DevBasis db;
    std::memset(&db, 0, sizeof(db));
    for (int i = 0; i < b.np * b.np; ++i) {
        db.D[i] = b.D[i]; db.D2[i] = b.D2[i]; db.S[i] = b.S[i];
        db.Df[i] = (float)b.D[i]; db.D2f[i] = (float)b.D2[i]; db.Sf[i] = (float)b.S[i];
    }
    for (int i = 0; i < b.np; ++i) {
        db.w[i] = b.w[i]; db.x[i] = b.x[i];
        db.wf[i] = (float)b.w[i]; db.xf[i] = (float)b.x[i];
    }
    // (D + e_0 e_0^T / w_0)^-1 by Gauss-Jordan elimination with partial pivoting
    {
        const int n = b.np;
        std::vector<double> A(b.D), I((size_t)n * n, 0.0);
        A[0] += 1.0 / b.w[0];
        for (int i = 0; i < n; ++i) I[(size_t)i * n + i] = 1.0;
        for (int c = 0; c < n; ++c) {
            int pr = c;
            for (int r = c + 1; r < n; ++r)
                if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)pr * n + c])) pr = r;
            for (int k = 0; k < n; ++k) {
                std::swap(A[(size_t)c * n + k], A[(size_t)pr * n + k]);
                std::swap(I[(size_t)c * n + k], I[(size_t)pr * n + k]);
            }
            const double d = A[(size_t)c * n + c];
            for (int k = 0; k < n; ++k) {
                A[(size_t)c * n + k] /= d;
                I[(size_t)c * n + k] /= d;
            }
            for (int r = 0; r < n; ++r) {
                if (r == c) continue;
                const double f = A[(size_t)r * n + c];
                for (int k = 0; k < n; ++k) {
                    A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
                    I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
                }
            }
        }
        for (int i = 0; i < n * n; ++i) {
            db.Ai[i] = I[i];
            db.Aif[i] = (float)I[i];
        }
        for (int k = 0; k < n; ++k) {
            db.a0[k] = I[(size_t)k * n] / b.w[0];
            db.a0f[k] = (float)db.a0[k];
        }
    }
    DRF_CUDA(cudaMemcpyToSymbol(cBs, &db, sizeof(db), (size_t)b.np * sizeof(DevBasis)));
    if (dev < 64) done[dev][b.np] = true;
}

template <typename T>
void to_device(drf_dg *m, void *dst, const double *src) {
    if constexpr (std::is_same_v<T, double>) {
        DRF_CUDA(cudaMemcpyAsync(dst, src, m->n3 * 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
    } else {
        std::vector<float> tmp(m->n3);
        for (int64_t i = 0; i < m->n3; ++i) tmp[i] = (float)src[i];
        DRF_CUDA(cudaMemcpyAsync(dst, tmp.data(), m->n3 * 4, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
    }
}

void from_device(drf_dg *m, double *dst, const void *src) {
    if (!m->mixed) {
        DRF_CUDA(cudaMemcpyAsync(dst, src, m->n3 * 8, cudaMemcpyDeviceToHost, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
    } else {
        std::vector<float> tmp(m->n3);
        DRF_CUDA(cudaMemcpyAsync(tmp.data(), src, m->n3 * 4, cudaMemcpyDeviceToHost, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        for (int64_t i = 0; i < m->n3; ++i) dst[i] = (double)tmp[i];
    }
}

void check_model(drf_dg *m) { DRF_CHECK(m != nullptr, DRF_E_INVALID, "null model handle"); }

// surfaces a status word set on the device (a bounded wait that gave up)
void check_device_status(drf_dg *m) {
    int st = 0;
    DRF_CUDA(cudaMemcpyAsync(&st, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    DRF_CUDA(cudaStreamSynchronize(m->stream));
    if (st != 0) {
        DRF_CUDA(cudaMemsetAsync(m->err, 0, sizeof(int), m->stream));
        throw Error(st, "a device-side wait gave up (status " + std::to_string(st) + ")");
    }
}

}  // namespace
}  // namespace drf

// Host-side set-up shared by a model and an ensemble member: argument checks, basis tables,
// geometry constants and the stage kernel's shared-memory size. No device memory is touched.
void drf_dg::setup(const drf_mesh_desc *mesh, const drf_dg_params *params, const double *h_,
                   const double *f_, const double *taux_, const double *tauy_) {
    DRF_CHECK(mesh->nx >= 1 && mesh->ny >= 1 && mesh->nz >= 1, DRF_E_INVALID,
              "mesh must have at least one element per direction");
    DRF_CHECK(mesh->Lx > 0 && mesh->Ly > 0, DRF_E_INVALID, "basin extent must be positive");
    DRF_CHECK(params->flux2d >= 0 && params->flux2d <= 2, DRF_E_INVALID, "unknown flux kind");
    DRF_CHECK(params->precision == DRF_PREC_FP64 || params->precision == DRF_PREC_MIXED,
              DRF_E_INVALID, "unknown precision");
    for (int s = 0; s < 4; ++s)
        DRF_CHECK(params->bc[s] == DRF_BC_WALL || params->bc[s] == DRF_BC_TIDE, DRF_E_INVALID,
                  "unknown boundary type");
    this->mesh = *mesh;  // (the parameters shadow the members of the same name)
    this->prm = *params;
    basis = make_lgl_basis(mesh->order);
    np = basis.np; np2 = np * np; np3 = np2 * np;
    ncol = mesh->nx * mesh->ny;
    n2 = (int64_t)ncol * np2;
    n3 = n2 * mesh->nz * np;
    mixed = params->precision == DRF_PREC_MIXED;
    tsz = mixed ? 4 : 8;
    for (const double *a : {h_, f_, taux_, tauy_})
        DRF_CHECK(all_finite(a, n2), DRF_E_NONFINITE, "non-finite value in a 2D field");
    for (int64_t i = 0; i < n2; ++i)
        DRF_CHECK(h_[i] > 0.0, DRF_E_INVALID, "bathymetry must be positive (no dry nodes)");
    const double dx = mesh->Lx / mesh->nx, dy = mesh->Ly / mesh->ny, ds = 1.0 / mesh->nz;
    const double wend = basis.w[0];
    G.nx = mesh->nx; G.ny = mesh->ny; G.nz = mesh->nz; G.flux2d = params->flux2d;
    for (int s = 0; s < 4; ++s) G.bc[s] = params->bc[s];
    G.cx = 2.0 / dx; G.cy = 2.0 / dy; G.cs = 2.0 / ds;
    G.Lx = G.cx / wend; G.Ly = G.cy / wend; G.Ls = G.cs / wend; G.dsig = ds;
    G.g = params->g; G.rho0 = params->rho0; G.nu_h = params->nu_h; G.nu_v = params->nu_v;
    G.kT = params->kappa_v_T; G.kS = params->kappa_v_S; G.cd = params->cd;
    G.tide_amp = params->tide_amp;
    G.tide_w = params->tide_period != 0.0 ? 2.0 * M_PI / params->tide_period : 0.0;
    G.alpha = params->alpha; G.beta = params->beta; G.T0 = params->T0; G.S0 = params->S0;
    G.Tref_s = params->Tref_s; G.Tref_dz = params->Tref_dz;
    G.eos = (params->alpha != 0.0 || params->beta != 0.0) ? 1 : 0;
    upload_phys_basis(basis);
    // shared memory of the stage kernel: 9 column arrays + per-layer bases + 2D scalars
    smem = stage_smem_bytes(mesh->nz, np, tsz);
    int dev = 0, maxsm = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    DRF_CUDA(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    DRF_CHECK(smem + 512 <= (size_t)maxsm, DRF_E_UNSUPPORTED,
              "water column too tall for one CTA: nz*(N+1)^3 too large");
    // the limit is a property of the kernel, shared by every model in the process: allow the
    // device maximum (the shared memory a launch actually asks for sets its occupancy)
    with_types([&](auto tv, auto npc) {
        using T = decltype(tv);
        constexpr int NP = decltype(npc)::value;
        dispatch_stage_nz<T, NP>(mesh->nz, [&](auto kern) {
            allow_max_dynamic_smem(reinterpret_cast<const void *>(kern), maxsm);
            int per_sm = 0, nsm = 0;
            DRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            DRF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, stage_threads(), smem));
            stage_pf_unit = per_sm * nsm;
            const char *pe = std::getenv("DRIFTER_B200_STAGE_PREFETCH");
            const char *tn = std::getenv("DRIFTER_B200_TUNE");
            stage_hw = pe ? std::max(std::atoi(pe), 0) : ((tn && tn[0] == '0') ? 1 : -1);
            stage_pf = (stage_hw < 0 ? 1 : stage_hw) * stage_pf_unit / 2;
        });
    });
}

// Autotuner of the barotropic tile (water columns per CTA of the subcycle kernels): times the
// predictor kernel, which writes only scratch arrays, at every candidate tile on the model's
// stream (two warm-up launches, then ten between CUDA events) and keeps the fastest. Choices
// are cached per (device, order, flux, number of columns) for the life of the process.
// DRIFTER_B200_TUNE=0 in the environment keeps the default tile.
void drf_dg::tune_baro() {
    if (baro_cpb) return;
    const char *env = std::getenv("DRIFTER_B200_TUNE");
    if (env && env[0] == '0') {
        baro_cpb = BARO_CPB;
        return;
    }
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, std::pair<int, std::array<double, 4>>> cache;
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, np, G.flux2d, ncol);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            baro_cpb = it->second.first;
            for (int i = 0; i < 4; ++i) baro_ms[i] = it->second.second[i];
            return;
        }
    }
    cudaEvent_t e0, e1;
    DRF_CUDA(cudaEventCreate(&e0));
    DRF_CUDA(cudaEventCreate(&e1));
    int best = BARO_CPB;
    double best_ms = 1e300;
    dispatch_np(np, [&](auto npc) {
        constexpr int NP = decltype(npc)::value;
        dispatch_flux(G.flux2d, [&](auto fk) {
            constexpr int FK = decltype(fk)::value;
            for (int i = 0; i < 4; ++i)
                dispatch_cpb(BARO_TILES[i], [&](auto cpbc) {
                    constexpr int CPB = decltype(cpbc)::value;
                    const unsigned nbt = (unsigned)((ncol + CPB - 1) / CPB);
                    auto launch = [&]() {
                        baro_pred_kernel<NP, FK, CPB><<<nbt, CPB * NP * NP, 0, stream>>>(
                            baro<NP>(eta, HU, HV, true, 0.0), 1.0, k1[0], k1[1], k1[2], us[0], us[1], us[2]);
                        DRF_LAUNCHED();
                    };
                    launch();
                    launch();
                    DRF_CUDA(cudaEventRecord(e0, stream));
                    for (int r = 0; r < 10; ++r) launch();
                    DRF_CUDA(cudaEventRecord(e1, stream));
                    DRF_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    DRF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    baro_ms[i] = ms / 10.0;
                    if (baro_ms[i] < best_ms) {
                        best_ms = baro_ms[i];
                        best = CPB;
                    }
                });
        });
    });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    baro_cpb = best;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = {best, {baro_ms[0], baro_ms[1], baro_ms[2], baro_ms[3]}};
}

// Stage-launch tuner: the L2 prefetch distance (0, 1/2 or 1 wave of resident CTAs), each timed
// on a non-first LSRK stage written into the spare buffers (two warm-up launches, then five
// between CUDA events; the model state is not modified), the fastest kept. Cached per
// (device, order, layers, columns, precision, equation of state).
void drf_dg::tune_stage() {
    if (stage_hw >= 0) return;
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int, int>, std::pair<int, std::array<double, 3>>> cache;
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, np, G.nz, ncol, (int)tsz, G.eos);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            stage_hw = it->second.first;
            for (int i = 0; i < 3; ++i) stage_ms[i] = it->second.second[i];
            stage_pf = stage_hw * stage_pf_unit / 2;
            return;
        }
    }
    cudaEvent_t e0, e1;
    DRF_CUDA(cudaEventCreate(&e0));
    DRF_CUDA(cudaEventCreate(&e1));
    int best = 1;
    double best_ms = 1e300;
    with_types([&](auto tv, auto npc) {
        using T = decltype(tv);
        constexpr int NP = decltype(npc)::value;
        for (int w = 0; w < 3; ++w) {
            stage_pf = w * stage_pf_unit / 2;
            auto launch = [&] {
                launch_stage<T, NP>(cur, 1 - cur, 1, 1e-6, 0, nullptr, nullptr, nullptr, eta, 0.0);
            };
            launch();
            launch();
            DRF_CUDA(cudaEventRecord(e0, stream));
            for (int r = 0; r < 5; ++r) launch();
            DRF_CUDA(cudaEventRecord(e1, stream));
            DRF_CUDA(cudaEventSynchronize(e1));
            float t = 0.f;
            DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
            stage_ms[w] = t / 5.0;
            if (stage_ms[w] < best_ms) {
                best_ms = stage_ms[w];
                best = w;
            }
        }
    });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    stage_hw = best;
    stage_pf = best * stage_pf_unit / 2;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = {best, {stage_ms[0], stage_ms[1], stage_ms[2]}};
}

extern "C" {

int drf_dg_create(const drf_mesh_desc *mesh, const drf_dg_params *params, const double *h,
                  const double *f, const double *taux, const double *tauy, drf_dg **out) {
    return guard([&] {
        DRF_CHECK(mesh && params && h && f && taux && tauy && out, DRF_E_INVALID, "null argument");
        *out = nullptr;
        auto m = std::make_unique<drf_dg>();
        m->setup(mesh, params, h, f, taux, tauy);
        DRF_CUDA(cudaStreamCreateWithFlags(&m->own, cudaStreamNonBlocking));
        m->stream = m->own;
        m->errbuf.alloc(1);
        DRF_CUDA(cudaMemset(m->errbuf.p, 0, sizeof(int)));
        m->syncbuf.alloc(4);
        DRF_CUDA(cudaMemset(m->syncbuf.p, 0, 4 * sizeof(unsigned)));
        m->q3.alloc((size_t)16 * m->n3 * m->tsz);
        DRF_CUDA(cudaMemset(m->q3.p, 0, m->q3.n));
        m->d2.alloc((size_t)drf_dg::N2ARRAYS * m->n2 + 8);
        DRF_CUDA(cudaMemset(m->d2.p, 0, m->d2.n * 8));
        m->bind(m->q3.p, m->n3, m->d2.p, m->n2, m->d2.p + (size_t)(drf_dg::N2ARRAYS - 1) * m->n2,
                m->errbuf.p);
        DRF_CUDA(cudaMemcpy(m->h, h, m->n2 * 8, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(m->f, f, m->n2 * 8, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(m->taux, taux, m->n2 * 8, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(m->tauy, tauy, m->n2 * 8, cudaMemcpyHostToDevice));
        *out = m.release();
    });
}

int drf_dg_destroy(drf_dg *m) {
    return guard([&] {
        if (!m) return;
        DRF_CHECK(!m->view, DRF_E_INVALID, "an ensemble member is destroyed with its ensemble");
        if (m->stream) cudaStreamSynchronize(m->stream);
        delete m;
    });
}

int drf_dg_set_stream(drf_dg *m, void *s) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(!m->view, DRF_E_INVALID, "set the stream of the ensemble, not of a member");
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        m->drop_graphs();
        m->stream = s ? (cudaStream_t)s : m->own;
    });
}

int drf_dg_sync(drf_dg *m) {
    return guard([&] {
        check_model(m);
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        check_device_status(m);
    });
}

int drf_dg_upload_state(drf_dg *m, const double *const *q4, const double *eta, double t) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(q4 && eta, DRF_E_INVALID, "null argument");
        for (int v = 0; v < 4; ++v)
            DRF_CHECK(q4[v] && all_finite(q4[v], m->n3), DRF_E_NONFINITE, "non-finite state value");
        DRF_CHECK(all_finite(eta, m->n2), DRF_E_NONFINITE, "non-finite eta");
        if (!m->view) m->cur = 0;  // an ensemble member keeps the ensemble's buffer parity
        for (int v = 0; v < 4; ++v) {
            if (m->mixed) to_device<float>(m, m->q(m->cur, v), q4[v]);
            else to_device<double>(m, m->q(m->cur, v), q4[v]);
        }
        DRF_CUDA(cudaMemcpyAsync(m->eta, eta, m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaMemcpyAsync(m->eta_avg, eta, m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        // barotropic transports = depth integrals of the FP64 input (exact, on the host)
        const int np = m->np, np2 = m->np2, np3 = m->np3, nz = m->mesh.nz;
        std::vector<double> hu(m->n2, 0.0), hv(m->n2, 0.0);
        for (int c = 0; c < m->ncol; ++c)
            for (int a = 0; a < np2; ++a) {
                double su = 0.0, sv = 0.0;
                for (int ez = 0; ez < nz; ++ez)
                    for (int k = 0; k < np; ++k) {
                        const size_t n = ((size_t)c * nz + ez) * np3 + a + np2 * k;
                        const double w = 0.5 * m->G.dsig * m->basis.w[k];
                        su += w * q4[0][n];
                        sv += w * q4[1][n];
                    }
                hu[(size_t)c * np2 + a] = su;
                hv[(size_t)c * np2 + a] = sv;
            }
        DRF_CUDA(cudaMemcpyAsync(m->HU, hu.data(), m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaMemcpyAsync(m->HV, hv.data(), m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaMemcpyAsync(m->tdev, &t, 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaMemsetAsync(m->corrU, 0, m->n2 * 8, m->stream));
        DRF_CUDA(cudaMemsetAsync(m->corrV, 0, m->n2 * 8, m->stream));
        DRF_CUDA(cudaMemsetAsync(m->corrR, 0, m->n2 * 8, m->stream));
        m->pending = false;
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        m->drop_graphs();
    });
}

int drf_dg_download_state(drf_dg *m, double *const *q4, double *eta, double *HU, double *HV,
                          double *eta_avg, double *t) {
    return guard([&] {
        check_model(m);
        m->materialize();
        check_device_status(m);
        if (q4)
            for (int v = 0; v < 4; ++v)
                if (q4[v]) from_device(m, q4[v], m->q(m->cur, v));
        if (eta) DRF_CUDA(cudaMemcpy(eta, m->eta, m->n2 * 8, cudaMemcpyDeviceToHost));
        if (HU) DRF_CUDA(cudaMemcpy(HU, m->HU, m->n2 * 8, cudaMemcpyDeviceToHost));
        if (HV) DRF_CUDA(cudaMemcpy(HV, m->HV, m->n2 * 8, cudaMemcpyDeviceToHost));
        if (eta_avg) DRF_CUDA(cudaMemcpy(eta_avg, m->eta_avg, m->n2 * 8, cudaMemcpyDeviceToHost));
        if (t) DRF_CUDA(cudaMemcpy(t, m->tdev, 8, cudaMemcpyDeviceToHost));
    });
}

// Asynchronous output staging (the step either side of the output calls around
// SimulationDriver's loop, src/io/vtk_writer.cpp): the state is folded (pending transport
// correction) and snapshot in FP64 on the model's stream, then copied to the caller's host
// buffers on a copy stream of the model; the model keeps stepping while the copy runs. A new
// snapshot waits for the previous copy.
int drf_dg_output_stage(drf_dg *m, double *const *q4, double *eta, double *HU, double *HV) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(!m->view, DRF_E_INVALID, "stage ensemble members' output through their ensemble's stream");
        if (!m->ostream) {
            DRF_CUDA(cudaStreamCreateWithFlags(&m->ostream, cudaStreamNonBlocking));
            DRF_CUDA(cudaEventCreateWithFlags(&m->ev_snap, cudaEventDisableTiming));
            DRF_CUDA(cudaEventCreateWithFlags(&m->ev_copied, cudaEventDisableTiming));
        }
        if (q4 && m->out3.n < (size_t)4 * m->n3) m->out3.alloc((size_t)4 * m->n3);
        if (m->out2.n < (size_t)3 * m->n2 + 1) m->out2.alloc((size_t)3 * m->n2 + 1);
        if (m->out_pending) DRF_CUDA(cudaStreamWaitEvent(m->stream, m->ev_copied, 0));
        m->materialize();
        if (q4)
            m->with_types([&](auto tv, auto) {
                using T = decltype(tv);
                for (int v = 0; v < 4; ++v)
                    if (q4[v]) {
                        widen_kernel<T><<<blocks_for(m->n3), 256, 0, m->stream>>>(
                            m->n3, (const T *)m->q(m->cur, v), m->out3.p + (size_t)v * m->n3);
                        DRF_LAUNCHED();
                    }
            });
        const double *src2[3] = {m->eta, m->HU, m->HV};
        for (int k = 0; k < 3; ++k)
            DRF_CUDA(cudaMemcpyAsync(m->out2.p + (size_t)k * m->n2, src2[k], m->n2 * 8, cudaMemcpyDeviceToDevice,
                                     m->stream));
        DRF_CUDA(cudaMemcpyAsync(m->out2.p + (size_t)3 * m->n2, m->tdev, 8, cudaMemcpyDeviceToDevice, m->stream));
        DRF_CUDA(cudaEventRecord(m->ev_snap, m->stream));
        DRF_CUDA(cudaStreamWaitEvent(m->ostream, m->ev_snap, 0));
        if (q4)
            for (int v = 0; v < 4; ++v)
                if (q4[v])
                    DRF_CUDA(cudaMemcpyAsync(q4[v], m->out3.p + (size_t)v * m->n3, m->n3 * 8,
                                             cudaMemcpyDeviceToHost, m->ostream));
        double *dst2[3] = {eta, HU, HV};
        for (int k = 0; k < 3; ++k)
            if (dst2[k])
                DRF_CUDA(cudaMemcpyAsync(dst2[k], m->out2.p + (size_t)k * m->n2, m->n2 * 8, cudaMemcpyDeviceToHost,
                                         m->ostream));
        DRF_CUDA(cudaEventRecord(m->ev_copied, m->ostream));
        m->out_pending = true;
    });
}

int drf_dg_output_wait(drf_dg *m, double *t) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(m->out_pending, DRF_E_INVALID, "no output staged (drf_dg_output_stage)");
        DRF_CUDA(cudaEventSynchronize(m->ev_copied));
        if (t) DRF_CUDA(cudaMemcpy(t, m->out2.p + (size_t)3 * m->n2, 8, cudaMemcpyDeviceToHost));
        m->out_pending = false;
        check_device_status(m);
    });
}

int drf_dg_compute_rhs(drf_dg *m, double *const *r4, double *omega, double *deta) {
    return guard([&] {
        check_model(m);
        m->materialize();
        void *rout[4] = {m->tmp(0), m->tmp(1), m->tmp(2), m->tmp(3)};
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            m->template launch_stage<T, NP>(m->cur, 1 - m->cur, 1, 0.0, 1, rout, (T *)m->res(0),
                                            m->scratch2, m->eta, 0.0);
        });
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        if (r4)
            for (int v = 0; v < 4; ++v)
                if (r4[v]) from_device(m, r4[v], rout[v]);
        if (omega) from_device(m, omega, m->res(0));
        if (deta) DRF_CUDA(cudaMemcpy(deta, m->scratch2, m->n2 * 8, cudaMemcpyDeviceToHost));
    });
}

int drf_dg_compute_rhs2d(drf_dg *m, const double *Fx, const double *Fy, double time, double *ke,
                         double *khu, double *khv) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(Fx && Fy && ke && khu && khv, DRF_E_INVALID, "null argument");
        DRF_CUDA(cudaMemcpyAsync(m->Fx, Fx, m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaMemcpyAsync(m->Fy, Fy, m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        double tcur = 0.0;
        DRF_CUDA(cudaMemcpyAsync(&tcur, m->tdev, 8, cudaMemcpyDeviceToHost, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        dispatch_np(m->np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            dispatch_flux(m->G.flux2d, [&](auto fk) {
                constexpr int FK = decltype(fk)::value;
                baro_rhs_kernel<NP, FK, BARO_CPB><<<(unsigned)((m->ncol + BARO_CPB - 1) / BARO_CPB), BARO_CPB * NP * NP,
                                          0, m->stream>>>(m->baro<NP>(m->eta, m->HU, m->HV, true, time - tcur),
                                                          m->k1[0], m->k1[1], m->k1[2]);
            });
        });
        DRF_LAUNCHED();
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        DRF_CUDA(cudaMemcpy(ke, m->k1[0], m->n2 * 8, cudaMemcpyDeviceToHost));
        DRF_CUDA(cudaMemcpy(khu, m->k1[1], m->n2 * 8, cudaMemcpyDeviceToHost));
        DRF_CUDA(cudaMemcpy(khv, m->k1[2], m->n2 * 8, cudaMemcpyDeviceToHost));
    });
}

int drf_dg_step_modesplit(drf_dg *m, double dt, int nsub, int nsteps) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(!m->view, DRF_E_INVALID, "ensemble members are stepped together (drf_ens_step)");
        DRF_CHECK(nsub >= 1, DRF_E_INVALID, "nsub must be >= 1");
        DRF_CHECK(dt > 0.0 && std::isfinite(dt), DRF_E_INVALID, "dt must be positive");
        DRF_CHECK(nsteps >= 0, DRF_E_INVALID, "nsteps must be >= 0");
        m->tune_baro();  // first step only: outside any capture
        m->tune_stage();
        if (m->graph_nsub != nsub || m->graph_dt != dt) {
            m->drop_graphs();
            const char *pe = std::getenv("DRIFTER_B200_BARO_PERSISTENT");
            m->baro_persist = pe && pe[0] == '1';
            const char *ph = std::getenv("DRIFTER_B200_DEBUG_HOLD_ARRIVAL");
            m->debug_hold = ph && ph[0] ? std::atoi(ph) : -1;
            for (int in = 0; in < 2; ++in)
                m->graph[in] = capture_graph(m->stream, [&] {
                    m->with_types([&](auto tv, auto npc) {
                        using T = decltype(tv);
                        constexpr int NP = decltype(npc)::value;
                        m->template enqueue_step<T, NP>(in, dt, nsub);
                    });
                }, &m->graph_kernels[in]);
            m->graph_nsub = nsub;
            m->graph_dt = dt;
        }
        for (int s = 0; s < nsteps; ++s) {
            DRF_CUDA(cudaGraphLaunch(m->graph[m->cur], m->stream));
            launch_counter().fetch_add(m->graph_kernels[m->cur]);
            m->cur = 1 - m->cur;
            m->pending = true;
        }
    });
}

int drf_dg_rk_step(drf_dg *m, int scheme, double dt, int nsteps) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(scheme >= 0 && scheme <= 5, DRF_E_INVALID, "unknown RK scheme");
        DRF_CHECK(dt > 0.0 && std::isfinite(dt), DRF_E_INVALID, "dt must be positive");
        m->materialize();
        // Stage storage: up to 6 RHS evaluations of (q[4], eta). The 3D parts live in a
        // separately allocated buffer; this path is the generic (non-split) reference driver.
        const int nk = scheme == DRF_RK_DOPRI ? 6 : (scheme == DRF_RK_RK4 ? 4 : 2);
        DevBuf<unsigned char> k3((size_t)(nk + 2) * 4 * m->n3 * m->tsz);
        DevBuf<double> k2d((size_t)(nk + 2) * m->n2);
        auto K3 = [&](int s, int v) { return (void *)(k3.p + ((size_t)s * 4 + v) * m->n3 * m->tsz); };
        auto K2 = [&](int s) { return k2d.p + (size_t)s * m->n2; };
        const int U0 = nk, UT = nk + 1;  // slots: U^n copy, stage input
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            auto rhs = [&](int in_slot, int kslot, double toff) {
                // copy stage input into ping buffer 1-cur so the stage kernel can read it
                void *rout[4] = {K3(kslot, 0), K3(kslot, 1), K3(kslot, 2), K3(kslot, 3)};
                for (int v = 0; v < 4; ++v)
                    DRF_CUDA(cudaMemcpyAsync(m->q(1 - m->cur, v), K3(in_slot, v), m->n3 * m->tsz,
                                             cudaMemcpyDeviceToDevice, m->stream));
                m->template launch_stage<T, NP>(1 - m->cur, m->cur, 1, 0.0, 1, rout, (T *)m->res(0),
                                                K2(kslot), K2(in_slot), toff);
            };
            auto comb = [&](int out_slot, std::initializer_list<std::pair<int, double>> terms) {
                Comb<T> c3{};
                Comb<double> c2{};
                for (int v = 0; v < 4; ++v) {
                    int i = 0;
                    for (auto &tm : terms) {
                        c3.in[i] = (const T *)K3(tm.first, v);
                        c3.coef[i] = tm.second;
                        ++i;
                    }
                    c3.nin = i;
                    c3.out = (T *)K3(out_slot, v);
                    combine_kernel<T><<<blocks_for(m->n3), 256, 0, m->stream>>>(m->n3, c3);
                    DRF_LAUNCHED();
                }
                int i = 0;
                for (auto &tm : terms) {
                    c2.in[i] = K2(tm.first);
                    c2.coef[i] = tm.second;
                    ++i;
                }
                c2.nin = i;
                c2.out = K2(out_slot);
                combine_kernel<double><<<blocks_for(m->n2), 256, 0, m->stream>>>(m->n2, c2);
                DRF_LAUNCHED();
            };
            for (int step = 0; step < nsteps; ++step) {
                for (int v = 0; v < 4; ++v)
                    DRF_CUDA(cudaMemcpyAsync(K3(U0, v), m->q(m->cur, v), m->n3 * m->tsz,
                                             cudaMemcpyDeviceToDevice, m->stream));
                DRF_CUDA(cudaMemcpyAsync(K2(U0), m->eta, m->n2 * 8, cudaMemcpyDeviceToDevice, m->stream));
                const double h1 = dt;
                switch (scheme) {
                case DRF_RK_EULER:
                    rhs(U0, 0, 0.0);
                    comb(U0, {{U0, 1.0}, {0, h1}});
                    break;
                case DRF_RK_MIDPOINT:
                    rhs(U0, 0, 0.0);
                    comb(UT, {{U0, 1.0}, {0, 0.5 * h1}});
                    rhs(UT, 1, 0.5 * h1);
                    comb(U0, {{U0, 1.0}, {1, h1}});
                    break;
                case DRF_RK_SSP3:
                    rhs(U0, 0, 0.0);
                    comb(UT, {{U0, 1.0}, {0, h1}});            // U1
                    rhs(UT, 1, h1);
                    comb(UT, {{U0, 0.75}, {UT, 0.25}, {1, 0.25 * h1}});  // U2
                    rhs(UT, 0, 0.5 * h1);
                    comb(U0, {{U0, 1.0 / 3.0}, {UT, 2.0 / 3.0}, {0, 2.0 / 3.0 * h1}});
                    break;
                case DRF_RK_RK4:
                    rhs(U0, 0, 0.0);
                    comb(UT, {{U0, 1.0}, {0, 0.5 * h1}});
                    rhs(UT, 1, 0.5 * h1);
                    comb(UT, {{U0, 1.0}, {1, 0.5 * h1}});
                    rhs(UT, 2, 0.5 * h1);
                    comb(UT, {{U0, 1.0}, {2, h1}});
                    rhs(UT, 3, h1);
                    comb(U0, {{U0, 1.0}, {0, h1 / 6.0}, {1, h1 / 3.0}, {2, h1 / 3.0}, {3, h1 / 6.0}});
                    break;
                case DRF_RK_LSRK45:
                    // slot 1 holds the 2N register
                    for (int s = 0; s < 5; ++s) {
                        rhs(U0, 0, LSRK_C[s] * h1);
                        if (s == 0) comb(1, {{0, h1}});
                        else comb(1, {{1, LSRK_A[s]}, {0, h1}});
                        comb(U0, {{U0, 1.0}, {1, LSRK_B[s]}});
                    }
                    break;
                case DRF_RK_DOPRI:
                    rhs(U0, 0, 0.0);
                    comb(UT, {{U0, 1.0}, {0, h1 / 5.0}});
                    rhs(UT, 1, h1 / 5.0);
                    comb(UT, {{U0, 1.0}, {0, h1 * 3.0 / 40.0}, {1, h1 * 9.0 / 40.0}});
                    rhs(UT, 2, 3.0 * h1 / 10.0);
                    comb(UT, {{U0, 1.0}, {0, h1 * 44.0 / 45.0}, {1, -h1 * 56.0 / 15.0}, {2, h1 * 32.0 / 9.0}});
                    rhs(UT, 3, 4.0 * h1 / 5.0);
                    comb(UT, {{U0, 1.0}, {0, h1 * 19372.0 / 6561.0}, {1, -h1 * 25360.0 / 2187.0},
                              {2, h1 * 64448.0 / 6561.0}, {3, -h1 * 212.0 / 729.0}});
                    rhs(UT, 4, 8.0 * h1 / 9.0);
                    comb(UT, {{U0, 1.0}, {0, h1 * 9017.0 / 3168.0}, {1, -h1 * 355.0 / 33.0},
                              {2, h1 * 46732.0 / 5247.0}, {3, h1 * 49.0 / 176.0}, {4, -h1 * 5103.0 / 18656.0}});
                    rhs(UT, 5, h1);
                    comb(U0, {{U0, 1.0}, {0, h1 * 35.0 / 384.0}, {2, h1 * 500.0 / 1113.0},
                              {3, h1 * 125.0 / 192.0}, {4, -h1 * 2187.0 / 6784.0}, {5, h1 * 11.0 / 84.0}});
                    break;
                }
                for (int v = 0; v < 4; ++v)
                    DRF_CUDA(cudaMemcpyAsync(m->q(m->cur, v), K3(U0, v), m->n3 * m->tsz,
                                             cudaMemcpyDeviceToDevice, m->stream));
                DRF_CUDA(cudaMemcpyAsync(m->eta, K2(U0), m->n2 * 8, cudaMemcpyDeviceToDevice, m->stream));
                column_integral_kernel<T, NP><<<blocks_for(m->n2), 256, 0, m->stream>>>(
                    m->n2, m->G.nz, m->G.dsig, (const T *)m->q(m->cur, 0), m->HU);
                DRF_LAUNCHED();
                column_integral_kernel<T, NP><<<blocks_for(m->n2), 256, 0, m->stream>>>(
                    m->n2, m->G.nz, m->G.dsig, (const T *)m->q(m->cur, 1), m->HV);
                DRF_LAUNCHED();
                // advance device time by dt
                double tnow = 0.0;
                DRF_CUDA(cudaMemcpyAsync(&tnow, m->tdev, 8, cudaMemcpyDeviceToHost, m->stream));
                DRF_CUDA(cudaStreamSynchronize(m->stream));
                tnow += dt;
                DRF_CUDA(cudaMemcpyAsync(m->tdev, &tnow, 8, cudaMemcpyHostToDevice, m->stream));
            }
        });
        DRF_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int drf_dg_diagnostics(drf_dg *m, double *out10) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(out10, DRF_E_INVALID, "null output");
        int dev = 0, nsm = 0;
        DRF_CUDA(cudaGetDevice(&dev));
        DRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const unsigned nb3 = (unsigned)std::min<int64_t>(m->ncol, (int64_t)nsm * 8), nb2 = blocks_for(m->n2);
        if (m->diag.n < (size_t)nb3 * 6 + (size_t)nb2 * 5 + 10)
            m->diag.alloc((size_t)nb3 * 6 + (size_t)nb2 * 5 + 10);
        double *p3 = m->diag.p, *p2 = p3 + (size_t)nb3 * 6, *res10 = p2 + (size_t)nb2 * 5;
        const double dx = m->mesh.Lx / m->mesh.nx, dy = m->mesh.Ly / m->mesh.ny;
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            const int c = m->cur;
            diag3d_kernel<T, NP><<<nb3, 256, 0, m->stream>>>(
                m->ncol, m->G.nz, (const T *)m->q(c, 0), (const T *)m->q(c, 1), (const T *)m->q(c, 2),
                (const T *)m->q(c, 3), m->eta, m->h, m->pending ? m->corrU : nullptr,
                m->pending ? m->corrV : nullptr, m->pending ? m->corrR : nullptr,
                0.125 * dx * dy * m->G.dsig, p3);
            DRF_LAUNCHED();
            diag2d_kernel<NP><<<nb2, 256, 0, m->stream>>>(m->n2, m->G.nz, m->eta, m->h,
                                                         0.25 * dx * dy, m->G.g, p2);
            DRF_LAUNCHED();
        });
        diag_final_kernel<<<1, 256, 0, m->stream>>>(p3, nb3, p2, nb2, res10);
        DRF_LAUNCHED();
        double vals[10];
        DRF_CUDA(cudaMemcpyAsync(vals, res10, sizeof(vals), cudaMemcpyDeviceToHost, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        std::memcpy(out10, vals, sizeof(vals));
        for (int i = 0; i < 10; ++i)
            DRF_CHECK(std::isfinite(vals[i]), DRF_E_NONFINITE, "non-finite diagnostic (model blew up)");
    });
}

int drf_dg_time_copy(drf_dg *m, int nrep, double *ms, double *bytes) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(nrep >= 1 && ms, DRF_E_INVALID, "bad arguments");
        DRF_CHECK(((size_t)m->G.nz * m->np3 * m->tsz) % 16 == 0, DRF_E_UNSUPPORTED,
                  "column blocks are not 16-byte multiples");
        DRF_CHECK(m->smem >= 16 + (size_t)2 * m->np2 * 8 + (size_t)8 * m->G.nz * m->np3 * m->tsz,
                  DRF_E_UNSUPPORTED, "shared memory plan too small for the copy");
        m->materialize();
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            // reads the current state and the register, writes the spare ping-pong buffer and
            // the register back unchanged: the model state is not modified
            const StageArgs<T> a = m->template stage_args<T>(m->cur, 1 - m->cur, 1, 0.0, 0, nullptr, nullptr,
                                                             nullptr, m->eta, 0.0, false);
            allow_max_dynamic_smem(reinterpret_cast<const void *>(dg3d_copy_kernel<T, NP>), [] {
                int dev = 0, v = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
                return v;
            }());
            dg3d_copy_kernel<T, NP><<<m->ncol, m->stage_threads(), m->smem, m->stream>>>(a);
            DRF_LAUNCHED();
            DRF_CUDA(cudaEventRecord(e0, m->stream));
            for (int r = 0; r < nrep; ++r) {
                dg3d_copy_kernel<T, NP><<<m->ncol, m->stage_threads(), m->smem, m->stream>>>(a);
                DRF_LAUNCHED();
            }
            DRF_CUDA(cudaEventRecord(e1, m->stream));
        });
        DRF_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = (double)t / nrep;
        if (bytes) *bytes = 16.0 * (double)m->n3 * m->tsz;
        check_device_status(m);
    });
}

int drf_dg_time_stage(drf_dg *m, int nrep, double *ms, double *alg_bytes, double *ndof) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(nrep >= 1 && ms, DRF_E_INVALID, "bad arguments");
        m->materialize();
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            // a non-first LSRK stage (reads the 2N register) from the current state into the
            // spare ping-pong buffer: the model state is not modified.
            m->template launch_stage<T, NP>(m->cur, 1 - m->cur, 1, 1e-6, 0, nullptr, nullptr,
                                            nullptr, m->eta, 0.0);
            DRF_CUDA(cudaEventRecord(e0, m->stream));
            for (int r = 0; r < nrep; ++r)
                m->template launch_stage<T, NP>(m->cur, 1 - m->cur, 1, 1e-6, 0, nullptr, nullptr,
                                                nullptr, m->eta, 0.0);
            DRF_CUDA(cudaEventRecord(e1, m->stream));
        });
        DRF_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = (double)t / nrep;
        // algorithmic bytes of one stage: per 3D DOF (node x variable) state read + write and
        // 2N-register read + write, plus the horizontal face traces of the 4 neighbouring
        // columns (4/(N+1) of a state read); per 2D node eta, h, f (+ surface stress on the top
        // layer) reads and the FP64 column-increment read + write; with the baroclinic pressure
        // the stage elevation's read and write and its register's read and write per 2D node.
        const double s = (double)m->tsz;
        const double per_dof = s * (4.0 + 4.0 / m->np);
        const int n2words = 3 + 2 + 4 + (m->G.eos ? 4 : 0);
        if (alg_bytes) *alg_bytes = (double)m->n3 * 4.0 * per_dof + (double)m->n2 * 8.0 * n2words;
        if (ndof) *ndof = (double)m->n3 * 4.0;
    });
}

int drf_dg_set_forcing(drf_dg *m, const double *taux, const double *tauy) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(taux && tauy, DRF_E_INVALID, "null argument");
        DRF_CUDA(cudaMemcpyAsync(m->taux, taux, m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
        DRF_CUDA(cudaMemcpyAsync(m->tauy, tauy, m->n2 * 8, cudaMemcpyHostToDevice, m->stream));
    });
}

int drf_dg_download_surface(drf_dg *m, double *eta) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(eta, DRF_E_INVALID, "null argument");
        DRF_CUDA(cudaMemcpyAsync(eta, m->eta, m->n2 * 8, cudaMemcpyDeviceToHost, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int drf_dg_tuning(drf_dg *m, int *baro_cols_per_cta, double *baro_ms4) {
    return guard([&] {
        check_model(m);
        m->tune_baro();
        if (baro_cols_per_cta) *baro_cols_per_cta = m->baro_cpb;
        if (baro_ms4)
            for (int i = 0; i < 4; ++i) baro_ms4[i] = m->baro_ms[i];
    });
}

int drf_dg_stage_tuning(drf_dg *m, int *prefetch_half_waves, int *prefetch_columns, double *stage_ms3) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(!m->view, DRF_E_INVALID, "ensemble members use the ensemble's stage launch");
        m->tune_stage();
        if (prefetch_half_waves) *prefetch_half_waves = m->stage_hw;
        if (prefetch_columns) *prefetch_columns = m->stage_pf;
        if (stage_ms3)
            for (int i = 0; i < 3; ++i) stage_ms3[i] = m->stage_ms[i];
    });
}

int drf_dg_info(drf_dg *m, int64_t *n3d, int64_t *n2d, int *precision) {
    return guard([&] {
        check_model(m);
        if (n3d) *n3d = m->n3;
        if (n2d) *n2d = m->n2;
        if (precision) *precision = m->prm.precision;
    });
}

}  // extern "C"

// ----------------------------------------------------------------------------- ensembles
struct drf_ens {
    std::vector<std::unique_ptr<drf_dg>> mem;  // member views into the pools below
    DevBuf<unsigned char> q3;                  // 16 pooled 3D arrays
    DevBuf<double> d2;                         // 26 pooled 2D arrays + one clock per member
    DevBuf<int> errbuf;
    DevBuf<unsigned> syncbuf;  // grid-barrier words of the persistent barotropic launch
    bool baro_persist = false;
    // failure-detection check of the persistent barotropic launch: the CTA that withholds its
    // first grid-barrier arrival (-1 none); fixed when the step graphs are built, from
    // DRIFTER_B200_DEBUG_HOLD_ARRIVAL
    int debug_hold = -1;  // as drf_dg::baro_persist
    DevBuf<EnsMember> table;
    DevBuf<int2> items, tiles;
    std::vector<EnsMember> htab;
    // the stage items of one layer count (a contiguous run of the sorted item list), launched
    // with that height's CTA size and shared memory
    struct Group {
        int start, count, nz, threads;
        size_t smem;
    };
    std::vector<Group> groups;
    int nitems = 0, ntiles = 0, grid = 0;
    int64_t n3tot = 0, n2tot = 0;
    cudaStream_t stream = nullptr, own = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_kernels[2] = {0, 0};  // kernel nodes of each step graph
    int graph_nsub = 0;
    int cur = 0;

    void drop_graphs() {
        for (auto &g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        graph_nsub = 0;
    }
    ~drf_ens() {
        drop_graphs();
        if (own) cudaStreamDestroy(own);
    }

    // one baroclinic step of every member from ping-pong buffer `in`, as drf_dg::enqueue_step
    template <typename T, int NP>
    void enqueue(int in, int nsub) {
        drf_dg *m0 = mem[0].get();  // its arrays start the pools
        const int out = 1 - in;
        int src = in;
        for (int s = 0; s < 5; ++s) {
            const int dst = (s % 2 == 0) ? out : in;
            StageArgs<T> a = m0->template stage_args<T>(src, dst, s, 0.0, 0, nullptr, nullptr, nullptr,
                                                        m0->eta, 0.0, s == 0);
            a.pf = 0;  // the work items are not in column order
            for (const Group &g : groups) {
                dg3d_stage_ens_kernel<T, NP><<<g.count, g.threads, g.smem, stream>>>(a, table.p, items.p + g.start,
                                                                                     g.count);
                DRF_LAUNCHED();
            }
            src = dst;
        }
        if (baro_persist) {
            SubcycleArgs sa = m0->subcycle_args(0.0, nsub, ntiles);
            sa.mem = table.p;
            sa.tiles = tiles.p;
            sa.nmem = (int)mem.size();
            sa.sync = syncbuf.p;
            sa.err = errbuf.p;
            dispatch_flux(m0->G.flux2d, [&](auto fk) {
                constexpr int FK = decltype(fk)::value;
                launch_subcycles<NP, FK, BARO_CPB, true>(
                    m0->template baro<NP>(m0->eta, m0->HU, m0->HV, false, 0.0),
                    m0->template baro<NP>(m0->eta, m0->HU, m0->HV, true, 0.0),
                    m0->template baro<NP>(m0->us[0], m0->us[1], m0->us[2], true, 0.0), sa, stream);
            });
            return;
        }
        const int bt = BARO_CPB * NP * NP;
        dispatch_flux(m0->G.flux2d, [&](auto fk) {
            constexpr int FK = decltype(fk)::value;
            baro_force_ens_kernel<NP, FK><<<ntiles, bt, 0, stream>>>(
                m0->template baro<NP>(m0->eta, m0->HU, m0->HV, false, 0.0), BaroEns{table.p, tiles.p, nsub, 0},
                m0->dHU3, m0->dHV3, m0->Fx, m0->Fy, m0->HUo, m0->HVo);
            DRF_LAUNCHED();
            for (int sub = 0; sub < nsub; ++sub) {
                const BaroEns E{table.p, tiles.p, nsub, sub};
                baro_pred_ens_kernel<NP, FK><<<ntiles, bt, 0, stream>>>(
                    m0->template baro<NP>(m0->eta, m0->HU, m0->HV, true, 0.0), E, m0->k1[0], m0->k1[1],
                    m0->k1[2], m0->us[0], m0->us[1], m0->us[2]);
                DRF_LAUNCHED();
                baro_corr_ens_kernel<NP, FK><<<ntiles, bt, 0, stream>>>(
                    m0->template baro<NP>(m0->us[0], m0->us[1], m0->us[2], true, 0.0), E, m0->k1[0], m0->k1[1],
                    m0->k1[2], m0->eta, m0->HU, m0->HV, m0->esum);
                DRF_LAUNCHED();
            }
        });
        const int64_t nfin = n2tot > (int64_t)mem.size() ? n2tot : (int64_t)mem.size();
        baro_finish_ens_kernel<<<blocks_for(nfin), 256, 0, stream>>>(
            n2tot, nsub, table.p, (int)mem.size(), m0->esum, m0->eta_avg, m0->HU, m0->HV, m0->HUo, m0->HVo,
            m0->dHU3, m0->dHV3, m0->corrU, m0->corrV, m0->tdev, m0->eta, m0->etb[0], m0->h, m0->corrR);
        DRF_LAUNCHED();
    }
};

namespace {
void check_ens(drf_ens *e) { DRF_CHECK(e != nullptr, DRF_E_INVALID, "null ensemble handle"); }
}  // namespace

extern "C" {

int drf_ens_create(int nmembers, const drf_mesh_desc *meshes, const drf_dg_params *params,
                   const double *const *h, const double *const *f, const double *const *taux,
                   const double *const *tauy, drf_ens **out) {
    return guard([&] {
        DRF_CHECK(out && meshes && params && h && f && taux && tauy, DRF_E_INVALID, "null argument");
        *out = nullptr;
        DRF_CHECK(nmembers >= 1, DRF_E_INVALID, "an ensemble needs at least one member");
        auto e = std::make_unique<drf_ens>();
        // members: host set-up and pool offsets (3D slices padded to 64 values, 256 B in FP32,
        // so every member's column blocks keep the 16-byte alignment of the bulk copies)
        std::vector<int64_t> off3(nmembers), off2(nmembers);
        for (int i = 0; i < nmembers; ++i) {
            DRF_CHECK(h[i] && f[i] && taux[i] && tauy[i], DRF_E_INVALID, "null member field");
            auto m = std::make_unique<drf_dg>();
            m->setup(&meshes[i], &params[i], h[i], f[i], taux[i], tauy[i]);
            if (i > 0) {
                const drf_dg &m0 = *e->mem[0];
                DRF_CHECK(m->np == m0.np && m->mixed == m0.mixed && m->G.flux2d == m0.G.flux2d,
                          DRF_E_INVALID, "ensemble members must share order, precision and 2D flux");
            }
            m->view = true;
            off3[i] = e->n3tot;
            off2[i] = e->n2tot;
            e->n3tot += (m->n3 + 63) / 64 * 64;
            e->n2tot += m->n2;
            e->mem.push_back(std::move(m));
        }
        drf_dg &m0 = *e->mem[0];
        DRF_CUDA(cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking));
        e->stream = e->own;
        e->errbuf.alloc(1);
        DRF_CUDA(cudaMemset(e->errbuf.p, 0, sizeof(int)));
        e->syncbuf.alloc(4);
        DRF_CUDA(cudaMemset(e->syncbuf.p, 0, 4 * sizeof(unsigned)));
        e->q3.alloc((size_t)16 * e->n3tot * m0.tsz);
        DRF_CUDA(cudaMemset(e->q3.p, 0, e->q3.n));
        e->d2.alloc((size_t)(drf_dg::N2ARRAYS - 1) * e->n2tot + nmembers);
        DRF_CUDA(cudaMemset(e->d2.p, 0, e->d2.n * 8));
        double *tdev = e->d2.p + (size_t)(drf_dg::N2ARRAYS - 1) * e->n2tot;
        // work lists: stage items (member, column), tallest columns first; barotropic tiles
        std::vector<int2> items, tiles;
        for (int i = 0; i < nmembers; ++i) {
            drf_dg &m = *e->mem[i];
            m.bind(e->q3.p + (size_t)off3[i] * m.tsz, e->n3tot, e->d2.p + off2[i], e->n2tot, tdev + i, e->errbuf.p);
            m.stream = e->stream;
            DRF_CUDA(cudaMemcpy(m.h, h[i], m.n2 * 8, cudaMemcpyHostToDevice));
            DRF_CUDA(cudaMemcpy(m.f, f[i], m.n2 * 8, cudaMemcpyHostToDevice));
            DRF_CUDA(cudaMemcpy(m.taux, taux[i], m.n2 * 8, cudaMemcpyHostToDevice));
            DRF_CUDA(cudaMemcpy(m.tauy, tauy[i], m.n2 * 8, cudaMemcpyHostToDevice));
            EnsMember t{};
            t.off3 = off3[i];
            t.off2 = off2[i];
            t.G = m.G;
            t.dt = 0.0;
            t.ncol = m.ncol;
            t.bulk = ((size_t)m.G.nz * m.np3 * m.tsz) % 16 == 0 && ((size_t)off3[i] * m.tsz) % 16 == 0 &&
                     ((size_t)e->n3tot * m.tsz) % 16 == 0;
            e->htab.push_back(t);
            for (int c = 0; c < m.ncol; ++c) items.push_back(make_int2(i, c));
            for (int b = 0; b < (m.ncol + BARO_CPB - 1) / BARO_CPB; ++b) tiles.push_back(make_int2(i, b));
        }
        std::stable_sort(items.begin(), items.end(), [&](int2 a, int2 b) {
            return e->mem[a.x]->G.nz > e->mem[b.x]->G.nz;
        });
        e->nitems = (int)items.size();
        e->ntiles = (int)tiles.size();
        // one stage launch per layer count, with that height's CTA size and shared memory
        for (int i = 0; i < e->nitems; ++i) {
            const drf_dg &m = *e->mem[items[i].x];
            if (e->groups.empty() || e->groups.back().nz != m.G.nz)
                e->groups.push_back({i, 0, m.G.nz, m.stage_threads_generic(), m.smem});
            ++e->groups.back().count;
        }
        e->table.alloc(nmembers);
        DRF_CUDA(cudaMemcpy(e->table.p, e->htab.data(), nmembers * sizeof(EnsMember), cudaMemcpyHostToDevice));
        e->items.alloc(items.size());
        DRF_CUDA(cudaMemcpy(e->items.p, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
        e->tiles.alloc(tiles.size());
        DRF_CUDA(cudaMemcpy(e->tiles.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
        // the stage kernel must fit on an SM with the tallest member's shared memory
        int dev = 0, nsm = 0, per_sm = 0;
        DRF_CUDA(cudaGetDevice(&dev));
        DRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        m0.with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            int maxsm = 0;
            DRF_CUDA(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            allow_max_dynamic_smem(reinterpret_cast<const void *>(dg3d_stage_ens_kernel<T, NP>), maxsm);
            for (const auto &g : e->groups) {
                DRF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dg3d_stage_ens_kernel<T, NP>,
                                                                       g.threads, g.smem));
                DRF_CHECK(per_sm >= 1, DRF_E_UNSUPPORTED, "ensemble stage kernel does not fit on an SM");
            }
        });
        e->grid = e->nitems;  // one CTA per (member, column) item, over the groups' launches
        *out = e.release();
    });
}

int drf_ens_destroy(drf_ens *e) {
    return guard([&] {
        if (!e) return;
        if (e->stream) cudaStreamSynchronize(e->stream);
        delete e;
    });
}

int drf_ens_member(drf_ens *e, int i, drf_dg **member) {
    return guard([&] {
        check_ens(e);
        DRF_CHECK(member, DRF_E_INVALID, "null output");
        DRF_CHECK(i >= 0 && i < (int)e->mem.size(), DRF_E_INVALID, "member index out of range");
        *member = e->mem[i].get();
    });
}

int drf_ens_set_stream(drf_ens *e, void *s) {
    return guard([&] {
        check_ens(e);
        DRF_CUDA(cudaStreamSynchronize(e->stream));
        e->drop_graphs();
        e->stream = s ? (cudaStream_t)s : e->own;
        for (auto &m : e->mem) {
            m->drop_graphs();
            m->stream = e->stream;
        }
    });
}

int drf_ens_sync(drf_ens *e) {
    return guard([&] {
        check_ens(e);
        DRF_CUDA(cudaStreamSynchronize(e->stream));
        check_device_status(e->mem[0].get());
    });
}

int drf_ens_step(drf_ens *e, const double *dt, int nsub, int nsteps) {
    return guard([&] {
        check_ens(e);
        DRF_CHECK(dt, DRF_E_INVALID, "null argument");
        DRF_CHECK(nsub >= 1, DRF_E_INVALID, "nsub must be >= 1");
        DRF_CHECK(nsteps >= 0, DRF_E_INVALID, "nsteps must be >= 0");
        bool changed = false;
        for (size_t i = 0; i < e->mem.size(); ++i) {
            DRF_CHECK(dt[i] > 0.0 && std::isfinite(dt[i]), DRF_E_INVALID, "dt must be positive");
            DRF_CHECK(e->mem[i]->cur == e->cur, DRF_E_INVALID, "ensemble member out of step");
            if (e->htab[i].dt != dt[i]) {
                e->htab[i].dt = dt[i];
                changed = true;
            }
        }
        if (changed)  // step sizes live in the member table the graphs read
            DRF_CUDA(cudaMemcpyAsync(e->table.p, e->htab.data(), e->htab.size() * sizeof(EnsMember),
                                     cudaMemcpyHostToDevice, e->stream));
        if (e->graph_nsub != nsub) {
            e->drop_graphs();
            const char *pe = std::getenv("DRIFTER_B200_BARO_PERSISTENT");
            e->baro_persist = pe && pe[0] == '1';
            for (int in = 0; in < 2; ++in)
                e->graph[in] = capture_graph(e->stream, [&] {
                    e->mem[0]->with_types([&](auto tv, auto npc) {
                        using T = decltype(tv);
                        constexpr int NP = decltype(npc)::value;
                        e->template enqueue<T, NP>(in, nsub);
                    });
                }, &e->graph_kernels[in]);
            e->graph_nsub = nsub;
        }
        for (int s = 0; s < nsteps; ++s) {
            DRF_CUDA(cudaGraphLaunch(e->graph[e->cur], e->stream));
            launch_counter().fetch_add(e->graph_kernels[e->cur]);
            e->cur = 1 - e->cur;
        }
        for (auto &m : e->mem) {
            m->cur = e->cur;
            if (nsteps > 0) m->pending = true;
        }
    });
}

int drf_ens_info(drf_ens *e, int64_t *n3d, int *items, int *grid) {
    return guard([&] {
        check_ens(e);
        if (n3d) {
            int64_t s = 0;
            for (auto &m : e->mem) s += m->n3;
            *n3d = s;
        }
        if (items) *items = e->nitems;
        if (grid) *grid = e->grid;
    });
}

}  // extern "C"
