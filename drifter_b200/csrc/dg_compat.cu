// Reference-semantics DG kernels (FP64): the element-local right-hand side of
// PrimitiveEquationsSolver::compute_rhs and the element-local ModeSplittingSolver::step,
// including the reference's index conventions, plus the batched numerical flux.
//
// One CTA per element, one thread per LGL node; tensor-product derivatives are applied
// sum-factorized ((N+1) terms per direction) instead of the reference's dense
// (N+1)^3 x (N+1)^3 Kronecker matvecs (src/dg/basis_hexahedron.cpp:321); the summation
// order matches the dense product's non-zero order, so results agree to rounding.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "flux.cuh"

namespace drf {

namespace {

__constant__ double cD[MAXNP * MAXNP];
__constant__ double cW[MAXNP];

struct CompatP {
    double g, rho0, alpha, beta, nu_h, nu_v, kT, kS;
};

void upload_basis(const HostBasis &b) {
    // one upload per (device, order); constant memory is per module and per device
    static std::mutex mu;
    static int cur_order[64] = {0};
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && cur_order[dev] == b.order) return;
    double D[MAXNP * MAXNP] = {0}, W[MAXNP] = {0};
    for (int i = 0; i < b.np * b.np; ++i) D[i] = b.D[i];
    for (int i = 0; i < b.np; ++i) W[i] = b.w[i];
    DRF_CUDA(cudaMemcpyToSymbol(cD, D, sizeof(D)));
    DRF_CUDA(cudaMemcpyToSymbol(cW, W, sizeof(W)));
    if (dev < 64) cur_order[dev] = b.order;
}

template <int NP>
__global__ void __launch_bounds__(NP *NP *NP) compat_rhs_kernel(
    int nel, const double *__restrict__ Hu_, const double *__restrict__ Hv_,
    const double *__restrict__ eta_, const double *__restrict__ HT_, const double *__restrict__ HS_,
    const double *__restrict__ om_, const double *__restrict__ h_, const double *__restrict__ f_,
    CompatP p, double *__restrict__ dHu_, double *__restrict__ dHv_, double *__restrict__ deta_,
    double *__restrict__ dHT_, double *__restrict__ dHS_) {
    constexpr int ND = NP * NP * NP, NH = NP * NP, NV = NP;
    __shared__ double s[20][ND];
    __shared__ double sHUb[NH], sHVb[NH];
    double *Hu = s[0], *Hv = s[1], *eta = s[2], *HT = s[3], *HS = s[4], *om = s[5], *H = s[6],
           *iH = s[7], *u = s[8], *v = s[9], *T = s[10], *S = s[11];
    double *gxu = s[12], *gyu = s[13], *gxv = s[14], *gyv = s[15], *gzu = s[16], *gzv = s[17],
           *gzT = s[18], *gzS = s[19];
    const int e = blockIdx.x, n = threadIdx.x;
    if (e >= nel) return;
    const size_t o = (size_t)e * ND + n;
    const int i = n % NP, j = (n / NP) % NP, k = n / NH;
    Hu[n] = Hu_[o]; Hv[n] = Hv_[o]; eta[n] = eta_[o]; HT[n] = HT_[o]; HS[n] = HS_[o]; om[n] = om_[o];
    const double fn = f_[o];
    H[n] = eta[n] + h_[o];
    iH[n] = (H[n] > 1e-10) ? 1.0 / H[n] : 0.0;
    u[n] = Hu[n] * iH[n]; v[n] = Hv[n] * iH[n]; T[n] = HT[n] * iH[n]; S[n] = HS[n] * iH[n];
    __syncthreads();
    auto X = [&](const double *a, int m) { return a[m + NP * (j + NP * k)]; };
    auto Y = [&](const double *a, int m) { return a[i + NP * (m + NP * k)]; };
    auto Z = [&](const double *a, int m) { return a[i + NP * (j + NP * m)]; };
    {
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0;
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            const double dx = cD[i * NP + m], dy = cD[j * NP + m], dz = cD[k * NP + m];
            a0 += dx * X(u, m); a1 += dy * Y(u, m); a2 += dx * X(v, m); a3 += dy * Y(v, m);
            a4 += dz * Z(u, m); a5 += dz * Z(v, m); a6 += dz * Z(T, m); a7 += dz * Z(S, m);
        }
        gxu[n] = a0; gyu[n] = a1; gxv[n] = a2; gyv[n] = a3;
        gzu[n] = a4; gzv[n] = a5; gzT[n] = a6; gzS[n] = a7;
    }
    __syncthreads();
    // advection in divergence form (src/physics/primitive_equations.cpp:275-305, :377-393)
    double ax[4] = {0, 0, 0, 0}, ay[4] = {0, 0, 0, 0}, az[4] = {0, 0, 0, 0};
    const double *qv[4] = {Hu, Hv, HT, HS};
    double dex = 0, dey = 0, gxx = 0, gyy = 0, hxx = 0, hyy = 0, uzz = 0, vzz = 0, Tzz = 0, Szz = 0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const double dx = cD[i * NP + m], dy = cD[j * NP + m], dz = cD[k * NP + m];
        const double ux = X(u, m), vy = Y(v, m), oz = Z(om, m);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ax[q] += dx * (X(qv[q], m) * ux);
            ay[q] += dy * (Y(qv[q], m) * vy);
            az[q] += dz * (Z(qv[q], m) * oz);
        }
        dex += dx * X(eta, m); dey += dy * Y(eta, m);
        gxx += dx * X(gxu, m); gyy += dy * Y(gyu, m); hxx += dx * X(gxv, m); hyy += dy * Y(gyv, m);
        uzz += dz * Z(gzu, m); vzz += dz * Z(gzv, m); Tzz += dz * Z(gzT, m); Szz += dz * Z(gzS, m);
    }
    double rHu = 0.0 - ((ax[0] + ay[0]) + az[0]);
    double rHv = 0.0 - ((ax[1] + ay[1]) + az[1]);
    rHu += fn * Hv[n];
    rHv += -fn * Hu[n];
    rHu += -p.g * H[n] * dex;
    rHv += -p.g * H[n] * dey;
    if (p.nu_h > 0.0) {
        rHu += H[n] * (p.nu_h * gxx + p.nu_h * gyy);
        rHv += H[n] * (p.nu_h * hxx + p.nu_h * hyy);
    }
    if (p.nu_v > 0.0) {
        rHu += p.nu_v * uzz * iH[n];
        rHv += p.nu_v * vzz * iH[n];
    }
    double rHT = 0.0 - ((ax[2] + ay[2]) + az[2]);
    double rHS = 0.0 - ((ax[3] + ay[3]) + az[3]);
    if (p.kT > 0.0) rHT += p.kT * Tzz * iH[n];
    if (p.kS > 0.0) rHS += p.kS * Szz * iH[n];
    dHu_[o] = rHu; dHv_[o] = rHv; dHT_[o] = rHT; dHS_[o] = rHS;
    // free surface (src/physics/primitive_equations.cpp:229-273); column index
    // i_h*n_vert + k as in the reference
    if (n < NH) {
        double su = 0.0, sv = 0.0;
#pragma unroll
        for (int kk = 0; kk < NV; ++kk) {
            su += (0.5 * cW[kk]) * Hu[n * NV + kk];
            sv += (0.5 * cW[kk]) * Hv[n * NV + kk];
        }
        sHUb[n] = su; sHVb[n] = sv;
    }
    __syncthreads();
    if (n < NH) {
        const int ii = n % NP, jj = n / NP;
        double dx = 0.0, dy = 0.0;
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            dx += cD[ii * NP + m] * sHUb[m + jj * NP];
            dy += cD[jj * NP + m] * sHVb[ii + m * NP];
        }
        const double d2 = -(dx + dy);
#pragma unroll
        for (int kk = 0; kk < NV; ++kk) deta_[(size_t)e * ND + n * NV + kk] = d2;
    }
}

template <int NP>
__global__ void __launch_bounds__(NP *NP *NP) compat_modesplit_kernel(
    int nel, double dt, int nsub, double *Hu_, double *Hv_, double *eta_, double *HT_,
    double *HS_, double *H_, double *u_, double *v_, double *T_, double *S_, double *om_,
    double *rho_, const double *__restrict__ h_, const double *__restrict__ f_, CompatP p) {
    constexpr int ND = NP * NP * NP, NH = NP * NP, NV = NP;
    __shared__ double u[ND], v[ND], H[ND], up[ND], vp[ND];
    __shared__ double Ub[NH], Vb[NH], beta[NH], HUb[NH], HVb[NH], bH[NH], eavg[NH];
    __shared__ double Es[NH], Us[NH], Vs[NH], Hs[NH], hh[NH], ff[NH], div2[NH];
    const int e = blockIdx.x, n = threadIdx.x;
    if (e >= nel) return;
    const size_t o0 = (size_t)e * ND, o = o0 + n;
    double sw[NV], swsum = 0.0;
#pragma unroll
    for (int kk = 0; kk < NV; ++kk) { sw[kk] = 0.5 * cW[kk]; }
    u[n] = u_[o]; v[n] = v_[o]; H[n] = H_[o];
    const double HTn = HT_[o], HSn = HS_[o];
    if (n < NH) { hh[n] = h_[o0 + n]; ff[n] = f_[o0 + n]; beta[n] = eta_[o0 + n]; bH[n] = H_[o0 + n]; }
    __syncthreads();
    (void)swsum;
    // decompose (src/physics/mode_splitting.cpp:359): depth_average :136, depth_integrate :151
    if (n < NH) {
        double s1 = 0, w1 = 0, s2 = 0, w2 = 0, s3 = 0, s4 = 0;
#pragma unroll
        for (int kk = 0; kk < NV; ++kk) {
            const int idx = n * NV + kk;
            s1 += sw[kk] * u[idx]; w1 += sw[kk];
            s2 += sw[kk] * v[idx]; w2 += sw[kk];
            s3 += sw[kk] * H[idx] * u[idx];
            s4 += sw[kk] * H[idx] * v[idx];
        }
        Ub[n] = s1 / w1; Vb[n] = s2 / w2; HUb[n] = s3; HVb[n] = s4;
    }
    __syncthreads();
    {
        const int ih = n / NV;
        up[n] = u[n] - Ub[ih];
        vp[n] = v[n] - Vb[ih];
    }
    // barotropic subcycles (src/physics/mode_splitting.cpp:319, :293, :213)
    const int i = n % NP, j = n / NP;
    auto dx2 = [&](const double *X) {
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < NP; ++m) s += cD[i * NP + m] * X[m + j * NP];
        return s;
    };
    auto dy2 = [&](const double *X) {
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < NP; ++m) s += cD[j * NP + m] * X[i + m * NP];
        return s;
    };
    const double dtb = dt / nsub;
    if (n < NH) eavg[n] = 0.0;
    __syncthreads();
    for (int sub = 0; sub < nsub; ++sub) {
        double dE = 0, dU = 0, dV = 0;
        if (n < NH) {
            dE = -(dx2(HUb) + dy2(HVb));
            dU = -p.g * bH[n] * dx2(beta) + ff[n] * HVb[n] + 0.0;
            dV = -p.g * bH[n] * dy2(beta) + -ff[n] * HUb[n] + 0.0;
            Es[n] = beta[n] + dtb * dE; Us[n] = HUb[n] + dtb * dU; Vs[n] = HVb[n] + dtb * dV;
            Hs[n] = Es[n] + hh[n];
        }
        __syncthreads();
        double sE = 0, sU = 0, sV = 0;
        if (n < NH) {
            sE = -(dx2(Us) + dy2(Vs));
            sU = -p.g * Hs[n] * dx2(Es) + ff[n] * Vs[n] + 0.0;
            sV = -p.g * Hs[n] * dy2(Es) + -ff[n] * Us[n] + 0.0;
        }
        __syncthreads();
        if (n < NH) {
            const double hdt = 0.5 * dtb;
            beta[n] += hdt * (dE + sE);
            HUb[n] += hdt * (dU + sU);
            HVb[n] += hdt * (dV + sV);
            bH[n] = beta[n] + hh[n];
            const double Hi = (bH[n] > 1e-10) ? 1.0 / bH[n] : 0.0;
            Ub[n] = HUb[n] * Hi; Vb[n] = HVb[n] * Hi;
            eavg[n] += beta[n];
        }
        __syncthreads();
    }
    if (n < NH) eavg[n] /= (double)nsub;
    __syncthreads();
    // update_baroclinic (src/physics/mode_splitting.cpp:487-600)
    const int ih = n / NV;
    const double Hn = eavg[ih] + hh[ih];
    // U2 = depth_average of the current u (still the input u)
    __shared__ double U2[NH], V2[NH];
    if (n < NH) {
        double s1 = 0, w1 = 0, s2 = 0, w2 = 0;
#pragma unroll
        for (int kk = 0; kk < NV; ++kk) {
            s1 += sw[kk] * u[n * NV + kk]; w1 += sw[kk];
            s2 += sw[kk] * v[n * NV + kk]; w2 += sw[kk];
        }
        U2[n] = s1 / w1; V2[n] = s2 / w2;
    }
    __syncthreads();
    const double ut = U2[ih] + up[n], vt = V2[ih] + vp[n];
    const double Hun = Hn * ut, Hvn = Hn * vt;
    const double Hi = (Hn > 1e-10) ? 1.0 / Hn : 0.0;
    const double Tn = HTn * Hi, Sn = HSn * Hi;
    const double cHT = Hn * Tn, cHS = Hn * Sn;
    __syncthreads();
    u[n] = ut; v[n] = vt; H[n] = Hn;
    __syncthreads();
    if (n < NH) {
        double s3 = 0, s4 = 0;
#pragma unroll
        for (int kk = 0; kk < NV; ++kk) {
            const int idx = n * NV + kk;
            s3 += sw[kk] * H[idx] * u[idx];
            s4 += sw[kk] * H[idx] * v[idx];
        }
        Es[n] = s3; Us[n] = s4;  // reuse as HU_bar, HV_bar of the updated state
    }
    __syncthreads();
    if (n < NH) div2[n] = dx2(Es) + dy2(Us);
    __syncthreads();
    const int kk = n % NV;
    const double Hval = H[ih * NV];
    const double Hvi = (Hval > 1e-10) ? 1.0 / Hval : 0.0;
    const double sf = (double)kk / (double)(NV - 1);
    const double omn = -sf * div2[ih] * Hvi;
    const double rhon = p.rho0 * (1.0 - p.alpha * (Tn - 10.0) + p.beta * (Sn - 35.0));
    // recombine (src/physics/mode_splitting.cpp:398)
    u_[o] = Ub[ih] + up[n];
    v_[o] = Vb[ih] + vp[n];
    eta_[o] = beta[ih];
    Hu_[o] = Hun; Hv_[o] = Hvn; H_[o] = Hn;
    T_[o] = Tn; S_[o] = Sn; HT_[o] = cHT; HS_[o] = cHS;
    om_[o] = omn; rho_[o] = rhon;
}

__global__ void flux_batch_kernel(int kind, int64_t n, const double *UL, const double *UR,
                                  const double *nrm, double g, double *F) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    double a[3] = {UL[3 * t], UL[3 * t + 1], UL[3 * t + 2]};
    double b[3] = {UR[3 * t], UR[3 * t + 1], UR[3 * t + 2]};
    double r[3];
    sw_flux(kind, a, b, nrm[2 * t], nrm[2 * t + 1], g, r);
    F[3 * t] = r[0]; F[3 * t + 1] = r[1]; F[3 * t + 2] = r[2];
}

CompatP compat_params(const double *p8) {
    CompatP p;
    p.g = p8[0]; p.rho0 = p8[1]; p.alpha = p8[2]; p.beta = p8[3];
    p.nu_h = p8[4]; p.nu_v = p8[5]; p.kT = p8[6]; p.kS = p8[7];
    return p;
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

}  // namespace
}  // namespace drf

using namespace drf;

extern "C" {

int drf_sw_flux_batch(int kind, int64_t n, const double *UL, const double *UR,
                      const double *normals, double g, double *F) {
    return guard([&] {
        DRF_CHECK(n >= 0 && (n == 0 || (UL && UR && normals && F)), DRF_E_INVALID, "bad arguments");
        DRF_CHECK(kind >= 0 && kind <= 2, DRF_E_INVALID, "unknown flux kind");
        if (n == 0) return;
        DevBuf<double> a(3 * n), b(3 * n), c(2 * n), r(3 * n);
        DRF_CUDA(cudaMemcpy(a.p, UL, 24 * n, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(b.p, UR, 24 * n, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(c.p, normals, 16 * n, cudaMemcpyHostToDevice));
        flux_batch_kernel<<<(unsigned)((n + 255) / 256), 256>>>(kind, n, a.p, b.p, c.p, g, r.p);
        DRF_LAUNCHED();
        DRF_CUDA(cudaMemcpy(F, r.p, 24 * n, cudaMemcpyDeviceToHost));
    });
}

int drf_compat_compute_rhs(int order, int nel, const double *const *in6, const double *h,
                           const double *f, const double *params8, double *const *out5) {
    return guard([&] {
        DRF_CHECK(nel >= 0 && in6 && out5 && h && f && params8, DRF_E_INVALID, "bad arguments");
        HostBasis b = make_lgl_basis(order);
        const size_t nd = (size_t)b.np * b.np * b.np, N = nd * nel;
        if (nel == 0) return;
        for (int q = 0; q < 6; ++q)
            DRF_CHECK(all_finite(in6[q], N), DRF_E_NONFINITE, "non-finite value in state input");
        upload_basis(b);
        DevBuf<double> buf(N * 13);
        double *d[13];
        for (int q = 0; q < 13; ++q) d[q] = buf.p + q * N;
        for (int q = 0; q < 6; ++q) DRF_CUDA(cudaMemcpy(d[q], in6[q], 8 * N, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(d[6], h, 8 * N, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(d[7], f, 8 * N, cudaMemcpyHostToDevice));
        CompatP p = compat_params(params8);
        dispatch_np(b.np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            compat_rhs_kernel<NP><<<nel, NP * NP * NP>>>(nel, d[0], d[1], d[2], d[3], d[4], d[5],
                                                         d[6], d[7], p, d[8], d[9], d[10], d[11], d[12]);
        });
        DRF_LAUNCHED();
        for (int q = 0; q < 5; ++q) DRF_CUDA(cudaMemcpy(out5[q], d[8 + q], 8 * N, cudaMemcpyDeviceToHost));
    });
}

int drf_compat_time_rhs(int order, int nsrc, const double *const *in6, const double *h,
                        const double *f, const double *params8, int nel, int nrep, double *ms) {
    return guard([&] {
        DRF_CHECK(nsrc >= 1 && nel >= nsrc && nrep >= 1 && in6 && h && f && params8 && ms,
                  DRF_E_INVALID, "bad arguments");
        HostBasis b = make_lgl_basis(order);
        const size_t nd = (size_t)b.np * b.np * b.np, S = nd * nsrc, N = nd * nel;
        for (int q = 0; q < 6; ++q)
            DRF_CHECK(all_finite(in6[q], S), DRF_E_NONFINITE, "non-finite value in state input");
        upload_basis(b);
        DevBuf<double> buf(N * 13);
        double *d[13];
        for (int q = 0; q < 13; ++q) d[q] = buf.p + q * N;
        // the nsrc source elements, repeated to nel elements on the device (doubling copies)
        const double *src[8] = {in6[0], in6[1], in6[2], in6[3], in6[4], in6[5], h, f};
        for (int q = 0; q < 8; ++q) {
            DRF_CUDA(cudaMemcpy(d[q], src[q], 8 * S, cudaMemcpyHostToDevice));
            for (size_t have = S; have < N;) {
                const size_t c = std::min(have, N - have);
                DRF_CUDA(cudaMemcpy(d[q] + have, d[q], 8 * c, cudaMemcpyDeviceToDevice));
                have += c;
            }
        }
        CompatP p = compat_params(params8);
        cudaEvent_t e0, e1;
        DRF_CUDA(cudaEventCreate(&e0));
        DRF_CUDA(cudaEventCreate(&e1));
        auto launch = [&] {
            dispatch_np(b.np, [&](auto npc) {
                constexpr int NP = decltype(npc)::value;
                compat_rhs_kernel<NP><<<nel, NP * NP * NP>>>(nel, d[0], d[1], d[2], d[3], d[4], d[5],
                                                             d[6], d[7], p, d[8], d[9], d[10], d[11],
                                                             d[12]);
            });
            DRF_LAUNCHED();
        };
        for (int r = 0; r < 3; ++r) launch();  // warm-up
        DRF_CUDA(cudaEventRecord(e0));
        for (int r = 0; r < nrep; ++r) launch();
        DRF_CUDA(cudaEventRecord(e1));
        DRF_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = (double)t / nrep;
    });
}

int drf_compat_modesplit_step(int order, int nel, double dt, int nsub, double *const *st12,
                              const double *h, const double *f, const double *params8) {
    return guard([&] {
        DRF_CHECK(nel >= 0 && st12 && h && f && params8, DRF_E_INVALID, "bad arguments");
        DRF_CHECK(nsub >= 1, DRF_E_INVALID, "nsub must be >= 1");
        DRF_CHECK(order >= 1, DRF_E_INVALID, "order must be >= 1");
        HostBasis b = make_lgl_basis(order);
        const size_t nd = (size_t)b.np * b.np * b.np, N = nd * nel;
        if (nel == 0) return;
        for (int q = 0; q < 12; ++q)
            DRF_CHECK(all_finite(st12[q], N), DRF_E_NONFINITE, "non-finite value in state input");
        upload_basis(b);
        DevBuf<double> buf(N * 14);
        double *d[14];
        for (int q = 0; q < 14; ++q) d[q] = buf.p + q * N;
        for (int q = 0; q < 12; ++q) DRF_CUDA(cudaMemcpy(d[q], st12[q], 8 * N, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(d[12], h, 8 * N, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(d[13], f, 8 * N, cudaMemcpyHostToDevice));
        CompatP p = compat_params(params8);
        dispatch_np(b.np, [&](auto npc) {
            constexpr int NP = decltype(npc)::value;
            compat_modesplit_kernel<NP><<<nel, NP * NP * NP>>>(nel, dt, nsub, d[0], d[1], d[2], d[3],
                                                               d[4], d[5], d[6], d[7], d[8], d[9],
                                                               d[10], d[11], d[12], d[13], p);
        });
        DRF_LAUNCHED();
        for (int q = 0; q < 12; ++q) DRF_CUDA(cudaMemcpy(st12[q], d[q], 8 * N, cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"
