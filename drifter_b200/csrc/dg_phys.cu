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
//   baro_force, (baro_pred, baro_corr) x nsub, baro_finish, correct3d.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "flux.cuh"

namespace drf {
namespace {

__constant__ DevBasis cB;

template <typename T>
struct BT;
template <>
struct BT<double> {
    __device__ static double D(int i) { return cB.D[i]; }
    __device__ static double D2(int i) { return cB.D2[i]; }
    __device__ static double S(int i) { return cB.S[i]; }
    __device__ static double w(int i) { return cB.w[i]; }
    __device__ static double x(int i) { return cB.x[i]; }
};
template <>
struct BT<float> {
    __device__ static float D(int i) { return cB.Df[i]; }
    __device__ static float D2(int i) { return cB.D2f[i]; }
    __device__ static float S(int i) { return cB.Sf[i]; }
    __device__ static float w(int i) { return cB.wf[i]; }
    __device__ static float x(int i) { return cB.xf[i]; }
};

struct Geo {
    int nx, ny, nz, flux2d;
    int bc[4];
    double cx, cy, cs, Lx, Ly, Ls, dsig;
    double g, rho0, nu_h, nu_v, kT, kS, cd;
    double tide_amp, tide_w;
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
    double toff;
    double *dHU3, *dHV3;
    T *omega_out;
    double *deta_out;
    T A, B, dt;
    int mode;   // 0: LSRK stage update, 1: write the right-hand side into res[]
    int first;  // 1: A = 0 stage (res not read, column increments overwritten)
    Geo G;
};

template <typename T, int NP>
__global__ void __launch_bounds__(256) dg3d_stage_kernel(StageArgs<T> a) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP, N = NP - 1;
    using B = BT<T>;
    const Geo &G = a.G;
    const int nz = G.nz, ncn = nz * NP3;
    const int c = blockIdx.x, ex = c % G.nx, ey = c / G.nx;
    const size_t base = (size_t)c * ncn;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sQ = reinterpret_cast<T *>(smem_raw);  // [4][ncn]
    T *sU = sQ + 4 * ncn, *sV = sU + ncn, *sOm = sV + ncn, *sW = sOm + ncn, *sW2 = sW + ncn;
    T *sBase = sW2 + ncn;                     // [nz][NP2]
    T *sIH = sBase + nz * NP2;                // [NP2]
    T *sItot = sIH + NP2;                     // [NP2]
    double *sEta = reinterpret_cast<double *>(
        (reinterpret_cast<uintptr_t>(sItot + NP2) + 15) & ~uintptr_t(15));
    double *sH = sEta + NP2;

    const double tnow = a.tdev[0] + a.toff;
    const double etide = tide_at(G, tnow);

    for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
#pragma unroll
        for (int v = 0; v < 4; ++v) sQ[v * ncn + n] = a.qin[v][base + n];
    }
    for (int t = threadIdx.x; t < NP2; t += blockDim.x) {
        const double e = a.eta[(size_t)c * NP2 + t];
        const double H = e + a.h[(size_t)c * NP2 + t];
        sEta[t] = e;
        sH[t] = H;
        sIH[t] = (T)(1.0 / H);
    }
    __syncthreads();
    for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
        const int an = (n % NP3) % NP2;
        sU[n] = sQ[n] * sIH[an];
        sV[n] = sQ[ncn + n] * sIH[an];
    }
    __syncthreads();

    // horizontal neighbour (or ghost) state across side s for own node (ez, i, j, k).
    auto outside = [&](int s, int ez, int i, int j, int k, int n, T qp[4], T &etap, T &Hp) {
        int nc = -1, ni = i, nj = j;
        if (s == 0 && ex > 0) { nc = c - 1; ni = N; }
        if (s == 1 && ex < G.nx - 1) { nc = c + 1; ni = 0; }
        if (s == 2 && ey > 0) { nc = c - G.nx; nj = N; }
        if (s == 3 && ey < G.ny - 1) { nc = c + G.nx; nj = 0; }
        const int an = i + NP * j;
        if (nc >= 0) {
            const size_t nb = (size_t)nc * ncn + (size_t)ez * NP3 + ni + NP * (nj + NP * k);
#pragma unroll
            for (int v = 0; v < 4; ++v) qp[v] = a.qin[v][nb];
            const size_t n2 = (size_t)nc * NP2 + ni + NP * nj;
            const double e = a.eta[n2];
            etap = (T)e;
            Hp = (T)(e + a.h[n2]);
            return;
        }
        if (G.bc[s] == DRF_BC_TIDE) {
            const double Hpd = etide + a.h[(size_t)c * NP2 + an];
            etap = (T)etide;
            Hp = (T)Hpd;
            const T r = (T)Hpd * sIH[an];
#pragma unroll
            for (int v = 0; v < 4; ++v) qp[v] = sQ[v * ncn + n] * r;
        } else {
            etap = (T)sEta[an];
            Hp = (T)sH[an];
#pragma unroll
            for (int v = 0; v < 4; ++v) qp[v] = sQ[v * ncn + n];
            if (s <= 1) qp[0] = -qp[0]; else qp[1] = -qp[1];
        }
    };

    const T cx = (T)G.cx, cy = (T)G.cy, cs = (T)G.cs;
    const T Lx = (T)G.Lx, Ly = (T)G.Ly, Ls = (T)G.Ls;

    // ---- horizontal divergence of (Hu, Hv), central face flux
    for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
        const int ez = n / NP3, ln = n % NP3, i = ln % NP, j = (ln / NP) % NP, k = ln / NP2;
        const int eb = ez * NP3;
        T sx = 0, sy = 0;
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            sx += B::D(i * NP + m) * sQ[eb + m + NP * (j + NP * k)];
            sy += B::D(j * NP + m) * sQ[ncn + eb + i + NP * (m + NP * k)];
        }
        T d = cx * sx + cy * sy;
        if (i == 0 || i == N || j == 0 || j == N) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const bool on = (s == 0 && i == 0) || (s == 1 && i == N) || (s == 2 && j == 0) ||
                                (s == 3 && j == N);
                if (!on) continue;
                T qp[4], ep, Hp;
                outside(s, ez, i, j, k, n, qp, ep, Hp);
                const int comp = s <= 1 ? 0 : 1;
                const T nrm = (s == 0 || s == 2) ? T(-1) : T(1);
                const T L = s <= 1 ? Lx : Ly;
                const T qm = sQ[comp * ncn + n];
                const T fm = qm * nrm;
                const T fs = T(0.5) * (qm + qp[comp]) * nrm;
                d += L * (fs - fm);
            }
        }
        sW[n] = d;
    }
    __syncthreads();
    // ---- layer integrals J_k = (dsig/2) sum_m S[k][m] delta_m
    const T hds = (T)(0.5 * G.dsig);
    for (int t = threadIdx.x; t < nz * NP2; t += blockDim.x) {
        const int ez = t / NP2, an = t % NP2;
        T del[NP];
#pragma unroll
        for (int m = 0; m < NP; ++m) del[m] = sW[ez * NP3 + an + NP2 * m];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            T s = 0;
#pragma unroll
            for (int m = 0; m < NP; ++m) s += B::S(k * NP + m) * del[m];
            sW[ez * NP3 + an + NP2 * k] = (k == 0) ? T(0) : hds * s;
        }
    }
    __syncthreads();
    for (int an = threadIdx.x; an < NP2; an += blockDim.x) {
        T Ib = 0;
        for (int ez = 0; ez < nz; ++ez) {
            sBase[ez * NP2 + an] = Ib;
            Ib = Ib + sW[ez * NP3 + an + NP2 * N];
        }
        sItot[an] = Ib;
        if (a.mode == 1 && a.deta_out) a.deta_out[(size_t)c * NP2 + an] = -(double)Ib;
    }
    __syncthreads();
    for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
        const int ez = n / NP3, ln = n % NP3, an = ln % NP2, k = ln / NP2;
        const T I = sBase[ez * NP2 + an] + sW[n];
        T s1 = (T)(G.dsig * (ez + 0.5 * ((double)B::x(k) + 1.0)));
        if (ez == nz - 1 && k == N) s1 = T(1);
        const T Hw = -I + s1 * sItot[an];
        const T om = Hw * sIH[an];
        sOm[n] = om;
        if (a.mode == 1 && a.omega_out) a.omega_out[base + n] = om;
    }
    __syncthreads();

    // ---- right-hand side and stage update
    const T g = (T)G.g;
    for (int n = threadIdx.x; n < ncn; n += blockDim.x) {
        const int ez = n / NP3, ln = n % NP3, i = ln % NP, j = (ln / NP) % NP, k = ln / NP2;
        const int an = i + NP * j, eb = ez * NP3;
        const T iH = sIH[an], Hh = (T)sH[an];
        T r[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const T *q = sQ + v * ncn + eb;
            T ax = 0, ay = 0, as = 0;
#pragma unroll
            for (int m = 0; m < NP; ++m) {
                const int px = m + NP * (j + NP * k), py = i + NP * (m + NP * k), pz = an + NP2 * m;
                ax += B::D(i * NP + m) * q[px] * sU[eb + px];
                ay += B::D(j * NP + m) * q[py] * sV[eb + py];
                as += B::D(k * NP + m) * q[pz] * sOm[eb + pz];
            }
            r[v] = -(cx * ax + cy * ay + cs * as);
        }
        const T fa = (T)a.f[(size_t)c * NP2 + an];
        T gex = 0, gey = 0;
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            gex += B::D(i * NP + m) * (T)sEta[m + NP * j];
            gey += B::D(j * NP + m) * (T)sEta[i + NP * m];
        }
        const T Hu = sQ[n], Hv = sQ[ncn + n];
        r[0] += fa * Hv - g * Hh * cx * gex;
        r[1] += -fa * Hu - g * Hh * cy * gey;
        if (G.nu_h > 0.0) {
            T uxx = 0, uyy = 0, vxx = 0, vyy = 0;
#pragma unroll
            for (int l = 0; l < NP; ++l) {
                const int px = eb + l + NP * (j + NP * k), py = eb + i + NP * (l + NP * k);
                uxx += B::D2(i * NP + l) * sU[px];
                uyy += B::D2(j * NP + l) * sU[py];
                vxx += B::D2(i * NP + l) * sV[px];
                vyy += B::D2(j * NP + l) * sV[py];
            }
            const T nh = (T)G.nu_h;
            r[0] += nh * Hh * (cx * cx * uxx + cy * cy * uyy);
            r[1] += nh * Hh * (cx * cx * vxx + cy * cy * vyy);
        }
        {
            const T kap[4] = {(T)G.nu_v, (T)G.nu_v, (T)G.kT, (T)G.kS};
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if (!(kap[v] > T(0))) continue;
                const T *q = sQ + v * ncn + eb;
                T szz = 0;
#pragma unroll
                for (int l = 0; l < NP; ++l) szz += B::D2(k * NP + l) * (q[an + NP2 * l] * iH);
                r[v] += kap[v] * iH * cs * cs * szz;
            }
        }
        if (i == 0 || i == N || j == 0 || j == N) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const bool on = (s == 0 && i == 0) || (s == 1 && i == N) || (s == 2 && j == 0) ||
                                (s == 3 && j == N);
                if (!on) continue;
                T qp[4], ep, Hp;
                outside(s, ez, i, j, k, n, qp, ep, Hp);
                const T nx = s == 0 ? T(-1) : (s == 1 ? T(1) : T(0));
                const T ny = s == 2 ? T(-1) : (s == 3 ? T(1) : T(0));
                const T L = s <= 1 ? Lx : Ly;
                const T unm = (Hu * nx + Hv * ny) * iH;
                const T unp = (qp[0] * nx + qp[1] * ny) / Hp;
                const T lam = fmax(fabs(unm), fabs(unp));
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const T qm = sQ[v * ncn + n];
                    const T fs = T(0.5) * (qm * unm + qp[v] * unp) - T(0.5) * lam * (qp[v] - qm);
                    r[v] -= L * (fs - qm * unm);
                }
                const T pj = g * Hh * T(0.5) * (ep - (T)sEta[an]);
                r[0] -= L * pj * nx;
                r[1] -= L * pj * ny;
            }
        }
        if (k == 0 || k == N) {
            const T nrm = k == 0 ? T(-1) : T(1);
            const T wm = sOm[n] * nrm;
            const bool interior = (k == 0 && ez > 0) || (k == N && ez < nz - 1);
            if (interior) {
                const int n2 = k == 0 ? (ez - 1) * NP3 + an + NP2 * N : (ez + 1) * NP3 + an;
                const T wp = sOm[n2] * nrm;
                const T lam = fmax(fabs(wm), fabs(wp));
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const T qm = sQ[v * ncn + n], qpp = sQ[v * ncn + n2];
                    const T fs = T(0.5) * (qm * wm + qpp * wp) - T(0.5) * lam * (qpp - qm);
                    r[v] -= Ls * (fs - qm * wm);
                }
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) r[v] -= Ls * (T(0) - sQ[v * ncn + n] * wm);
                if (k == 0) {
                    const T uu = Hu * iH, vv = Hv * iH;
                    const T sp = sqrt(uu * uu + vv * vv);
                    r[0] -= Ls * (T)G.cd * sp * uu;
                    r[1] -= Ls * (T)G.cd * sp * vv;
                } else {
                    r[0] += Ls * (T)(a.taux[(size_t)c * NP2 + an] / G.rho0);
                    r[1] += Ls * (T)(a.tauy[(size_t)c * NP2 + an] / G.rho0);
                }
            }
        }
        const size_t gi = base + n;
        if (a.mode == 1) {
#pragma unroll
            for (int v = 0; v < 4; ++v) a.res[v][gi] = r[v];
        } else {
            T rn[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                rn[v] = (a.first ? T(0) : a.A * a.res[v][gi]) + a.dt * r[v];
                a.res[v][gi] = rn[v];
                a.qout[v][gi] = sQ[v * ncn + n] + a.B * rn[v];
            }
            sW[n] = B::w(k) * (a.B * rn[0]);
            sW2[n] = B::w(k) * (a.B * rn[1]);
        }
    }
    if (a.mode == 0) {
        __syncthreads();
        for (int an = threadIdx.x; an < NP2; an += blockDim.x) {
            double su = 0.0, sv = 0.0;
            for (int ez = 0; ez < nz; ++ez)
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    su += (double)sW[ez * NP3 + an + NP2 * k];
                    sv += (double)sW2[ez * NP3 + an + NP2 * k];
                }
            const size_t i2 = (size_t)c * NP2 + an;
            const double hd = 0.5 * G.dsig;
            a.dHU3[i2] = (a.first ? 0.0 : a.dHU3[i2]) + hd * su;
            a.dHV3[i2] = (a.first ? 0.0 : a.dHV3[i2]) + hd * sv;
        }
    }
}

// ------------------------------------------------------------------------- barotropic (FP64)
struct BaroArgs {
    const double *e, *hu, *hv, *h, *f, *Fx, *Fy, *tdev;
    double toff;
    Geo G;
};

template <int NP>
__device__ void baro_phi(const BaroArgs &a, int c, int an, double &re, double &ru, double &rv) {
    constexpr int NP2 = NP * NP, N = NP - 1;
    const Geo &G = a.G;
    const int ex = c % G.nx, ey = c / G.nx, i = an % NP, j = an / NP;
    const size_t o = (size_t)c * NP2;
    const double H = a.e[o + an] + a.h[o + an];
    double dhu = 0, dhv = 0, auu = 0, auv = 0, avu = 0, avv = 0, gex = 0, gey = 0;
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const size_t px = o + m + NP * j, py = o + i + NP * m;
        const double Hx = a.e[px] + a.h[px], Hy = a.e[py] + a.h[py];
        const double dxm = cB.D[i * NP + m], dym = cB.D[j * NP + m];
        dhu += dxm * a.hu[px];
        dhv += dym * a.hv[py];
        auu += dxm * a.hu[px] * a.hu[px] / Hx;
        avu += dxm * a.hv[px] * a.hu[px] / Hx;
        auv += dym * a.hu[py] * a.hv[py] / Hy;
        avv += dym * a.hv[py] * a.hv[py] / Hy;
        gex += dxm * a.e[px];
        gey += dym * a.e[py];
    }
    re = -(G.cx * dhu + G.cy * dhv);
    ru = -(G.cx * auu + G.cy * auv) - G.g * H * G.cx * gex + a.f[o + an] * a.hv[o + an] +
         (a.Fx ? a.Fx[o + an] : 0.0);
    rv = -(G.cx * avu + G.cy * avv) - G.g * H * G.cy * gey - a.f[o + an] * a.hu[o + an] +
         (a.Fy ? a.Fy[o + an] : 0.0);
    if (!(i == 0 || i == N || j == 0 || j == N)) return;
    const double etide = tide_at(G, a.tdev[0] + a.toff);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const bool on = (s == 0 && i == 0) || (s == 1 && i == N) || (s == 2 && j == 0) ||
                        (s == 3 && j == N);
        if (!on) continue;
        const double nx = s == 0 ? -1.0 : (s == 1 ? 1.0 : 0.0);
        const double ny = s == 2 ? -1.0 : (s == 3 ? 1.0 : 0.0);
        const double L = s <= 1 ? G.Lx : G.Ly;
        int nc = -1, ni = i, nj = j;
        if (s == 0 && ex > 0) { nc = c - 1; ni = N; }
        if (s == 1 && ex < G.nx - 1) { nc = c + 1; ni = 0; }
        if (s == 2 && ey > 0) { nc = c - G.nx; nj = N; }
        if (s == 3 && ey < G.ny - 1) { nc = c + G.nx; nj = 0; }
        double UL[3] = {H, a.hu[o + an], a.hv[o + an]}, UR[3];
        if (nc >= 0) {
            const size_t q = (size_t)nc * NP2 + ni + NP * nj;
            UR[0] = a.e[q] + a.h[q]; UR[1] = a.hu[q]; UR[2] = a.hv[q];
        } else if (G.bc[s] == DRF_BC_TIDE) {
            UR[0] = etide + a.h[o + an];
            const double r = UR[0] / H;
            UR[1] = UL[1] * r; UR[2] = UL[2] * r;
        } else {
            UR[0] = H; UR[1] = UL[1]; UR[2] = UL[2];
            if (s <= 1) UR[1] = -UL[1]; else UR[2] = -UL[2];
        }
        double Fs[3], Fm[3];
        sw_flux(G.flux2d, UL, UR, nx, ny, G.g, Fs);
        sw_phys_flux(UL, nx, ny, G.g, Fm);
        re -= L * (Fs[0] - Fm[0]);
        ru -= L * (Fs[1] - Fm[1]);
        rv -= L * (Fs[2] - Fm[2]);
    }
}

template <int NP>
__global__ void baro_rhs_kernel(BaroArgs a, int64_t n2, double *ke, double *ku, double *kv) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n2) return;
    double re, ru, rv;
    baro_phi<NP>(a, (int)(t / (NP * NP)), (int)(t % (NP * NP)), re, ru, rv);
    ke[t] = re; ku[t] = ru; kv[t] = rv;
}

// F = (3D-integrated increment)/dt - Phi(U^n); keeps HU^n, HV^n for the transport correction.
template <int NP>
__global__ void baro_force_kernel(BaroArgs a, int64_t n2, double dt, const double *dHU3,
                                  const double *dHV3, double *Fx, double *Fy, double *HUo,
                                  double *HVo) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n2) return;
    double re, ru, rv;
    baro_phi<NP>(a, (int)(t / (NP * NP)), (int)(t % (NP * NP)), re, ru, rv);
    Fx[t] = dHU3[t] / dt - ru;
    Fy[t] = dHV3[t] / dt - rv;
    HUo[t] = a.hu[t];
    HVo[t] = a.hv[t];
}

template <int NP>
__global__ void baro_pred_kernel(BaroArgs a, int64_t n2, double dtb, double *k1e, double *k1u,
                                 double *k1v, double *es, double *us, double *vs) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n2) return;
    double re, ru, rv;
    baro_phi<NP>(a, (int)(t / (NP * NP)), (int)(t % (NP * NP)), re, ru, rv);
    k1e[t] = re; k1u[t] = ru; k1v[t] = rv;
    es[t] = a.e[t] + dtb * re;
    us[t] = a.hu[t] + dtb * ru;
    vs[t] = a.hv[t] + dtb * rv;
}

template <int NP>
__global__ void baro_corr_kernel(BaroArgs a, int64_t n2, double dtb, const double *k1e,
                                 const double *k1u, const double *k1v, double *e, double *hu,
                                 double *hv, double *esum, int first) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n2) return;
    double re, ru, rv;
    baro_phi<NP>(a, (int)(t / (NP * NP)), (int)(t % (NP * NP)), re, ru, rv);
    const double hd = 0.5 * dtb;
    const double en = e[t] + hd * (k1e[t] + re);
    e[t] = en;
    hu[t] = hu[t] + hd * (k1u[t] + ru);
    hv[t] = hv[t] + hd * (k1v[t] + rv);
    esum[t] = (first ? 0.0 : esum[t]) + en;
}

__global__ void baro_finish_kernel(int64_t n2, int nsub, double dt, const double *esum,
                                   double *eta_avg, const double *HU, const double *HV,
                                   const double *HUo, const double *HVo, double *dHU3, double *dHV3,
                                   double *tdev) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t == 0) tdev[0] = tdev[0] + dt;
    if (t >= n2) return;
    eta_avg[t] = esum[t] / nsub;
    dHU3[t] = HU[t] - (HUo[t] + dHU3[t]);
    dHV3[t] = HV[t] - (HVo[t] + dHV3[t]);
}

template <typename T, int NP>
__global__ void correct3d_kernel(int64_t n3, int nz, T *Hu, T *Hv, const double *cu,
                                 const double *cv) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const int64_t c = t / ((int64_t)nz * NP3);
    const int an = (int)((t % NP3) % NP2);
    const int64_t i2 = c * NP2 + an;
    Hu[t] = Hu[t] + (T)cu[i2];
    Hv[t] = Hv[t] + (T)cv[i2];
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
            s += 0.5 * dsig * cB.w[k] * (double)q[(c * nz + ez) * NP3 + an + NP2 * k];
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
template <typename T, int NP>
__global__ void diag3d_kernel(int64_t n3, int nz, const T *Hu, const T *Hv, const T *HT,
                              const T *HS, const double *eta, const double *h, double wvol,
                              double *part) {
    constexpr int NP2 = NP * NP, NP3 = NP2 * NP;
    __shared__ double red[6][256];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double en = 0, heat = 0, salt = 0, um = 0, Tmax = -1e300, Tmin = 1e300;
    if (t < n3) {
        const int64_t c = t / ((int64_t)nz * NP3);
        const int ln = (int)(t % NP3), an = ln % NP2, i = an % NP, j = an / NP, k = ln / NP2;
        const int64_t i2 = c * NP2 + an;
        const double H = eta[i2] + h[i2];
        const double wv = wvol * cB.w[i] * cB.w[j] * cB.w[k];
        const double hu = Hu[t], hv = Hv[t];
        en = wv * 0.5 * (hu * hu + hv * hv) / H;
        heat = wv * (double)HT[t];
        salt = wv * (double)HS[t];
        um = sqrt(hu * hu + hv * hv) / H;
        Tmax = Tmin = (double)HT[t] / H;
    }
    red[0][threadIdx.x] = en; red[1][threadIdx.x] = heat; red[2][threadIdx.x] = salt;
    red[3][threadIdx.x] = um; red[4][threadIdx.x] = Tmax; red[5][threadIdx.x] = Tmin;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
            red[3][threadIdx.x] = fmax(red[3][threadIdx.x], red[3][threadIdx.x + s]);
            red[4][threadIdx.x] = fmax(red[4][threadIdx.x], red[4][threadIdx.x + s]);
            red[5][threadIdx.x] = fmin(red[5][threadIdx.x], red[5][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) part[blockIdx.x * 6 + q] = red[q][0];
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
        const double H = eta[t] + h[t], wa = warea * cB.w[i] * cB.w[j];
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

const double LSRK_A[5] = {0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257};
const double LSRK_B[5] = {0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488,
                          0.1530572479681};
const double LSRK_C[5] = {0.0, 0.1496590219993, 0.3704009573644, 0.6222557631345, 0.9582821306748};

inline unsigned blocks_for(int64_t n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

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
    double *h = nullptr, *f = nullptr, *taux = nullptr, *tauy = nullptr, *eta = nullptr,
           *HU = nullptr, *HV = nullptr, *eta_avg = nullptr, *esum = nullptr, *Fx = nullptr,
           *Fy = nullptr, *HUo = nullptr, *HVo = nullptr, *k1[3] = {}, *us[3] = {}, *dHU3 = nullptr,
           *dHV3 = nullptr, *tdev = nullptr, *scratch2 = nullptr;
    int cur = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_dt = 0.0;
    int graph_nsub = 0;
    size_t smem = 0;

    void *q(int buf, int v) { return q3.p + ((size_t)buf * 4 + v) * n3 * tsz; }
    void *res(int v) { return q3.p + ((size_t)8 + v) * n3 * tsz; }
    void *tmp(int v) { return q3.p + ((size_t)12 + v) * n3 * tsz; }

    void drop_graphs() {
        for (auto &g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        graph_nsub = 0;
    }
    ~drf_dg() {
        drop_graphs();
        if (own) cudaStreamDestroy(own);
    }

    template <typename T, int NP>
    void launch_stage(int in, int out, int s, double dt, int mode, void *const *rout,
                      T *omega_out, double *deta_out, const double *eta_use, double toff) {
        StageArgs<T> a{};
        for (int v = 0; v < 4; ++v) {
            a.qin[v] = (const T *)q(in, v);
            a.qout[v] = (T *)q(out, v);
            a.res[v] = mode == 1 ? (T *)rout[v] : (T *)res(v);
        }
        a.eta = eta_use; a.h = h; a.f = f; a.taux = taux; a.tauy = tauy; a.tdev = tdev;
        a.toff = toff;
        a.dHU3 = dHU3; a.dHV3 = dHV3;
        a.omega_out = omega_out; a.deta_out = deta_out;
        a.A = (T)LSRK_A[s]; a.B = (T)LSRK_B[s]; a.dt = (T)dt;
        a.mode = mode; a.first = (s == 0);
        a.G = G;
        dg3d_stage_kernel<T, NP><<<ncol, 256, smem, stream>>>(a);
        DRF_LAUNCHED();
    }

    template <int NP>
    BaroArgs baro(const double *e, const double *u, const double *v, bool forced, double toff) {
        BaroArgs b{};
        b.e = e; b.hu = u; b.hv = v; b.h = h; b.f = f;
        b.Fx = forced ? Fx : nullptr; b.Fy = forced ? Fy : nullptr;
        b.tdev = tdev; b.toff = toff; b.G = G;
        return b;
    }

    template <typename T, int NP>
    void enqueue_step(int in, double dt, int nsub) {
        const int out = 1 - in;
        int src = in;
        for (int s = 0; s < 5; ++s) {
            const int dst = (s % 2 == 0) ? out : in;
            launch_stage<T, NP>(src, dst, s, dt, 0, nullptr, nullptr, nullptr, eta, 0.0);
            src = dst;
        }
        // after 5 stages the state is in `out`
        const unsigned nb2 = blocks_for(n2);
        baro_force_kernel<NP><<<nb2, 256, 0, stream>>>(baro<NP>(eta, HU, HV, false, 0.0), n2, dt,
                                                       dHU3, dHV3, Fx, Fy, HUo, HVo);
        DRF_LAUNCHED();
        const double dtb = dt / nsub;
        for (int m = 0; m < nsub; ++m) {
            baro_pred_kernel<NP><<<nb2, 256, 0, stream>>>(baro<NP>(eta, HU, HV, true, m * dtb), n2,
                                                          dtb, k1[0], k1[1], k1[2], us[0], us[1], us[2]);
            DRF_LAUNCHED();
            baro_corr_kernel<NP><<<nb2, 256, 0, stream>>>(
                baro<NP>(us[0], us[1], us[2], true, m * dtb + dtb), n2, dtb, k1[0], k1[1], k1[2],
                eta, HU, HV, esum, m == 0);
            DRF_LAUNCHED();
        }
        baro_finish_kernel<<<nb2, 256, 0, stream>>>(n2, nsub, dt, esum, eta_avg, HU, HV, HUo, HVo,
                                                    dHU3, dHV3, tdev);
        DRF_LAUNCHED();
        correct3d_kernel<T, NP><<<blocks_for(n3), 256, 0, stream>>>(n3, G.nz, (T *)q(out, 0),
                                                                  (T *)q(out, 1), dHU3, dHV3);
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

void upload_phys_basis(const HostBasis &b) {
    static std::mutex mu;
    static int cur_order[64] = {0};
    int dev = 0;
    DRF_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && cur_order[dev] == b.order) return;
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
    DRF_CUDA(cudaMemcpyToSymbol(cB, &db, sizeof(db)));
    if (dev < 64) cur_order[dev] = b.order;
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

}  // namespace
}  // namespace drf

extern "C" {

int drf_dg_create(const drf_mesh_desc *mesh, const drf_dg_params *params, const double *h,
                  const double *f, const double *taux, const double *tauy, drf_dg **out) {
    return guard([&] {
        DRF_CHECK(mesh && params && h && f && taux && tauy && out, DRF_E_INVALID, "null argument");
        *out = nullptr;
        DRF_CHECK(mesh->nx >= 1 && mesh->ny >= 1 && mesh->nz >= 1, DRF_E_INVALID,
                  "mesh must have at least one element per direction");
        DRF_CHECK(mesh->Lx > 0 && mesh->Ly > 0, DRF_E_INVALID, "basin extent must be positive");
        DRF_CHECK(params->flux2d >= 0 && params->flux2d <= 2, DRF_E_INVALID, "unknown flux kind");
        DRF_CHECK(params->precision == DRF_PREC_FP64 || params->precision == DRF_PREC_MIXED,
                  DRF_E_INVALID, "unknown precision");
        for (int s = 0; s < 4; ++s)
            DRF_CHECK(params->bc[s] == DRF_BC_WALL || params->bc[s] == DRF_BC_TIDE, DRF_E_INVALID,
                      "unknown boundary type");
        auto m = std::make_unique<drf_dg>();
        m->mesh = *mesh;
        m->prm = *params;
        m->basis = make_lgl_basis(mesh->order);
        m->np = m->basis.np; m->np2 = m->np * m->np; m->np3 = m->np2 * m->np;
        m->ncol = mesh->nx * mesh->ny;
        m->n2 = (int64_t)m->ncol * m->np2;
        m->n3 = m->n2 * mesh->nz * m->np;
        m->mixed = params->precision == DRF_PREC_MIXED;
        m->tsz = m->mixed ? 4 : 8;
        for (const double *a : {h, f, taux, tauy})
            DRF_CHECK(all_finite(a, m->n2), DRF_E_NONFINITE, "non-finite value in a 2D field");
        for (int64_t i = 0; i < m->n2; ++i)
            DRF_CHECK(h[i] > 0.0, DRF_E_INVALID, "bathymetry must be positive (no dry nodes)");
        Geo &G = m->G;
        const double dx = mesh->Lx / mesh->nx, dy = mesh->Ly / mesh->ny, ds = 1.0 / mesh->nz;
        const double wend = m->basis.w[0];
        G.nx = mesh->nx; G.ny = mesh->ny; G.nz = mesh->nz; G.flux2d = params->flux2d;
        for (int s = 0; s < 4; ++s) G.bc[s] = params->bc[s];
        G.cx = 2.0 / dx; G.cy = 2.0 / dy; G.cs = 2.0 / ds;
        G.Lx = G.cx / wend; G.Ly = G.cy / wend; G.Ls = G.cs / wend; G.dsig = ds;
        G.g = params->g; G.rho0 = params->rho0; G.nu_h = params->nu_h; G.nu_v = params->nu_v;
        G.kT = params->kappa_v_T; G.kS = params->kappa_v_S; G.cd = params->cd;
        G.tide_amp = params->tide_amp;
        G.tide_w = params->tide_period != 0.0 ? 2.0 * M_PI / params->tide_period : 0.0;
        upload_phys_basis(m->basis);
        DRF_CUDA(cudaStreamCreateWithFlags(&m->own, cudaStreamNonBlocking));
        m->stream = m->own;
        // shared memory of the stage kernel: 9 column arrays + per-layer bases + 2D scalars
        const int ncn = mesh->nz * m->np3;
        m->smem = (size_t)(9 * ncn + mesh->nz * m->np2 + 2 * m->np2) * m->tsz + 16 + 2 * m->np2 * 8 + 16;
        int dev = 0, maxsm = 0;
        DRF_CUDA(cudaGetDevice(&dev));
        DRF_CUDA(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        DRF_CHECK(m->smem <= (size_t)maxsm, DRF_E_UNSUPPORTED,
                  "water column too tall for one CTA: nz*(N+1)^3 too large");
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            DRF_CUDA(cudaFuncSetAttribute(dg3d_stage_kernel<T, NP>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem));
        });
        m->q3.alloc((size_t)16 * m->n3 * m->tsz);
        DRF_CUDA(cudaMemset(m->q3.p, 0, m->q3.n));
        const int n2arrays = 25;
        m->d2.alloc((size_t)n2arrays * m->n2 + 8);
        DRF_CUDA(cudaMemset(m->d2.p, 0, m->d2.n * 8));
        double *p = m->d2.p;
        auto take = [&]() { double *r = p; p += m->n2; return r; };
        m->h = take(); m->f = take(); m->taux = take(); m->tauy = take(); m->eta = take();
        m->HU = take(); m->HV = take(); m->eta_avg = take(); m->esum = take(); m->Fx = take();
        m->Fy = take(); m->HUo = take(); m->HVo = take();
        for (int i = 0; i < 3; ++i) m->k1[i] = take();
        for (int i = 0; i < 3; ++i) m->us[i] = take();
        m->dHU3 = take(); m->dHV3 = take(); m->scratch2 = take();
        m->tdev = p;
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
        if (m->stream) cudaStreamSynchronize(m->stream);
        delete m;
    });
}

int drf_dg_set_stream(drf_dg *m, void *s) {
    return guard([&] {
        check_model(m);
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        m->drop_graphs();
        m->stream = s ? (cudaStream_t)s : m->own;
    });
}

int drf_dg_sync(drf_dg *m) {
    return guard([&] {
        check_model(m);
        DRF_CUDA(cudaStreamSynchronize(m->stream));
    });
}

int drf_dg_upload_state(drf_dg *m, const double *const *q4, const double *eta, double t) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(q4 && eta, DRF_E_INVALID, "null argument");
        for (int v = 0; v < 4; ++v)
            DRF_CHECK(q4[v] && all_finite(q4[v], m->n3), DRF_E_NONFINITE, "non-finite state value");
        DRF_CHECK(all_finite(eta, m->n2), DRF_E_NONFINITE, "non-finite eta");
        m->cur = 0;
        for (int v = 0; v < 4; ++v) {
            if (m->mixed) to_device<float>(m, m->q(0, v), q4[v]);
            else to_device<double>(m, m->q(0, v), q4[v]);
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
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        m->drop_graphs();
    });
}

int drf_dg_download_state(drf_dg *m, double *const *q4, double *eta, double *HU, double *HV,
                          double *eta_avg, double *t) {
    return guard([&] {
        check_model(m);
        DRF_CUDA(cudaStreamSynchronize(m->stream));
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

int drf_dg_compute_rhs(drf_dg *m, double *const *r4, double *omega, double *deta) {
    return guard([&] {
        check_model(m);
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
            baro_rhs_kernel<NP><<<blocks_for(m->n2), 256, 0, m->stream>>>(
                m->baro<NP>(m->eta, m->HU, m->HV, true, time - tcur), m->n2, m->k1[0], m->k1[1],
                m->k1[2]);
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
        DRF_CHECK(nsub >= 1, DRF_E_INVALID, "nsub must be >= 1");
        DRF_CHECK(dt > 0.0 && std::isfinite(dt), DRF_E_INVALID, "dt must be positive");
        DRF_CHECK(nsteps >= 0, DRF_E_INVALID, "nsteps must be >= 0");
        if (m->graph_nsub != nsub || m->graph_dt != dt) {
            m->drop_graphs();
            for (int in = 0; in < 2; ++in) {
                cudaGraph_t g = nullptr;
                DRF_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    m->with_types([&](auto tv, auto npc) {
                        using T = decltype(tv);
                        constexpr int NP = decltype(npc)::value;
                        m->template enqueue_step<T, NP>(in, dt, nsub);
                    });
                } catch (...) {
                    cudaStreamEndCapture(m->stream, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                DRF_CUDA(cudaStreamEndCapture(m->stream, &g));
                cudaError_t e = cudaGraphInstantiate(&m->graph[in], g, 0);
                cudaGraphDestroy(g);
                DRF_CUDA(e);
            }
            m->graph_nsub = nsub;
            m->graph_dt = dt;
        }
        for (int s = 0; s < nsteps; ++s) {
            DRF_CUDA(cudaGraphLaunch(m->graph[m->cur], m->stream));
            launch_counter().fetch_add(5 + 3 + 2 * (uint64_t)nsub);
            m->cur = 1 - m->cur;
        }
    });
}

int drf_dg_rk_step(drf_dg *m, int scheme, double dt, int nsteps) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(scheme >= 0 && scheme <= 5, DRF_E_INVALID, "unknown RK scheme");
        DRF_CHECK(dt > 0.0 && std::isfinite(dt), DRF_E_INVALID, "dt must be positive");
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
        const unsigned nb3 = blocks_for(m->n3), nb2 = blocks_for(m->n2);
        DevBuf<double> part((size_t)nb3 * 6 + (size_t)nb2 * 5);
        const double dx = m->mesh.Lx / m->mesh.nx, dy = m->mesh.Ly / m->mesh.ny;
        m->with_types([&](auto tv, auto npc) {
            using T = decltype(tv);
            constexpr int NP = decltype(npc)::value;
            const int c = m->cur;
            diag3d_kernel<T, NP><<<nb3, 256, 0, m->stream>>>(
                m->n3, m->G.nz, (const T *)m->q(c, 0), (const T *)m->q(c, 1), (const T *)m->q(c, 2),
                (const T *)m->q(c, 3), m->eta, m->h, 0.125 * dx * dy * m->G.dsig, part.p);
            DRF_LAUNCHED();
            diag2d_kernel<NP><<<nb2, 256, 0, m->stream>>>(m->n2, m->G.nz, m->eta, m->h,
                                                         0.25 * dx * dy, m->G.g, part.p + (size_t)nb3 * 6);
            DRF_LAUNCHED();
        });
        std::vector<double> hp(part.n);
        DRF_CUDA(cudaMemcpyAsync(hp.data(), part.p, part.n * 8, cudaMemcpyDeviceToHost, m->stream));
        DRF_CUDA(cudaStreamSynchronize(m->stream));
        double en = 0, heat = 0, salt = 0, um = 0, Tmax = -1e300, Tmin = 1e300;
        for (unsigned b = 0; b < nb3; ++b) {
            en += hp[b * 6]; heat += hp[b * 6 + 1]; salt += hp[b * 6 + 2];
            um = std::max(um, hp[b * 6 + 3]); Tmax = std::max(Tmax, hp[b * 6 + 4]);
            Tmin = std::min(Tmin, hp[b * 6 + 5]);
        }
        double mw = 0, mu = 0, pe = 0, emax = -1e300, emin = 1e300;
        const double *p2 = hp.data() + (size_t)nb3 * 6;
        for (unsigned b = 0; b < nb2; ++b) {
            mw += p2[b * 5]; mu += p2[b * 5 + 1]; pe += p2[b * 5 + 2];
            emax = std::max(emax, p2[b * 5 + 3]); emin = std::min(emin, p2[b * 5 + 4]);
        }
        const double vals[10] = {mw, mu, en + pe, heat, salt, um, emax, emin, Tmax, Tmin};
        std::memcpy(out10, vals, sizeof(vals));
        for (int i = 0; i < 10; ++i)
            DRF_CHECK(std::isfinite(vals[i]), DRF_E_NONFINITE, "non-finite diagnostic (model blew up)");
    });
}

int drf_dg_time_stage(drf_dg *m, int nrep, double *ms, double *alg_bytes, double *ndof) {
    return guard([&] {
        check_model(m);
        DRF_CHECK(nrep >= 1 && ms, DRF_E_INVALID, "bad arguments");
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
        // layer) reads and the FP64 column-increment read + write.
        const double s = (double)m->tsz;
        const double per_dof = s * (4.0 + 4.0 / m->np);
        if (alg_bytes) *alg_bytes = (double)m->n3 * 4.0 * per_dof + (double)m->n2 * 8.0 * (3 + 2 + 4);
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

int drf_dg_info(drf_dg *m, int64_t *n3d, int64_t *n2d, int *precision) {
    return guard([&] {
        check_model(m);
        if (n3d) *n3d = m->n3;
        if (n2d) *n2d = m->n2;
        if (precision) *precision = m->prm.precision;
    });
}

}  // extern "C"
