// Device shallow-water numerical fluxes F*(U_L, U_R, n), U = (h, hu, hv), n = (nx, ny).
// Same formulas as the reference's flux set: Lax-Friedrichs with the factory's wave speed
// max(|u_n| + sqrt(g h)) (src/flux/numerical_flux.cpp:134-180,
// include/flux/numerical_flux.hpp:222), HLLC with Einfeldt speeds
// (include/flux/numerical_flux.hpp:272-390), Roe with Harten's entropy fix, delta = 0.1 c
// (src/flux/numerical_flux.cpp:13-131). Dry states are clamped to h = 1e-10 as there.
#pragma once
#include <cuda_runtime.h>

namespace drf {

__device__ __forceinline__ void sw_phys_flux(const double U[3], double nx, double ny, double g,
                                             double F[3]) {
    const double h = U[0] < 1e-10 ? 1e-10 : U[0];
    const double u = U[1] / h, v = U[2] / h, un = u * nx + v * ny;
    F[0] = h * un;
    F[1] = h * u * un + 0.5 * g * h * h * nx;
    F[2] = h * v * un + 0.5 * g * h * h * ny;
}

__device__ __forceinline__ void sw_flux_lf(const double UL[3], const double UR[3], double nx,
                                           double ny, double g, double F[3]) {
    const double hLc = UL[0] < 1e-10 ? 1e-10 : UL[0], hRc = UR[0] < 1e-10 ? 1e-10 : UR[0];
    const double uL = UL[1] / hLc, vL = UL[2] / hLc, uR = UR[1] / hRc, vR = UR[2] / hRc;
    // normal components of the Cartesian physical fluxes
    const double FxL[3] = {UL[1], UL[1] * uL + 0.5 * g * hLc * hLc, UL[1] * vL};
    const double FyL[3] = {UL[2], UL[2] * uL, UL[2] * vL + 0.5 * g * hLc * hLc};
    const double FxR[3] = {UR[1], UR[1] * uR + 0.5 * g * hRc * hRc, UR[1] * vR};
    const double FyR[3] = {UR[2], UR[2] * uR, UR[2] * vR + 0.5 * g * hRc * hRc};
    const double unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
    const double lam = fmax(fabs(unL) + sqrt(g * hLc), fabs(unR) + sqrt(g * hRc));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double FnL = FxL[i] * nx + FyL[i] * ny, FnR = FxR[i] * nx + FyR[i] * ny;
        F[i] = 0.5 * (FnL + FnR) - 0.5 * lam * (UR[i] - UL[i]);
    }
}

__device__ __forceinline__ void sw_flux_hllc(const double UL[3], const double UR[3], double nx,
                                             double ny, double g, double F[3]) {
    const double hL = UL[0] < 1e-10 ? 1e-10 : UL[0], hR = UR[0] < 1e-10 ? 1e-10 : UR[0];
    const double huL = UL[1], hvL = UL[2], huR = UR[1], hvR = UR[2];
    const double uL = huL / hL, vL = hvL / hL, uR = huR / hR, vR = hvR / hR;
    const double unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
    const double cL = sqrt(g * hL), cR = sqrt(g * hR);
    const double SL = fmin(unL - cL, unR - cR), SR = fmax(unL + cL, unR + cR);
    const double den = hL * (SL - unL) - hR * (SR - unR);
    double Ss;
    if (fabs(den) > 1e-10)
        Ss = (hL * unL * (SL - unL) - hR * unR * (SR - unR) + 0.5 * g * (hR * hR - hL * hL)) / den;
    else
        Ss = 0.5 * (unL + unR);
    const double FL[3] = {hL * unL, hL * uL * unL + 0.5 * g * hL * hL * nx,
                          hL * vL * unL + 0.5 * g * hL * hL * ny};
    const double FR[3] = {hR * unR, hR * uR * unR + 0.5 * g * hR * hR * nx,
                          hR * vR * unR + 0.5 * g * hR * hR * ny};
    if (SL >= 0) { F[0] = FL[0]; F[1] = FL[1]; F[2] = FL[2]; return; }
    if (SR <= 0) { F[0] = FR[0]; F[1] = FR[1]; F[2] = FR[2]; return; }
    if (Ss >= 0) {
        const double hs = hL * (SL - unL) / (SL - Ss);
        const double Us[3] = {hs, hs * (uL + (Ss - unL) * nx), hs * (vL + (Ss - unL) * ny)};
        const double Uv[3] = {hL, huL, hvL};
#pragma unroll
        for (int i = 0; i < 3; ++i) F[i] = FL[i] + SL * (Us[i] - Uv[i]);
    } else {
        const double hs = hR * (SR - unR) / (SR - Ss);
        const double Us[3] = {hs, hs * (uR + (Ss - unR) * nx), hs * (vR + (Ss - unR) * ny)};
        const double Uv[3] = {hR, huR, hvR};
#pragma unroll
        for (int i = 0; i < 3; ++i) F[i] = FR[i] + SR * (Us[i] - Uv[i]);
    }
}

__device__ __forceinline__ void sw_flux_roe(const double UL[3], const double UR[3], double nx,
                                            double ny, double g, double F[3]) {
    const double efix = 0.1;
    const double hL = UL[0] < 1e-10 ? 1e-10 : UL[0], hR = UR[0] < 1e-10 ? 1e-10 : UR[0];
    const double uL = UL[1] / hL, vL = UL[2] / hL, uR = UR[1] / hR, vR = UR[2] / hR;
    const double unL = uL * nx + vL * ny, utL = -uL * ny + vL * nx;
    const double unR = uR * nx + vR * ny, utR = -uR * ny + vR * nx;
    const double sL = sqrt(hL), sR = sqrt(hR), den = sL + sR;
    const double hr = 0.5 * (hL + hR), ur = (sL * uL + sR * uR) / den, vr = (sL * vL + sR * vR) / den;
    const double unr = ur * nx + vr * ny, cr = sqrt(g * hr);
    double l1 = unr - cr, l2 = unr, l3 = unr + cr;
    const double delta = efix * cr;
    if (fabs(l1) < delta) { l1 = (l1 * l1 + delta * delta) / (2.0 * delta); if (l1 < 0) l1 = -l1; }
    if (fabs(l3) < delta) { l3 = (l3 * l3 + delta * delta) / (2.0 * delta); if (l3 < 0) l3 = -l3; }
    const double dh = hR - hL, dun = unR - unL, dut = utR - utL;
    const double a1 = 0.5 * (dh - hr / cr * dun), a2 = hr * dut, a3 = 0.5 * (dh + hr / cr * dun);
    const double F1L = hL * unL, F2L = hL * uL * unL + 0.5 * g * hL * hL * nx,
                 F3L = hL * vL * unL + 0.5 * g * hL * hL * ny;
    const double F1R = hR * unR, F2R = hR * uR * unR + 0.5 * g * hR * hR * nx,
                 F3R = hR * vR * unR + 0.5 * g * hR * hR * ny;
    const double al1 = fabs(l1), al2 = fabs(l2), al3 = fabs(l3);
    const double r11 = a1, r12 = a1 * (ur - cr * nx), r13 = a1 * (vr - cr * ny);
    const double r21 = 0.0, r22 = a2 * (-ny), r23 = a2 * nx;
    const double r31 = a3, r32 = a3 * (ur + cr * nx), r33 = a3 * (vr + cr * ny);
    F[0] = 0.5 * (F1L + F1R) - 0.5 * (al1 * r11 + al2 * r21 + al3 * r31);
    F[1] = 0.5 * (F2L + F2R) - 0.5 * (al1 * r12 + al2 * r22 + al3 * r32);
    F[2] = 0.5 * (F3L + F3R) - 0.5 * (al1 * r13 + al2 * r23 + al3 * r33);
}

__device__ __forceinline__ void sw_flux(int kind, const double UL[3], const double UR[3],
                                        double nx, double ny, double g, double F[3]) {
    if (kind == DRF_FLUX_HLLC) sw_flux_hllc(UL, UR, nx, ny, g, F);
    else if (kind == DRF_FLUX_ROE) sw_flux_roe(UL, UR, nx, ny, g, F);
    else sw_flux_lf(UL, UR, nx, ny, g, F);
}

}  // namespace drf
