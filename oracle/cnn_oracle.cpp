// ORACLE — test infrastructure only (see oracle.hpp). CPU reference of the learned
// preconditioner network: 4 conv3x3 layers (zero padding 1), NHWC, channels padded as on the
// GPU (16 -> 32 -> 32 -> 32 -> 16), ReLU after layers 1-3. No counterpart in the reference
// ("parity unpinned"): this file is the judge for the GPU forward/backward kernels.
//
// Precision model mirrored from the GPU: weights and the activations that feed a convolution
// are rounded to bfloat16 (round-to-nearest-even), products accumulate in FP64 here (FP32 on
// the GPU), the last layer's output is kept unrounded. With round_bf16 = 0 everything is FP64
// (used for the finite-difference check of the backward pass).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

static double bf16r(double x) {
    float f = (float)x;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;  // inf/nan untouched
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    u &= 0xffff0000u;
    std::memcpy(&f, &u, 4);
    return f;
}

static const int CH[5] = {16, 32, 32, 32, 16};

// W layout per layer: [co][tap = dy*3+dx][ci]; bias [co]
struct CnnW {
    std::vector<double> W[4], b[4];
};

static void conv(const std::vector<double> &X, int H, int Wd, int ci_n, const std::vector<double> &Wt,
                 const std::vector<double> *bias, int co_n, std::vector<double> &Y) {
    Y.assign((size_t)H * Wd * co_n, 0.0);
    for (int h = 0; h < H; ++h)
        for (int w = 0; w < Wd; ++w)
            for (int co = 0; co < co_n; ++co) {
                double s = bias ? (*bias)[co] : 0.0;
                for (int t = 0; t < 9; ++t) {
                    const int hh = h + t / 3 - 1, ww = w + t % 3 - 1;
                    if (hh < 0 || hh >= H || ww < 0 || ww >= Wd) continue;
                    const double *xp = &X[((size_t)hh * Wd + ww) * ci_n];
                    const double *wp = &Wt[((size_t)co * 9 + t) * ci_n];
                    for (int ci = 0; ci < ci_n; ++ci) s += wp[ci] * xp[ci];
                }
                Y[((size_t)h * Wd + w) * co_n + co] = s;
            }
}

// forward; keeps the layer inputs A[l] (post-rounding) and pre-activations Z[l]
static void forward(const CnnW &P, const std::vector<double> &X0, int H, int Wd, bool rnd,
                    std::vector<double> A[5], std::vector<double> Z[4]) {
    A[0] = X0;
    if (rnd)
        for (auto &v : A[0]) v = bf16r(v);
    for (int l = 0; l < 4; ++l) {
        std::vector<double> Wl = P.W[l];
        if (rnd)
            for (auto &v : Wl) v = bf16r(v);
        conv(A[l], H, Wd, CH[l], Wl, &P.b[l], CH[l + 1], Z[l]);
        A[l + 1] = Z[l];
        if (l < 3)
            for (auto &v : A[l + 1]) {
                v = v > 0.0 ? v : 0.0;
                if (rnd) v = bf16r(v);
            }
    }
}

}  // namespace orc

using namespace orc;

extern "C" {

// params: 4 layers, W[l] size CH[l+1]*9*CH[l], b[l] size CH[l+1], packed in that order.
long orc_cnn_nparams() {
    long n = 0;
    for (int l = 0; l < 4; ++l) n += (long)CH[l + 1] * 9 * CH[l] + CH[l + 1];
    return n;
}

static void unpack(const double *p, CnnW &P) {
    for (int l = 0; l < 4; ++l) {
        const size_t nw = (size_t)CH[l + 1] * 9 * CH[l];
        P.W[l].assign(p, p + nw);
        p += nw;
        P.b[l].assign(p, p + CH[l + 1]);
        p += CH[l + 1];
    }
}

// out: H*W*16; returns loss = mean over (pixels x 9 real channels) of (out - target)^2 when
// target != null, and grads (packed like params) when grad != null.
double orc_cnn_forward_backward(const double *params, const double *X0, int H, int Wd,
                                const double *target, double *out, double *grad, int round_bf16) {
    CnnW P;
    unpack(params, P);
    std::vector<double> A[5], Z[4];
    std::vector<double> x0(X0, X0 + (size_t)H * Wd * CH[0]);
    forward(P, x0, H, Wd, round_bf16 != 0, A, Z);
    const size_t np = (size_t)H * Wd;
    if (out) std::memcpy(out, A[4].data(), sizeof(double) * np * CH[4]);
    if (!target) return 0.0;
    const double cnt = (double)np * 9.0;
    double loss = 0.0;
    std::vector<double> dA(np * CH[4], 0.0);
    for (size_t p = 0; p < np; ++p)
        for (int c = 0; c < 9; ++c) {
            const double d = A[4][p * CH[4] + c] - target[p * CH[4] + c];
            loss += d * d;
            dA[p * CH[4] + c] = 2.0 * d / cnt;
        }
    loss /= cnt;
    if (!grad) return loss;
    std::vector<double> dZ = dA;
    double *g = grad;
    std::vector<double> gl[4], gb[4];
    for (int l = 3; l >= 0; --l) {
        // dZ -> dW, db
        const int ci_n = CH[l], co_n = CH[l + 1];
        gl[l].assign((size_t)co_n * 9 * ci_n, 0.0);
        gb[l].assign(co_n, 0.0);
        for (int h = 0; h < H; ++h)
            for (int w = 0; w < Wd; ++w)
                for (int co = 0; co < co_n; ++co) {
                    const double dz = dZ[((size_t)h * Wd + w) * co_n + co];
                    if (dz == 0.0) continue;
                    gb[l][co] += dz;
                    for (int t = 0; t < 9; ++t) {
                        const int hh = h + t / 3 - 1, ww = w + t % 3 - 1;
                        if (hh < 0 || hh >= H || ww < 0 || ww >= Wd) continue;
                        const double *xp = &A[l][((size_t)hh * Wd + ww) * ci_n];
                        double *gp = &gl[l][((size_t)co * 9 + t) * ci_n];
                        for (int ci = 0; ci < ci_n; ++ci) gp[ci] += dz * xp[ci];
                    }
                }
        if (l == 0) break;
        // dA_l = conv^T(dZ, W) then ReLU mask -> dZ_{l-1}
        std::vector<double> Wl = P.W[l];
        if (round_bf16)
            for (auto &v : Wl) v = bf16r(v);
        std::vector<double> dX((size_t)np * ci_n, 0.0);
        std::vector<double> dz_r = dZ;
        if (round_bf16)
            for (auto &v : dz_r) v = bf16r(v);
        for (int h = 0; h < H; ++h)
            for (int w = 0; w < Wd; ++w)
                for (int co = 0; co < co_n; ++co) {
                    const double dz = dz_r[((size_t)h * Wd + w) * co_n + co];
                    if (dz == 0.0) continue;
                    for (int t = 0; t < 9; ++t) {
                        const int hh = h + t / 3 - 1, ww = w + t % 3 - 1;
                        if (hh < 0 || hh >= H || ww < 0 || ww >= Wd) continue;
                        double *dxp = &dX[((size_t)hh * Wd + ww) * ci_n];
                        const double *wp = &Wl[((size_t)co * 9 + t) * ci_n];
                        for (int ci = 0; ci < ci_n; ++ci) dxp[ci] += dz * wp[ci];
                    }
                }
        dZ.assign(np * ci_n, 0.0);
        for (size_t i = 0; i < np * ci_n; ++i) dZ[i] = Z[l - 1][i] > 0.0 ? dX[i] : 0.0;
    }
    for (int l = 0; l < 4; ++l) {
        std::memcpy(g, gl[l].data(), sizeof(double) * gl[l].size());
        g += gl[l].size();
        std::memcpy(g, gb[l].data(), sizeof(double) * gb[l].size());
        g += gb[l].size();
    }
    return loss;
}

}  // extern "C"
