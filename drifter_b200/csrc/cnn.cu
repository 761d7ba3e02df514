// Learned preconditioner for the Bezier smoother's CG: a 4-layer conv3x3 network on 3x3
// "superpixels" of the control-point grid (space-to-depth exposes the element structure:
// superpixel (I, J) holds the 9 control points 3I..3I+2 x 3J..3J+2 as channels), BF16
// activations and weights with FP32 accumulation on the tensor cores, trained on the GPU by the
// backward kernels below with Adam. Two forms of the conv, bit-identical in their results:
//  * conv3x3_kernel (default): warp-level mma.sync m16n8k16 implicit GEMM (M = 16 pixels of a
//    row, N = output channels, K = 9 taps x input channels);
//  * conv3x3_tc_kernel (DRIFTER_B200_CNN_MMA=tcgen05): tcgen05 MMAs (M = 128 pixels) from
//    shared-memory descriptors into TMEM, TMA halo copies, warp-specialised.
//
// Channels (padded for the MMA shapes): 16 (9 used) -> 32 -> 32 -> 32 -> 16 (9 used); ReLU
// after layers 1-3. Layouts: activations NHWC [b][h][w][c]; weights [co][tap][ci] (tap = dy*3+dx).
#include <algorithm>
#include <cuda.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstdlib>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <random>
#include <vector>

#include "cnn.hpp"
#include "common.cuh"

namespace drf {
namespace {

using bf16 = __nv_bfloat16;
constexpr int CH[5] = {16, 32, 32, 32, 16};
constexpr int TH = 8, TW = 16;  // CTA tile: 8 rows x 16 pixels, one warp per row

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// 16-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}

// four 8x8 bf16 matrices from shared memory, one row address per lane
__device__ __forceinline__ void ldsm_x4(const bf16 *p, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"((uint32_t)__cvta_generic_to_shared(p)));
}

// Y = conv3x3(X, W) (+ bias) (+ ReLU); X, W bf16; Y bf16 (OUTF32 = false) or f32.
// Persistent over tiles of TH x TW pixels: a CTA stages the layer's weights once, then walks
// tiles (b, ty, tx) = blockIdx.x, blockIdx.x + gridDim.x, ... staging each tile's input halo.
// Shared memory: input halo (TH+2) x (TW+2) pixels with pixel stride CIN+8, and the weights
// with output-channel stride 9*CIN+8 (both paddings remove shared-memory bank conflicts of
// the fragment loads).
// conv tiles: TH rows x CTW pixels, one warp per row computing two 16-pixel MMA tiles (the B
// fragments of the weights are shared by both)
constexpr int CTW = 32;
template <int CIN, int COUT>
constexpr size_t conv_smem_bytes() {
    return (size_t)2 * (TH + 2) * (CTW + 2) * (CIN + 8) * 2 + (size_t)COUT * (9 * CIN + 8) * 2;
}

template <int CIN, int COUT, bool RELU, bool OUTF32>
__global__ void __launch_bounds__(256) conv3x3_kernel(int B, int H, int W, const bf16 *__restrict__ X,
                                                      const bf16 *__restrict__ Wt,
                                                      const float *__restrict__ bias, void *Yv,
                                                      const int *stop) {
    if (stop && *stop) return;  // a preconditioner apply queued after its solve converged
    constexpr int PS = CIN + 8, WS = 9 * CIN + 8, HP = TH + 2, WP = CTW + 2, C8 = CIN / 8;
    extern __shared__ __align__(16) unsigned char conv_smem[];
    bf16 *Xs0 = reinterpret_cast<bf16 *>(conv_smem);  // double-buffered input halo
    bf16 *Ws = Xs0 + 2 * HP * WP * PS;
    const int ntx = (W + CTW - 1) / CTW, nty = (H + TH - 1) / TH;
    const int64_t ntiles = (int64_t)ntx * nty * B;
    // asynchronous 16-byte copies of the tile's halo into buffer `buf` (zeros outside the image)
    auto stage_halo = [&](int64_t tile, int buf) {
        const int b = (int)(tile / ((int64_t)ntx * nty)), r2 = (int)(tile % ((int64_t)ntx * nty));
        const int h0 = (r2 / ntx) * TH, w0 = (r2 % ntx) * CTW;
        const bf16 *Xb = X + (size_t)b * H * W * CIN;
        bf16 *Xs = Xs0 + buf * HP * WP * PS;
        for (int i = threadIdx.x; i < HP * WP * C8; i += blockDim.x) {
            const int pix = i / C8, c8 = i % C8;
            const int hh = h0 - 1 + pix / WP, ww = w0 - 1 + pix % WP;
            const bool in = hh >= 0 && hh < H && ww >= 0 && ww < W;
            cp_async16(&Xs[pix * PS + 8 * c8], in ? Xb + ((size_t)hh * W + ww) * CIN + 8 * c8 : Xb, in ? 16 : 0);
        }
    };
    // the layer's weights, once per CTA, together with the first tile's halo
    for (int i = threadIdx.x; i < COUT * 9 * C8; i += blockDim.x) {
        const int co = i / (9 * C8), c8 = i % (9 * C8);
        cp_async16(&Ws[co * WS + 8 * c8], Wt + (size_t)co * 9 * CIN + 8 * c8, 16);
    }
    if (blockIdx.x < ntiles) stage_halo(blockIdx.x, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, g = lane >> 2, t = lane & 3;
    // fragments by ldmatrix.x4: lane l addresses row (l % 8) + 8 ((l / 8) % 2) of the A tile
    // (pixels of the strip) at channel offset 8 (l / 16), and output channel
    // 8 (j + l / 16) + l % 8 of the B tile at k offset 8 ((l / 8) % 2)
    const int arow = (lane & 7) + 8 * ((lane >> 3) & 1), acol = 8 * (lane >> 4);
    const int brow = (lane & 7) + 8 * (lane >> 4), bcol = 8 * ((lane >> 3) & 1);
    int buf = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, buf ^= 1) {
        const int b = (int)(tile / ((int64_t)ntx * nty)), r2 = (int)(tile % ((int64_t)ntx * nty));
        const int h0 = (r2 / ntx) * TH, w0 = (r2 % ntx) * CTW;
        // prefetch the next tile's halo into the other buffer (last read in the previous
        // iteration, behind its closing barrier)
        if (tile + gridDim.x < ntiles) stage_halo(tile + gridDim.x, buf ^ 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");  // all but the newest group
        __syncthreads();
        const bf16 *Xs = Xs0 + buf * HP * WP * PS;
        const int h = h0 + warp;
        float acc[2][COUT / 8][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int j = 0; j < COUT / 8; ++j) acc[mt][j][0] = acc[mt][j][1] = acc[mt][j][2] = acc[mt][j][3] = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3, dx = tap % 3;
            // pixel m of the strip reads halo pixel (warp + dy, m + dx)
            const bf16 *xa = &Xs[((warp + dy) * WP + (arow + dx)) * PS + acol];
#pragma unroll
            for (int kc = 0; kc < CIN; kc += 16) {
                uint32_t a[2][4];
                ldsm_x4(xa + kc, a[0][0], a[0][1], a[0][2], a[0][3]);
                ldsm_x4(xa + 16 * PS + kc, a[1][0], a[1][1], a[1][2], a[1][3]);
#pragma unroll
                for (int j = 0; j < COUT / 8; j += 2) {
                    uint32_t b0, b1, b2, b3;
                    ldsm_x4(&Ws[(8 * j + brow) * WS + tap * CIN + kc + bcol], b0, b1, b2, b3);
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        mma_bf16(acc[mt][j], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b0, b1);
                        mma_bf16(acc[mt][j + 1], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b2, b3);
                    }
                }
            }
        }
        if (h < H) {
#pragma unroll
            for (int j = 0; j < COUT / 8; ++j) {
                const int co = 8 * j + 2 * t;
                const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
#pragma unroll
                for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                    for (int half = 0; half < 2; ++half) {
                        const int w = w0 + 16 * mt + g + 8 * half;
                        if (w >= W) continue;
                        float v0 = acc[mt][j][2 * half] + b0, v1 = acc[mt][j][2 * half + 1] + b1;
                        if (RELU) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                        const size_t o = (((size_t)b * H + h) * W + w) * COUT + co;
                        if (OUTF32) {
                            float *Y = static_cast<float *>(Yv);
                            Y[o] = v0;
                            Y[o + 1] = v1;
                        } else {
                            bf16 *Y = static_cast<bf16 *>(Yv);
                            *reinterpret_cast<__nv_bfloat162 *>(&Y[o]) = __floats2bfloat162_rn(v0, v1);
                        }
                    }
            }
        }
        __syncthreads();  // every warp is done with this buffer before it is refilled
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// ------------------------------------------------------------ tcgen05 (5th-generation) conv
// The same conv3x3 as conv3x3_kernel as an implicit GEMM on Blackwell's tcgen05 tensor cores:
// M = 128 output pixels (a 16 x 8 tile), N = COUT, K = 9 taps x CIN in steps of 16. Operands
// are read by the tensor core from shared memory through matrix descriptors; the FP32
// accumulator lives in tensor memory (TMEM) and is read back with tcgen05.ld for the epilogue.
//
// Shared-memory operand layouts (K-major, no swizzle: "core matrices" of 8 rows x 16 bytes,
// the 8 rows 16 bytes apart):
//  * input halo, 18 x 10 pixels, planar by 8-channel chunk: [c8][pixel][8 channels]. For tap
//    (dy, dx) the A rows of output row r are halo pixels (r + dy) * 10 + dx + 0..7, consecutive,
//    so the 16 eight-row groups are 10 pixels (160 B) apart (the stride byte offset) and the
//    two channel chunks of one K step a plane apart (the leading byte offset);
//  * weights [tap][c8][co][8 channels]: eight-row groups of output channels 128 B apart, the
//    two chunks of a K step COUT x 16 B apart.
// Persistent CTAs of 4 warps walk tiles; per tile one thread issues the 9 x CIN/16 MMAs into
// one of two TMEM accumulators and commits them to an mbarrier, while all threads write the
// previous tile from the other accumulator. Halos rotate through three buffers: the next tile's
// halo is requested (cp.async) at the start of an iteration, a whole iteration before its MMAs.
constexpr int TCH = 16, TCW = 8;  // tile rows x pixels per row (M = 128)

__device__ __forceinline__ uint32_t sh_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading and stride byte offsets (all >> 4),
// descriptor version 1 (bits 46-47), base offset 0, no swizzle (layout type 0, bits 61-63)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28
template <int M, int N>
constexpr uint32_t umma_idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sh_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 16 consecutive 32-bit TMEM columns of this thread's lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
template <int CIN, int COUT>
struct TcConv {
    static constexpr int C8 = CIN / 8, HP = TCH + 2, WP = TCW + 2, PLANE = HP * WP;
    // one 8-channel plane of the halo as the tensor copy writes it ([HP][WP][8] bf16), its
    // stride rounded up to 128 B (the alignment of a tensor copy's destination)
    static constexpr uint32_t PLANE_TX = (uint32_t)PLANE * 16, PLANE_B = (PLANE_TX + 127) / 128 * 128;
    static constexpr uint32_t HALO_B = (uint32_t)C8 * PLANE_B;  // one halo stage
    static constexpr uint32_t W_B = 9u * C8 * COUT * 16;
    static constexpr int NS = 3;  // halo stages
    static constexpr int NA = 4;  // TMEM accumulators
    static constexpr uint32_t NCOL = NA * COUT <= 32 ? 32 : (NA * COUT <= 64 ? 64 : 128);
    // mbarriers: full[NS], empty[NS], acc_full[NA], acc_empty[NA]; then the TMEM address, an
    // abort flag and the bias
    static constexpr uint32_t BAR_B = 8u * (2 * NS + 2 * NA) + 16 + 4 * COUT;
    // at least 46 KB per CTA, so that at most 4 CTAs share an SM and their TMEM (4 x 128 of
    // 512 columns) is always free: a CTA never waits in tcgen05.alloc
    static constexpr size_t NEED = NS * (size_t)HALO_B + W_B + BAR_B;
    static constexpr size_t SMEM = NEED < 47104 ? 47104 : NEED;
    static constexpr int THREADS = 192;  // warp 0 producer, warp 1 MMA issuer, warps 2-5 epilogue
};

// bounded wait on an mbarrier phase that also gives up when another role set the abort flag
// (abort may be null: then only the bound ends it)
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort) {
    const uint32_t a = sh_u32(bar);
    for (long it = 0; it < (1L << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && abort && *abort) return false;
    }
    return false;
}
__device__ __forceinline__ void tc_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sh_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_bar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sh_u32(bar)), "r"(count) : "memory");
}

// Warp-specialised persistent CTA; every CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// (local index k):
//  * warp 0, one lane, stages halo k into stage k % NS (after the MMAs of tile k - NS released
//    it) with one tensor copy (TMA) per 8-channel plane; the copies complete full[stage] by
//    their byte count, and pixels outside the image arrive as zeros;
//  * warp 1, one lane, waits on full[stage] and on acc_empty[k % NA], issues the tile's MMAs
//    into accumulator k % NA and commits them to empty[stage] and acc_full[k % NA];
//  * warps 2-5 wait on acc_full, read the accumulator (warp w reads TMEM lanes 32 (w % 4) ..),
//    release it on acc_empty (one arrival per warp) and write the tile.
template <int CIN, int COUT, bool RELU, bool OUTF32>
__global__ void __launch_bounds__(192) conv3x3_tc_kernel(int B, int H, int W, const __grid_constant__ CUtensorMap xmap,
                                                         const bf16 *__restrict__ Wt,
                                                         const float *__restrict__ bias, void *Yv, int *err,
                                                         const int *stop) {
    // a preconditioner apply queued after its solve converged: every thread leaves before any
    // barrier, copy or tensor-memory allocation
    if (stop && *stop) return;
    using P = TcConv<CIN, COUT>;
    constexpr int C8 = P::C8, WP = P::WP, NS = P::NS, NA = P::NA;
    constexpr uint32_t IDESC = umma_idesc_bf16<128, COUT>();
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 32, "tcgen05 conv shape");
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char *halo = tc_smem;                   // [NS][C8][PLANE_B]
    unsigned char *wsm = tc_smem + NS * P::HALO_B;  // [9][C8][COUT][16 B]
    uint64_t *full = reinterpret_cast<uint64_t *>(wsm + P::W_B);
    uint64_t *empty = full + NS, *acc_full = empty + NS, *acc_empty = acc_full + NA;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_empty + NA);
    volatile int *abort = reinterpret_cast<volatile int *>(tmem_slot + 1);
    float *sbias = reinterpret_cast<float *>(tmem_slot + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntx = (W + TCW - 1) / TCW, nty = (H + TCH - 1) / TCH;
    const int64_t per_img = (int64_t)ntx * nty, ntiles = per_img * B;
    const int nloc = blockIdx.x < ntiles ? (int)((ntiles - 1 - blockIdx.x) / gridDim.x) + 1 : 0;

    // the layer's weights (and bias) once per CTA, by every thread, visible to the async proxy
    for (int i = threadIdx.x; i < COUT * 9 * C8; i += blockDim.x) {
        const int co = i / (9 * C8), r = i % (9 * C8), tap = r / C8, c8 = r % C8;
        cp_async16(wsm + ((size_t)(tap * C8 + c8) * COUT + co) * 16, Wt + (size_t)co * 9 * CIN + tap * CIN + 8 * c8,
                   16);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int i = threadIdx.x; i < COUT; i += blockDim.x) sbias[i] = bias ? bias[i] : 0.f;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) { tc_bar_init(&full[i], 1); tc_bar_init(&empty[i], 1); }
        for (int i = 0; i < NA; ++i) { tc_bar_init(&acc_full[i], 1); tc_bar_init(&acc_empty[i], 4); }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sh_u32(tmem_slot)),
                     "r"(P::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp == 0) {
        // ---- producer: halo k into stage k % NS by C8 tensor copies, one per channel plane
        if (lane == 0) {
            const uint64_t map = reinterpret_cast<uint64_t>(&xmap);
            for (int k = 0; k < nloc && ok; ++k) {
                const int s = k % NS;
                if (k >= NS) ok = tc_wait(&empty[s], (uint32_t)(((k / NS) - 1) & 1), abort);
                if (!ok) break;
                const int64_t tile = blockIdx.x + (int64_t)k * gridDim.x;
                const int b = (int)(tile / per_img), r2 = (int)(tile % per_img);
                const int h0 = (r2 / ntx) * TCH, w0 = (r2 % ntx) * TCW;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sh_u32(&full[s])),
                             "r"((uint32_t)(C8 * P::PLANE_TX))
                             : "memory");
#pragma unroll
                for (int c8 = 0; c8 < C8; ++c8)
                    asm volatile(
                        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(sh_u32(halo + s * P::HALO_B + c8 * P::PLANE_B)),
                        "l"(map), "r"(0), "r"(c8), "r"(w0 - 1), "r"(h0 - 1), "r"(b), "r"(sh_u32(&full[s]))
                        : "memory");
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint32_t wb = sh_u32(wsm);
            for (int k = 0; k < nloc && ok; ++k) {
                const int s = k % NS, a = k % NA;
                ok = tc_wait(&full[s], (uint32_t)((k / NS) & 1), abort);
                if (ok && k >= NA) ok = tc_wait(&acc_empty[a], (uint32_t)(((k / NA) - 1) & 1), abort);
                if (!ok) break;
                tc_fence_after();
                const uint32_t hb = sh_u32(halo + s * P::HALO_B), d = tmem + (uint32_t)(a * COUT);
#pragma unroll
                for (int tap = 0; tap < 9; ++tap) {
                    const int dy = tap / 3, dx = tap % 3;
#pragma unroll
                    for (int ks = 0; ks < C8 / 2; ++ks) {
                        const uint64_t ad = umma_desc(hb + (uint32_t)(2 * ks * P::PLANE_B + (dy * WP + dx) * 16),
                                                      P::PLANE_B, WP * 16);
                        const uint64_t bd = umma_desc(wb + (uint32_t)((tap * C8 + 2 * ks) * COUT * 16), COUT * 16, 128);
                        umma_bf16(d, ad, bd, IDESC, (tap | ks) != 0);
                    }
                }
                umma_commit(&empty[s]);
                umma_commit(&acc_full[a]);
            }
            // nothing may be in flight when TMEM is freed: the last commit's phase, waited for
            // even after an abort (bounded)
            if (nloc > 0) tc_wait(&acc_full[(nloc - 1) % NA], (uint32_t)(((nloc - 1) / NA) & 1), nullptr);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 = tile pixels m
        const int q = warp & 3, m = 32 * q + lane;
        for (int k = 0; k < nloc && ok; ++k) {
            const int a = k % NA;
            ok = tc_wait(&acc_full[a], (uint32_t)((k / NA) & 1), abort);
            if (__any_sync(0xffffffffu, !ok)) { ok = false; break; }
            tc_fence_after();
            float f[COUT];
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * COUT + c0), v);
                tmem_ld_wait();
#pragma unroll
                for (int j = 0; j < 16; ++j) f[c0 + j] = __uint_as_float(v[j]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) tc_arrive(&acc_empty[a]);  // the accumulator may be overwritten
            const int64_t tile = blockIdx.x + (int64_t)k * gridDim.x;
            const int b = (int)(tile / per_img), r2 = (int)(tile % per_img);
            const int h = (r2 / ntx) * TCH + m / TCW, w = (r2 % ntx) * TCW + m % TCW;
            if (h >= H || w >= W) continue;
            const size_t o = (((size_t)b * H + h) * W + w) * COUT;
#pragma unroll
            for (int j = 0; j < COUT; ++j) {
                f[j] += sbias[j];
                if (RELU) f[j] = fmaxf(f[j], 0.f);
            }
            if (OUTF32) {
                float4 *Y = reinterpret_cast<float4 *>(static_cast<float *>(Yv) + o);
#pragma unroll
                for (int j = 0; j < COUT / 4; ++j) Y[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
            } else {
                uint32_t p[COUT / 2];
#pragma unroll
                for (int j = 0; j < COUT / 2; ++j) {
                    __nv_bfloat162 t2 = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
                    p[j] = *reinterpret_cast<uint32_t *>(&t2);
                }
                uint4 *Y = reinterpret_cast<uint4 *>(static_cast<bf16 *>(Yv) + o);
#pragma unroll
                for (int j = 0; j < COUT / 8; ++j) Y[j] = make_uint4(p[4 * j], p[4 * j + 1], p[4 * j + 2], p[4 * j + 3]);
            }
        }
    }
    if (!ok) {
        *abort = 1;
        atomicExch(err, DRF_E_TIMEOUT);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P::NCOL) : "memory");
    }
}

// dW partials of one layer for one CTA tile: dW[co][tap][ci] += dZ[p][co] * A[p + shift][ci],
// db[co] += dZ[p][co]; FP32, one partial row per tile (reduced in a fixed order afterwards).
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) dw_partial_kernel(int H, int W, const float *__restrict__ dZ,
                                                         const bf16 *__restrict__ A, float *part) {
    constexpr int HP = TH + 2, WP = TW + 2, NW = COUT * 9 * CIN + COUT;
    __shared__ float dzs[TH * TW * COUT];
    __shared__ float as[HP * WP * CIN];
    const int b = blockIdx.z;
    const int h0 = blockIdx.y * TH, w0 = blockIdx.x * TW;
    for (int i = threadIdx.x; i < TH * TW * COUT; i += blockDim.x) {
        const int p = i / COUT, co = i % COUT;
        const int hh = h0 + p / TW, ww = w0 + p % TW;
        dzs[i] = (hh < H && ww < W) ? dZ[(((size_t)b * H + hh) * W + ww) * COUT + co] : 0.f;
    }
    for (int i = threadIdx.x; i < HP * WP * CIN; i += blockDim.x) {
        const int pix = i / CIN, ci = i % CIN;
        const int hh = h0 - 1 + pix / WP, ww = w0 - 1 + pix % WP;
        as[i] = (hh >= 0 && hh < H && ww >= 0 && ww < W)
                    ? __bfloat162float(A[(((size_t)b * H + hh) * W + ww) * CIN + ci])
                    : 0.f;
    }
    __syncthreads();
    const size_t tile = ((size_t)b * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    for (int e = threadIdx.x; e < NW; e += blockDim.x) {
        float s = 0.f;
        if (e < COUT * 9 * CIN) {
            const int co = e / (9 * CIN), r = e % (9 * CIN), tap = r / CIN, ci = r % CIN;
            const int dy = tap / 3, dx = tap % 3;
            for (int p = 0; p < TH * TW; ++p) {
                const int ph = p / TW, pw = p % TW;
                s += dzs[p * COUT + co] * as[((ph + dy) * WP + (pw + dx)) * CIN + ci];
            }
        } else {
            const int co = e - COUT * 9 * CIN;
            for (int p = 0; p < TH * TW; ++p) s += dzs[p * COUT + co];
        }
        part[tile * NW + e] = s;
    }
}

__global__ void reduce_cols_kernel(int nrows, int ncols, const float *part, float *out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ncols) return;
    float s = 0.f;
    for (int r = 0; r < nrows; ++r) s += part[(size_t)r * ncols + e];
    out[e] = s;
}

// dOut = 2 (out - target) / count on the 9 used channels; per-block loss partials
__global__ void loss_grad_kernel(int64_t npix, const float *out, const float *tgt, float *dout,
                                 float inv_cnt, double *lpart) {
    __shared__ double red[256];
    double l = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix * 16;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % 16);
        float d = 0.f;
        if (c < 9) {
            d = out[i] - tgt[i];
            l += (double)d * d;
        }
        dout[i] = 2.f * d * inv_cnt;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}

// dZ_{l-1} = dX * (Z_{l-1} > 0); keeps an FP32 copy (for dW) and a BF16 copy (next conv input)
__global__ void relu_back_kernel(int64_t n, const float *dX, const bf16 *Apost, float *dZ,
                                 bf16 *dZb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    // A_post = relu(Z) rounded; Z > 0 <=> A_post > 0 except values that rounded to 0
    const float v = __bfloat162float(Apost[i]) > 0.f ? dX[i] : 0.f;
    dZ[i] = v;
    dZb[i] = __float2bfloat16_rn(v);
}

__global__ void f32_to_bf16_kernel(int64_t n, const float *a, bf16 *b) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

// bf16 weights of a layer and the flipped/transposed copy used by the input-gradient conv
__global__ void cast_weights_kernel(int cin, int cout, const float *Wm, bf16 *W, bf16 *Wflip) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= cout * 9 * cin) return;
    const int co = e / (9 * cin), r = e % (9 * cin), tap = r / cin, ci = r % cin;
    const bf16 v = __float2bfloat16_rn(Wm[e]);
    W[e] = v;
    if (Wflip) Wflip[(ci * 9 + (8 - tap)) * cout + co] = v;
}

__global__ void adam_kernel(int n, float *w, float *m, float *v, const float *g, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// random crops of the device dataset into a batch (X bf16, target f32)
__global__ void crop_kernel(int B, int ch, int cw, int H, int W, const int *sel, const float *Xd,
                            const float *Td, bf16 *Xb, float *Tb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * ch * cw * 16) return;
    const int c = (int)(i % 16);
    const int64_t p = i / 16;
    const int w = (int)(p % cw), h = (int)((p / cw) % ch), b = (int)(p / ((int64_t)cw * ch));
    const int k = sel[3 * b], oy = sel[3 * b + 1], ox = sel[3 * b + 2];
    const int64_t s = ((((int64_t)k * H) + oy + h) * W + ox + w) * 16 + c;
    Xb[i] = __float2bfloat16_rn(Xd[s]);
    Tb[i] = Td[s];
}

// superpixel packing of a control-point field (nd x nd, nd = 3n + 1) scaled by 1/rms
__global__ void pack_kernel(int n, const double *r, const double *rr_ptr, double inv_len, bf16 *X,
                            const int *stop) {
    if (stop && *stop) return;
    // one thread per superpixel (I, J): its 9 control points 3I..3I+2 x 3J..3J+2 (three runs of
    // three consecutive values) become channels 0..8, channels 9..15 are zero; one 32-byte store
    const int S = n + 1, nd = 3 * n + 1;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S * S) return;
    const int I = p % S, J = p / S;
    const double rr = *rr_ptr;
    const double sc = rr > 0 ? 1.0 / sqrt(rr * inv_len) : 0.0;
    __align__(16) bf16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16_rn(0.f);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const int gj = 3 * J + b;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int gi = 3 * I + a;
            if (gi < nd && gj < nd) v[a + 3 * b] = __float2bfloat16_rn((float)(r[gi + (int64_t)nd * gj] * sc));
        }
    }
    uint4 *dst = reinterpret_cast<uint4 *>(X + (size_t)p * 16);
    dst[0] = reinterpret_cast<const uint4 *>(v)[0];
    dst[1] = reinterpret_cast<const uint4 *>(v)[1];
}

// z (+)= rms(r) out_scale Y on the control points (add = 1 adds to a base already in z; with
// jr, jd non-null the base is the Jacobi step jr / jd instead); one thread per superpixel
// writes its (up to) 9 control points
__global__ void __launch_bounds__(256) unpack_kernel(int n, const float *Y, const double *rr_ptr, double inv_len,
                                                     double out_scale, double *z, int add, const int *stop,
                                                     const double *jr, const double *jd, const double *dq,
                                                     double *part) {
    // with part non-null, also the block partials of z.jr (part[block]) and z.dq
    // (part[gridDim.x + block]): the dot products of flexible CG, in the pass that forms z
    __shared__ double red[2][8];
    if (stop && *stop) return;
    const int S = n + 1, nd = 3 * n + 1;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double s1 = 0.0, s2 = 0.0;
    if (p < S * S) {
        const int I = p % S, J = p / S;
        const double rr = *rr_ptr;
        const double sc = sqrt(rr * inv_len);
        const float4 *src = reinterpret_cast<const float4 *>(Y + (size_t)p * 16);
        const float4 y0 = src[0], y1 = src[1], y2 = src[2];
        const float y[9] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w, y2.x};
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int gj = 3 * J + b;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int gi = 3 * I + a;
                if (gi < nd && gj < nd) {
                    const size_t t = gi + (size_t)nd * gj;
                    const double v = (double)y[a + 3 * b] * sc * out_scale;
                    const double zn = jr ? jr[t] / jd[t] + v : (add ? z[t] + v : v);
                    z[t] = zn;
                    if (part) {
                        s1 += zn * jr[t];
                        s2 += zn * dq[t];
                    }
                }
            }
        }
    }
    if (!part) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = s1;
        red[1][threadIdx.x >> 5] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        part[blockIdx.x] = a;
        part[gridDim.x + blockIdx.x] = b;
    }
}

inline unsigned nb(int64_t n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

// the tcgen05 conv: persistent, as many CTAs as are resident (at most one per tile)
// Tensor map of an NHWC bf16 activation tensor for the conv's halo copies: dimensions
// (8 channels, CIN/8 channel chunks, W, H, B), box (8, 1, TCW + 2, TCH + 2, 1): one copy brings
// one 8-channel plane of a tile's halo; coordinates outside the image read zeros.
template <int CIN>
CUtensorMap conv_halo_map(const bf16 *X, int B, int H, int W) {
    CUtensorMap m;
    const cuuint64_t dims[5] = {8, (cuuint64_t)(CIN / 8), (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[4] = {16, (cuuint64_t)CIN * 2, (cuuint64_t)W * CIN * 2, (cuuint64_t)H * W * CIN * 2};
    const cuuint32_t box[5] = {8, 1, TCW + 2, TCH + 2, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    // the driver's encoder, looked up through the runtime (the library does not link the driver)
    using Encode = decltype(&cuTensorMapEncodeTiled);
    static Encode encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        DRF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        DRF_CHECK(fn && q == cudaDriverEntryPointSuccess, DRF_E_CUDA, "cuTensorMapEncodeTiled not available");
        return reinterpret_cast<Encode>(fn);
    }();
    const CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(X), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    DRF_CHECK(r == CUDA_SUCCESS, DRF_E_CUDA, "cuTensorMapEncodeTiled failed for the conv input");
    return m;
}

template <int CIN, int COUT, bool RELU, bool OUTF32>
void conv_tc(cudaStream_t s, int B, int H, int W, const bf16 *X, const bf16 *Wt, const float *bias, void *Y,
             int *err, const int *stop) {
    constexpr size_t smem = TcConv<CIN, COUT>::SMEM;
    static int resident = 0;
    if (!resident) {
        int dev = 0, nsm = 0, smpm = 0, rsv = 0;
        DRF_CUDA(cudaGetDevice(&dev));
        DRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        DRF_CUDA(cudaDeviceGetAttribute(&smpm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        DRF_CUDA(cudaDeviceGetAttribute(&rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
        DRF_CUDA(cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT, RELU, OUTF32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // CTAs per SM: 2 (the fastest of 1-4 measured at C4), fewer if shared memory or the 512
        // TMEM columns allow fewer; DRIFTER_B200_CONV_CTAS_PER_SM sets it within those limits
        int per = std::min(smpm / (int)(smem + rsv), 512 / (int)TcConv<CIN, COUT>::NCOL);
        const int cap = per;
        per = std::max(1, std::min(per, 2));
        if (const char *e = std::getenv("DRIFTER_B200_CONV_CTAS_PER_SM"))
            per = std::max(1, std::min(cap, std::atoi(e)));
        resident = nsm * per;
    }
    const int64_t ntiles = (int64_t)((W + TCW - 1) / TCW) * ((H + TCH - 1) / TCH) * B;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, resident);
    DRF_CHECK(reinterpret_cast<uintptr_t>(X) % 16 == 0, DRF_E_INVALID, "conv input not 16-byte aligned");
    const CUtensorMap xmap = conv_halo_map<CIN>(X, B, H, W);
    conv3x3_tc_kernel<CIN, COUT, RELU, OUTF32><<<grid, TcConv<CIN, COUT>::THREADS, smem, s>>>(B, H, W, xmap, Wt, bias,
                                                                                          Y, err, stop);
    DRF_LAUNCHED();
}

// Conv form per (layer, batch, height, width): 0 the warp-level mma.sync kernel, 1 the tcgen05
// kernel. Both compute bit-identical outputs. DRIFTER_B200_CNN_MMA=tcgen05 or =mma_sync forces
// a form; otherwise the autotuner (cnn_tune) times both at the preconditioner's size and keeps
// the faster, and untuned shapes (the training batches) take mma.sync.
inline int forced_conv_form() {
    static const int v = [] {
        const char *e = std::getenv("DRIFTER_B200_CNN_MMA");
        if (e && std::strcmp(e, "tcgen05") == 0) return 1;
        if (e && std::strcmp(e, "mma_sync") == 0) return 0;
        return -1;
    }();
    return v;
}
std::mutex &conv_form_mu() {
    static std::mutex m;
    return m;
}
std::map<std::array<int, 4>, int> &conv_form_table() {
    static std::map<std::array<int, 4>, int> t;
    return t;
}
int conv_form(int l, int B, int H, int W) {
    const int f = forced_conv_form();
    if (f >= 0) return f;
    std::lock_guard<std::mutex> lk(conv_form_mu());
    const auto it = conv_form_table().find({l, B, H, W});
    return it == conv_form_table().end() ? 0 : it->second;
}

template <int CIN, int COUT, bool RELU, bool OUTF32>
void conv(cudaStream_t s, int B, int H, int W, const bf16 *X, const bf16 *Wt, const float *bias,
          void *Y, int *err, int form, const int *stop = nullptr) {
    if (form == 1) {
        conv_tc<CIN, COUT, RELU, OUTF32>(s, B, H, W, X, Wt, bias, Y, err, stop);
        return;
    }
    // persistent grid: as many CTAs as are resident at once (the weights are staged once each)
    constexpr size_t smem = conv_smem_bytes<CIN, COUT>();
    static int resident = 0;
    if (!resident) {
        int dev = 0, nsm = 0, per = 0;
        DRF_CUDA(cudaGetDevice(&dev));
        DRF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        DRF_CUDA(cudaFuncSetAttribute(conv3x3_kernel<CIN, COUT, RELU, OUTF32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        DRF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, conv3x3_kernel<CIN, COUT, RELU, OUTF32>, 256, smem));
        resident = nsm * (per > 0 ? per : 1);
    }
    const int64_t ntiles = (int64_t)((W + CTW - 1) / CTW) * ((H + TH - 1) / TH) * B;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, resident);
    conv3x3_kernel<CIN, COUT, RELU, OUTF32><<<grid, 256, smem, s>>>(B, H, W, X, Wt, bias, Y, stop);
    DRF_LAUNCHED();
}

// form -1: the tuned (or forced, or default) form of this layer and shape; stop (device, may be
// null): the launch returns at once when it is set
void conv_layer(cudaStream_t s, int l, int B, int H, int W, const bf16 *X, const bf16 *Wt,
                const float *bias, void *Y, int *err, int form = -1, const int *stop = nullptr) {
    if (form < 0) form = conv_form(l, B, H, W);
    switch (l) {
    case 0: conv<16, 32, true, false>(s, B, H, W, X, Wt, bias, Y, err, form, stop); break;
    case 1: conv<32, 32, true, false>(s, B, H, W, X, Wt, bias, Y, err, form, stop); break;
    case 2: conv<32, 32, true, false>(s, B, H, W, X, Wt, bias, Y, err, form, stop); break;
    default: conv<32, 16, false, true>(s, B, H, W, X, Wt, bias, Y, err, form, stop); break;
    }
}

// input-gradient conv of layer l (l = 1..3): dX (CIN_l channels, f32) = conv(dZ_l, Wflip_l)
void conv_back(cudaStream_t s, int l, int B, int H, int W, const bf16 *dZb, const bf16 *Wf, float *dX,
               int *err) {
    switch (l) {
    case 3: conv<16, 32, false, true>(s, B, H, W, dZb, Wf, nullptr, dX, err, forced_conv_form() == 1); break;
    default: conv<32, 32, false, true>(s, B, H, W, dZb, Wf, nullptr, dX, err, forced_conv_form() == 1); break;
    }
}

void dw_layer(cudaStream_t s, int l, int B, int H, int W, const float *dZ, const bf16 *A, float *part) {
    dim3 grid((W + TW - 1) / TW, (H + TH - 1) / TH, B);
    switch (l) {
    case 0: dw_partial_kernel<16, 32><<<grid, 256, 0, s>>>(H, W, dZ, A, part); break;
    case 3: dw_partial_kernel<32, 16><<<grid, 256, 0, s>>>(H, W, dZ, A, part); break;
    default: dw_partial_kernel<32, 32><<<grid, 256, 0, s>>>(H, W, dZ, A, part); break;
    }
    DRF_LAUNCHED();
}

size_t layer_w(int l) { return (size_t)CH[l + 1] * 9 * CH[l]; }

}  // namespace

// ------------------------------------------------------------------------------ network object
struct CnnNet {
    cudaStream_t stream = nullptr, own = nullptr;
    // FP32 masters (packed like the oracle: per layer W then b), Adam moments, gradients
    DevBuf<float> wm, am, av, grad;
    DevBuf<int> status;  // device status word (DRF_E_TIMEOUT when a bounded wait gave up)
    DevBuf<bf16> wb, wflip;
    size_t off_w[4], off_b[4], off_wb[4], nparam = 0, nwb = 0;
    int64_t adam_t = 0;
    // activation buffers (sized on demand)
    int64_t cap_pix = 0;
    DevBuf<bf16> act[4], dzb;
    DevBuf<float> out, dout, dx, dz;
    DevBuf<float> part;
    DevBuf<double> lpart;
    // dataset
    DevBuf<float> dsX, dsT;
    DevBuf<int> sel;
    DevBuf<bf16> bx;
    DevBuf<float> bt;
    int ds_n = 0, ds_h = 0, ds_w = 0;

    CnnNet() {
        size_t o = 0, ob = 0;
        for (int l = 0; l < 4; ++l) {
            off_w[l] = o; o += layer_w(l);
            off_b[l] = o; o += CH[l + 1];
            off_wb[l] = ob; ob += layer_w(l);
        }
        nparam = o;
        nwb = ob;
        for (auto *b : {&wm, &am, &av, &grad}) b->alloc(nparam);
        wb.alloc(nwb);
        wflip.alloc(nwb);
        status.alloc(1);
        DRF_CUDA(cudaMemset(status.p, 0, sizeof(int)));
        DRF_CUDA(cudaMemset(am.p, 0, nparam * 4));
        DRF_CUDA(cudaMemset(av.p, 0, nparam * 4));
        DRF_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        stream = own;
    }
    ~CnnNet() {
        if (own) cudaStreamDestroy(own);
    }
    void cast() {
        for (int l = 0; l < 4; ++l) {
            cast_weights_kernel<<<nb(layer_w(l)), 256, 0, stream>>>(CH[l], CH[l + 1], wm.p + off_w[l],
                                                                    wb.p + off_wb[l], wflip.p + off_wb[l]);
            DRF_LAUNCHED();
        }
    }
    void ensure(int64_t pix) {
        if (pix <= cap_pix) return;
        for (int l = 0; l < 4; ++l) act[l].alloc(pix * CH[l]);
        dzb.alloc(pix * 32);
        out.alloc(pix * 16);
        dout.alloc(pix * 16);
        dx.alloc(pix * 32);
        dz.alloc(pix * 32);
        lpart.alloc(1024);
        cap_pix = pix;
    }
    // forward from act[0]; output f32 in `out` (every launch skipped when *stop is set)
    void forward(int B, int H, int W, const int *stop = nullptr) {
        for (int l = 0; l < 3; ++l)
            conv_layer(stream, l, B, H, W, act[l].p, wb.p + off_wb[l], wm.p + off_b[l], act[l + 1].p, status.p,
                       -1, stop);
        conv_layer(stream, 3, B, H, W, act[3].p, wb.p + off_wb[3], wm.p + off_b[3], out.p, status.p, -1, stop);
    }
    // backward of the mean-square loss against tgt; fills grad; returns device loss partials
    void backward(int B, int H, int W, const float *tgt) {
        const int64_t pix = (int64_t)B * H * W;
        loss_grad_kernel<<<1024, 256, 0, stream>>>(pix, out.p, tgt, dout.p, 1.f / (float)(pix * 9), lpart.p);
        DRF_LAUNCHED();
        const int tiles = ((W + TW - 1) / TW) * ((H + TH - 1) / TH) * B;
        const float *dZ = dout.p;
        for (int l = 3; l >= 0; --l) {
            const size_t nw = layer_w(l) + CH[l + 1];
            if (part.n < (size_t)tiles * nw) part.alloc((size_t)tiles * nw);
            dw_layer(stream, l, B, H, W, dZ, act[l].p, part.p);
            reduce_cols_kernel<<<nb(nw), 256, 0, stream>>>(tiles, (int)nw, part.p, grad.p + off_w[l]);
            DRF_LAUNCHED();
            if (l == 0) break;
            // dZ_l in bf16 for the input-gradient conv
            f32_to_bf16_kernel<<<nb(pix * CH[l + 1]), 256, 0, stream>>>(pix * CH[l + 1], dZ, dzb.p);
            DRF_LAUNCHED();
            conv_back(stream, l, B, H, W, dzb.p, wflip.p + off_wb[l], dx.p, status.p);
            // dZ_{l-1} = dX * relu'(Z_{l-1}) into dz (the previous dZ is no longer read)
            relu_back_kernel<<<nb(pix * CH[l]), 256, 0, stream>>>(pix * CH[l], dx.p, act[l].p, dz.p, dzb.p);
            DRF_LAUNCHED();
            dZ = dz.p;
        }
    }
    double loss_host() {
        std::vector<double> lp(1024);
        DRF_CUDA(cudaMemcpyAsync(lp.data(), lpart.p, 1024 * 8, cudaMemcpyDeviceToHost, stream));
        DRF_CUDA(cudaStreamSynchronize(stream));
        double s = 0.0;
        for (double v : lp) s += v;
        return s;
    }
};

// packs r (control points) and runs the network; z (+)= rms(r) * out_scale * net(r / rms(r))
int cnn_precondition(CnnNet *net, cudaStream_t s, int n, const double *r, const double *rr_dev,
                     double out_scale, double *z, int add, const int *stop, const double *jac_diag,
                     const double *dq, double *part) {
    const int S = n + 1;
    const int64_t pix = (int64_t)S * S, nd = 3 * n + 1;
    cudaStream_t keep = net->stream;
    net->stream = s;
    net->ensure(pix);
    // after convergence (stop set) every launch of the apply returns at once
    pack_kernel<<<nb(pix), 256, 0, s>>>(n, r, rr_dev, 1.0 / (double)(nd * nd), net->act[0].p, stop);
    DRF_LAUNCHED();
    net->forward(1, S, S, stop);
    DRF_CHECK(!part || jac_diag, DRF_E_INVALID, "the fused dot products need the Jacobi base (r)");
    unpack_kernel<<<nb(pix), 256, 0, s>>>(n, net->out.p, rr_dev, 1.0 / (double)(nd * nd), out_scale,
                                              z, add, stop, jac_diag ? r : nullptr, jac_diag, dq, part);
    DRF_LAUNCHED();
    net->stream = keep;
    return (int)nb(pix);
}

void cnn_prepare(CnnNet *net, int n) { net->ensure((int64_t)(n + 1) * (n + 1)); }

// Autotuner of the conv form at the preconditioner's size ((n + 1)^2 superpixels, batch 1):
// every layer is timed in both forms on the net's stream (two warm-up launches, then ten
// between CUDA events) and the faster kept for the life of the process. Must run outside any
// stream capture. DRIFTER_B200_TUNE=0 (or a forced form) skips it.
void cnn_tune(CnnNet *net, int n, double ms_out[4][2], int form_out[4]) {
    const int S = n + 1;
    for (int l = 0; l < 4; ++l) {
        form_out[l] = conv_form(l, 1, S, S);
        ms_out[l][0] = ms_out[l][1] = 0.0;
    }
    const char *te = std::getenv("DRIFTER_B200_TUNE");
    if ((te && te[0] == '0') || forced_conv_form() >= 0) return;
    net->ensure((int64_t)S * S);
    cudaStream_t st = net->stream;
    cudaEvent_t e0, e1;
    DRF_CUDA(cudaEventCreate(&e0));
    DRF_CUDA(cudaEventCreate(&e1));
    for (int l = 0; l < 4; ++l) {
        const bf16 *X = net->act[l].p;
        void *Y = l < 3 ? (void *)net->act[l + 1].p : (void *)net->out.p;
        for (int form = 0; form < 2; ++form) {
            for (int w = 0; w < 2; ++w)
                conv_layer(st, l, 1, S, S, X, net->wb.p + net->off_wb[l], net->wm.p + net->off_b[l], Y,
                           net->status.p, form);
            DRF_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < 10; ++r)
                conv_layer(st, l, 1, S, S, X, net->wb.p + net->off_wb[l], net->wm.p + net->off_b[l], Y,
                           net->status.p, form);
            DRF_CUDA(cudaEventRecord(e1, st));
            DRF_CUDA(cudaEventSynchronize(e1));
            float t = 0.f;
            DRF_CUDA(cudaEventElapsedTime(&t, e0, e1));
            ms_out[l][form] = t / 10.0;
        }
        form_out[l] = ms_out[l][1] < ms_out[l][0] ? 1 : 0;
        std::lock_guard<std::mutex> lk(conv_form_mu());
        conv_form_table()[{l, 1, S, S}] = form_out[l];
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cnn_check(net, st);
}

void cnn_check(CnnNet *net, cudaStream_t s) {
    int st = 0;
    DRF_CUDA(cudaMemcpyAsync(&st, net->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    DRF_CUDA(cudaStreamSynchronize(s));
    if (st != 0) {
        DRF_CUDA(cudaMemsetAsync(net->status.p, 0, sizeof(int), s));
        throw Error(st, "a device-side wait of the network gave up (status " + std::to_string(st) + ")");
    }
}

}  // namespace drf

using namespace drf;

struct drf_cnn {
    std::unique_ptr<CnnNet> net;
};

extern "C" {

int64_t drf_cnn_nparams(void) {
    int64_t n = 0;
    for (int l = 0; l < 4; ++l) n += (int64_t)CH[l + 1] * 9 * CH[l] + CH[l + 1];
    return n;
}

int drf_cnn_create(uint64_t seed, drf_cnn **out) {
    return guard([&] {
        DRF_CHECK(out, DRF_E_INVALID, "null argument");
        auto h = std::make_unique<drf_cnn>();
        h->net = std::make_unique<CnnNet>();
        // He-normal initialisation of the used input channels, zero biases
        std::mt19937_64 rng(seed);
        std::vector<float> w(h->net->nparam, 0.f);
        for (int l = 0; l < 4; ++l) {
            const int cin_used = l == 0 ? 9 : CH[l], cout_used = l == 3 ? 9 : CH[l + 1];
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (9.f * cin_used)));
            for (int co = 0; co < cout_used; ++co)
                for (int tap = 0; tap < 9; ++tap)
                    for (int ci = 0; ci < cin_used; ++ci)
                        w[h->net->off_w[l] + ((size_t)co * 9 + tap) * CH[l] + ci] = nd(rng) * (l == 3 ? 0.1f : 1.f);
        }
        DRF_CUDA(cudaMemcpy(h->net->wm.p, w.data(), w.size() * 4, cudaMemcpyHostToDevice));
        h->net->cast();
        DRF_CUDA(cudaStreamSynchronize(h->net->stream));
        *out = h.release();
    });
}

int drf_cnn_destroy(drf_cnn *h) {
    return guard([&] {
        if (!h) return;
        cudaStreamSynchronize(h->net->stream);
        delete h;
    });
}

int drf_cnn_get_params(drf_cnn *h, double *p) {
    return guard([&] {
        DRF_CHECK(h && p, DRF_E_INVALID, "null argument");
        std::vector<float> w(h->net->nparam);
        DRF_CUDA(cudaMemcpyAsync(w.data(), h->net->wm.p, w.size() * 4, cudaMemcpyDeviceToHost, h->net->stream));
        DRF_CUDA(cudaStreamSynchronize(h->net->stream));
        for (size_t i = 0; i < w.size(); ++i) p[i] = w[i];
    });
}

int drf_cnn_set_params(drf_cnn *h, const double *p) {
    return guard([&] {
        DRF_CHECK(h && p, DRF_E_INVALID, "null argument");
        DRF_CHECK(all_finite(p, h->net->nparam), DRF_E_NONFINITE, "non-finite parameter");
        std::vector<float> w(h->net->nparam);
        for (size_t i = 0; i < w.size(); ++i) w[i] = (float)p[i];
        DRF_CUDA(cudaMemcpyAsync(h->net->wm.p, w.data(), w.size() * 4, cudaMemcpyHostToDevice, h->net->stream));
        h->net->cast();
        DRF_CUDA(cudaStreamSynchronize(h->net->stream));
    });
}

// forward (and optional loss/gradient) of B images H x W x 16 given on the host (FP64)
int drf_cnn_forward_backward(drf_cnn *h, int B, int H, int W, const double *X, const double *T,
                             double *Y, double *grad, double *loss) {
    return guard([&] {
        DRF_CHECK(h && X && B > 0 && H > 0 && W > 0, DRF_E_INVALID, "bad arguments");
        CnnNet &n = *h->net;
        const int64_t pix = (int64_t)B * H * W;
        n.ensure(pix);
        std::vector<bf16> xb(pix * 16);
        for (int64_t i = 0; i < pix * 16; ++i) xb[i] = __float2bfloat16_rn((float)X[i]);
        DRF_CUDA(cudaMemcpyAsync(n.act[0].p, xb.data(), pix * 16 * 2, cudaMemcpyHostToDevice, n.stream));
        n.forward(B, H, W);
        if (Y) {
            std::vector<float> y(pix * 16);
            DRF_CUDA(cudaMemcpyAsync(y.data(), n.out.p, pix * 16 * 4, cudaMemcpyDeviceToHost, n.stream));
            DRF_CUDA(cudaStreamSynchronize(n.stream));
            for (int64_t i = 0; i < pix * 16; ++i) Y[i] = y[i];
        }
        if (T) {
            std::vector<float> t(pix * 16);
            for (int64_t i = 0; i < pix * 16; ++i) t[i] = (float)T[i];
            DevBuf<float> td(pix * 16);
            DRF_CUDA(cudaMemcpyAsync(td.p, t.data(), pix * 16 * 4, cudaMemcpyHostToDevice, n.stream));
            n.backward(B, H, W, td.p);
            const double l = n.loss_host() / (double)(pix * 9);
            if (loss) *loss = l;
            if (grad) {
                std::vector<float> g(n.nparam);
                DRF_CUDA(cudaMemcpyAsync(g.data(), n.grad.p, g.size() * 4, cudaMemcpyDeviceToHost, n.stream));
                DRF_CUDA(cudaStreamSynchronize(n.stream));
                for (size_t i = 0; i < g.size(); ++i) grad[i] = g[i];
            }
        }
        cnn_check(&n, n.stream);
    });
}

// training set of N samples H x W x 16 (inputs X, targets T), kept on the device in FP32
int drf_cnn_set_dataset(drf_cnn *h, int N, int H, int W, const double *X, const double *T) {
    return guard([&] {
        DRF_CHECK(h && X && T && N > 0 && H > 0 && W > 0, DRF_E_INVALID, "bad arguments");
        CnnNet &n = *h->net;
        const size_t cnt = (size_t)N * H * W * 16;
        std::vector<float> a(cnt), b(cnt);
        for (size_t i = 0; i < cnt; ++i) { a[i] = (float)X[i]; b[i] = (float)T[i]; }
        n.dsX.alloc(cnt);
        n.dsT.alloc(cnt);
        DRF_CUDA(cudaMemcpy(n.dsX.p, a.data(), cnt * 4, cudaMemcpyHostToDevice));
        DRF_CUDA(cudaMemcpy(n.dsT.p, b.data(), cnt * 4, cudaMemcpyHostToDevice));
        n.ds_n = N; n.ds_h = H; n.ds_w = W;
    });
}

// Adam on random crops (batch x crop x crop) of the device dataset; returns the mean loss of
// the last `report` steps.
int drf_cnn_train(drf_cnn *h, int steps, int batch, int crop, double lr, uint64_t seed,
                  double *loss) {
    return guard([&] {
        DRF_CHECK(h && steps >= 0 && batch > 0 && crop > 0, DRF_E_INVALID, "bad arguments");
        CnnNet &n = *h->net;
        DRF_CHECK(n.ds_n > 0, DRF_E_INVALID, "no dataset (drf_cnn_set_dataset)");
        DRF_CHECK(crop <= n.ds_h && crop <= n.ds_w, DRF_E_INVALID, "crop larger than the samples");
        const int64_t pix = (int64_t)batch * crop * crop;
        n.ensure(pix);
        n.sel.alloc(3 * batch);
        n.bx.alloc(pix * 16);
        n.bt.alloc(pix * 16);
        std::mt19937_64 rng(seed);
        std::vector<int> sel(3 * batch);
        double acc = 0.0;
        int nacc = 0;
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        for (int s = 0; s < steps; ++s) {
            for (int b = 0; b < batch; ++b) {
                sel[3 * b] = (int)(rng() % n.ds_n);
                sel[3 * b + 1] = (int)(rng() % (n.ds_h - crop + 1));
                sel[3 * b + 2] = (int)(rng() % (n.ds_w - crop + 1));
            }
            DRF_CUDA(cudaMemcpyAsync(n.sel.p, sel.data(), sel.size() * 4, cudaMemcpyHostToDevice, n.stream));
            crop_kernel<<<nb(pix * 16), 256, 0, n.stream>>>(batch, crop, crop, n.ds_h, n.ds_w, n.sel.p,
                                                          n.dsX.p, n.dsT.p, n.bx.p, n.bt.p);
            DRF_LAUNCHED();
            DRF_CUDA(cudaMemcpyAsync(n.act[0].p, n.bx.p, pix * 16 * 2, cudaMemcpyDeviceToDevice, n.stream));
            n.forward(batch, crop, crop);
            n.backward(batch, crop, crop, n.bt.p);
            ++n.adam_t;
            const float c1 = 1.f - std::pow(b1, (float)n.adam_t), c2 = 1.f - std::pow(b2, (float)n.adam_t);
            adam_kernel<<<nb(n.nparam), 256, 0, n.stream>>>((int)n.nparam, n.wm.p, n.am.p, n.av.p,
                                                           n.grad.p, (float)lr, b1, b2, eps, c1, c2);
            DRF_LAUNCHED();
            n.cast();
            if (s >= steps - 10) {
                acc += n.loss_host() / (double)(pix * 9);
                ++nacc;
            }
        }
        cnn_check(&n, n.stream);
        if (loss) *loss = nacc ? acc / nacc : 0.0;
    });
}

}  // extern "C"

namespace drf {
CnnNet *cnn_net(drf_cnn *h) { return h ? h->net.get() : nullptr; }
}  // namespace drf
