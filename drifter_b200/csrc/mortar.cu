// Mortar coupling of non-conforming hexahedral faces (directional AMR) on the GPU: the coarse
// face trace and the 1..4 fine face traces are L2-projected onto a mortar space on the coarse
// face, a scalar numerical flux is taken at the mortar nodes, and the result is lifted back to
// the coarse face and, with the opposite sign, to the fine faces. Operators and semantics follow
// MortarSpace (src/dg/mortar.cpp:13-258) and DG3DIntegration::compute_interface_flux_nonconforming
// (src/dg/operators_3d.cpp:345-390):
//  * mortar order = element order p (both sides share it), mortar basis = tensor LGL Lagrange,
//    mortar quadrature (2p + 1)^2 Gauss-Legendre points on the coarse face;
//  * fine coupling B_f = sum over the mortar quadrature points inside the closed sub-face of
//    w_q phi_m(q) psi_j(map_f(q)) (points on a split line count for both halves, as in the
//    reference); P = M^-1 B, L = B^T for both sides;
//  * flux at mortar node m from (P_c U_c)_m and (sum_f P_f U_f)_m with the coarse face's
//    outward axis normal; coarse lift L_c M^-1 F, fine lifts -L_f M^-1 F.
// Device work: one warp per interface computes all lifted face values into a staging buffer;
// a second kernel adds them into the element right-hand sides, one thread per element node,
// in interface order (deterministic, no atomics).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "common.cuh"
#include "mortar_internal.hpp"

namespace drf {
namespace {

constexpr int MORTAR_TYPES = 6;  // FaceConnectionType SameLevel .. Fine2x2 (face_connection.hpp:15)
constexpr int MAXNM = MAXNP * MAXNP;
constexpr int SLOTS = 5;         // coarse side + up to 4 fine faces
constexpr int MW = 8;            // warps per CTA of the face kernel

int type_num_fine(int t) {
    static const int n[MORTAR_TYPES] = {1, 2, 2, 3, 3, 4};
    return n[t];
}

// sub-face rectangles (min t1, min t2, max t1, max t2) in the coarse face's [-1, 1]^2
// (MortarSpace::compute_subface_bounds, src/dg/mortar.cpp:27)
void subface_bounds(int t, double b[4][4]) {
    auto set = [&](int f, double a0, double a1, double c0, double c1) {
        b[f][0] = a0; b[f][1] = a1; b[f][2] = c0; b[f][3] = c1;
    };
    switch (t) {
    case 0: set(0, -1, -1, 1, 1); break;
    case 1: set(0, -1, -1, 0, 1); set(1, 0, -1, 1, 1); break;
    case 2: set(0, -1, -1, 1, 0); set(1, -1, 0, 1, 1); break;
    case 3: set(0, -1, -1, 0, 0); set(1, 0, -1, 1, 0); set(2, -1, 0, 1, 1); break;
    case 4: set(0, -1, -1, 0, 0); set(1, -1, 0, 0, 1); set(2, 0, -1, 1, 1); break;
    default: set(0, -1, -1, 0, 0); set(1, 0, -1, 1, 0); set(2, -1, 0, 0, 1); set(3, 0, 0, 1, 1); break;
    }
}

// n-point Gauss-Legendre on [-1, 1], ascending
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double d = p1 / dp;
            z -= d;
            if (std::abs(d) < 1e-16) break;
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
    for (int i = 0; i < n / 2; ++i) {  // exact symmetry
        const double s = 0.5 * (x[n - 1 - i] - x[i]);
        x[i] = -s;
        x[n - 1 - i] = s;
    }
}

// Lagrange basis on nodes at point z (barycentric; exactly 1 / 0 at a node)
void lagrange(const std::vector<double> &nodes, double z, double *phi) {
    const int n = (int)nodes.size();
    for (int j = 0; j < n; ++j)
        if (std::abs(z - nodes[j]) < 1e-15) {
            for (int k = 0; k < n; ++k) phi[k] = k == j ? 1.0 : 0.0;
            return;
        }
    double s = 0.0;
    for (int j = 0; j < n; ++j) {
        double bw = 1.0;
        for (int k = 0; k < n; ++k)
            if (k != j) bw *= nodes[j] - nodes[k];
        phi[j] = 1.0 / (bw * (z - nodes[j]));
        s += phi[j];
    }
    for (int j = 0; j < n; ++j) phi[j] /= s;
}

std::vector<double> inverse(const std::vector<double> &A, int n) {
    std::vector<double> M = A, I((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(M[r * n + c]) > std::abs(M[piv * n + c])) piv = r;
        DRF_CHECK(std::abs(M[piv * n + c]) > 0.0, DRF_E_INVALID, "singular mortar mass matrix");
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(M[c * n + k], M[piv * n + k]);
                std::swap(I[c * n + k], I[piv * n + k]);
            }
        const double d = 1.0 / M[c * n + c];
        for (int k = 0; k < n; ++k) { M[c * n + k] *= d; I[c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = M[r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) { M[r * n + k] -= f * M[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
        }
    }
    return I;
}

// Operators of one connection type, row-major: M, Minv (nm x nm), Pc (nm x nf), Lc (nf x nm),
// Pf[f] (nm x nf), Lf[f] (nf x nm); nm = nf = (p + 1)^2
struct HostOps {
    int nfine = 0;
    std::vector<double> M, Minv, Pc, Lc, Pf[4], Lf[4];
};

HostOps build_ops(int order, int t) {
    const HostBasis lgl = make_lgl_basis(order);
    const int np = order + 1, nm = np * np, nf = nm, nq1 = 2 * order + 1, nq = nq1 * nq1;
    std::vector<double> gx, gw;
    gauss_legendre(nq1, gx, gw);
    std::vector<double> I1((size_t)nq1 * np);
    for (int q = 0; q < nq1; ++q) lagrange(lgl.x, gx[q], &I1[q * np]);
    std::vector<double> Phi((size_t)nq * nm), W(nq);
    for (int qj = 0; qj < nq1; ++qj)
        for (int qi = 0; qi < nq1; ++qi) {
            const int q = qi + nq1 * qj;
            W[q] = gw[qi] * gw[qj];
            for (int j = 0; j < np; ++j)
                for (int i = 0; i < np; ++i) Phi[(size_t)q * nm + i + np * j] = I1[qi * np + i] * I1[qj * np + j];
        }
    HostOps o;
    o.nfine = type_num_fine(t);
    o.M.assign((size_t)nm * nm, 0.0);
    for (int q = 0; q < nq; ++q)
        for (int a = 0; a < nm; ++a)
            for (int b = 0; b < nm; ++b) o.M[(size_t)a * nm + b] += W[q] * Phi[(size_t)q * nm + a] * Phi[(size_t)q * nm + b];
    o.Minv = inverse(o.M, nm);
    auto project = [&](const std::vector<double> &B, std::vector<double> &P, std::vector<double> &L) {
        P.assign((size_t)nm * nf, 0.0);
        L.assign((size_t)nf * nm, 0.0);
        for (int r = 0; r < nm; ++r)
            for (int k = 0; k < nm; ++k)
                for (int c = 0; c < nf; ++c) P[(size_t)r * nf + c] += o.Minv[(size_t)r * nm + k] * B[(size_t)k * nf + c];
        for (int r = 0; r < nm; ++r)
            for (int c = 0; c < nf; ++c) L[(size_t)c * nm + r] = B[(size_t)r * nf + c];
    };
    std::vector<double> B((size_t)nm * nf, 0.0);
    for (int q = 0; q < nq; ++q)
        for (int m = 0; m < nm; ++m)
            for (int j = 0; j < nf; ++j) B[(size_t)m * nf + j] += W[q] * Phi[(size_t)q * nm + m] * Phi[(size_t)q * nm + j];
    project(B, o.Pc, o.Lc);
    double sb[4][4];
    subface_bounds(t, sb);
    double pt[MAXNP], ps[MAXNP];
    for (int f = 0; f < o.nfine; ++f) {
        std::fill(B.begin(), B.end(), 0.0);
        for (int qj = 0; qj < nq1; ++qj)
            for (int qi = 0; qi < nq1; ++qi) {
                const double x0 = gx[qi], x1 = gx[qj];
                if (!(x0 >= sb[f][0] && x0 <= sb[f][2] && x1 >= sb[f][1] && x1 <= sb[f][3])) continue;
                const int q = qi + nq1 * qj;
                lagrange(lgl.x, 2.0 * (x0 - sb[f][0]) / (sb[f][2] - sb[f][0]) - 1.0, pt);
                lagrange(lgl.x, 2.0 * (x1 - sb[f][1]) / (sb[f][3] - sb[f][1]) - 1.0, ps);
                for (int m = 0; m < nm; ++m)
                    for (int jf = 0; jf < np; ++jf)
                        for (int i = 0; i < np; ++i)
                            B[(size_t)m * nf + i + np * jf] += W[q] * Phi[(size_t)q * nm + m] * pt[i] * ps[jf];
            }
        project(B, o.Pf[f], o.Lf[f]);
    }
    return o;
}

// device operator block of one type: Minv | Pc | Lc | Pf[4] | Lf[4], each nm * nm doubles,
// stored transposed (column-major)
constexpr int OPS_MATS = 11;
__host__ __device__ inline size_t ops_stride(int nm) { return (size_t)OPS_MATS * nm * nm; }

struct MortarDev {
    int np, nm, nd;
    int64_t n_if;
    const double *ops;                 // MORTAR_TYPES blocks of ops_stride(nm)
    const int *type, *cface, *fface;   // fface: 4 per interface
    const int64_t *celem, *felem;      // felem: 4 per interface
};

__device__ __forceinline__ int type_num_fine_dev(int t) { return t == 0 ? 1 : (t <= 2 ? 2 : (t <= 4 ? 3 : 4)); }

__device__ __forceinline__ int face_node(int np, int f, int it, int jt) {
    const int axis = f >> 1, b = (f & 1) ? np - 1 : 0;
    if (axis == 0) return b + np * (it + np * jt);
    if (axis == 1) return it + np * (b + np * jt);
    return it + np * (jt + np * b);
}

// scalar fluxes for u_t + div(a u) = 0 (include/flux/numerical_flux.hpp: CentralFlux :244,
// UpwindFlux :264, LaxFriedrichsFlux :222 with speed |a.n|)
__device__ __forceinline__ double scalar_flux(int kind, double uL, double uR, double vn) {
    if (kind == DRF_MORTAR_FLUX_CENTRAL) return 0.5 * (vn * uL + vn * uR);
    if (kind == DRF_MORTAR_FLUX_UPWIND) return vn * (vn >= 0 ? uL : uR);
    return 0.5 * (vn * uL + vn * uR) - 0.5 * fabs(vn) * (uR - uL);
}

// NP (nodes per direction) is a compile-time constant so the small dense products unroll and
// their operator loads pipeline.
template <int NP>
__global__ void __launch_bounds__(32 * MW) mortar_face_kernel(MortarDev D, int kind, double a0, double a1,
                                                              double a2, const double *__restrict__ U,
                                                              double *__restrict__ contrib) {
    constexpr int nm = NP * NP, nf = NP * NP, np = NP;
    __shared__ double sU[MW][SLOTS][nm];
    __shared__ double sF[MW][nm], sG[MW][nm];
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int64_t i = blockIdx.x * (int64_t)MW + w; i < D.n_if; i += (int64_t)gridDim.x * MW) {
        const int t = D.type[i], nfine = type_num_fine_dev(t);
        const double *op = D.ops + (size_t)t * ops_stride(nm);
        const double *Minv = op, *Pc = op + nm * nm, *Lc = op + 2 * nm * nm;
        const double *Pf = op + 3 * nm * nm, *Lf = op + 7 * nm * nm;
        const int cf = D.cface[i];
        for (int j = lane; j < nf; j += 32) {
            sU[w][0][j] = U[D.celem[i] * D.nd + face_node(np, cf, j % np, j / np)];
            for (int f = 0; f < nfine; ++f)
                sU[w][1 + f][j] = U[D.felem[4 * i + f] * D.nd + face_node(np, D.fface[4 * i + f], j % np, j / np)];
        }
        __syncwarp();
        const int axis = cf >> 1;
        const double vn = ((cf & 1) ? 1.0 : -1.0) * (axis == 0 ? a0 : (axis == 1 ? a1 : a2));
        for (int m = lane; m < nm; m += 32) {
            double uc = 0.0, uf = 0.0;
#pragma unroll
            for (int j = 0; j < nf; ++j) uc += Pc[j * nm + m] * sU[w][0][j];
            for (int f = 0; f < nfine; ++f) {
                double s = 0.0;
                const double *P = Pf + (size_t)f * nm * nm + m;
#pragma unroll
                for (int j = 0; j < nf; ++j) s += P[j * nm] * sU[w][1 + f][j];
                uf += s;
            }
            sF[w][m] = scalar_flux(kind, uc, uf, vn);
        }
        __syncwarp();
        for (int m = lane; m < nm; m += 32) {
            double g = 0.0;
#pragma unroll
            for (int k = 0; k < nm; ++k) g += Minv[k * nm + m] * sF[w][k];
            sG[w][m] = g;
        }
        __syncwarp();
        double *out = contrib + (size_t)i * SLOTS * nf;
        for (int j = lane; j < nf; j += 32) {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < nm; ++m) s += Lc[m * nf + j] * sG[w][m];
            out[j] = s;
            for (int f = 0; f < nfine; ++f) {
                const double *L = Lf + (size_t)f * nm * nm + j;
                double sf = 0.0;
#pragma unroll
                for (int m = 0; m < nm; ++m) sf += L[m * nf] * sG[w][m];
                out[(1 + f) * nf + j] = -sf;
            }
        }
        __syncwarp();
    }
}

// rhs[e][v] += every staged face value of element e that lands on node v, in interface order.
// touched[u]: element; ent[ptr[u] .. ptr[u+1]): (interface, slot, face) triples
__global__ void __launch_bounds__(256) mortar_lift_kernel(int np, int nd, int64_t n_touched,
                                                          const int64_t *__restrict__ touched,
                                                          const int64_t *__restrict__ ptr,
                                                          const int *__restrict__ ent,
                                                          const double *__restrict__ contrib,
                                                          double *__restrict__ rhs) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n_touched * nd) return;
    const int64_t u = t / nd;
    const int v = (int)(t % nd);
    const int vi = v % np, vj = (v / np) % np, vk = v / (np * np);
    const int nf = np * np;
    bool any = false;
    double acc = rhs[touched[u] * nd + v];
    for (int64_t k = ptr[u]; k < ptr[u + 1]; ++k) {
        const int iface = ent[3 * k], slot = ent[3 * k + 1], f = ent[3 * k + 2];
        const int axis = f >> 1, b = (f & 1) ? np - 1 : 0;
        int on, it, jt;
        if (axis == 0) { on = vi; it = vj; jt = vk; }
        else if (axis == 1) { on = vj; it = vi; jt = vk; }
        else { on = vk; it = vi; jt = vj; }
        if (on != b) continue;
        acc += contrib[((size_t)iface * SLOTS + slot) * nf + it + np * jt];
        any = true;
    }
    if (any) rhs[touched[u] * nd + v] = acc;
}

}  // namespace
}  // namespace drf

using namespace drf;

struct drf_mortar {
    int order = 0, np = 0, nm = 0, nd = 0;
    int64_t n_if = 0, n_elem = 0, n_touched = 0;
    cudaStream_t stream = nullptr, own = nullptr;
    DevBuf<double> ops, contrib, U, rhs;
    DevBuf<int> type, cface, fface, ent;
    DevBuf<int64_t> celem, felem, touched, ptr;
    ~drf_mortar() {
        if (own) cudaStreamDestroy(own);
    }
    MortarDev dev() const {
        MortarDev D;
        D.np = np; D.nm = nm; D.nd = nd; D.n_if = n_if;
        D.ops = ops.p; D.type = type.p; D.cface = cface.p; D.fface = fface.p;
        D.celem = celem.p; D.felem = felem.p;
        return D;
    }
    void run(int kind, const double a[3], const double *dU, double *drhs) {
        if (n_if == 0) return;
        stage_faces(kind, a, dU);
        const int64_t nt = n_touched * nd;
        mortar_lift_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, stream>>>(np, nd, n_touched, touched.p, ptr.p,
                                                                             ent.p, contrib.p, drhs);
        DRF_LAUNCHED();
    }
    void stage_faces(int kind, const double a[3], const double *dU) {
        if (n_if == 0) return;
        const unsigned g = (unsigned)std::min<int64_t>((n_if + MW - 1) / MW, 148 * 16);
        switch (np) {
        case 2: mortar_face_kernel<2><<<g, 32 * MW, 0, stream>>>(dev(), kind, a[0], a[1], a[2], dU, contrib.p); break;
        case 3: mortar_face_kernel<3><<<g, 32 * MW, 0, stream>>>(dev(), kind, a[0], a[1], a[2], dU, contrib.p); break;
        case 4: mortar_face_kernel<4><<<g, 32 * MW, 0, stream>>>(dev(), kind, a[0], a[1], a[2], dU, contrib.p); break;
        case 5: mortar_face_kernel<5><<<g, 32 * MW, 0, stream>>>(dev(), kind, a[0], a[1], a[2], dU, contrib.p); break;
        default: mortar_face_kernel<6><<<g, 32 * MW, 0, stream>>>(dev(), kind, a[0], a[1], a[2], dU, contrib.p); break;
        }
        DRF_LAUNCHED();
    }
};

namespace drf {
void mortar_stage_faces(drf_mortar *h, int kind, const double a[3], const double *d_U) {
    h->stage_faces(kind, a, d_U);
}
MortarLifts mortar_lifts(const drf_mortar *h) {
    MortarLifts L;
    L.contrib = h->contrib.p;
    L.touched = h->touched.p;
    L.ptr = h->ptr.p;
    L.ent = h->ent.p;
    L.n_touched = h->n_touched;
    L.slots = SLOTS;
    return L;
}
}  // namespace drf

namespace {
template <class T>
void upload(DevBuf<T> &d, const std::vector<T> &v) {
    d.alloc(std::max<size_t>(v.size(), 1));
    if (!v.empty()) DRF_CUDA(cudaMemcpy(d.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}
void check_flux(int kind, const double *a) {
    DRF_CHECK(kind == DRF_MORTAR_FLUX_CENTRAL || kind == DRF_MORTAR_FLUX_UPWIND || kind == DRF_MORTAR_FLUX_LF,
              DRF_E_INVALID, "unknown mortar flux kind");
    DRF_CHECK(a && std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]), DRF_E_INVALID,
              "advection velocity must be finite");
}
}  // namespace

extern "C" {

int drf_mortar_ops(int order, int type, double *M, double *Minv, double *Pc, double *Lc, double *Pf,
                   double *Lf, int *nfine) {
    return guard([&] {
        DRF_CHECK(type >= 0 && type < MORTAR_TYPES, DRF_E_INVALID, "connection type must be 0..5");
        const HostOps o = build_ops(order, type);
        const size_t n2 = o.M.size();
        if (M) std::memcpy(M, o.M.data(), n2 * 8);
        if (Minv) std::memcpy(Minv, o.Minv.data(), n2 * 8);
        if (Pc) std::memcpy(Pc, o.Pc.data(), n2 * 8);
        if (Lc) std::memcpy(Lc, o.Lc.data(), n2 * 8);
        for (int f = 0; f < o.nfine; ++f) {
            if (Pf) std::memcpy(Pf + f * n2, o.Pf[f].data(), n2 * 8);
            if (Lf) std::memcpy(Lf + f * n2, o.Lf[f].data(), n2 * 8);
        }
        if (nfine) *nfine = o.nfine;
    });
}

int drf_mortar_create(int order, int64_t n_if, const int *type, const int64_t *coarse_elem,
                      const int *coarse_face, const int64_t *fine_elem, const int *fine_face,
                      int64_t n_elem, drf_mortar **out) {
    return guard([&] {
        DRF_CHECK(out, DRF_E_INVALID, "null output");
        *out = nullptr;
        DRF_CHECK(n_if >= 0 && n_elem > 0, DRF_E_INVALID, "bad interface or element count");
        DRF_CHECK(n_if == 0 || (type && coarse_elem && coarse_face && fine_elem && fine_face), DRF_E_INVALID,
                  "null interface array");
        auto h = std::make_unique<drf_mortar>();
        h->order = order;
        h->np = order + 1;
        h->nm = h->np * h->np;
        h->nd = h->np * h->nm;
        h->n_if = n_if;
        h->n_elem = n_elem;
        // operators of every connection type
        std::vector<double> ops(MORTAR_TYPES * ops_stride(h->nm), 0.0);
        for (int t = 0; t < MORTAR_TYPES; ++t) {
            const HostOps o = build_ops(order, t);
            double *dst = ops.data() + t * ops_stride(h->nm);
            const int nm = h->nm;
            const size_t n2 = (size_t)nm * nm;
            // stored transposed: in the face kernel lane m reads row m, so column-major storage
            // makes a warp's reads of one column consecutive addresses
            auto put_t = [&](double *d, const std::vector<double> &A) {
                for (int r = 0; r < nm; ++r)
                    for (int c = 0; c < nm; ++c) d[(size_t)c * nm + r] = A[(size_t)r * nm + c];
            };
            put_t(dst, o.Minv);
            put_t(dst + n2, o.Pc);
            put_t(dst + 2 * n2, o.Lc);
            for (int f = 0; f < o.nfine; ++f) {
                put_t(dst + (3 + f) * n2, o.Pf[f]);
                put_t(dst + (7 + f) * n2, o.Lf[f]);
            }
        }
        // interfaces, validated; per-element entries in interface order
        std::vector<int> ty(n_if), cf(n_if), ff(4 * n_if, 0);
        std::vector<int64_t> ce(n_if), fe(4 * n_if, 0);
        std::map<int64_t, std::vector<int>> per_elem;
        for (int64_t i = 0; i < n_if; ++i) {
            DRF_CHECK(type[i] >= 0 && type[i] < MORTAR_TYPES, DRF_E_INVALID,
                      "interface " + std::to_string(i) + ": connection type must be 0..5");
            DRF_CHECK(coarse_face[i] >= 0 && coarse_face[i] < 6, DRF_E_INVALID, "face id must be 0..5");
            DRF_CHECK(coarse_elem[i] >= 0 && coarse_elem[i] < n_elem, DRF_E_INVALID, "element index out of range");
            ty[i] = type[i];
            cf[i] = coarse_face[i];
            ce[i] = coarse_elem[i];
            auto &pc = per_elem[ce[i]];
            pc.insert(pc.end(), {(int)i, 0, cf[i]});
            for (int f = 0; f < type_num_fine(ty[i]); ++f) {
                DRF_CHECK(fine_face[4 * i + f] >= 0 && fine_face[4 * i + f] < 6, DRF_E_INVALID, "face id must be 0..5");
                DRF_CHECK(fine_elem[4 * i + f] >= 0 && fine_elem[4 * i + f] < n_elem, DRF_E_INVALID,
                          "element index out of range");
                ff[4 * i + f] = fine_face[4 * i + f];
                fe[4 * i + f] = fine_elem[4 * i + f];
                auto &pf = per_elem[fe[4 * i + f]];
                pf.insert(pf.end(), {(int)i, 1 + f, ff[4 * i + f]});
            }
        }
        std::vector<int64_t> touched, ptr{0};
        std::vector<int> ent;
        for (auto &kv : per_elem) {
            touched.push_back(kv.first);
            ent.insert(ent.end(), kv.second.begin(), kv.second.end());
            ptr.push_back((int64_t)ent.size() / 3);
        }
        h->n_touched = (int64_t)touched.size();
        DRF_CUDA(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
        h->stream = h->own;
        upload(h->ops, ops);
        upload(h->type, ty); upload(h->cface, cf); upload(h->fface, ff);
        upload(h->celem, ce); upload(h->felem, fe);
        upload(h->touched, touched); upload(h->ptr, ptr); upload(h->ent, ent);
        h->contrib.alloc(std::max<size_t>((size_t)n_if * SLOTS * h->nm, 1));
        *out = h.release();
    });
}

int drf_mortar_destroy(drf_mortar *h) {
    return guard([&] {
        if (!h) return;
        if (h->stream) cudaStreamSynchronize(h->stream);
        delete h;
    });
}

int drf_mortar_set_stream(drf_mortar *h, void *stream) {
    return guard([&] {
        DRF_CHECK(h, DRF_E_INVALID, "null mortar handle");
        DRF_CUDA(cudaStreamSynchronize(h->stream));
        h->stream = stream ? (cudaStream_t)stream : h->own;
    });
}

int drf_mortar_apply_device(drf_mortar *h, int flux_kind, const double *a, const double *d_U, double *d_rhs) {
    return guard([&] {
        DRF_CHECK(h && d_U && d_rhs, DRF_E_INVALID, "null argument");
        check_flux(flux_kind, a);
        h->run(flux_kind, a, d_U, d_rhs);
    });
}

int drf_mortar_apply(drf_mortar *h, int flux_kind, const double *a, const double *U, double *rhs) {
    return guard([&] {
        DRF_CHECK(h && U && rhs, DRF_E_INVALID, "null argument");
        check_flux(flux_kind, a);
        const size_t n = (size_t)h->n_elem * h->nd;
        DRF_CHECK(all_finite(U, n), DRF_E_NONFINITE, "non-finite state");
        if (h->U.n < n) { h->U.alloc(n); h->rhs.alloc(n); }
        DRF_CUDA(cudaMemcpyAsync(h->U.p, U, n * 8, cudaMemcpyHostToDevice, h->stream));
        DRF_CUDA(cudaMemcpyAsync(h->rhs.p, rhs, n * 8, cudaMemcpyHostToDevice, h->stream));
        h->run(flux_kind, a, h->U.p, h->rhs.p);
        DRF_CUDA(cudaMemcpyAsync(rhs, h->rhs.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
        DRF_CUDA(cudaStreamSynchronize(h->stream));
    });
}

}  // extern "C"
