// Shared runtime pieces of libdrifter_b200: status codes, error capture, launch
// accounting, and the nodal basis tables kept in constant memory.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/drifter_b200.h"

namespace drf {

// ----------------------------------------------------------------------------- errors
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
void set_last_error(const std::string &msg);
std::atomic<uint64_t> &launch_counter();
// Device allocations made by this library (every cudaMalloc goes through DevBuf::alloc).
std::atomic<uint64_t> &alloc_counter();
// Nonzero while the calling thread is capturing a stream into a graph: kernels queued then are
// counted when the graph is launched, not when they are queued.
int &capture_depth();

#define DRF_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw ::drf::Error(DRF_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define DRF_CHECK(cond, code, msg)                  \
    do {                                            \
        if (!(cond)) throw ::drf::Error(code, msg); \
    } while (0)

// After every kernel launch: count it (unless it was only queued into a graph being
// captured) and surface launch-configuration errors.
#define DRF_LAUNCHED()                                                      \
    do {                                                                    \
        if (::drf::capture_depth() == 0) ::drf::launch_counter().fetch_add(1); \
        DRF_CUDA(cudaGetLastError());                                       \
    } while (0)

// C-ABI wrapper: converts exceptions into status codes.
template <class F>
int guard(F &&f) {
    try {
        f();
        return DRF_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return DRF_E_NOMEM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return DRF_E_INVALID;
    }
}

// ----------------------------------------------------------------------------- basis (host)
// Legendre-Gauss-Lobatto basis on [-1, 1] computed in FP64 on the host: nodes, weights,
// derivative matrix D (D[i][m] = l_m'(x_i)), its square D2 = D*D, and the integration
// matrix S[k][m] = int_{-1}^{x_k} l_m(x) dx.
struct HostBasis {
    int order = 0, np = 0;
    std::vector<double> x, w, D, D2, S;
};
HostBasis make_lgl_basis(int order);

constexpr int MAXNP = 6;

// Basis tables for device code (both precisions), uploaded once per process. Ai is the
// inverse of the strong-form derivative with the value at x = -1 lifted in,
// (D + e_0 e_0^T / w_0)^-1, and a0 = Ai e_0 / w_0: the sigma velocity that is consistent with
// the discrete tracer divergence is solved with them.
struct DevBasis {
    double D[MAXNP * MAXNP], D2[MAXNP * MAXNP], S[MAXNP * MAXNP], w[MAXNP], x[MAXNP];
    double Ai[MAXNP * MAXNP], a0[MAXNP];
    float Df[MAXNP * MAXNP], D2f[MAXNP * MAXNP], Sf[MAXNP * MAXNP], wf[MAXNP], xf[MAXNP];
    float Aif[MAXNP * MAXNP], a0f[MAXNP];
};

// Device-memory RAII buffer.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) {
            alloc_counter().fetch_add(1);
            cudaError_t e = cudaMalloc(&p, count * sizeof(T));
            if (e != cudaSuccess) {
                p = nullptr;
                n = 0;
                (void)cudaGetLastError();
                throw Error(DRF_E_NOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) +
                                             " bytes failed: " + cudaGetErrorString(e));
            }
        }
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        release();
        p = o.p; n = o.n; o.p = nullptr; o.n = 0;
        return *this;
    }
};

bool all_finite(const double *x, size_t n);

// Captures what `enqueue` queues on `stream` (thread-local capture mode) into an executable
// graph. `kernels` receives the number of kernel nodes in it, which a caller adds to the launch
// counter per replay. The capture is ended, and the partial graph destroyed, if `enqueue` throws.
template <class F>
cudaGraphExec_t capture_graph(cudaStream_t stream, F &&enqueue, uint64_t *kernels) {
    cudaGraph_t g = nullptr;
    DRF_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    ++capture_depth();
    try {
        enqueue();
    } catch (...) {
        --capture_depth();
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    --capture_depth();
    DRF_CUDA(cudaStreamEndCapture(stream, &g));
    size_t nn = 0;
    cudaError_t e = cudaGraphGetNodes(g, nullptr, &nn);
    uint64_t nk = 0;
    if (e == cudaSuccess && nn) {
        std::vector<cudaGraphNode_t> nodes(nn);
        e = cudaGraphGetNodes(g, nodes.data(), &nn);
        for (size_t i = 0; e == cudaSuccess && i < nn; ++i) {
            cudaGraphNodeType t;
            e = cudaGraphNodeGetType(nodes[i], &t);
            if (e == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
        }
    }
    cudaGraphExec_t x = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    DRF_CUDA(e);
    if (kernels) *kernels = nk;
    return x;
}

}  // namespace drf
