// Learned preconditioner network (cnn.cu) as used by the Bezier PCG (bz.cu).
#pragma once
#include <cuda_runtime.h>

#include "../../include/drifter_b200.h"

namespace drf {
struct CnnNet;
CnnNet *cnn_net(drf_cnn *h);
void cnn_prepare(CnnNet *net, int n);
// z (+)= rms(r) * out_scale * net(r / rms(r)) on the control-point grid of n x n elements
// (add = 1 adds to the base already in z); rr_dev points to r.r on the device; kernels return
// early when *stop is set.
// z (+)= the network's correction of r; with jac_diag non-null z = r / jac_diag + correction
// (the Jacobi base and the correction in one pass)
// With dq and part non-null (and jac_diag set), the unpack pass also writes per-block partials
// of z.r (part[block]) and z.dq (part[nblocks + block]); returns the number of blocks.
int cnn_precondition(CnnNet *net, cudaStream_t s, int n, const double *r, const double *rr_dev,
                     double out_scale, double *z, int add, const int *stop, const double *jac_diag = nullptr,
                     const double *dq = nullptr, double *part = nullptr);
// surfaces (and clears) the network's device status word: throws when a bounded wait gave up
void cnn_check(CnnNet *net, cudaStream_t s);
// autotunes the conv form (mma.sync or tcgen05) of every layer at the preconditioner's size
// (n x n elements); ms[l][form] the timed launches, form[l] the choice (outside any capture)
void cnn_tune(CnnNet *net, int n, double ms[4][2], int form[4]);
}  // namespace drf
