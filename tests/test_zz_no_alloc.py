"""The allocation-free Bezier solve (drf_bz_jacobi_pcg_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory: they own the right-hand side and
solution buffers, and the solve keeps its vectors in a fixed scratch array inside the
library. This file is collected last so a run stopping at the first failure has run every
other test first; it passes alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import pyoracle as O
from drifter_b200._abi import alloc_count, check, lib
from drifter_b200.bezier import BezierSmoother, BzGridDesc

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8  # the PCG parity tolerance of tests/test_bz_gpu.py


def _data(n, L, seed):
    rng = np.random.default_rng(seed)
    X, Y = O.gauss_points(n, n, 0, 0, L, L)
    d = 1000.0 + 500.0 * np.sin(2 * np.pi * X / L + rng.uniform(0, 6)) * np.cos(2 * np.pi * Y / L)
    return d + rng.standard_normal(d.shape)


def _noalloc_solve(desc, b, torch):
    L = lib()
    L.drf_bz_jacobi_pcg_noalloc.argtypes = [C.POINTER(BzGridDesc), C.c_void_p, C.c_void_p,
                                            C.c_double, C.c_int, C.c_void_p,
                                            C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.drf_bz_jacobi_pcg_noalloc.restype = C.c_int
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros_like(db)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    n0 = alloc_count()
    it, rr = C.c_int(), C.c_double()
    check(L.drf_bz_jacobi_pcg_noalloc(C.byref(desc), C.c_void_p(db.data_ptr()),
                                      C.c_void_p(dx.data_ptr()), 1e-10, 5000,
                                      C.c_void_p(stream.cuda_stream), C.byref(it), C.byref(rr)))
    n1 = alloc_count()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return dx.cpu().numpy(), it.value, rr.value, n1 - n0, free0 - free1


def test_noalloc_matches_existing_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    deltas = []
    for n, L, seed in ((24, 3000.0, 5), (16, 1200.0, 9)):
        s = BezierSmoother(n, n, L, L, _data(n, L, seed), lam=1.0, ridge_epsilon=1e-4)
        b = s.rhs()
        x_ref, info = s.solve("jacobi", tol=1e-10, maxit=5000)
        x, it, rr, nalloc, dmem = _noalloc_solve(s.desc, b, torch)
        # no cudaMalloc inside the library on either call (its own allocation counter)
        assert nalloc == 0
        deltas.append(dmem)
        assert rr <= 1e-10
        assert abs(it - info["iters"]) <= 1
        assert np.abs(x - x_ref).max() / np.abs(x_ref).max() < REL_TOL
        s.close()
    # loose extra check (free memory is device-wide, so other users of the GPU move it): the
    # second call runs already-loaded kernels and should leave it unchanged
    assert abs(deltas[1]) <= 2 << 20


def test_noalloc_rejects_oversized_grid():
    L = lib()
    L.drf_bz_jacobi_pcg_noalloc.argtypes = [C.POINTER(BzGridDesc), C.c_void_p, C.c_void_p,
                                            C.c_double, C.c_int, C.c_void_p,
                                            C.POINTER(C.c_int), C.POINTER(C.c_double)]
    desc = BzGridDesc(171, 171, 0.0, 0.0, 1.0, 1.0, 1.0, 1e-4)
    it, rr = C.c_int(), C.c_double()
    rc = L.drf_bz_jacobi_pcg_noalloc(C.byref(desc), C.c_void_p(16), C.c_void_p(16), 1e-10, 10,
                                     None, C.byref(it), C.byref(rr))
    assert rc == 5  # DRF_E_UNSUPPORTED, before any device work
