"""Host mirror of DRIFTER's cubic Bezier smoother interfaces over the C ABI.

  * BezierSmoother  ~ CGBezierSmootherBase assembly + solve (src/bathymetry/cg_bezier_smoother_base.cpp)
  * BezierMultigridPreconditioner.setup/apply (include/bathymetry/bezier_multigrid_preconditioner.hpp:240,246)
  * solve(...) = PCG on Q x = b (FP64) with preconditioner "none" | "jacobi" | "mg" | "cnn"
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import check, dptr, lib

PRECOND = {"none": 0, "jacobi": 1, "mg": 2, "cnn": 3, "mg_reference": 4}


class BzGridDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("x0", C.c_double), ("y0", C.c_double),
                ("Lx", C.c_double), ("Ly", C.c_double), ("lam", C.c_double),
                ("ridge_epsilon", C.c_double)]


def _setup_sigs():
    L = lib()
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    sigs = {
        "drf_bz_create": [C.POINTER(BzGridDesc), dp, C.POINTER(C.c_void_p)],
        "drf_bz_destroy": [vp], "drf_bz_set_stream": [vp, vp],
        "drf_bz_info": [vp, C.POINTER(C.c_int64), dp, C.POINTER(C.c_int)],
        "drf_bz_get_rhs": [vp, dp], "drf_bz_apply_Q": [vp, dp, dp],
        "drf_mg_setup": [vp, C.c_int, C.c_int, C.c_int], "drf_mg_apply": [vp, dp, dp],
        "drf_mg_apply_reference": [vp, dp, dp, C.c_double, C.c_int, C.POINTER(C.c_int), dp],
        "drf_bz_cnn_tuning": [vp, C.POINTER(C.c_int), dp],
        "drf_bz_precondition": [vp, C.c_int, dp, dp],
        "drf_pcg_solve": [vp, dp, dp, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int), dp, dp],
        "drf_bz_constraints_apply": [vp, C.c_int, dp, dp],
        "drf_bz_constrained_solve": [vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, dp,
                                     C.POINTER(C.c_int), dp, dp],
        "drf_bz_element_errors": [vp, dp, dp, C.c_int, dp, dp],
        "drf_bz_mesh_element_errors": [C.c_int64, dp, dp, dp, C.c_int, dp, dp],
        "drf_bz_mesh_data_fitting": [C.c_int64, dp, dp, dp, C.c_int, dp, dp, dp],
    }
    for k, a in sigs.items():
        getattr(L, k).argtypes = a
        getattr(L, k).restype = C.c_int
    return L


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def mesh_element_errors(bounds, coeffs, zdata, ngauss: int = 4):
    """AdaptiveCGCubicBezierSmoother::compute_element_l2_error / estimate_element_error
    (src/bathymetry/adaptive_cg_cubic_bezier_smoother.cpp:100,142) for every element of a
    quadtree mesh: bounds (n, 4) as (xmin, ymin, xmax, ymax), coeffs (n, 16) the element's
    resolved control values, zdata (n, ngauss**2) the data at its Gauss points ([qj][qi]).
    Returns (l2, normalized)."""
    L = _setup_sigs()
    b = _c(bounds).reshape(-1, 4)
    n = len(b)
    l2, nrm = np.empty(n), np.empty(n)
    check(L.drf_bz_mesh_element_errors(n, dptr(b), dptr(_c(coeffs)), dptr(_c(zdata)), ngauss, dptr(l2),
                                       dptr(nrm)))
    return l2, nrm


def mesh_data_fitting(bounds, zdata, ngauss: int = 4, relax=None):
    """The element part of CGBezierSmootherBase::assemble_data_fitting_global
    (src/bathymetry/cg_bezier_smoother_base.cpp:308) on a quadtree mesh: (BtWB (n, 16, 16),
    BtWd (n, 16), dTWd (n,)); the scatter through the DOF map stays with the caller."""
    L = _setup_sigs()
    b = _c(bounds).reshape(-1, 4)
    n = len(b)
    K, r, dd = np.empty((n, 16, 16)), np.empty((n, 16)), np.empty(n)
    rel = dptr(_c(relax)) if relax is not None else None
    check(L.drf_bz_mesh_data_fitting(n, dptr(b), dptr(_c(zdata)), rel, ngauss, dptr(K), dptr(r), dptr(dd)))
    return K, r, dd


class BezierSmoother:
    """Uniform-grid cubic Bezier smoother resident on the GPU."""

    def __init__(self, nx, ny, Lx, Ly, dgauss, lam=1.0, ridge_epsilon=1e-4, x0=0.0, y0=0.0):
        L = _setup_sigs()
        self.desc = BzGridDesc(nx, ny, x0, y0, Lx, Ly, lam, ridge_epsilon)
        d = np.ascontiguousarray(dgauss, dtype=np.float64)
        h = C.c_void_p()
        check(L.drf_bz_create(C.byref(self.desc), dptr(d), C.byref(h)))
        self.h = h
        n, a, nl = C.c_int64(), C.c_double(), C.c_int()
        check(L.drf_bz_info(self.h, C.byref(n), C.byref(a), C.byref(nl)))
        self.ndof, self.alpha = n.value, a.value

    def close(self):
        if getattr(self, "h", None):
            lib().drf_bz_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, ptr):
        check(lib().drf_bz_set_stream(self.h, C.c_void_p(ptr or 0)))

    def rhs(self):
        b = np.empty(self.ndof)
        check(lib().drf_bz_get_rhs(self.h, dptr(b)))
        return b

    def apply_Q(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.ndof)
        check(lib().drf_bz_apply_Q(self.h, dptr(x), dptr(y)))
        return y

    def mg_setup(self, coarsest_n=2, pre=1, post=1):
        check(lib().drf_mg_setup(self.h, coarsest_n, pre, post))

    def mg_apply(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.ndof)
        check(lib().drf_mg_apply(self.h, dptr(r), dptr(z)))
        return z

    def mg_apply_reference(self, r, tol=1e-6, max_vcycles=100):
        """BezierMultigridPreconditioner::apply as the reference computes it: V-cycles with the
        row-normalised restriction and one colour order, repeated to tol. Returns (z, cycles,
        relres)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.ndof)
        cyc, rel = C.c_int(), C.c_double()
        check(lib().drf_mg_apply_reference(self.h, dptr(r), dptr(z), tol, max_vcycles,
                                           C.byref(cyc), C.byref(rel)))
        return z, cyc.value, rel.value

    def cnn_tuning(self) -> dict:
        """The attached network's conv form per layer (mma_sync or tcgen05, timed at this size)."""
        f = (C.c_int * 4)()
        ms = np.zeros(8)
        check(lib().drf_bz_cnn_tuning(self.h, f, dptr(ms)))
        names = ("mma_sync", "tcgen05")
        return {"forms": [names[v] for v in f],
                "ms": {names[k]: [round(float(ms[2 * l + k]), 5) for l in range(4)] for k in (0, 1)}}

    def precondition(self, r, kind="jacobi"):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.ndof)
        check(lib().drf_bz_precondition(self.h, PRECOND[kind], dptr(r), dptr(z)))
        return z

    def solve(self, precond="mg", tol=1e-10, maxit=1000, b=None, x0=None):
        x = np.zeros(self.ndof) if x0 is None else np.array(x0, dtype=np.float64)
        bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
        it, rr, ms = C.c_int(), C.c_double(), C.c_double()
        check(lib().drf_pcg_solve(self.h, dptr(bb) if bb is not None else None, dptr(x), tol,
                                  maxit, PRECOND[precond], C.byref(it), C.byref(rr), C.byref(ms)))
        return x, dict(iters=it.value, relres=rr.value, ms=ms.value)

    def element_errors(self, x, zdata, ngauss=4):
        """Per-element L2 misfit of the surface x to the data sampled at the ngauss x ngauss
        Gauss points of every element (AdaptiveCGCubicBezierSmoother::compute_element_l2_error
        and the normalized error of estimate_element_error): returns (l2, normalized)."""
        xx = np.ascontiguousarray(x, dtype=np.float64)
        zd = np.ascontiguousarray(zdata, dtype=np.float64)
        ne = self.desc.nx * self.desc.ny
        if zd.size != ne * ngauss * ngauss:
            raise ValueError("zdata must hold ngauss^2 samples per element")
        l2, nrm = np.empty(ne), np.empty(ne)
        check(lib().drf_bz_element_errors(self.h, dptr(xx), dptr(zd), ngauss, dptr(l2), dptr(nrm)))
        return l2, nrm

    def constraints_apply(self, x, edge_ngauss=4):
        """C1 edge-constraint rows A x (2 n (n - 1) edge_ngauss values, vertical edges first)."""
        n = self.desc.nx
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(2 * n * (n - 1) * edge_ngauss)
        check(lib().drf_bz_constraints_apply(self.h, edge_ngauss, dptr(x), dptr(y)))
        return y

    def solve_constrained(self, edge_ngauss=4, tol=1e-10, maxit=5000, inner="mg", inner_tol=1e-12):
        """Constrained minimiser (CGCubicBezierBathymetrySmoother::solve with C1 edge
        constraints): CG on the Schur complement A Q^-1 A^T, each Q^-1 a PCG solve."""
        x = np.empty(self.ndof)
        it, rr, ms = C.c_int(), C.c_double(), C.c_double()
        check(lib().drf_bz_constrained_solve(self.h, edge_ngauss, PRECOND[inner], tol, maxit,
                                             inner_tol, dptr(x), C.byref(it), C.byref(rr),
                                             C.byref(ms)))
        return x, dict(outer_iters=it.value, relres=rr.value, ms=ms.value)


class BezierMultigridPreconditioner:
    """setup()/apply() over a BezierSmoother's operator (one symmetric V-cycle per apply)."""

    def __init__(self, smoother: BezierSmoother, coarsest_n=2, pre=1, post=1):
        self.s = smoother
        self.cfg = (coarsest_n, pre, post)

    def setup(self):
        self.s.mg_setup(*self.cfg)

    def apply(self, r):
        return self.s.mg_apply(r)
