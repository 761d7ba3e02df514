"""Mortar coupling of non-conforming faces (MortarSpace, src/dg/mortar.cpp; the non-conforming
face flux of DG3DIntegration, src/dg/operators_3d.cpp:345) on the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import check, dptr, lib

SAME_LEVEL, FINE_2X1, FINE_1X2, FINE_3_2PLUS1, FINE_3_1PLUS2, FINE_2X2 = range(6)
NUM_FINE = {0: 1, 1: 2, 2: 2, 3: 3, 4: 3, 5: 4}
FLUX = {"central": 0, "upwind": 1, "lf": 2}


def _sigs():
    L = lib()
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    sigs = {
        "drf_mortar_ops": [C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, ip],
        "drf_mortar_create": [C.c_int, C.c_int64, vp, vp, vp, vp, vp, C.c_int64, C.POINTER(vp)],
        "drf_mortar_destroy": [vp], "drf_mortar_set_stream": [vp, vp],
        "drf_mortar_apply": [vp, C.c_int, dp, dp, dp],
        "drf_mortar_apply_device": [vp, C.c_int, dp, vp, vp],
    }
    for k, a in sigs.items():
        getattr(L, k).argtypes = a
        getattr(L, k).restype = C.c_int
    return L


def mortar_ops(order: int, ctype: int) -> dict:
    """M, M^-1, P_c, L_c and the per-fine-face P_f, L_f of one connection type."""
    L = _sigs()
    nm = (order + 1) ** 2
    nfine = NUM_FINE[ctype]
    M, Minv, Pc, Lc = (np.empty((nm, nm)) for _ in range(4))
    Pf, Lf = np.empty((nfine, nm, nm)), np.empty((nfine, nm, nm))
    nf = C.c_int()
    check(L.drf_mortar_ops(order, ctype, dptr(M), dptr(Minv), dptr(Pc), dptr(Lc), dptr(Pf),
                           dptr(Lf), C.byref(nf)))
    return dict(M=M, Minv=Minv, Pc=Pc, Lc=Lc, Pf=Pf, Lf=Lf)


class MortarInterfaceManager:
    """The non-conforming interfaces of a mesh of n_elem hexahedra of order p and their mortar
    operators (MortarInterfaceManager, include/dg/mortar.hpp:145); apply() adds the mortar
    flux lifts of every interface to a right-hand side."""

    def __init__(self, order: int, ifaces, n_elem: int):
        L = _sigs()
        n = len(ifaces)
        self.order, self.n_elem = order, n_elem
        t = np.zeros(n, np.int32)
        ce = np.zeros(n, np.int64)
        cf = np.zeros(n, np.int32)
        fe = -np.ones((n, 4), np.int64)
        ff = -np.ones((n, 4), np.int32)
        for i, (ty, e, f, fes, ffs) in enumerate(ifaces):
            t[i], ce[i], cf[i] = ty, e, f
            fe[i, :len(fes)] = fes
            ff[i, :len(ffs)] = ffs
        self._keep = (t, ce, cf, fe, ff)
        h = C.c_void_p()
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        check(L.drf_mortar_create(order, n, ptr(t), ptr(ce), ptr(cf), ptr(fe), ptr(ff), n_elem,
                                  C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().drf_mortar_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        check(lib().drf_mortar_set_stream(self.h, C.c_void_p(stream_ptr)))

    def apply(self, U, a, flux="lf", rhs=None):
        """rhs (zeros by default) + the lifted mortar fluxes for the scalar field U
        (n_elem x (p+1)^3) advected with velocity a."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = np.zeros_like(U) if rhs is None else np.array(rhs, dtype=np.float64)
        av = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().drf_mortar_apply(self.h, FLUX[flux], dptr(av), dptr(U), dptr(out)))
        return out

    def apply_device(self, d_U: int, d_rhs: int, a, flux="lf"):
        """Enqueue rhs += lifts on device buffers (raw device pointers)."""
        av = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().drf_mortar_apply_device(self.h, FLUX[flux], dptr(av), C.c_void_p(d_U),
                                            C.c_void_p(d_rhs)))
