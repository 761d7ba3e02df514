"""DG3DIntegration (include/dg/operators_3d.hpp:153) on directionally refined hexahedral meshes
over the C ABI: compute_rhs (src/dg/operators_3d.cpp:228) of the scalar conservation law
u_t + div(a u) = 0, with the non-conforming faces coupled by mortars, and an LSRK45 stepper
whose steps are CUDA graphs. All compute runs in libdrifter_b200.so on the GPU."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._abi import check, dptr, lib
from .mortar import FLUX

MODES = {"reference": 0, "complete": 1}


def _sigs():
    L = lib()
    vp, dp, i64 = C.c_void_p, C.POINTER(C.c_double), C.c_int64
    sigs = {
        "drf_amr_create": [C.c_int, i64, i64, vp, i64, vp, i64, vp, vp, vp, vp, vp, C.POINTER(vp)],
        "drf_amr_destroy": [vp], "drf_amr_set_stream": [vp, vp], "drf_amr_sync": [vp],
        "drf_amr_compute_rhs": [vp, C.c_int, C.c_int, dp, dp, dp],
        "drf_amr_upload": [vp, dp], "drf_amr_download": [vp, dp],
        "drf_amr_step": [vp, C.c_int, C.c_int, dp, C.c_double, C.c_int],
        "drf_amr_time_rhs": [vp, C.c_int, C.c_int, dp, C.c_int, dp, dp],
        "drf_amr_build_mesh": [C.c_int, C.c_int, vp, vp, vp, C.c_double, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                               vp, vp, vp],
        "drf_amr_estimate": [vp, dp, C.c_double, C.c_double, C.c_double, dp, vp, vp],
        "drf_amr_refine_levels": [C.c_int, C.c_int, vp, vp, vp, i64, vp, vp, C.c_int, C.c_int, vp, vp, vp, vp],
        "drf_amr_transfer": [vp, vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp],
    }
    for k, a in sigs.items():
        getattr(L, k).argtypes = a
        getattr(L, k).restype = C.c_int
    return L


def build_mesh(lx, ly, lz, L: float = 1.0) -> dict:
    """Elements and face connections of a column-wise directionally refined mesh from the
    native builder (drf_amr_build_mesh, the producer of OctreeAdapter::build_face_connections'
    tables, src/mesh/octree_adapter.cpp:369). lx, ly, lz: (ny, nx) per-column levels. Returns
    the dict of configs.amr_mesh (n_elem, level, box, conf, bnd, ifaces, col_levels) plus the
    interfaces as the arrays drf_amr_create takes ("if_arrays")."""
    Lb = _sigs()
    lx, ly, lz = (np.ascontiguousarray(a, np.int32) for a in (lx, ly, lz))
    ny, nx = lx.shape
    ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
    cnt = [C.c_int64() for _ in range(4)]
    args = [nx, ny, ptr(lx), ptr(ly), ptr(lz), float(L)] + [C.c_void_p(C.addressof(c)) for c in cnt]
    check(Lb.drf_amr_build_mesh(*args, *([None] * 9)))
    ne, nc, nb, ni = (c.value for c in cnt)
    level = np.zeros((ne, 3), np.int32)
    box = np.zeros((ne, 6))
    conf = np.zeros((nc, 4), np.int64)
    bnd = np.zeros((nb, 2), np.int64)
    t = np.zeros(ni, np.int32)
    ce = np.zeros(ni, np.int64)
    cf = np.zeros(ni, np.int32)
    fe = np.zeros((ni, 4), np.int64)
    ff = np.zeros((ni, 4), np.int32)
    check(Lb.drf_amr_build_mesh(*args, ptr(level), ptr(box), ptr(conf), ptr(bnd), ptr(t), ptr(ce), ptr(cf),
                                ptr(fe), ptr(ff)))
    ifaces = [(int(t[i]), int(ce[i]), int(cf[i]), [int(v) for v in fe[i] if v >= 0],
               [int(v) for v in ff[i] if v >= 0]) for i in range(ni)]
    col_levels = np.stack([lx.ravel(), ly.ravel(), lz.ravel()], 1).astype(np.int64)
    return dict(n_elem=ne, level=level.astype(np.int64), box=box, conf=conf, bnd=bnd, ifaces=ifaces,
                col_levels=col_levels, if_arrays=(t, ce, cf, fe, ff))


class DG3DIntegration:
    """The reference class's compute_rhs for one mesh (the dict of configs.amr_mesh: elements,
    conforming pairs, boundary faces and non-conforming interfaces) at polynomial order N."""

    def __init__(self, order: int, mesh: dict):
        L = _sigs()
        self.order, self.n_elem = order, int(mesh["n_elem"])
        self.nd = (order + 1) ** 3
        conf = np.ascontiguousarray(mesh["conf"], np.int64).reshape(-1, 4)
        bnd = np.ascontiguousarray(mesh["bnd"], np.int64).reshape(-1, 2)
        if "if_arrays" in mesh:  # the native builder's arrays
            t, ce, cf, fe, ff = (np.ascontiguousarray(a) for a in mesh["if_arrays"])
            n = len(t)
        else:
            ifs = mesh["ifaces"]
            n = len(ifs)
            t = np.zeros(n, np.int32)
            ce = np.zeros(n, np.int64)
            cf = np.zeros(n, np.int32)
            fe = -np.ones((n, 4), np.int64)
            ff = -np.ones((n, 4), np.int32)
            for i, (ty, e, f, fes, ffs) in enumerate(ifs):
                t[i], ce[i], cf[i] = ty, e, f
                fe[i, :len(fes)] = fes
                ff[i, :len(ffs)] = ffs
        self._keep = (conf, bnd, t, ce, cf, fe, ff)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        h = C.c_void_p()
        check(L.drf_amr_create(order, self.n_elem, len(conf), ptr(conf), len(bnd), ptr(bnd), n, ptr(t),
                               ptr(ce), ptr(cf), ptr(fe), ptr(ff), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().drf_amr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(lib().drf_amr_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def sync(self):
        check(lib().drf_amr_sync(self.h))

    def compute_rhs(self, U, a, flux: str = "lf", mode: str = "reference") -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.n_elem, self.nd)
        out = np.empty_like(U)
        av = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().drf_amr_compute_rhs(self.h, MODES[mode], FLUX[flux], dptr(av), dptr(U), dptr(out)))
        return out

    def upload(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.n_elem, self.nd)
        check(lib().drf_amr_upload(self.h, dptr(U)))

    def download(self) -> np.ndarray:
        out = np.empty((self.n_elem, self.nd))
        check(lib().drf_amr_download(self.h, dptr(out)))
        return out

    def step(self, a, dt: float, nsteps: int = 1, flux: str = "lf", mode: str = "reference"):
        """nsteps LSRK45 steps of du/dt = -compute_rhs(u), each one CUDA graph."""
        av = np.ascontiguousarray(a, dtype=np.float64)
        check(lib().drf_amr_step(self.h, MODES[mode], FLUX[flux], dptr(av), dt, nsteps))

    def time_rhs(self, a, nrep: int = 20, flux: str = "lf", mode: str = "reference") -> dict:
        av = np.ascontiguousarray(a, dtype=np.float64)
        ms, ab = C.c_double(), C.c_double()
        check(lib().drf_amr_time_rhs(self.h, MODES[mode], FLUX[flux], dptr(av), nrep, C.byref(ms),
                                     C.byref(ab)))
        return dict(ms=ms.value, alg_bytes=ab.value)


@dataclass
class RefinementParams:
    """RefinementParams (include/amr/refinement.hpp:63)."""
    refine_threshold: float = 0.1
    coarsen_threshold: float = 0.01
    max_level: int = 8
    min_level: int = 0
    smoothness_factor: float = 0.5


def _iptr(a):
    return a.ctypes.data_as(C.c_void_p)


def element_lengths(mesh: dict) -> np.ndarray:
    """Characteristic length cbrt(volume) of every element (estimate_element's h,
    src/amr/refinement.cpp:84-87), from the mesh's element boxes."""
    b = np.asarray(mesh["box"], dtype=np.float64)
    return np.cbrt((b[:, 3] - b[:, 0]) * (b[:, 4] - b[:, 1]) * (b[:, 5] - b[:, 2]))


class AdaptiveMeshRefinement:
    """AdaptiveMeshRefinement (include/amr/refinement.hpp, src/amr/refinement.cpp:413) for the
    column-wise refined meshes of build_mesh: the gradient estimator on the GPU, the column
    levels (marking, refine / coarsen and 2:1 balance) on the host, the face tables rebuilt by
    the native builder and the solution carried over on the GPU."""

    def __init__(self, order: int, params: RefinementParams | None = None):
        self.order = order
        self.params = params or RefinementParams()

    def estimate(self, model: DG3DIntegration, mesh: dict):
        """GradientErrorEstimator::estimate of the model's device state: (value, mask, flags)."""
        Lb = _sigs()
        p = self.params
        hchar = np.ascontiguousarray(element_lengths(mesh))
        ne = model.n_elem
        val = np.zeros(ne)
        mask = np.zeros(ne, np.int32)
        flags = np.zeros(ne, np.int32)
        check(Lb.drf_amr_estimate(model.h, dptr(hchar), p.refine_threshold, p.coarsen_threshold,
                                  p.smoothness_factor, dptr(val), _iptr(mask), _iptr(flags)))
        return val, mask, flags

    def refine_levels(self, levels, mask, flags):
        """New per-column levels (lx, ly, lz as (ny, nx) arrays) from the element marks, with the
        number of columns that changed."""
        Lb = _sigs()
        lx, ly, lz = (np.ascontiguousarray(a, np.int32) for a in levels)
        ny, nx = lx.shape
        out = [np.zeros_like(lx) for _ in range(3)]
        ch = C.c_int()
        mask = np.ascontiguousarray(mask, np.int32)
        flags = np.ascontiguousarray(flags, np.int32)
        check(Lb.drf_amr_refine_levels(nx, ny, _iptr(lx), _iptr(ly), _iptr(lz), len(mask), _iptr(mask),
                                       _iptr(flags), self.params.max_level, self.params.min_level,
                                       *[_iptr(a) for a in out], C.byref(ch)))
        return tuple(out), ch.value

    def transfer(self, old: DG3DIntegration, new: DG3DIntegration, old_levels, new_levels):
        """The device state of `old` carried into `new` (transfer_solution with the projections)."""
        Lb = _sigs()
        ol = [np.ascontiguousarray(a, np.int32) for a in old_levels]
        nl = [np.ascontiguousarray(a, np.int32) for a in new_levels]
        ny, nx = ol[0].shape
        check(Lb.drf_amr_transfer(old.h, new.h, nx, ny, *[_iptr(a) for a in ol], *[_iptr(a) for a in nl]))

    def adapt(self, model: DG3DIntegration, mesh: dict, levels, L: float = 1.0):
        """One adaptation (AdaptiveMeshRefinement::adapt, src/amr/refinement.cpp:422): returns
        (model, mesh, levels, columns changed); the model is a new one on the new mesh holding the
        carried-over state, or the same one when nothing changed."""
        _, mask, flags = self.estimate(model, mesh)
        new_levels, changed = self.refine_levels(levels, mask, flags)
        if changed == 0:
            return model, mesh, levels, 0
        new_mesh = build_mesh(*new_levels, L=L)
        new_model = DG3DIntegration(self.order, new_mesh)
        self.transfer(model, new_model, levels, new_levels)
        return new_model, new_mesh, new_levels, changed
