"""ctypes binding of libdrifter_b200.so (the C ABI declared in include/drifter_b200.h).

The shared library is built in-tree (drifter_b200/libdrifter_b200.so). Loading fails loudly
when it is missing: there is no CPU fallback for any operator of this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdrifter_b200.so")

DRF_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "non-finite value", 5: "unsupported", 6: "timeout"}

FLUX = {"lf": 0, "hllc": 1, "roe": 2}
PREC = {"fp64": 0, "mixed": 1}
BC = {"wall": 0, "tide": 1}
RK = {"euler": 0, "midpoint": 1, "ssp3": 2, "rk4": 3, "lsrk45": 4, "dopri": 5}

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)


class DrfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"drifter_b200 error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("order", C.c_int32),
                ("Lx", C.c_double), ("Ly", C.c_double)]


class DGParams(C.Structure):
    _fields_ = [("g", C.c_double), ("rho0", C.c_double), ("nu_h", C.c_double),
                ("nu_v", C.c_double), ("kappa_v_T", C.c_double), ("kappa_v_S", C.c_double),
                ("cd", C.c_double), ("flux2d", C.c_int32), ("precision", C.c_int32),
                ("bc", C.c_int32 * 4), ("tide_amp", C.c_double), ("tide_period", C.c_double),
                ("alpha", C.c_double), ("beta", C.c_double), ("T0", C.c_double), ("S0", C.c_double),
                ("Tref_s", C.c_double), ("Tref_dz", C.c_double)]


_lib = None

# (name, restype, argtypes) of every exported symbol this binding uses
_SIGS = {
    "drf_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "drf_version": (C.c_char_p, []),
    "drf_kernel_launch_count": (C.c_uint64, []),
    "drf_device_alloc_count": (C.c_uint64, []),
    "drf_sw_flux_batch": (C.c_int, [C.c_int, C.c_int64, _dp, _dp, _dp, C.c_double, _dp]),
    "drf_compat_compute_rhs": (C.c_int, [C.c_int, C.c_int, C.POINTER(_dp), _dp, _dp, _dp,
                                         C.POINTER(_dp)]),
    "drf_compat_time_rhs": (C.c_int, [C.c_int, C.c_int, C.POINTER(_dp), _dp, _dp, _dp, C.c_int,
                                      C.c_int, _dp]),
    "drf_compat_modesplit_step": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_int,
                                            C.POINTER(_dp), _dp, _dp, _dp]),
    "drf_dg_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(DGParams), _dp, _dp, _dp, _dp,
                                C.POINTER(C.c_void_p)]),
    "drf_dg_destroy": (C.c_int, [C.c_void_p]),
    "drf_dg_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "drf_dg_sync": (C.c_int, [C.c_void_p]),
    "drf_dg_upload_state": (C.c_int, [C.c_void_p, C.POINTER(_dp), _dp, C.c_double]),
    "drf_dg_download_state": (C.c_int, [C.c_void_p, C.POINTER(_dp), _dp, _dp, _dp, _dp, _dp]),
    "drf_dg_output_stage": (C.c_int, [C.c_void_p, C.POINTER(_dp), _dp, _dp, _dp]),
    "drf_dg_output_wait": (C.c_int, [C.c_void_p, _dp]),
    "drf_dg_compute_rhs": (C.c_int, [C.c_void_p, C.POINTER(_dp), _dp, _dp]),
    "drf_dg_compute_rhs2d": (C.c_int, [C.c_void_p, _dp, _dp, C.c_double, _dp, _dp, _dp]),
    "drf_dg_step_modesplit": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int]),
    "drf_dg_rk_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int]),
    "drf_dg_diagnostics": (C.c_int, [C.c_void_p, _dp]),
    "drf_dg_time_stage": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp]),
    "drf_dg_set_forcing": (C.c_int, [C.c_void_p, _dp, _dp]),
    "drf_dg_download_surface": (C.c_int, [C.c_void_p, _dp]),
    "drf_dg_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                              C.POINTER(C.c_int)]),
    "drf_dg_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), _dp]),
    "drf_dg_stage_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
    "drf_dg_time_copy": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "drf_ens_create": (C.c_int, [C.c_int, C.POINTER(MeshDesc), C.POINTER(DGParams),
                                 C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp),
                                 C.POINTER(C.c_void_p)]),
    "drf_ens_destroy": (C.c_int, [C.c_void_p]),
    "drf_ens_member": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "drf_ens_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "drf_ens_sync": (C.c_int, [C.c_void_p]),
    "drf_ens_step": (C.c_int, [C.c_void_p, _dp, C.c_int, C.c_int]),
    "drf_ens_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                               C.POINTER(C.c_int)]),
}


def lib() -> C.CDLL:
    """Loads the CUDA library (once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m drifter_b200.build` "
                              "(the package has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols(header: str | None = None) -> list[str]:
    """Function names declared in include/*.h (used to check the exports)."""
    import re
    import glob
    inc = os.path.join(HERE, "..", "include")
    names = []
    for h in sorted(glob.glob(os.path.join(inc, "*.h"))) if header is None else [header]:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(drf_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def check(code: int) -> None:
    if code != DRF_OK:
        buf = C.create_string_buffer(1024)
        lib().drf_last_error(buf, 1024)
        raise DrfError(code, buf.value.decode(errors="replace"))


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "expected contiguous float64"
    return a.ctypes.data_as(_dp)


def dptr_array(arrs):
    return (_dp * len(arrs))(*[dptr(a) if a is not None else _dp() for a in arrs])


def launch_count() -> int:
    return int(lib().drf_kernel_launch_count())


def alloc_count() -> int:
    """Device allocations (cudaMalloc) the library has made since it was loaded."""
    return int(lib().drf_device_alloc_count())
