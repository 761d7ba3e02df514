"""CPU-side checks of the C ABI: the library loads, exports every symbol include/*.h declares,
and rejects bad arguments with status codes before touching the GPU."""
import ctypes as C
import os

import numpy as np
import pytest

from drifter_b200 import _abi
from drifter_b200._abi import DrfError, check, dptr, dptr_array, lib


def test_library_loads_and_exports_all_declared_symbols():
    L = lib()
    declared = _abi.declared_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if getattr(L, s, None) is None]
    assert not missing, missing
    assert b"sm_100a" in L.drf_version()


def test_header_declarations_are_cited():
    # every entry point of the drop-in boundary cites the reference interface it replaces
    # (or states that it has none)
    text = open(os.path.join(os.path.dirname(_abi.HERE), "include", "drifter_b200.h")).read()
    assert "include/physics/mode_splitting.hpp:241" in text
    assert "include/physics/primitive_equations.hpp:240" in text
    assert "include/flux/numerical_flux.hpp:25" in text


def test_invalid_arguments_return_status_without_gpu():
    L = lib()
    nd = 64
    arrs = [np.zeros((1, nd)) for _ in range(12)]
    h = np.full((1, nd), 10.0)
    f = np.zeros((1, nd))
    p = np.array([9.81, 1025, 2e-4, 7.6e-4, 1, 1e-4, 1e-5, 1e-5])
    # nsub = 0 -> invalid (the reference would divide by zero)
    rc = L.drf_compat_modesplit_step(3, 1, 1.0, 0, dptr_array(arrs), dptr(h), dptr(f), dptr(p))
    assert rc == 1
    with pytest.raises(DrfError, match="nsub"):
        check(rc)
    # order out of range -> unsupported
    rc = L.drf_compat_compute_rhs(9, 1, dptr_array(arrs[:6]), dptr(h), dptr(f), dptr(p),
                                  dptr_array(arrs[6:11]))
    assert rc == 5
    # empty mesh -> invalid
    mesh = _abi.MeshDesc(0, 4, 2, 3, 1e3, 1e3)
    prm = _abi.DGParams()
    hd = C.c_void_p()
    z = np.zeros(10)
    rc = L.drf_dg_create(C.byref(mesh), C.byref(prm), dptr(z), dptr(z), dptr(z), dptr(z),
                         C.byref(hd))
    assert rc == 1 and not hd.value
    # null handle
    assert L.drf_dg_sync(None) == 1
    assert L.drf_dg_step_modesplit(None, 1.0, 1, 1) == 1


def test_nonfinite_input_rejected_without_gpu():
    L = lib()
    nd = 27
    arrs = [np.zeros((1, nd)) for _ in range(12)]
    arrs[0][0, 3] = np.nan
    h = np.full((1, nd), 10.0)
    f = np.zeros((1, nd))
    p = np.array([9.81, 1025, 2e-4, 7.6e-4, 1, 1e-4, 1e-5, 1e-5])
    rc = L.drf_compat_modesplit_step(2, 1, 1.0, 2, dptr_array(arrs), dptr(h), dptr(f), dptr(p))
    assert rc == 4
