"""C3 on the GPU through the C ABI: DG3DIntegration::compute_rhs (src/dg/operators_3d.cpp:228)
on the seeded AMR mesh against the FP64 oracle, in the reference's semantics (mode 0) and with
conforming and boundary faces (mode 1), and the LSRK45 step (one CUDA graph per step).
Tolerance: 1e-12 relative to the field's largest magnitude (the GPU applies the volume
quadrature sum-factorized, the oracle point by point)."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs, launch_count
from drifter_b200._abi import DrfError
from drifter_b200.amr import DG3DIntegration

pytestmark = pytest.mark.gpu

FLUXES = {"central": 0, "upwind": 1, "lf": 2}


def relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def small():
    return configs.c3(nb=8)


@pytest.mark.parametrize("mode", ["reference", "complete"])
@pytest.mark.parametrize("flux", ["central", "upwind", "lf"])
def test_compute_rhs_matches_oracle(small, mode, flux):
    c = small
    gpu = DG3DIntegration(c["order"], c["mesh"])
    g = gpu.compute_rhs(c["U"], c["a"], flux=flux, mode=mode)
    r = O.amr_rhs(c["order"], c["mesh"], {"reference": 0, "complete": 1}[mode], FLUXES[flux], c["a"], c["U"])
    assert relerr(g, r) < 1e-12
    gpu.close()


@pytest.mark.parametrize("order", [1, 2, 4, 5])
def test_compute_rhs_other_orders(order):
    c = configs.c3(nb=6, order=order)
    gpu = DG3DIntegration(order, c["mesh"])
    rng = np.random.default_rng(order)
    U = rng.standard_normal(c["U"].shape)
    for mode in (0, 1):
        g = gpu.compute_rhs(U, c["a"], flux="lf", mode=("reference", "complete")[mode])
        r = O.amr_rhs(order, c["mesh"], mode, 2, c["a"], U)
        assert relerr(g, r) < 1e-12, mode


def test_c3_full_size_rhs_matches_oracle():
    """C3 in full: the 256 x 256 base grid refined to the coastline (about 2.6e5 hexes)."""
    c = configs.c3()
    assert 2.0e5 <= c["mesh"]["n_elem"] <= 3.0e5
    gpu = DG3DIntegration(c["order"], c["mesh"])
    g = gpu.compute_rhs(c["U"], c["a"], flux="lf", mode="complete")
    r = O.amr_rhs(c["order"], c["mesh"], 1, 2, c["a"], c["U"])
    assert relerr(g, r) < 1e-12
    gpu.close()


@pytest.mark.parametrize("mode", ["reference", "complete"])
def test_lsrk_steps_match_oracle(small, mode):
    c = small
    gpu = DG3DIntegration(c["order"], c["mesh"])
    gpu.upload(c["U"])
    dt = 2e-4
    gpu.step(c["a"], dt, 0, flux="upwind", mode=mode)  # captures the step graph
    before = launch_count()
    gpu.step(c["a"], dt, 3, flux="upwind", mode=mode)
    g = gpu.download()
    # per stage: the mortar face kernel, then volume, faces, mortar lifts and update in one kernel
    assert launch_count() - before == 3 * 5 * 2
    r = O.amr_lsrk(c["order"], c["mesh"], {"reference": 0, "complete": 1}[mode], 1, c["a"], c["U"], dt, 3)
    assert relerr(g, r) < 1e-12
    gpu.close()


def test_bad_inputs_are_rejected(small):
    m = small["mesh"]
    gpu = DG3DIntegration(3, m)
    with pytest.raises(DrfError):
        gpu.step(small["a"], -1.0, 1)
    bad = np.array(small["U"])
    bad[3, 5] = np.nan
    with pytest.raises(DrfError):
        gpu.compute_rhs(bad, small["a"])
    twice = dict(m)
    twice["bnd"] = np.concatenate([m["bnd"], m["bnd"][:1]])
    with pytest.raises(DrfError):
        DG3DIntegration(3, twice)
    gpu.close()
