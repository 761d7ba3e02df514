"""Config C2 (the benched workload) against the FP64 oracle: 128 x 128 x 16 hexes, N = 4,
200 x 200 km, depth 20 m + 32 seeded Gaussians clipped to [20, 2000] m, M2 tide of 1 m on the
west side, linear temperature stratification (which drives the baroclinic pressure gradient),
20 barotropic subcycles per step.

- The FP64 GPU step equals the oracle at full size (2 steps; the oracle's 3D right-hand side
  runs on the host's threads) to 1e-9 relative, and to 1e-8 with the baroclinic pressure
  gradient on.
- The mixed-precision surface elevation is within 1e-6 of the FP64 oracle over the config's
  500 steps on the same physics cut to 16 x 16 x 16 hexes over 25 km, with C2's seamount widths
  (and so its slopes) kept (the full size is compared against the FP64 GPU form over 500 steps
  in bench.py).
"""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs
from drifter_b200.dg import OceanModel

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _pair(case):
    cfg = case["cfg"]
    gpu = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    gpu.upload_state(case["q"], case["eta"])
    ref = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    ref.set_state(case["q"], case["eta"])
    return gpu, ref


@pytest.mark.parametrize("baroclinic", [False, True])
def test_c2_full_size_fp64_step_matches_oracle(baroclinic):
    """Both forms of C2: the benched one (stratification passive) and the one with the
    baroclinic pressure gradient on. At full size (409,600 surface nodes, 2000 m columns) the
    FP64 summation orders of the GPU and the oracle differ by 2.4e-10 of eta after two steps
    (1e-9 tolerance); with the pressure gradient, whose force is a difference of nearly equal
    products over 2000 m columns, by 1.0e-9 of HU (1e-8 tolerance)."""
    case = configs.c2(precision="fp64", baroclinic=baroclinic)
    gpu, ref = _pair(case)
    gpu.step(case["dt"], case["nsub"], 2)
    ref.split_steps(case["dt"], case["nsub"], 2)
    g, r = gpu.download_state(), ref.get_state()
    assert np.abs(r["eta"]).max() > 1e-3  # the tide has come in
    assert np.abs(r["Hu"]).max() > 1e-3  # and the flow moves
    tol = 1e-8 if baroclinic else 1e-9
    for k in ("eta", "eta_avg", "HT", "HS"):
        assert relerr(g[k], r[k]) < tol, (k, relerr(g[k], r[k]))
    # transports as vectors: the cross-basin component is small after two tidal steps, so each
    # pair is measured against the larger of its components
    for a, b in (("HU", "HV"), ("Hu", "Hv")):
        den = max(np.abs(r[a]).max(), np.abs(r[b]).max())
        for k in (a, b):
            assert np.abs(g[k] - r[k]).max() / den < tol, (k, np.abs(g[k] - r[k]).max() / den)
    gpu.close()


def test_c2_physics_mixed_eta_within_1e6_of_oracle_over_500_steps():
    case = configs.c2(nx=16, ny=16, nz=16, precision="mixed", Lx=25e3, wscale=1.0)
    gpu, ref = _pair(case)
    steps = case["steps"]
    assert steps == 500
    gpu.step(case["dt"], case["nsub"], steps)
    ref.split_steps(case["dt"], case["nsub"], steps)
    g, r = gpu.download_state(), ref.get_state()
    err = np.linalg.norm(g["eta"] - r["eta"]) / np.linalg.norm(r["eta"])
    assert np.abs(r["eta"]).max() > 0.1  # 500 steps of the M2 tide
    assert err <= 1e-6, err
    gpu.close()
