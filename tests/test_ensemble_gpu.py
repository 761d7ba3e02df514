"""Uneven ensembles (C5 layout) on the GPU, through the C ABI.

An ensemble steps all members with one stage launch per LSRK stage and layer count and one launch
per barotropic pass over every member's tiles; each member must end where the same model stepped
alone ends (both evaluate the same formulas per node; the ensemble's barotropic kernels are
separately compiled instances, whose multiply-add fusion may differ, so they agree to 1e-11
relative), and an FP64 member must match the FP64 oracle to 1e-10 relative, the tolerance of
the single-model split-step test.
"""
import dataclasses

import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs, launch_count
from drifter_b200._abi import DrfError
from drifter_b200.dg import Ensemble, OceanModel

pytestmark = pytest.mark.gpu


def relerr(a, b):
    den = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / den


def _members(precision, sizes, order=3):
    cases = [configs.perturb(configs.c5_member(i, nx, ny, nz, order=order, precision=precision), seed=11 + i)
             for i, (nx, ny, nz) in enumerate(sizes)]
    # member 1 has an open tidal side, so the members' boundary tables differ too
    cases[1]["cfg"] = dataclasses.replace(cases[1]["cfg"], bc=("wall", "tide", "wall", "wall"),
                                          tide_amp=0.5, tide_period=30000.0)
    return cases


SIZES = [(5, 4, 3), (3, 6, 5), (7, 3, 2), (4, 4, 4)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_members_equal_single_runs(precision):
    cases = _members(precision, SIZES)
    ens = Ensemble(cases)
    for m, c in zip(ens.members, cases):
        m.upload_state(c["q"], c["eta"])
    dts = [c["dt"] for c in cases]
    ens.step(dts, 20, 0)  # captures the step graphs (their launches are counted at capture)
    before = launch_count()
    ens.step(dts, 20, 3)
    ens.sync()
    # per step: 5 stages, each one launch per layer count of the members, then force, 2 per
    # subcycle and finish, for all members together
    groups = len({c["cfg"].nz for c in cases})
    assert launch_count() - before == 3 * (5 * groups + 2 + 2 * 20)
    for m, c in zip(ens.members, cases):
        g = m.download_state()
        solo = OceanModel(c["cfg"], c["h"], c["f"], c["taux"], c["tauy"])
        solo.upload_state(c["q"], c["eta"])
        solo.step(c["dt"], 20, 3)
        s = solo.download_state()
        assert g["t"] == s["t"]
        # the ensemble and the single-model kernels inline the same column function, which the
        # compiler may contract differently: FP64 members agree to 1e-11, FP32-bulk members to
        # the FP32 rounding their three steps amplify (1e-5)
        tol = 1e-11 if precision == "fp64" else 1e-5
        for k in ("eta", "HU", "HV", "eta_avg", "Hu", "Hv", "HT", "HS"):
            assert relerr(g[k], s[k]) <= tol, (c["name"], k, relerr(g[k], s[k]))
        solo.close()
    ens.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_persistent_barotropic_agrees_with_per_pass_launches(monkeypatch, precision):
    """The ensemble's barotropic step as one cooperative launch over every member's tiles
    (DRIFTER_B200_BARO_PERSISTENT=1) agrees with the per-pass launches to rounding: the same
    formulas per node, in kernels the compiler may contract differently."""
    cases = _members(precision, SIZES)
    per = Ensemble(cases)
    for m, c in zip(per.members, cases):
        m.upload_state(c["q"], c["eta"])
    dts = [c["dt"] for c in cases]
    per.step(dts, 20, 3)
    monkeypatch.setenv("DRIFTER_B200_BARO_PERSISTENT", "1")
    pers = Ensemble(cases)
    for m, c in zip(pers.members, cases):
        m.upload_state(c["q"], c["eta"])
    pers.step(dts, 20, 0)
    before = launch_count()
    pers.step(dts, 20, 3)
    pers.sync()
    assert launch_count() - before == 3 * (5 * len({c["cfg"].nz for c in cases}) + 1)
    for ma, mb in zip(pers.members, per.members):
        a, b = ma.download_state(), mb.download_state()
        assert a["t"] == b["t"]
        for k in ("eta", "HU", "HV", "eta_avg", "Hu", "Hv", "HT", "HS"):
            assert relerr(a[k], b[k]) <= 1e-11, (k, relerr(a[k], b[k]))
    pers.close()
    per.close()


def test_ensemble_fp64_member_matches_oracle():
    cases = _members("fp64", SIZES[:3])
    ens = Ensemble(cases)
    for m, c in zip(ens.members, cases):
        m.upload_state(c["q"], c["eta"])
    ens.step([c["dt"] for c in cases], 20, 2)
    c = cases[1]
    ref = O.PhysOracle(c["cfg"], c["h"], c["f"], c["taux"], c["tauy"])
    ref.set_state(c["q"], c["eta"])
    ref.split_steps(c["dt"], 20, 2)
    g, r = ens.members[1].download_state(), ref.get_state()
    assert abs(g["t"] - r["t"]) < 1e-9
    for k in ("eta", "HU", "HV", "Hu", "Hv", "HT", "HS"):
        assert relerr(g[k], r[k]) < 1e-10, k
    ens.close()


def test_ensemble_download_between_steps_and_diagnostics():
    """Reading a member back (which folds its pending transport correction in) between
    ensemble steps leaves the trajectory unchanged."""
    cases = _members("mixed", SIZES[:2])
    a, b = Ensemble(cases), Ensemble(cases)
    for e in (a, b):
        for m, c in zip(e.members, cases):
            m.upload_state(c["q"], c["eta"])
    dts = [c["dt"] for c in cases]
    a.step(dts, 20, 2)
    b.step(dts, 20, 1)
    b.members[0].download_state()
    d = b.members[1].diagnostics()
    assert np.isfinite(list(d.values())).all()
    b.step(dts, 20, 1)
    for ma, mb in zip(a.members, b.members):
        sa, sb = ma.download_state(), mb.download_state()
        for k in ("eta", "Hu", "HT"):
            assert relerr(sb[k], sa[k]) <= 1e-15, k
    a.close()
    b.close()


def test_ensemble_rejects_member_stepping_and_bad_mixes():
    cases = _members("mixed", SIZES[:2])
    ens = Ensemble(cases)
    with pytest.raises(DrfError):
        ens.members[0].step(cases[0]["dt"], 4, 1)
    with pytest.raises(DrfError):
        ens.step([cases[0]["dt"], -1.0], 4, 1)
    with pytest.raises(ValueError):
        ens.step([cases[0]["dt"]], 4, 1)
    ens.close()
    mixed = [cases[0], configs.c5_member(5, 3, 3, 2, precision="fp64")]
    with pytest.raises(DrfError):
        Ensemble(mixed)
    other_order = [cases[0], configs.c5_member(6, 3, 3, 2, order=4, precision="mixed")]
    with pytest.raises(DrfError):
        Ensemble(other_order)


def test_models_of_different_orders_coexist():
    """The basis tables are kept per order: a model of order 4 created after one of order 3
    does not change the older model's results."""
    c3 = configs.perturb(configs.c5_member(0, 4, 3, 2, order=3, precision="fp64"))
    ref = OceanModel(c3["cfg"], c3["h"], c3["f"], c3["taux"], c3["tauy"])
    ref.upload_state(c3["q"], c3["eta"])
    ref.step(c3["dt"], 20, 1)
    r = ref.download_state()
    m3 = OceanModel(c3["cfg"], c3["h"], c3["f"], c3["taux"], c3["tauy"])
    c4 = configs.perturb(configs.c5_member(1, 3, 3, 2, order=4, precision="fp64"))
    m4 = OceanModel(c4["cfg"], c4["h"], c4["f"], c4["taux"], c4["tauy"])
    m4.upload_state(c4["q"], c4["eta"])
    m4.step(c4["dt"], 20, 1)
    m3.upload_state(c3["q"], c3["eta"])
    m3.step(c3["dt"], 20, 1)
    g = m3.download_state()
    for k in ("eta", "Hu", "HT"):
        assert relerr(g[k], r[k]) <= 1e-15, k


def test_models_of_different_heights_coexist():
    """The stage kernel's shared-memory limit is shared by all models: a model with short
    columns created after one with tall columns must not stop the tall one from launching."""
    tall = configs.c5_member(0, 3, 3, 8, precision="mixed")
    short = configs.c5_member(1, 3, 3, 2, precision="mixed")
    mt = OceanModel(tall["cfg"], tall["h"], tall["f"], tall["taux"], tall["tauy"])
    ms = OceanModel(short["cfg"], short["h"], short["f"], short["taux"], short["tauy"])
    for m, c in ((mt, tall), (ms, short)):
        m.upload_state(c["q"], c["eta"])
    mt.step(tall["dt"], 20, 1)
    ms.step(short["dt"], 20, 1)
    assert np.isfinite(mt.download_state()["eta"]).all()
