"""GPU parity of the DG path against the FP64 oracle, through the C ABI.

Tolerances: FP64 kernels 1e-10 relative to the field's max magnitude (sum-factorized vs dense
products, FMA contraction); mixed precision (FP32 3D bulk) 2e-4 on 3D fields; the surface
elevation of the mixed run is held to the stated 1e-6 relative error against the FP64 oracle.
"""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs, launch_count
from drifter_b200.dg import ModeSplittingSolver, OceanModel, PrimitiveEquationsSolver, numerical_flux

pytestmark = pytest.mark.gpu


def relerr(a, b):
    den = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / den


# ---------------------------------------------------------------- fluxes
@pytest.mark.parametrize("kind", ["lf", "hllc", "roe"])
def test_flux_batch_matches_oracle(kind):
    rng = np.random.default_rng(3)
    n = 257
    UL = np.stack([rng.uniform(0.5, 3, n), rng.normal(0, 1, n), rng.normal(0, 1, n)], 1)
    UR = np.stack([rng.uniform(0.5, 3, n), rng.normal(0, 1, n), rng.normal(0, 1, n)], 1)
    UL[:8, 0] = 1e-12  # dry cells
    th = rng.uniform(0, 2 * np.pi, n)
    nr = np.stack([np.cos(th), np.sin(th)], 1)
    F = numerical_flux(kind, UL, UR, nr)
    ref = np.array([O.sw_flux(kind, UL[i], UR[i], nr[i, 0], nr[i, 1]) for i in range(n)])
    assert np.isfinite(F).all()
    # dry cells (h clamped to 1e-10) produce ~1e14 fluxes: rounding amplified to ~3e-12 relative
    np.testing.assert_allclose(F, ref, rtol=1e-10, atol=1e-12)


def test_flux_batch_empty():
    assert numerical_flux("lf", np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 2))).shape == (0, 3)


# ---------------------------------------------------------------- reference-semantics DG
def _compat_state(order, nel, seed=1):
    rng = np.random.default_rng(seed)
    nd = (order + 1) ** 3
    h = 100.0 + rng.uniform(0, 20, (nel, nd))
    f = 1e-4 + 1e-6 * rng.standard_normal((nel, nd))
    eta = 0.1 * rng.standard_normal((nel, nd))
    H = eta + h
    u, v = 0.2 * rng.standard_normal((2, nel, nd))
    T = 10.0 + rng.standard_normal((nel, nd))
    S = 35.0 + 0.1 * rng.standard_normal((nel, nd))
    om = 1e-4 * rng.standard_normal((nel, nd))
    st = dict(Hu=H * u, Hv=H * v, eta=eta, HT=H * T, HS=H * S, H=H, u=u, v=v, T=T, S=S, omega=om,
              rho=np.zeros((nel, nd)))
    return st, h, f


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_compat_rhs_matches_oracle(order):
    st, h, f = _compat_state(order, 9)
    gpu = PrimitiveEquationsSolver(order, h, f).compute_rhs(st)
    ref = O.compat_rhs(order, st, h, f)
    for k in ref:
        assert relerr(gpu[k], ref[k]) < 1e-11, k


@pytest.mark.parametrize("order,nsub", [(2, 7), (3, 20), (4, 5)])
def test_compat_modesplit_matches_oracle(order, nsub):
    st, h, f = _compat_state(order, 6, seed=order)
    # the reference's isolated-element barotropic solve is only stable for small reference-space
    # CFL (no inter-element coupling): dt = 0.05 s keeps c*dt_b/dxi << 1
    ref = O.compat_modesplit(order, 0.05, nsub, st, h, f)
    gst = {k: v.copy() for k, v in st.items()}
    ModeSplittingSolver(order, h, f, subcycles=nsub).step(0.05, gst)
    for k in ref:
        assert np.isfinite(ref[k]).all(), k
        assert relerr(gst[k], ref[k]) < 1e-11, k


def test_compat_empty_batch():
    st, h, f = _compat_state(3, 0)
    out = PrimitiveEquationsSolver(3, h, f).compute_rhs(st)
    assert out["dHu_dt"].shape == (0, 64)


# ---------------------------------------------------------------- coupled model
def _pair(case):
    cfg = case["cfg"]
    gpu = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    gpu.upload_state(case["q"], case["eta"])
    ref = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    ref.set_state(case["q"], case["eta"])
    return gpu, ref


def _tidal_small(precision, order=3, nx=5, ny=4, nz=3, flux2d="lf"):
    case = configs.c2(nx=nx, ny=ny, nz=nz, order=order, precision=precision, Lx=40e3, flux2d=flux2d,
                      baroclinic=True)
    case = configs.perturb(case)
    case["taux"][:] = 0.05
    return case


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_phys_rhs_fp64_matches_oracle(order):
    case = _tidal_small("fp64", order=order)
    gpu, ref = _pair(case)
    g, r = gpu.compute_rhs(), ref.rhs()
    assert relerr(g["omega"], r["omega"]) < 1e-10
    assert relerr(g["deta"], r["deta"]) < 1e-10
    for k in ("dHu", "dHv", "dHT", "dHS"):
        assert relerr(g[k], r[k]) < 1e-10, k


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-4)])
@pytest.mark.parametrize("order", [1, 4])
def test_baroclinic_pgf_of_a_front_is_exact_on_gpu(precision, tol, order):
    """Flat bed (H = 100 m), at rest, temperature T0 + gamma x through the whole column: the
    only tendency is the baroclinic force on Hu, -g H^2 alpha gamma sigma, exactly (the same
    case pins the oracle in test_oracle_dg.py)."""
    gamma = 1e-4
    cfg = configs.DGConfig(nx=6, ny=3, nz=3, order=order, Lx=20e3, Ly=10e3, precision=precision)
    X, Y, Sg = configs.node_coords(cfg)
    h = np.full(cfg.n2, 100.0)
    H3 = configs.expand_2d_to_3d(cfg, h)
    X3 = configs.expand_2d_to_3d(cfg, X)
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), (10.0 + gamma * X3) * H3, cfg.S0 * H3]
    z2 = np.zeros(cfg.n2)
    gpu = OceanModel(cfg, h, z2, z2, z2)
    gpu.upload_state(q, z2)
    r = gpu.compute_rhs()
    expect = -cfg.g * H3 ** 2 * cfg.alpha * gamma * Sg
    assert np.abs(r["dHu"] - expect).max() <= tol * np.abs(expect).max()
    assert np.abs(r["dHv"]).max() <= tol * np.abs(expect).max()
    gpu.close()


@pytest.mark.parametrize("baroclinic,tol", [(False, 2e-4), (True, 1e-3)])
def test_phys_rhs_mixed_matches_oracle(baroclinic, tol):
    """Mixed precision (FP32 3D state and arithmetic) against the FP64 oracle. With the
    baroclinic pressure on, the FP32 state limits the density anomaly: HS = 35 H rounds S to
    ~2e-6, i.e. the anomaly to ~1.5e-9, and the force differences the pressure of that anomaly
    across ~400 m; the momentum tendencies then hold 1e-3 instead of 2e-4."""
    case = _tidal_small("mixed", order=4)
    if not baroclinic:
        case["cfg"] = configs.DGConfig(**{**case["cfg"].__dict__, "alpha": 0.0, "beta": 0.0})
    gpu, ref = _pair(case)
    g, r = gpu.compute_rhs(), ref.rhs()
    for k in ("dHu", "dHv", "omega"):
        assert relerr(g[k], r[k]) < tol, (k, relerr(g[k], r[k]))


@pytest.mark.parametrize("flux2d", ["lf", "hllc", "roe"])
def test_phys_rhs2d_matches_oracle(flux2d):
    case = _tidal_small("fp64", flux2d=flux2d)
    gpu, ref = _pair(case)
    rng = np.random.default_rng(1)
    Fx, Fy = 1e-3 * rng.standard_normal((2, case["cfg"].n2))
    g = gpu.compute_rhs2d(Fx, Fy, 1234.5)
    r = ref.rhs2d(Fx, Fy, 1234.5)
    for a, b in zip(g, r):
        assert relerr(a, b) < 1e-11


@pytest.mark.parametrize("flux2d", ["lf", "hllc", "roe"])
def test_split_step_fp64_matches_oracle(flux2d):
    case = _tidal_small("fp64", flux2d=flux2d)
    gpu, ref = _pair(case)
    gpu.step(case["dt"], case["nsub"], 3)
    ref.split_steps(case["dt"], case["nsub"], 3)
    g, r = gpu.download_state(), ref.get_state()
    assert abs(g["t"] - r["t"]) < 1e-9
    for k in ("eta", "HU", "HV", "eta_avg"):
        assert relerr(g[k], r[k]) < 1e-10, k
    for k in ("Hu", "Hv", "HT", "HS"):
        assert relerr(g[k], r[k]) < 1e-10, k


def test_c1_mixed_eta_error_within_1e6():
    """C1 in full (16x16x4, N=3, 20 subcycles, 100 steps): mixed-precision surface elevation
    against the FP64 oracle; the target is <= 1e-6 relative."""
    case = configs.c1(precision="mixed")
    gpu, ref = _pair(case)
    gpu.step(case["dt"], case["nsub"], case["steps"])
    ref.split_steps(case["dt"], case["nsub"], case["steps"])
    g, r = gpu.download_state(), ref.get_state()
    err = np.linalg.norm(g["eta"] - r["eta"]) / np.linalg.norm(r["eta"])
    assert np.abs(r["eta"]).max() > 1e-4  # the wind has set up a surface slope
    assert err <= 1e-6, err
    # and the FP64 GPU form matches to rounding
    case64 = configs.c1(precision="fp64")
    g64 = OceanModel(case64["cfg"], case64["h"], case64["f"], case64["taux"], case64["tauy"])
    g64.upload_state(case64["q"], case64["eta"])
    g64.step(case64["dt"], case64["nsub"], case64["steps"])
    s64 = g64.download_state()
    assert np.linalg.norm(s64["eta"] - r["eta"]) / np.linalg.norm(r["eta"]) < 1e-9


@pytest.mark.parametrize("scheme", ["euler", "midpoint", "ssp3", "rk4", "lsrk45", "dopri"])
def test_rk_step_matches_oracle(scheme):
    case = _tidal_small("fp64", nx=3, ny=3, nz=2)
    gpu, ref = _pair(case)
    dt = case["dt"] / case["nsub"]
    gpu.rk_step(scheme, dt, 2)
    ref.rk_steps(scheme, dt, 2)
    g, r = gpu.download_state(), ref.get_state()
    for k in ("eta", "Hu", "Hv", "HT", "HU"):
        assert relerr(g[k], r[k]) < 1e-10, k


def test_diagnostics_match_oracle():
    case = _tidal_small("fp64")
    gpu, ref = _pair(case)
    gpu.step(case["dt"], case["nsub"], 2)
    ref.split_steps(case["dt"], case["nsub"], 2)
    g, r = gpu.diagnostics(), ref.diagnostics()
    for k in r:
        assert abs(g[k] - r[k]) <= 1e-10 * max(abs(r[k]), 1e-12), k


def test_lake_at_rest_stays_at_rest_on_gpu():
    case = configs.c1(nx=6, ny=5, nz=3)
    case["taux"][:] = 0.0
    gpu = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    gpu.upload_state(case["q"], case["eta"])
    before = launch_count()
    gpu.step(case["dt"], case["nsub"], 4)
    s = gpu.download_state()
    assert launch_count() > before
    assert np.abs(s["eta"]).max() < 1e-12 and np.abs(s["Hu"]).max() < 1e-8


def test_launch_count_counts_graph_replays_not_capture(monkeypatch):
    """Kernels queued while the step graphs are captured are not launches; each replay of a
    step graph counts its kernel nodes (5 stages, force, predictor and corrector per subcycle,
    finish)."""
    monkeypatch.setenv("DRIFTER_B200_TUNE", "0")
    case = configs.c1(nx=6, ny=5, nz=3)
    gpu = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    gpu.upload_state(case["q"], case["eta"])
    gpu.sync()
    before = launch_count()
    gpu.step(case["dt"], case["nsub"], 1)  # captures both step graphs, replays one
    gpu.sync()
    assert launch_count() - before == 5 + 2 + 2 * case["nsub"]
    gpu.close()


def test_time_stage_reports_positive_rate():
    case = configs.c1(nx=8, ny=8, nz=4, precision="mixed")
    gpu = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    gpu.upload_state(case["q"], case["eta"])
    r = gpu.time_stage(5)
    assert r["ms"] > 0 and r["alg_bytes"] > 0 and r["ndof"] == 4 * case["cfg"].n3


def test_autotuned_barotropic_tile_matches_default_tile(monkeypatch):
    """The autotuner picks one of the candidate tiles by timing; every tile does the same
    arithmetic per 2D node, so the tuned step equals the default-tile step exactly. The stage
    kernel's L2 prefetch distance is tuned too (0, 1/2 or 1 wave); a prefetch changes no
    arithmetic."""
    case = _tidal_small("fp64", nx=9, ny=7)
    tuned = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    tuned.upload_state(case["q"], case["eta"])
    tuned.step(case["dt"], case["nsub"], 2)
    t = tuned.tuning()
    assert t["baro_cols_per_cta"] in (2, 4, 8, 16)
    assert all(v > 0 for v in t["candidates_ms"].values())
    assert t["stage_prefetch_half_waves"] in (0, 1, 2)
    assert all(v > 0 for v in t["stage_candidates_ms"].values())
    monkeypatch.setenv("DRIFTER_B200_TUNE", "0")
    fixed = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    fixed.upload_state(case["q"], case["eta"])
    fixed.step(case["dt"], case["nsub"], 2)
    ft = fixed.tuning()
    assert ft["baro_cols_per_cta"] == 8 and ft["stage_prefetch_half_waves"] == 1
    a, b = tuned.download_state(), fixed.download_state()
    for k in ("eta", "HU", "HV", "Hu", "HT"):
        assert relerr(a[k], b[k]) <= 1e-15, k


@pytest.mark.parametrize("precision,flux2d,nsub", [("fp64", "lf", 20), ("fp64", "hllc", 1), ("fp64", "roe", 3),
                                                    ("mixed", "lf", 20)])
def test_persistent_barotropic_step_agrees_with_per_pass_launches(monkeypatch, precision, flux2d, nsub):
    """DRIFTER_B200_BARO_PERSISTENT=1 runs the barotropic step as ONE cooperative launch with
    grid barriers between its passes, in place of one launch per pass. Every node evaluates the
    same formulas in both forms; the two kernels are compiled separately, so the compiler may
    fuse a multiply-add in one and not the other. A face-flux difference F* - F(U-) cancels ~1e6
    of its terms' magnitude (0.5 g h^2 against the jump), which lifts such a rounding difference
    to ~1e-12 of eta after two HLLC steps: the states agree to 1e-11 relative (the oracle
    comparisons hold 1e-10). 128 x 128 columns give more tiles than CTAs at every tile size, so
    CTAs walk several tiles per pass. The substep is the case's (dt scaled with nsub), so the
    run stays stable."""
    case = configs.c2(nx=128, ny=128, nz=1, order=3, precision=precision, Lx=400e3, flux2d=flux2d)
    case = configs.perturb(case)
    case["dt"] = case["dt"] * nsub / case["nsub"]
    per = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    per.upload_state(case["q"], case["eta"])
    per.step(case["dt"], nsub, 0)  # builds the step graphs
    before = launch_count()
    per.step(case["dt"], nsub, 2)
    per.sync()
    assert launch_count() - before == 2 * (5 + 2 + 2 * nsub)
    monkeypatch.setenv("DRIFTER_B200_BARO_PERSISTENT", "1")
    pers = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    pers.upload_state(case["q"], case["eta"])
    pers.step(case["dt"], nsub, 0)
    before = launch_count()
    pers.step(case["dt"], nsub, 2)
    pers.sync()
    assert launch_count() - before == 2 * 6  # 5 stages + one barotropic launch per step
    a, b = pers.download_state(), per.download_state()
    assert a["t"] == b["t"] and np.abs(a["eta"]).max() < 10.0
    for k in ("eta", "HU", "HV", "eta_avg", "Hu", "Hv", "HT", "HS"):
        assert relerr(a[k], b[k]) <= 1e-11, (k, relerr(a[k], b[k]))


def test_bounded_grid_barrier_wait_gives_up_and_the_model_stays_usable(monkeypatch):
    """Failure detection without a GPU fault. With DRIFTER_B200_DEBUG_HOLD_ARRIVAL=0 the
    persistent barotropic launch's CTA 0 withholds its arrival at the first grid barrier, so no
    CTA's bounded wait there can complete: each gives up after its iteration limit (about a
    second), sets the abort word and the model's status word, and returns. The host reads
    DRF_E_TIMEOUT at the next synchronisation, which clears the status word. The context stays
    usable: a model built afterwards in the same process steps normally and agrees with the
    per-pass launches."""
    from drifter_b200 import DrfError
    case = _tidal_small("fp64", nx=9, ny=7)
    monkeypatch.setenv("DRIFTER_B200_BARO_PERSISTENT", "1")
    monkeypatch.setenv("DRIFTER_B200_DEBUG_HOLD_ARRIVAL", "0")
    held = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    held.upload_state(case["q"], case["eta"])
    held.step(case["dt"], case["nsub"], 1)
    with pytest.raises(DrfError) as ei:
        held.sync()
    assert ei.value.code == 6  # DRF_E_TIMEOUT
    held.sync()  # the status word was cleared
    held.close()
    monkeypatch.delenv("DRIFTER_B200_DEBUG_HOLD_ARRIVAL")
    pers = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    pers.upload_state(case["q"], case["eta"])
    pers.step(case["dt"], case["nsub"], 2)
    pers.sync()
    monkeypatch.delenv("DRIFTER_B200_BARO_PERSISTENT")
    per = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    per.upload_state(case["q"], case["eta"])
    per.step(case["dt"], case["nsub"], 2)
    a, b = pers.download_state(), per.download_state()
    assert a["t"] == b["t"]
    for k in ("eta", "HU", "Hu", "HT"):
        assert relerr(a[k], b[k]) <= 1e-11, (k, relerr(a[k], b[k]))
    pers.close()
    per.close()


def test_time_copy_leaves_the_state_unchanged():
    case = _tidal_small("mixed", order=4, nx=6, ny=4, nz=4)
    gpu = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    gpu.upload_state(case["q"], case["eta"])
    gpu.step(case["dt"], case["nsub"], 1)
    before = gpu.download_state()
    r = gpu.time_copy(3)
    assert r["ms"] > 0 and r["bytes"] == 16 * 4 * case["cfg"].n3
    after = gpu.download_state()
    for k in ("Hu", "HT", "eta"):
        assert np.array_equal(before[k], after[k]), k


def test_diagnostics_with_pending_correction_equal_materialized():
    """Diagnostics add a pending transport correction on the fly; downloading (which folds it
    into the state) first must not change them."""
    case = _tidal_small("mixed", order=3)
    a = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    b = OceanModel(case["cfg"], case["h"], case["f"], case["taux"], case["tauy"])
    for m in (a, b):
        m.upload_state(case["q"], case["eta"])
        m.step(case["dt"], case["nsub"], 2)
    da = a.diagnostics()
    b.download_state()
    db = b.diagnostics()
    for k in da:
        assert da[k] == db[k], k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_output_staging_overlaps_steps_and_returns_the_snapshot(precision):
    """drf_dg_output_stage snapshots the state (its pending transport correction folded in) and
    copies it to pinned host buffers on the model's copy stream while the next steps run;
    after output_wait the buffers hold exactly the state download_state returns at that step."""
    torch = pytest.importorskip("torch")
    case = _tidal_small(precision, nx=9, ny=7)
    cfg = case["cfg"]
    a = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    b = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    for m in (a, b):
        m.upload_state(case["q"], case["eta"])
        m.step(case["dt"], case["nsub"], 2)
    pinned = {k: torch.empty(cfg.n3 if k in ("Hu", "Hv", "HT", "HS") else cfg.n2,
                             dtype=torch.float64).pin_memory().numpy()
              for k in ("Hu", "Hv", "HT", "HS", "eta", "HU", "HV")}
    a.output_stage(pinned)
    a.step(case["dt"], case["nsub"], 3)  # runs while the copy is in flight
    t = a.output_wait()
    ref = b.download_state()
    assert t == ref["t"]
    for k in pinned:
        assert np.array_equal(pinned[k], ref[k]), k
    # a second stage after further steps; the model itself is unaffected by staging
    a.output_stage(pinned)
    t2 = a.output_wait()
    b.step(case["dt"], case["nsub"], 3)
    ref2 = b.download_state()
    assert t2 == ref2["t"]
    for k in pinned:
        assert np.array_equal(pinned[k], ref2[k]), k
    a.close()
    b.close()
