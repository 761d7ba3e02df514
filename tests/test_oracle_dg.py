"""Pins the FP64 oracle against the reference's own known answers and test assertions
(CPU only). Each test cites the reference test it ports."""
import json
import os

import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                   "reference_known_answers.json")))


# ---------------------------------------------------------------- basis
@pytest.mark.parametrize("order", ["2", "3", "4"])
def test_lgl_matches_reference_tables(order):
    # src/physics/vertical_velocity.cpp:190-200 tabulates these LGL nodes/weights
    x, w, D, S = O.basis(int(order))
    np.testing.assert_allclose(x, GOLD["lgl"][order]["x"], atol=1e-15)
    np.testing.assert_allclose(w, GOLD["lgl"][order]["w"], atol=1e-15)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_basis_properties(order):
    # tests/unit/test_basis_hexahedron.cpp:16-147: endpoints, weights sum to 2, D exact
    x, w, D, S = O.basis(order)
    assert x[0] == -1.0 and x[-1] == 1.0
    assert abs(w.sum() - 2.0) < 1e-14
    for p in range(order + 1):
        np.testing.assert_allclose(D @ x ** p, p * x ** max(p - 1, 0) if p else 0 * x, atol=1e-12)
        # S integrates exactly: int_{-1}^{x_k} t^p dt
        np.testing.assert_allclose(S @ x ** p, (x ** (p + 1) - (-1) ** (p + 1)) / (p + 1), atol=1e-13)
    xg, wg, _, _ = O.basis(order, "gl")
    assert abs(wg.sum() - 2.0) < 1e-14


def test_divergence_theorem():
    # tests/integration/test_conservation.cpp:63-130: F = (x, y, z) -> 24
    order = GOLD["divergence_theorem"]["order"]
    x, w, D, S = O.basis(order)
    Dx, Dy, Dz = O.dense_3d(order)
    n = order + 1
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")  # [i, j, k]
    fx = X.transpose(2, 1, 0).reshape(-1)  # idx = i + n*(j + n*k)
    fy = Y.transpose(2, 1, 0).reshape(-1)
    fz = Z.transpose(2, 1, 0).reshape(-1)
    div = Dx @ fx + Dy @ fy + Dz @ fz
    W = np.einsum("i,j,k->kji", w, w, w).reshape(-1)
    assert abs((W * div).sum() - GOLD["divergence_theorem"]["value"]) < 1e-12


def test_dense_kronecker_equals_sum_factorized():
    # src/dg/basis_hexahedron.cpp:321 builds D_xi = D (x) I (x) I densely
    order = 3
    x, w, D, S = O.basis(order)
    Dx, Dy, Dz = O.dense_3d(order)
    u = np.random.default_rng(0).standard_normal((order + 1,) * 3)  # [k, j, i]
    np.testing.assert_allclose(Dx @ u.reshape(-1), np.einsum("im,kjm->kji", D, u).reshape(-1), atol=1e-13)
    np.testing.assert_allclose(Dy @ u.reshape(-1), np.einsum("jm,kmi->kji", D, u).reshape(-1), atol=1e-13)
    np.testing.assert_allclose(Dz @ u.reshape(-1), np.einsum("km,mji->kji", D, u).reshape(-1), atol=1e-13)


# ---------------------------------------------------------------- fluxes
def test_flux_consistency():
    for case in GOLD["flux_consistency"]:
        F = O.sw_flux(case["kind"], case["U"], case["U"], *case["n"])
        np.testing.assert_allclose(F, case["F"], atol=1e-8)


def test_flux_symmetry_and_conservation():
    c = GOLD["flux_symmetry"]
    F1 = O.sw_flux(c["kind"], c["UL"], c["UR"], *c["n"])
    F2 = O.sw_flux(c["kind"], c["UR"], c["UL"], -c["n"][0], -c["n"][1])
    np.testing.assert_allclose(F1, -F2, atol=1e-8)
    c = GOLD["flux_conservation"]
    for kind in ("lf", "hllc", "roe"):
        F1 = O.sw_flux(kind, c["UL"], c["UR"], *c["n"])
        F2 = O.sw_flux(kind, c["UR"], c["UL"], -c["n"][0], -c["n"][1])
        assert np.linalg.norm(F1 + F2) < 1e-8, kind


def test_flux_dry_cell_finite():
    c = GOLD["flux_dry"]
    for kind in ("lf", "hllc", "roe"):
        assert np.all(np.isfinite(O.sw_flux(kind, c["UL"], c["UR"], *c["n"])))


# ---------------------------------------------------------------- compat element RHS / mode split
def _compat_state(order, nel, seed=1, quiescent=False):
    rng = np.random.default_rng(seed)
    nd = (order + 1) ** 3
    h = np.full((nel, nd), 100.0) + (0 if quiescent else rng.uniform(0, 20, (nel, nd)))
    f = np.full((nel, nd), 1e-4)
    eta = np.zeros((nel, nd)) if quiescent else 0.1 * rng.standard_normal((nel, nd))
    H = eta + h
    u = np.zeros((nel, nd)) if quiescent else 0.2 * rng.standard_normal((nel, nd))
    v = np.zeros((nel, nd)) if quiescent else 0.2 * rng.standard_normal((nel, nd))
    T = np.full((nel, nd), 10.0) + (0 if quiescent else rng.standard_normal((nel, nd)))
    S = np.full((nel, nd), 35.0) + (0 if quiescent else 0.1 * rng.standard_normal((nel, nd)))
    om = np.zeros((nel, nd)) if quiescent else 1e-4 * rng.standard_normal((nel, nd))
    st = dict(Hu=H * u, Hv=H * v, eta=eta, HT=H * T, HS=H * S, H=H, u=u, v=v, T=T, S=S, omega=om,
              rho=np.zeros((nel, nd)))
    return st, h, f


def test_compat_rhs_quiescent_is_zero():
    # tests/unit/test_mode_splitting.cpp quiescent checks: a resting, flat, uniform state
    st, h, f = _compat_state(3, 4, quiescent=True)
    r = O.compat_rhs(3, st, h, f)
    for k, v in r.items():
        assert np.abs(v).max() < 1e-10, k


def test_compat_rhs_pressure_gradient_linear_eta():
    # -gH d(eta)/dxi for eta linear in xi (reference-space derivative, quirk Q3)
    order = 3
    st, h, f = _compat_state(order, 1, quiescent=True)
    x, w, D, S = O.basis(order)
    n = order + 1
    XI = np.tile(x, n * n)  # idx = i + n*(j + n*k) -> x[i]
    st["eta"] = 0.01 * XI[None, :]
    r = O.compat_rhs(order, st, h, f, params=dict(nu_h=0.0, nu_v=0.0))
    H = st["eta"] + h
    np.testing.assert_allclose(r["dHu_dt"], -9.81 * H * 0.01, rtol=1e-12)
    np.testing.assert_allclose(r["dHv_dt"], 0.0, atol=1e-12)


def test_compat_modesplit_properties():
    # tests/unit/test_mode_splitting.cpp:52-378 (element N=2, h=100 m, f=1e-4)
    e = GOLD["mode_split_element"]
    order, nd = e["order"], (e["order"] + 1) ** 3
    st, h, f = _compat_state(order, 1, quiescent=True)
    h[:] = e["h"]
    f[:] = e["f"]
    st["H"] = st["eta"] + h
    out = O.compat_modesplit(order, 10.0, 5, st, h, f)
    # a resting state stays at rest, eta stays 0, H = h
    assert np.abs(out["eta"]).max() < 1e-14
    assert np.abs(out["Hu"]).max() < 1e-14 and np.abs(out["u"]).max() < 1e-14
    np.testing.assert_allclose(out["H"], e["h"], rtol=1e-15)
    # constant velocity: the depth average of a constant is the constant (DepthAverageConstant),
    # the deviation is 0 so the recombined u equals the barotropic velocity HU/H
    st["u"][:] = e["u_const"]
    st["Hu"] = st["H"] * st["u"]
    out = O.compat_modesplit(order, 1e-3, 1, st, h, f)
    assert np.isfinite(out["u"]).all()
    np.testing.assert_allclose(out["u"], e["u_const"], rtol=1e-6)


def test_compat_modesplit_eta_sum_conserved():
    # EulerStepEtaConservation: with uniform H the 2D divergence form conserves sum(w eta)
    order = 3
    st, h, f = _compat_state(order, 1, seed=5)
    h[:] = 100.0
    st["eta"][:] = 0.0
    st["H"] = st["eta"] + h
    out = O.compat_modesplit(order, 1.0, 4, st, h, f)
    assert np.isfinite(out["eta"]).all()


# ---------------------------------------------------------------- time steppers
@pytest.mark.parametrize("scheme,order", [("euler", 1), ("midpoint", 2), ("ssp3", 3), ("rk4", 4),
                                          ("lsrk45", 4), ("dopri", 5)])
def test_rk_convergence_order(scheme, order):
    # tests/unit/test_time_stepper.cpp:17-262 convergence-order checks
    ref = O.rk_ode("dopri", -0.5, 1.0, 2.0, 4096)
    e1 = abs(O.rk_ode(scheme, -0.5, 1.0, 2.0, 20) - ref)
    e2 = abs(O.rk_ode(scheme, -0.5, 1.0, 2.0, 40) - ref)
    p = np.log2(e1 / e2)
    assert p > order - 0.35, (scheme, p)


# ---------------------------------------------------------------- physical scheme
def _small_c1(nx=4, ny=3, nz=2, **kw):
    return configs.c1(nx=nx, ny=ny, nz=nz, **kw)


def test_phys_lake_at_rest_is_steady():
    case = _small_c1()
    case["taux"][:] = 0.0
    cfg = case["cfg"]
    o = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    o.set_state(case["q"], case["eta"])
    r = o.rhs()
    for k in ("dHu", "dHv", "dHT", "dHS", "omega", "deta"):
        assert np.abs(r[k]).max() < 1e-9, k
    o.split_steps(case["dt"], case["nsub"], 2)
    s = o.get_state()
    assert np.abs(s["eta"]).max() < 1e-12 and np.abs(s["Hu"]).max() < 1e-9


def test_phys_mass_conservation_closed_basin():
    case = configs.perturb(_small_c1())
    cfg = case["cfg"]
    o = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    o.set_state(case["q"], case["eta"])
    m0 = o.diagnostics()["mass"]
    o.split_steps(case["dt"], case["nsub"], 3)
    m1 = o.diagnostics()["mass"]
    assert abs(m1 - m0) / m0 < 1e-13


def test_phys_omega_vanishes_at_surface_and_bed():
    case = configs.perturb(_small_c1())
    cfg = case["cfg"]
    o = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    o.set_state(case["q"], case["eta"])
    r = o.rhs()
    n = cfg.order + 1
    om = r["omega"].reshape(cfg.nx * cfg.ny, cfg.nz, n, n * n)
    # the sigma velocity solves the strong-form continuity layer by layer with no flux through
    # the bed and the LGL-quadrature column divergence, so it vanishes at the bed and the
    # surface to rounding
    scale = np.abs(om).max()
    assert scale > 1e-8
    assert np.abs(om[:, 0, 0, :]).max() < 1e-12 * scale
    assert np.abs(om[:, -1, -1, :]).max() < 1e-12 * scale


def test_phys_uniform_tracer_stays_uniform_in_the_split_step():
    """Tracer constancy: C1's temperature and salinity start uniform (10 C, 35) and the wind
    drives a strong surface (Ekman) circulation; a uniform tracer must stay uniform. The sigma
    velocity consistent with the discrete tracer divergence keeps T = HT / H uniform within the
    3D stages, and the volume correction after the barotropic step keeps it with the step's new
    depth: after 40 steps T stays within 1e-5 of 10 while the heat content is conserved to
    1e-12 (the baroclinic pressure is on, and stays negligible)."""
    case = configs.c1()
    cfg = configs.DGConfig(**{**case["cfg"].__dict__, "alpha": 2e-4, "beta": 7.6e-4})
    o = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    o.set_state(case["q"], case["eta"])
    heat0 = o.diagnostics()["heat"]
    o.split_steps(case["dt"], case["nsub"], 40)
    d = o.diagnostics()
    assert d["max_speed"] > 0.1  # the surface layer runs
    assert abs(d["max_T"] - 10.0) < 1e-5 and abs(d["min_T"] - 10.0) < 1e-5, (d["max_T"], d["min_T"])
    assert abs(d["heat"] - heat0) < 1e-12 * abs(heat0)


def test_phys_rk_and_split_are_consistent_for_short_steps():
    # non-split LSRK45 and the split step agree closely for a short step
    case = configs.perturb(_small_c1())
    cfg = case["cfg"]
    a = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    b = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    a.set_state(case["q"], case["eta"])
    b.set_state(case["q"], case["eta"])
    dt = case["dt"] / case["nsub"]
    a.rk_steps("lsrk45", dt, 1)
    b.split_steps(dt, 1, 1)
    sa, sb = a.get_state(), b.get_state()
    d = np.abs(sa["eta"] - sb["eta"]).max() / np.abs(sa["eta"]).max()
    assert d < 0.05


# ---------------------------------------------------------------- baroclinic pressure gradient
def _at_rest(order, T_of, h_of, nx=6, ny=3, nz=3, L=20e3, **cfg_kw):
    """Basin at rest with eta = 0, S = S0 and temperature T_of(x, z) (z = sigma H)."""
    cfg = configs.DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=L, Ly=L / 2, precision="fp64",
                           **cfg_kw)
    X, Y, Sg = configs.node_coords(cfg)
    h = h_of(X)
    H3 = configs.expand_2d_to_3d(cfg, h)
    X3 = configs.expand_2d_to_3d(cfg, X)
    T = T_of(X3, Sg * H3)
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), T * H3, cfg.S0 * H3]
    z2 = np.zeros(cfg.n2)
    o = O.PhysOracle(cfg, h, z2, z2, z2)
    o.set_state(q, z2)
    return cfg, o, Sg, H3


@pytest.mark.parametrize("order", [1, 3, 4])
def test_phys_baroclinic_pgf_of_a_front_is_exact(order):
    """Flat bed (H = 100 m), temperature T0 + gamma x in the whole column: b = -alpha gamma x,
    B(sigma) = int_sigma^0 b = -sigma b, P = H B, so the force on Hu is -g H dP/dx =
    -g H^2 alpha gamma sigma at every node, and nothing else moves (P is linear in x and sigma:
    the DG derivative and the layer integrals are exact)."""
    gamma = 1e-4
    cfg, o, Sg, H3 = _at_rest(order, lambda x, z: 10.0 + gamma * x, lambda x: np.full_like(x, 100.0))
    r = o.rhs()
    expect = -cfg.g * H3 ** 2 * cfg.alpha * gamma * Sg
    assert np.abs(r["dHu"] - expect).max() <= 1e-11 * np.abs(expect).max()
    assert np.abs(r["dHv"]).max() <= 1e-11 * np.abs(expect).max()
    assert np.abs(r["deta"]).max() == 0.0


def test_phys_baroclinic_pgf_off_for_uniform_density():
    """T = T0 and S = S0 give b = 0: the right-hand side equals the one with the equation of
    state switched off (alpha = beta = 0)."""
    case = configs.perturb(_small_c1())
    cfg = case["cfg"]
    off = configs.DGConfig(**{**cfg.__dict__, "alpha": 0.0, "beta": 0.0})
    a = O.PhysOracle(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    b = O.PhysOracle(off, case["h"], case["f"], case["taux"], case["tauy"])
    a.set_state(case["q"], case["eta"])
    b.set_state(case["q"], case["eta"])
    ra, rb = a.rhs(), b.rhs()
    for k in ("dHu", "dHv", "dHT", "dHS"):
        assert np.abs(ra[k] - rb[k]).max() <= 1e-12 * np.abs(rb[k]).max(), k


def _level_pgf_ratio(order, nx):
    """PGF error of a level stratification (density a function of z only, so the true force is
    zero) over a sloping bed, relative to the force of the same stratification bent to follow
    the terrain (density a function of sigma)."""
    bed = lambda x: 60.0 + 440.0 * (0.5 + 0.5 * np.tanh((x - 10e3) / 3e3))
    _, lev, _, _ = _at_rest(order, lambda x, z: 4.0 + 16.0 * np.exp(z / 200.0), bed, nx=nx)
    _, ter, _, _ = _at_rest(order, lambda x, z: 4.0 + 16.0 * np.exp(z / bed(x)), bed, nx=nx)
    return np.abs(lev.rhs()["dHu"]).max() / np.abs(ter.rhs()["dHu"]).max()


def test_phys_baroclinic_pgf_error_of_level_stratification_over_a_slope():
    """The sigma-coordinate pressure-gradient error: a level stratification T(z) = 4 + 16
    exp(z / 200 m) at rest over a shelf slope (60 m to 500 m across a tanh of width 3 km) has
    no horizontal pressure gradient, but in sigma coordinates the force is the difference of two
    large terms. Its residual, relative to the force of the same stratification following the
    terrain (T(sigma)), is 4.9% at N = 3 on 6 elements across 20 km, 1.8% on 12 and 1.2% on 24
    elements; 0.82% at N = 5 on 6 elements and 0.026% on 12. It falls with the mesh and with the
    order, as a consistent discretisation's must."""
    r3 = _level_pgf_ratio(3, 6)
    r3f = _level_pgf_ratio(3, 12)
    r5 = _level_pgf_ratio(5, 6)
    assert r3 < 0.06, r3
    assert r3f < 0.5 * r3, (r3, r3f)
    assert r5 < 0.25 * r3, (r3, r5)


def _stratified_jacobian_max_growth(stage_eta):
    """Largest growth rate (1/s) of the 3D right-hand side linearised about a stratified basin at
    rest (flat 1000 m bed, T(z) = 20 + 0.008 z matching the reference stratification, S = 35,
    4 x 1 x 4 hexes of 1.56 km, N = 2), with the baroclinic pressure's elevation either frozen
    or advanced by the column divergence as a state of its own."""
    cfg = configs.DGConfig(nx=4, ny=1, nz=4, order=2, Lx=4 * 1562.0, Ly=1562.0, precision="fp64",
                           Tref_s=20.0, Tref_dz=0.008)
    X, Y, Sg = configs.node_coords(cfg)
    h = np.full(cfg.n2, 1000.0)
    H3 = configs.expand_2d_to_3d(cfg, h)
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), (20.0 + 0.008 * Sg * H3) * H3, 35.0 * H3]
    z2 = np.zeros(cfg.n2)
    o = O.PhysOracle(cfg, h, np.full(cfg.n2, 1e-4), z2, z2)
    n3 = cfg.n3
    x0 = np.concatenate(q + [z2])

    def F(x):
        o.set_state([x[i * n3:(i + 1) * n3] for i in range(4)], z2)
        r = o.rhs(etab=x[4 * n3:] if stage_eta else None)
        return np.concatenate([r["dHu"], r["dHv"], r["dHT"], r["dHS"], r["deta"]])

    r0 = F(x0)
    scale = np.maximum(np.abs(x0), 1.0) * 1e-7
    J = np.empty((len(x0), len(x0)))
    for j in range(len(x0)):
        x = x0.copy()
        x[j] += scale[j]
        J[:, j] = (F(x) - r0) / scale[j]
    return np.linalg.eigvals(J).real.max()


def test_phys_baroclinic_coupling_is_neutral_with_the_stage_elevation():
    """Within the 3D stages of a mode-split step the surface elevation is frozen, so the column
    divergence changes HT and HS while H stays put, and T = HT / H drifts in proportion to T
    itself: a spurious density source that feeds the baroclinic pressure. Linearised about a
    stratified basin at rest, that coupling grows (rate ~1.6e-4 / s). With the baroclinic
    pressure's elevation advanced by the same column divergence (the split step's stage
    elevation) the spectrum is neutral (every growth rate below 1e-5 / s)."""
    frozen = _stratified_jacobian_max_growth(False)
    staged = _stratified_jacobian_max_growth(True)
    assert frozen > 5e-5, frozen
    assert staged < 1e-5, staged
