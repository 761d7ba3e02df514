"""GPU parity of the Bezier smoother path against the FP64 oracle, through the C ABI.
Tolerances: operator applications and multigrid cycles 1e-11 relative (FP64, different
summation order); PCG solutions 1e-8 relative at the 1e-10 residual."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs
from drifter_b200.bezier import BezierMultigridPreconditioner, BezierSmoother

pytestmark = pytest.mark.gpu


def fbm(n, L=5000.0, seed=3):
    rng = np.random.default_rng(seed)
    X, Y = O.gauss_points(n, n, 0, 0, L, L)
    d = np.zeros_like(X)
    for _ in range(12):
        k = rng.uniform(0.5, 6, 2) * 2 * np.pi / L
        d += rng.normal() / (k @ k) ** 0.5 * np.sin(k[0] * X + k[1] * Y + rng.uniform(0, 6.3))
    return 2000 + 1500 * d / np.abs(d).max()


def pair(n, L=5000.0, lam=1.0, eps=1e-4):
    d = fbm(n, L)
    return BezierSmoother(n, n, L, L, d, lam=lam, ridge_epsilon=eps), O.BezierOracle(n, n, L, L, d, lam=lam, eps=eps)


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("n", [1, 2, 5, 16])
def test_rhs_and_operator_match_oracle(n):
    g, o = pair(n)
    assert g.ndof == o.ndof
    assert abs(g.alpha - o.alpha) <= 1e-12 * o.alpha
    assert rel(g.rhs(), o.vec("b")) < 1e-12
    x = np.random.default_rng(1).standard_normal(g.ndof)
    assert rel(g.apply_Q(x), o.csr("Q") @ x) < 1e-12


@pytest.mark.parametrize("n", [4, 16, 32])
def test_vcycle_matches_oracle(n):
    g, o = pair(n)
    BezierMultigridPreconditioner(g, 2).setup()
    o.mg_setup(2)
    r = np.random.default_rng(2).standard_normal(g.ndof)
    assert rel(g.mg_apply(r), o.vcycle(r)) < 1e-11


@pytest.mark.parametrize("n", [4, 16, 32])
def test_reference_mg_apply_matches_oracle(n):
    """BezierMultigridPreconditioner::apply as written (row-normalised restriction, one colour
    order, V-cycles to the tolerance) against the oracle's restatement: the same number of
    cycles and the same result."""
    g, o = pair(n)
    g.mg_setup(2)
    o.mg_setup(2)
    b = o.vec("b")
    for tol in (1e-6, 1e-9):
        z, cycles, relres = g.mg_apply_reference(b, tol=tol)
        zo, co = o.mg_apply_ref(b, tol=tol)
        assert cycles == co and relres < tol
        assert rel(z, zo) < 1e-10


def test_flexible_cg_with_the_reference_mg_apply():
    """PCG kind 4: the reference's multigrid apply (a variable preconditioner) under flexible
    CG reaches the FP64 1e-10 residual and the oracle's direct-preconditioned solution."""
    g, o = pair(32)
    g.mg_setup(2)
    o.mg_setup(2)
    x, info = g.solve("mg_reference", tol=1e-10, maxit=200)
    xo, ito, rro = o.pcg(precond="mg", tol=1e-12, maxit=5000)
    assert info["relres"] <= 1e-10 and info["iters"] < 20
    assert rel(x, xo) < 1e-8


@pytest.mark.parametrize("precond", ["none", "jacobi", "mg"])
def test_pcg_solution_matches_oracle(precond):
    g, o = pair(32)
    g.mg_setup(2)
    o.mg_setup(2)
    x, info = g.solve(precond, tol=1e-10, maxit=5000)
    xo, ito, rro = o.pcg(precond=precond, tol=1e-10, maxit=5000)
    assert info["relres"] <= 1e-10
    assert rel(x, xo) < 1e-8
    assert abs(info["iters"] - ito) <= 1


def test_c4_full_size_operator_and_jacobi_pcg_match_oracle():
    """C4 at full size (512 x 512 elements, 2.36 M control points, seeded fBm): the assembled
    right-hand side and Q x to 1e-12, and the Jacobi-PCG solution at the 1e-10 residual to 1e-8
    with the same iteration count (+-1), GPU against the FP64 oracle."""
    c = configs.c4()
    g = BezierSmoother(c["n"], c["n"], c["L"], c["L"], c["d"], lam=c["lam"], ridge_epsilon=c["eps"])
    o = O.BezierOracle(c["n"], c["n"], c["L"], c["L"], c["d"], lam=c["lam"], eps=c["eps"])
    assert rel(g.rhs(), o.vec("b")) < 1e-12
    x = np.random.default_rng(5).uniform(-1, 1, g.ndof)
    assert rel(g.apply_Q(x), o.csr("Q") @ x) < 1e-12
    xs, info = g.solve("jacobi", tol=1e-10, maxit=5000)
    xo, ito, rro = o.pcg(precond="jacobi", tol=1e-10, maxit=5000)
    assert info["relres"] <= 1e-10 and rro <= 1e-10
    assert abs(info["iters"] - ito) <= 1
    assert rel(xs, xo) < 1e-8
    g.close()


def test_pcg_zero_rhs_and_maxit():
    g, o = pair(8)
    x, info = g.solve("jacobi", b=np.zeros(g.ndof))
    assert info["iters"] == 0 and np.all(x == 0)
    x, info = g.solve("none", tol=1e-14, maxit=3)
    assert info["iters"] == 3


def test_vcycle_element_thread_smoother_matches_oracle(monkeypatch):
    # the element-per-thread Schwarz kernel (large levels) on every grid-wide level
    monkeypatch.setenv("DRF_BZ_ELEM_SMOOTHER_MIN", "1")
    g, o = pair(32)
    g.mg_setup(2)
    o.mg_setup(2)
    r = np.random.default_rng(4).standard_normal(g.ndof)
    assert rel(g.mg_apply(r), o.vcycle(r)) < 1e-11


def _oracle_row_order(n, ng):
    """GPU row index of each oracle constraint row (oracle: per element, right edge then top)."""
    nv = n * (n - 1) * ng
    out = []
    for ey in range(n):
        for ex in range(n):
            if ex + 1 < n:
                out += [(ey * (n - 1) + ex) * ng + q for q in range(ng)]
            if ey + 1 < n:
                out += [nv + (ey * n + ex) * ng + q for q in range(ng)]
    return np.array(out)


@pytest.mark.parametrize("ng", [2, 4])
def test_constraint_rows_match_oracle(ng):
    n = 8
    g, o = pair(n)
    A = o.constraints(ng)
    x = np.random.default_rng(5).standard_normal(g.ndof)
    y = g.constraints_apply(x, ng)
    assert y.shape[0] == A.shape[0]
    assert rel(y[_oracle_row_order(n, ng)], A @ x) < 1e-12


@pytest.mark.parametrize("inner", ["mg", "jacobi"])
def test_constrained_solve_doc_known_answer(inner):
    # docs/cg_bezier_solver_verification.md:32-39: objective 25.235, ||x|| 61.715, data
    # residual 0.1398 for the 16 x 16 sin-exp case, against the oracle's direct Schur solve
    from test_oracle_bz import GOLD, doc_case, schur_solve
    k = GOLD["bezier_doc_16x16"]
    o = doc_case()
    X, Y = O.gauss_points(16, 16, 0, 0, 1000.0, 1000.0)
    d = np.exp(np.sin(2 * np.pi * X / 1000.0) * np.sin(2 * np.pi * Y / 1000.0))
    g = BezierSmoother(16, 16, 1000.0, 1000.0, d, lam=1.0, ridge_epsilon=1e-4)
    if inner == "mg":
        g.mg_setup(2)
    x, info = g.solve_constrained(4, tol=1e-10, inner=inner, inner_tol=1e-13)
    xo, A = schur_solve(o)
    assert info["relres"] < 1e-10 and info["outer_iters"] > 0
    assert rel(x, xo) < 1e-7
    obj, reg, dat = o.objective(x)
    assert abs(obj - k["objective"]) < 6e-4
    assert abs(np.linalg.norm(x) - k["x_norm"]) < 6e-4
    assert abs(dat - k["data_residual"]) < 6e-5
    assert np.abs(A @ x).max() < 1e-7


def test_constrained_solve_matches_oracle_at_48():
    """The constrained (C1, Schur-CG) solve on a 48 x 48 fBm case (21,025 control points, the
    reference's edge constraints at 4 Gauss points): the GPU's Schur CG with inner multigrid-PCG
    solves against the oracle's Schur CG with exact Q^-1 (SuperLU), 1e-7 relative."""
    from test_oracle_bz import schur_solve
    n = 48
    g, o = pair(n)
    g.mg_setup(2)
    x, info = g.solve_constrained(4, tol=1e-10, inner="mg", inner_tol=1e-13)
    xo, A = schur_solve(o)
    assert info["relres"] < 1e-10 and info["outer_iters"] > 0
    assert rel(x, xo) < 1e-7
    assert np.abs(A @ x).max() < 1e-6 * np.abs(x).max()


@pytest.mark.parametrize("ng", [3, 4, 5])
def test_element_errors_match_oracle(ng):
    """AdaptiveCGCubicBezierSmoother::compute_element_l2_error for every element on the GPU
    against the oracle, for the smoothed surface of a 16 x 16 grid."""
    c = configs.c4(n=16, L=1600.0)
    s = BezierSmoother(16, 16, c["L"], c["L"], c["d"], lam=c["lam"], ridge_epsilon=c["eps"])
    s.mg_setup(2)
    x, _ = s.solve("mg", tol=1e-10)
    rng = np.random.default_rng(ng)
    z = rng.uniform(0, 4000, 16 * 16 * ng * ng)
    l2, nrm = s.element_errors(x, z, ngauss=ng)
    r2, rn = O.bz_element_errors(16, 16, c["L"], c["L"], ng, x, z)
    assert np.abs(l2 - r2).max() <= 1e-12 * np.abs(r2).max()
    assert np.abs(nrm - rn).max() <= 1e-12 * np.abs(rn).max()
    s.close()


def test_element_errors_c4_full_size():
    """C4 (512 x 512): the misfit of the MG-PCG solution to the data at the 4 x 4 Gauss points,
    GPU against the oracle."""
    c = configs.c4()
    s = BezierSmoother(c["n"], c["n"], c["L"], c["L"], c["d"], lam=c["lam"], ridge_epsilon=c["eps"])
    s.mg_setup(2)
    x, inf = s.solve("mg", tol=1e-10)
    l2, nrm = s.element_errors(x, c["d"], ngauss=4)
    r2, rn = O.bz_element_errors(c["n"], c["n"], c["L"], c["L"], 4, x, c["d"])
    assert np.abs(l2 - r2).max() <= 1e-12 * np.abs(r2).max()
    assert l2.max() > 0
    s.close()
