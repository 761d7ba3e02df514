"""AMR refinement (src/amr/refinement.cpp): the oracle pinned to the reference's own unit tests
(tests/unit/test_amr.cpp), the column-wise level refinement of the native library (host-only,
no GPU), and on the GPU the estimator and the solution transfer against the oracle."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs
from drifter_b200.amr import (AdaptiveMeshRefinement, DG3DIntegration, RefinementParams, build_mesh,
                              element_lengths)


def _lgl(order):
    b = O.basis(order)
    return np.asarray(b["nodes"] if isinstance(b, dict) else b[0])


# ----------------------------------------------------------------- oracle pins (test_amr.cpp)
def test_projection_of_a_constant_to_children():
    """SolutionProjectionConstant: 42 everywhere in all 8 children (order 2, XYZ)."""
    ch = O.amr_project_children(2, np.full(27, 42.0), 7)
    assert ch.shape == (8, 27)
    assert np.abs(ch - 42.0).max() < 1e-12


@pytest.mark.parametrize("order", [2, 3, 4])
def test_projection_of_a_linear_field_is_exact(order):
    """SolutionProjectionLinear: x + y + z is reproduced in the first child, whose nodes sit at
    -1 + (x + 1) / 2 of the parent (and in every child, at any order)."""
    x = _lgl(order)
    n = order + 1
    idx = [(i, j, k) for k in range(n) for j in range(n) for i in range(n)]
    U = np.array([x[i] + x[j] + x[k] for i, j, k in idx])
    ch = O.amr_project_children(order, U, 7)
    for c in range(8):
        cx, cy, cz = c & 1, (c >> 1) & 1, c >> 2
        p = lambda t, cc: (-1.0 + cc) + 0.5 * (t + 1.0)
        exp = np.array([p(x[i], cx) + p(x[j], cy) + p(x[k], cz) for i, j, k in idx])
        assert np.abs(ch[c] - exp).max() < 1e-13


@pytest.mark.parametrize("order", [2, 3, 5])
@pytest.mark.parametrize("mask", [1, 3, 7, 4])
def test_projection_roundtrip(order, mask):
    """SolutionProjectionRoundtrip (within 10% in the reference's test): a polynomial of the
    element's order restricted to a child is still one, so to children and back is exact."""
    rng = np.random.default_rng(order + 10 * mask)
    U = rng.uniform(-1, 1, (order + 1) ** 3)
    back = O.amr_project_parent(order, O.amr_project_children(order, U, mask), mask)
    assert np.abs(back - U).max() < 1e-12


def test_directional_child_counts():
    """SolutionProjectionDirectionalX / XY and RefineMaskNumChildren."""
    for mask, n in ((0, 1), (1, 2), (2, 2), (4, 2), (3, 4), (5, 4), (6, 4), (7, 8)):
        assert O.amr_project_children(2, np.ones(27), mask).shape[0] == n


def test_gradient_estimator_constant_and_variable():
    """GradientErrorEstimatorConstant / Variable (order 2, 8 elements): zero for a constant; for
    u = dof index the largest range runs along z (0..18 against 0..6 along y and 0..2 along x), so
    the mask is Z alone (x, y below half of it), and the normalised value is 1 and refines."""
    v, m, f = O.amr_estimate(2, np.ones((8, 27)), np.full(8, 0.5))
    assert np.all(v == 0) and np.all(m == 0) and np.all(f == 0)
    v, m, f = O.amr_estimate(2, np.tile(np.arange(27.0), (8, 1)), np.full(8, 0.5))
    assert np.all(v == 1.0) and np.all(m == 4) and np.all(f == 1)


def test_estimator_thresholds_and_normalisation():
    """Values are normalised by the largest; refine above 0.1, coarsen below 0.01."""
    U = np.zeros((4, 64))
    for e, r in enumerate((1.0, 0.5, 0.05, 0.001)):
        U[e, 63] = r
    v, m, f = O.amr_estimate(3, U, np.ones(4))
    assert np.allclose(v, [1.0, 0.5, 0.05, 0.001])
    assert list(f) == [1, 1, 0, 2]


# ----------------------------------------------------------------- column levels (host C++)
def _levels(nb=16, seed=3):
    lx, ly, lz = configs.c3_levels(nb, seed=seed, lmax=2)
    return tuple(np.ascontiguousarray(a, np.int32) for a in (lx, ly, lz))


def _balanced(lx, ly, lz):
    ny, nx = lx.shape
    for iy in range(ny):
        for ix in range(nx):
            for dx, dy, t in ((1, 0, ly), (0, 1, lx)):
                jx, jy = ix + dx, iy + dy
                if jx >= nx or jy >= ny:
                    continue
                d = (int(t[jy, jx]) - int(t[iy, ix]), int(lz[jy, jx]) - int(lz[iy, ix]))
                if max(abs(d[0]), abs(d[1])) > 1 or d[0] * d[1] < 0:
                    return False
    return True


def test_refine_levels_follows_the_marks_and_stays_balanced():
    amr = AdaptiveMeshRefinement(3, RefinementParams(max_level=4))
    lv = _levels()
    m = build_mesh(*lv)
    ne = m["n_elem"]
    mask = np.zeros(ne, np.int32)
    flags = np.zeros(ne, np.int32)
    # refine the first element of one level-0 column along x; coarsen every element of a refined one
    col_lv = m["col_levels"]
    c0 = int(np.flatnonzero(col_lv.sum(1) == 0)[0])
    c1 = int(np.flatnonzero(col_lv[:, 0] >= 1)[0])
    ny, nx = lv[0].shape
    box = m["box"]
    colof = (np.floor(box[:, 0] * nx + 1e-9).astype(int) + nx * np.floor(box[:, 1] * ny + 1e-9).astype(int))
    e0 = int(np.flatnonzero(colof == c0)[0])
    mask[e0], flags[e0] = 1, 1
    flags[colof == c1] = 2
    new, changed = amr.refine_levels(lv, mask, flags)
    nlx, nly, nlz = (a.ravel() for a in new)
    assert nlx[c0] == 1 and nly[c0] <= 1  # refined along x (y, z only as the balance needs)
    assert nlx[c1] <= col_lv[c1, 0]
    assert changed >= 1
    assert _balanced(*new)
    build_mesh(*new)  # the builder accepts the new levels


def test_refine_levels_respects_max_and_min_level():
    amr = AdaptiveMeshRefinement(3, RefinementParams(max_level=1, min_level=0))
    one = np.ones((2, 2), np.int32)
    lv = (one, one, one)
    ne = build_mesh(*lv)["n_elem"]
    new, changed = amr.refine_levels(lv, np.full(ne, 7, np.int32), np.ones(ne, np.int32))
    assert changed == 0 and all((a == 1).all() for a in new)  # every level at max_level
    new, changed = amr.refine_levels(lv, np.zeros(ne, np.int32), np.full(ne, 2, np.int32))
    assert changed == 4 and all((a == 0).all() for a in new)  # coarsened to min_level
    z = np.zeros((2, 2), np.int32)
    new, changed = amr.refine_levels((z, z, z), np.zeros(4, np.int32), np.full(4, 2, np.int32))
    assert changed == 0  # nothing below min_level


def test_refine_levels_random_marks_always_give_a_buildable_mesh():
    amr = AdaptiveMeshRefinement(3, RefinementParams(max_level=3))
    rng = np.random.default_rng(7)
    lv = _levels(12, seed=5)
    for _ in range(4):
        ne = build_mesh(*lv)["n_elem"]
        mask = rng.integers(0, 8, ne).astype(np.int32)
        flags = rng.choice([0, 1, 2], ne, p=[0.8, 0.1, 0.1]).astype(np.int32)
        lv, _ = amr.refine_levels(lv, mask, flags)
        assert _balanced(*lv)
        build_mesh(*lv)


def test_oracle_transfer_matches_the_projections():
    """The column-wise remap restates project_to_children on a refined axis and
    project_from_children on a coarsened one."""
    order, nd = 3, 64
    rng = np.random.default_rng(2)
    one = np.ones((1, 1), np.int32)
    z = np.zeros((1, 1), np.int32)
    U = rng.uniform(-1, 1, (1, nd))
    ch = O.amr_transfer(order, np.stack([z, z, z], -1), np.stack([one, z, one], -1), U)
    assert np.array_equal(ch, O.amr_project_children(order, U[0], 5))
    back = O.amr_transfer(order, np.stack([one, z, one], -1), np.stack([z, z, z], -1), ch)
    assert np.array_equal(back[0], O.amr_project_parent(order, ch, 5))


# ----------------------------------------------------------------- GPU against the oracle
def _field(m, order, kind):
    x = _lgl(order)
    n = order + 1
    b = m["box"]
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))  # dof i + n (j + n k)
    X = b[:, 0:1] + 0.5 * (x[i][None, :] + 1) * (b[:, 3:4] - b[:, 0:1])
    Y = b[:, 1:2] + 0.5 * (x[j][None, :] + 1) * (b[:, 4:5] - b[:, 1:2])
    Z = b[:, 2:3] + 0.5 * (x[k][None, :] + 1) * (b[:, 5:6] - b[:, 2:3])
    if kind == "linear":
        return 1.0 + 2.0 * X - 3.0 * Y + 0.5 * Z
    return np.tanh((X - 0.5 + 0.1 * np.sin(6 * Y)) / 0.03) + 0.002 * Z


@pytest.mark.gpu
@pytest.mark.parametrize("order", [2, 3, 4])
def test_estimate_equals_oracle(order):
    lv = _levels(16, seed=1)
    m = build_mesh(*lv)
    U = _field(m, order, "front")
    model = DG3DIntegration(order, m)
    model.upload(U)
    amr = AdaptiveMeshRefinement(order)
    v, mask, flags = amr.estimate(model, m)
    rv, rm, rf = O.amr_estimate(order, U, element_lengths(m))
    assert np.array_equal(v, rv)
    assert np.array_equal(mask, rm)
    assert np.array_equal(flags, rf)
    assert flags.any() and (flags == 2).any()
    model.close()


@pytest.mark.gpu
@pytest.mark.parametrize("order", [2, 3, 4])
def test_transfer_equals_oracle(order):
    """Refined, coarsened and mixed columns; the GPU keeps the oracle's operations and order
    (the Lagrange rows of interpolate_3d, the sum in dof order without fused multiply-adds)."""
    lv = _levels(12, seed=4)
    m = build_mesh(*lv)
    U = _field(m, order, "front")
    rng = np.random.default_rng(order)
    amr = AdaptiveMeshRefinement(order, RefinementParams(max_level=3))
    mask = rng.integers(0, 8, m["n_elem"]).astype(np.int32)
    flags = rng.choice([0, 1, 2], m["n_elem"], p=[0.6, 0.2, 0.2]).astype(np.int32)
    new, changed = amr.refine_levels(lv, mask, flags)
    assert changed > 0
    ol = np.stack(lv, -1)
    nl = np.stack(new, -1)
    assert (nl > ol).any() and (nl < ol).any()
    m2 = build_mesh(*new)
    a, b = DG3DIntegration(order, m), DG3DIntegration(order, m2)
    a.upload(U)
    amr.transfer(a, b, lv, new)
    got = b.download()
    ref = O.amr_transfer(order, ol, nl, U)
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
    a.close()
    b.close()


@pytest.mark.gpu
def test_adapt_carries_a_linear_field_exactly_and_refines_at_a_front():
    order = 3
    lv = _levels(12, seed=6)
    m = build_mesh(*lv)
    amr = AdaptiveMeshRefinement(order, RefinementParams(max_level=3))
    lin = DG3DIntegration(order, m)
    lin.upload(_field(m, order, "linear"))
    new_model, m2, lv2, changed = amr.adapt(lin, m, lv)
    assert changed > 0
    got = new_model.download()
    assert np.abs(got - _field(m2, order, "linear")).max() < 1e-12
    # a front: the columns of the elements it marks for refinement gain a level, the smooth
    # rest coarsens, and the new model steps
    fr = DG3DIntegration(order, m)
    U = _field(m, order, "front")
    fr.upload(U)
    _, _, flags = amr.estimate(fr, m)
    ny, nx = lv[0].shape
    box = m["box"]
    colof = (np.floor(box[:, 0] * nx + 1e-9).astype(int) + nx * np.floor(box[:, 1] * ny + 1e-9).astype(int))
    marked = np.unique(colof[(flags & 1) == 1])
    f2, m3, lv3, ch = amr.adapt(fr, m, lv)
    old_sum = sum(a.ravel() for a in lv)
    new_sum = sum(a.ravel() for a in lv3)
    assert ch > 0 and len(marked) > 0
    assert np.all(new_sum[marked] > old_sum[marked])
    assert (new_sum < old_sum).any()
    f2.step([1.0, 0.0, 0.0], 1e-4, 2, mode="complete")
    assert np.isfinite(f2.download()).all()
    for mdl in (lin, new_model, fr, f2):
        mdl.close()
