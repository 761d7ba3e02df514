"""Pins the mortar oracle against the reference's mortar unit tests
(tests/unit/test_mortar.cpp) and the projection identities its construction implies (CPU)."""
import numpy as np
import pytest

import pyoracle as O


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_mortar_dofs_order_and_quadrature(order):
    # MortarSpaceConstructionSameLevel / 1To4: num_dofs (p+1)^2, order p; QuadraturePoints:
    # (2p+1)^2 mortar points (the mass matrix is exact: integrand degree 2p < 2(2p+1))
    for t in (0, 5):
        o = O.mortar_ops(order, t)
        assert o["M"].shape == ((order + 1) ** 2,) * 2
    # LGL Lagrange mass on [-1,1]^2: the exact mass integrates 1 to the face area 4
    assert abs(O.mortar_ops(order, 0)["M"].sum() - 4.0) < 1e-12


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_mass_matrix_symmetric_positive_definite(order):
    # MassMatrixPositiveDefinite
    M = O.mortar_ops(order, 0)["M"]
    np.testing.assert_allclose(M, M.T, atol=1e-14)
    assert np.linalg.eigvalsh(M).min() > 0


def test_num_fine_faces_per_connection_type():
    # FaceConnectionHelpers: SameLevel 1, Fine2x1 2, Fine3_2plus1 3, Fine2x2 4
    for t, n in O.MORTAR_NUM_FINE.items():
        assert O.mortar_ops(2, t)["Pf"].shape[0] == n


@pytest.mark.parametrize("order", [2, 3])
def test_projection_identities(order):
    # same order on both sides: the coarse projection is the identity, L = B^T = M P
    for t in range(6):
        o = O.mortar_ops(order, t)
        np.testing.assert_allclose(o["Pc"], np.eye(o["Pc"].shape[0]), atol=1e-12)
        np.testing.assert_allclose(o["Lc"], (o["M"] @ o["Pc"]).T, atol=1e-12)
        for f in range(o["Pf"].shape[0]):
            np.testing.assert_allclose(o["Lf"][f], (o["M"] @ o["Pf"][f]).T, atol=1e-12)
    # a conforming (SameLevel) mortar passes a constant through exactly
    o = O.mortar_ops(order, 0)
    one = np.ones(o["Pf"].shape[2])
    np.testing.assert_allclose(o["Pf"][0] @ one, one, atol=1e-12)


def test_fine_coupling_counts_split_line_points_twice():
    # mortar.cpp:176-200: the fine coupling sums full-face quadrature points inside the closed
    # sub-face; with 2p + 1 (odd) points the split line xi = 0 carries points that both halves
    # take. So sum_f B_f 1 exceeds B_c 1 by exactly the split-line points' contribution.
    order = 2
    o2 = O.mortar_ops(order, 1)  # Fine2x1: split in t1 at 0
    o0 = O.mortar_ops(order, 0)
    one = np.ones(o0["Pc"].shape[1])
    Bc1 = o0["Lc"].T @ one
    Bf1 = sum(o2["Lf"][f].T @ one for f in range(2))
    extra = Bf1 - Bc1
    assert np.abs(extra).max() > 1e-3  # the double count is visible
    # it equals the split line's quadrature points (xi_1 = 0) with their full weights
    n1 = 2 * order + 1
    gx, gw = np.polynomial.legendre.leggauss(n1)
    lgl = np.array([-1.0, 0.0, 1.0])
    def lag(x):
        return np.array([np.prod([(x - lgl[k]) / (lgl[j] - lgl[k]) for k in range(3) if k != j])
                         for j in range(3)])
    line = np.zeros(9)
    for qj in range(n1):
        w = gw[n1 // 2] * gw[qj]
        line += w * np.kron(lag(gx[qj]), lag(0.0))
    np.testing.assert_allclose(extra, line, atol=1e-12)


def test_apply_conserves_on_conforming_faces():
    # SameLevel mortar: coarse and fine lifts are equal and opposite, so the flux leaving one
    # element enters the other (sum over both faces' lifted values = 0)
    rng = np.random.default_rng(0)
    order, nd = 3, 64
    U = rng.standard_normal((2, nd))
    r = O.mortar_apply(order, [(0, 0, 1, [1], [0])], 2, [0.7, -0.2, 0.1], U)
    assert abs(r.sum()) < 1e-12 and np.abs(r).max() > 1e-3
