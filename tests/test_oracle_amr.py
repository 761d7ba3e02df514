"""C3 AMR mesh generator and the CPU oracle of DG3DIntegration::compute_rhs
(src/dg/operators_3d.cpp:228): face coverage, 2:1 connection types, the volume quadrature
restated against a dense per-element assembly, free-stream preservation on conforming meshes,
and the reference semantics (no conforming or boundary faces in mode 0)."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import configs

A = np.array([1.0, 0.6, 0.2])


@pytest.fixture(scope="module")
def small():
    return configs.c3(nb=8)


def test_every_face_is_covered_once(small):
    m = small["mesh"]
    seen = np.zeros((m["n_elem"], 6), np.int64)
    for e1, f1, e2, f2 in m["conf"]:
        seen[e1, f1] += 1
        seen[e2, f2] += 1
        assert f1 // 2 == f2 // 2 and f1 != f2
    for e, f in m["bnd"]:
        seen[e, f] += 1
    for t, ce, cf, fe, ff in m["ifaces"]:
        assert len(fe) == O.MORTAR_NUM_FINE[t] and t in (1, 2, 5)
        seen[ce, cf] += 1
        for e, f in zip(fe, ff):
            seen[e, f] += 1
            assert f // 2 == cf // 2 and f != cf
    assert (seen == 1).all()


def test_connection_geometry_matches_subface_order(small):
    """Fine faces lie in the sub-face rectangles of MortarSpace::compute_subface_bounds
    (src/dg/mortar.cpp:27) in the coarse face's tangential coordinates."""
    m = small["mesh"]
    box = m["box"]
    bounds = {1: [(-1, -1, 0, 1), (0, -1, 1, 1)], 2: [(-1, -1, 1, 0), (-1, 0, 1, 1)],
              5: [(-1, -1, 0, 0), (0, -1, 1, 0), (-1, 0, 0, 1), (0, 0, 1, 1)]}
    for t, ce, cf, fe, ff in m["ifaces"]:
        ax = cf // 2
        t1, t2 = [d for d in range(3) if d != ax]
        lo, hi = box[ce, :3], box[ce, 3:]
        for s, e in enumerate(fe):
            b = bounds[t][s]
            ref = lambda x, d: 2 * (x - lo[d]) / (hi[d] - lo[d]) - 1
            got = (ref(box[e, t1], t1), ref(box[e, t2], t2), ref(box[e, 3 + t1], t1), ref(box[e, 3 + t2], t2))
            assert np.allclose(got, b), (t, s)
            # the fine face touches the coarse face plane
            plane = box[ce, 3 + ax] if cf % 2 else box[ce, ax]
            fplane = box[e, 3 + ax] if ff[s] % 2 else box[e, ax]
            assert abs(plane - fplane) < 1e-12


def test_c3_mesh_size_and_levels():
    lx, ly, lz = configs.c3_levels(64)
    assert lx.max() == 3 and ly.max() == 3 and lz.max() == 1 and lx.min() == 0
    # 2:1 balance of the tangential levels across faces
    assert np.abs(np.diff(ly, axis=1)).max() <= 1 and np.abs(np.diff(lx, axis=0)).max() <= 1


def _dense_volume(order, a):
    """-sum_q w_q grad(phi_i)(x_q).a phi_j(x_q) assembled densely (volume_integral,
    src/dg/operators_3d.cpp:81) with numpy's Gauss-Legendre rule of N points."""
    npn = order + 1
    x = configs.lgl_nodes(order)
    gx, gw = np.polynomial.legendre.leggauss(order)
    def lag(xs, j):
        return np.prod([(xs - x[m]) / (x[j] - x[m]) for m in range(npn) if m != j], axis=0)
    def dlag(xs, j):
        s = 0.0
        for k in range(npn):
            if k == j:
                continue
            s = s + np.prod([(xs - x[m]) / (x[j] - x[m]) for m in range(npn) if m not in (j, k)], axis=0) / (x[j] - x[k])
        return s
    B = np.array([[lag(g, j) for j in range(npn)] for g in gx])
    Bd = np.array([[dlag(g, j) for j in range(npn)] for g in gx])
    W = np.einsum("a,b,c->abc", gw, gw, gw)
    V = (a[0] * np.einsum("ai,bj,ck->abcijk", Bd, B, B) + a[1] * np.einsum("ai,bj,ck->abcijk", B, Bd, B)
         + a[2] * np.einsum("ai,bj,ck->abcijk", B, B, Bd))
    P = np.einsum("ai,bj,ck->abcijk", B, B, B)
    K = -np.einsum("abc,abcIJK,abcijk->KJIkji", W, V, P).reshape(npn ** 3, npn ** 3)
    w = _lgl_w(order)
    return K, np.einsum("i,j,k->kji", w, w, w).ravel()


def _lgl_w(order):
    x = configs.lgl_nodes(order)
    from numpy.polynomial import legendre as L
    P = L.Legendre.basis(order)(x)
    return 2.0 / (order * (order + 1) * P * P)


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_volume_term_matches_dense_quadrature(order):
    """Mode 0 on a mesh without non-conforming faces is the volume term alone (the reference's
    TODO branches add nothing), i.e. M^-1 of the dense quadrature."""
    z = np.zeros((2, 3), np.int64)
    mesh = configs.amr_mesh(z, z, z)
    rng = np.random.default_rng(order)
    U = rng.standard_normal((mesh["n_elem"], (order + 1) ** 3))
    K, w3 = _dense_volume(order, A)
    ref = (U @ K.T) / w3
    got = O.amr_rhs(order, mesh, 0, 2, A, U)
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("flux", [0, 1, 2])
def test_free_stream_on_conforming_mesh(flux):
    z = np.zeros((3, 4), np.int64)
    mesh = configs.amr_mesh(z, z + 1, z)
    U = np.ones((mesh["n_elem"], 64))
    assert np.abs(O.amr_rhs(3, mesh, 1, flux, A, U)).max() < 1e-12


def test_rhs_is_linear(small):
    m = small["mesh"]
    rng = np.random.default_rng(2)
    U, V = rng.standard_normal((2, m["n_elem"], 64))
    for mode in (0, 1):
        r = O.amr_rhs(3, m, mode, 2, A, 2.0 * U - 3.0 * V)
        s = 2.0 * O.amr_rhs(3, m, mode, 2, A, U) - 3.0 * O.amr_rhs(3, m, mode, 2, A, V)
        assert np.abs(r - s).max() <= 1e-12 * np.abs(s).max()
