"""Element-list forms of the adaptive smoother's per-element work on quadtree meshes (hanging
nodes included): the L2 error estimate (compute_element_l2_error) and the element part of the
data-fitting assembly (assemble_data_fitting_global). The oracle is checked against properties
and the uniform-grid oracle on CPU; the GPU against the oracle on a refined quadtree."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200.bezier import BezierSmoother, mesh_data_fitting, mesh_element_errors


def _quadtree(L=1000.0):
    """A 4 x 4 grid with two cells split in four and one of those children split again: 25
    elements of three sizes, with hanging nodes along the split cells' sides."""
    cells = [(i * L / 4, j * L / 4, L / 4) for j in range(4) for i in range(4)]

    def split(c):
        x, y, h = c
        return [(x, y, h / 2), (x + h / 2, y, h / 2), (x, y + h / 2, h / 2), (x + h / 2, y + h / 2, h / 2)]

    out = []
    for k, c in enumerate(cells):
        if k in (5, 10):
            kids = split(c)
            if k == 5:
                kids = split(kids[3]) + kids[:3]
            out += kids
        else:
            out.append(c)
    return np.array([[x, y, x + h, y + h] for x, y, h in out])


def _gauss01(ng):
    x, w = np.polynomial.legendre.leggauss(ng)
    return 0.5 * (x + 1), 0.5 * w


def _data(bounds, ng, f):
    g, _ = _gauss01(ng)
    dx = bounds[:, 2] - bounds[:, 0]
    dy = bounds[:, 3] - bounds[:, 1]
    X = bounds[:, 0, None, None] + g[None, None, :] * dx[:, None, None]  # [e][qj][qi]
    Y = bounds[:, 1, None, None] + g[None, :, None] * dy[:, None, None]
    return f(X, Y).reshape(len(bounds), ng * ng)


def _bern(t):
    s = 1 - t
    return np.stack([s ** 3, 3 * t * s ** 2, 3 * t ** 2 * s, t ** 3], -1)


def test_oracle_error_of_data_on_the_patch_is_zero():
    b = _quadtree()
    rng = np.random.default_rng(0)
    c = rng.uniform(-50, 50, (len(b), 16))
    g, _ = _gauss01(4)
    Bu = _bern(g)
    # the patch at the Gauss points, [e][qj][qi]: sum_ab c[a + 4 b] Bu[qi, a] Bv[qj, b]
    zd = np.einsum("eba,ia,jb->eji", c.reshape(-1, 4, 4), Bu, Bu).reshape(len(b), 16)
    l2, nrm = O.bz_mesh_element_errors(b, c, zd, 4)
    assert np.abs(l2).max() < 1e-9
    zd2 = zd + 1.0  # a constant offset: l2 = sqrt(area), normalized = 1
    l2, nrm = O.bz_mesh_element_errors(b, c, zd2, 4)
    area = (b[:, 2] - b[:, 0]) * (b[:, 3] - b[:, 1])
    assert np.allclose(l2, np.sqrt(area), rtol=1e-9)
    assert np.allclose(nrm, 1.0, rtol=1e-9)


def test_oracle_mesh_error_equals_the_uniform_grid_oracle():
    """On a uniform grid the element list (coefficients gathered from the control grid) gives the
    uniform-grid estimate."""
    nx = ny = 5
    L = 800.0
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 100, (3 * ny + 1) * (3 * nx + 1))
    zd = rng.uniform(0, 100, (nx * ny, 16))
    b, c = [], []
    for ey in range(ny):
        for ex in range(nx):
            b.append([ex * L / nx, ey * L / ny, (ex + 1) * L / nx, (ey + 1) * L / ny])
            c.append([x[(3 * ex + i) + (3 * nx + 1) * (3 * ey + j)] for j in range(4) for i in range(4)])
    l2m, _ = O.bz_mesh_element_errors(np.array(b), np.array(c), zd, 4)
    l2u, _ = O.bz_element_errors(nx, ny, L, L, 4, x, zd)
    assert np.allclose(l2m, l2u, rtol=1e-12)


@pytest.mark.parametrize("ng,wsum", [(2, 1.0), (3, 1.0), (4, 0.5)])
def test_oracle_data_fitting_blocks(ng, wsum):
    """Partition of unity: the block sums to (sum of the rule's weights)^2 dx dy (relaxation 1),
    its row sums are BtWd for d = 1, and dTWd of d = 1 is the same total; the block is symmetric.
    gauss_legendre_01's 4-point weights sum to 1/2 (they are halved twice, :55-57), so the
    reference's default ngauss_data = 4 weighs the data a quarter of what n = 2 or 3 does; the
    oracle keeps that, as the uniform-grid path does."""
    b = _quadtree()
    area = (b[:, 2] - b[:, 0]) * (b[:, 3] - b[:, 1])
    K, r, dd = O.bz_mesh_data_fitting(b, np.ones((len(b), ng * ng)), ng)
    assert np.allclose(K.sum((1, 2)), wsum ** 2 * area, rtol=1e-13)
    assert np.allclose(K.sum(2), r, rtol=1e-12)
    assert np.allclose(K, K.transpose(0, 2, 1), rtol=0, atol=1e-12 * area.max())
    assert np.allclose(dd, wsum ** 2 * area, rtol=1e-13)
    rel = np.full((len(b), ng * ng), 0.5)
    K2, r2, dd2 = O.bz_mesh_data_fitting(b, np.ones((len(b), ng * ng)), ng, relax=rel)
    assert np.allclose(K2, 0.5 * K, rtol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("ng", [2, 4, 6])
def test_mesh_element_errors_match_oracle(ng):
    b = _quadtree()
    rng = np.random.default_rng(ng)
    c = rng.uniform(-50, 50, (len(b), 16))
    zd = _data(b, ng, lambda X, Y: 30 * np.sin(X / 130.0) * np.cos(Y / 170.0))
    l2, nrm = mesh_element_errors(b, c, zd, ng)
    rl2, rnrm = O.bz_mesh_element_errors(b, c, zd, ng)
    assert np.abs(l2 - rl2).max() <= 1e-13 * np.abs(rl2).max()
    assert np.abs(nrm - rnrm).max() <= 1e-13 * np.abs(rnrm).max()


@pytest.mark.gpu
@pytest.mark.parametrize("ng", [1, 3, 4])
def test_mesh_data_fitting_matches_oracle(ng):
    """Same points, same Bernstein recurrence, every term rounded in the reference's order:
    the blocks agree with the oracle to the last bit (or within 1e-15 of their scale)."""
    b = _quadtree()
    zd = _data(b, ng, lambda X, Y: 1000 + 300 * np.tanh((X - Y) / 90.0))
    rel = 0.5 + 0.5 * np.random.default_rng(ng).uniform(size=(len(b), ng * ng))
    K, r, dd = mesh_data_fitting(b, zd, ng, relax=rel)
    rK, rr, rdd = O.bz_mesh_data_fitting(b, zd, ng, relax=rel)
    for got, ref in ((K, rK), (r, rr), (dd, rdd)):
        assert np.abs(got - ref).max() <= 1e-15 * np.abs(ref).max()


@pytest.mark.gpu
def test_mesh_element_errors_equal_the_uniform_gpu_path():
    """The element list of a uniform grid reproduces the uniform-grid GPU estimate."""
    n = 8
    L = 1600.0
    rng = np.random.default_rng(4)
    data = rng.uniform(0, 100, n * n * 16)
    s = BezierSmoother(n, n, L, L, data, lam=1.0, ridge_epsilon=1e-4)
    x = rng.uniform(0, 100, s.ndof)
    zd = rng.uniform(0, 100, (n * n, 16))
    l2u, _ = s.element_errors(x, zd, 4)
    b, c = [], []
    for ey in range(n):
        for ex in range(n):
            b.append([ex * L / n, ey * L / n, (ex + 1) * L / n, (ey + 1) * L / n])
            c.append([x[(3 * ex + i) + (3 * n + 1) * (3 * ey + j)] for j in range(4) for i in range(4)])
    l2m, _ = mesh_element_errors(np.array(b), np.array(c), zd, 4)
    assert np.allclose(l2m, l2u, rtol=1e-12)
    s.close()
