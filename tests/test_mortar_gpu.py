"""Mortar coupling of non-conforming faces: the library's operators (host construction, CPU)
and its GPU flux/lift kernels against the FP64 oracle restatement of MortarSpace and
compute_interface_flux_nonconforming. Tolerance 1e-12 relative (FP64, different summation
order)."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200 import mortar as Mo


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_operators_match_oracle(order):
    for t in range(6):
        g, o = Mo.mortar_ops(order, t), O.mortar_ops(order, t)
        for k in ("M", "Minv", "Pc", "Lc", "Pf", "Lf"):
            assert rel(g[k], o[k]) < 1e-12, (order, t, k)


def test_create_rejects_bad_interfaces():
    from drifter_b200._abi import DrfError
    with pytest.raises(DrfError):
        Mo.MortarInterfaceManager(3, [(6, 0, 1, [1], [0])], 4)       # Boundary is not a mortar
    with pytest.raises(DrfError):
        Mo.MortarInterfaceManager(3, [(0, 0, 1, [9], [0])], 4)       # element out of range
    with pytest.raises(DrfError):
        Mo.MortarInterfaceManager(3, [(1, 0, 7, [1, 2], [0, 0])], 4)  # face id


def random_interfaces(n_if, n_elem, seed):
    """Interfaces of every connection type over random elements and faces (elements repeat,
    so per-element accumulation order matters)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_if):
        t = int(rng.integers(0, 6))
        k = Mo.NUM_FINE[t]
        els = rng.choice(n_elem, size=k + 1, replace=False)
        cf = int(rng.integers(0, 6))
        out.append((t, int(els[0]), cf, [int(e) for e in els[1:]],
                    [int(f) for f in rng.integers(0, 6, size=k)]))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("flux", ["central", "upwind", "lf"])
@pytest.mark.parametrize("order", [2, 3, 4])
def test_apply_matches_oracle(order, flux):
    n_elem = 60
    ifaces = random_interfaces(80, n_elem, seed=order)
    rng = np.random.default_rng(7)
    nd = (order + 1) ** 3
    U = rng.standard_normal((n_elem, nd))
    rhs0 = rng.standard_normal((n_elem, nd))
    a = np.array([0.8, -0.45, 0.3])
    m = Mo.MortarInterfaceManager(order, ifaces, n_elem)
    g = m.apply(U, a, flux, rhs=rhs0)
    o = O.mortar_apply(order, ifaces, Mo.FLUX[flux], a, U, rhs0)
    assert rel(g - rhs0, o - rhs0) < 1e-12
    m.close()


@pytest.mark.gpu
def test_apply_large_batch_matches_oracle():
    # a few thousand interfaces of an AMR-like mesh (every type, order 3)
    n_elem = 20000
    ifaces = random_interfaces(6000, n_elem, seed=11)
    U = np.random.default_rng(3).standard_normal((n_elem, 64))
    a = np.array([0.2, 1.0, -0.6])
    m = Mo.MortarInterfaceManager(3, ifaces, n_elem)
    g = m.apply(U, a, "lf")
    o = O.mortar_apply(3, ifaces, 2, a, U)
    assert rel(g, o) < 1e-12
    # conforming (SameLevel) interfaces alone conserve: lifts sum to zero
    same = [f for f in ifaces if f[0] == 0]
    m0 = Mo.MortarInterfaceManager(3, same, n_elem)
    assert abs(m0.apply(U, a, "lf").sum()) < 1e-9
