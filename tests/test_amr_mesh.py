"""The native face-connection builder (drf_amr_build_mesh) against the Python generator of the
same column-wise directional AMR meshes (configs.amr_mesh): identical elements, boxes,
conforming pairs, boundary faces and non-conforming interfaces in the same order; and the
argument checks. Host code only: runs without a GPU."""
import numpy as np
import pytest

from drifter_b200 import configs
from drifter_b200._abi import DrfError
from drifter_b200.amr import build_mesh


def _same(a, b):
    assert a["n_elem"] == b["n_elem"]
    assert np.array_equal(a["level"], b["level"])
    assert np.array_equal(a["box"], b["box"])  # the same IEEE operations: bit for bit
    assert np.array_equal(a["conf"], b["conf"])
    assert np.array_equal(a["bnd"], b["bnd"])
    assert len(a["ifaces"]) == len(b["ifaces"])
    for x, y in zip(a["ifaces"], b["ifaces"]):
        assert x[0] == y[0] and x[1] == y[1] and x[2] == y[2]
        assert list(x[3]) == list(y[3]) and list(x[4]) == list(y[4])
    assert np.array_equal(a["col_levels"], b["col_levels"])


@pytest.mark.parametrize("nb,seed", [(8, 1), (16, 2), (24, 7)])
def test_native_builder_equals_generator_on_coastline_meshes(nb, seed):
    lx, ly, lz = configs.c3_levels(nb, seed=seed)
    _same(build_mesh(lx, ly, lz), configs.amr_mesh(lx, ly, lz))


def test_native_builder_every_connection_type_and_nonsquare_base():
    # a 4 x 2 base grid: across each shared face the finer column is finer in one or both
    # tangential directions (Fine2x1, Fine1x2, Fine2x2) or in neither (conforming)
    levels = [[(0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 0)],
              [(1, 0, 0), (1, 1, 0), (0, 1, 1), (1, 0, 1)]]
    lx, ly, lz = (np.array([[c[d] for c in row] for row in levels]) for d in range(3))
    a, b = build_mesh(lx, ly, lz, L=3.0), configs.amr_mesh(lx, ly, lz, L=3.0)
    _same(a, b)
    assert {t for t, *_ in a["ifaces"]} == {1, 2, 5}


def test_native_builder_uniform_and_single_column():
    z = np.zeros((4, 6), int)
    m = build_mesh(z, z, z)
    _same(m, configs.amr_mesh(z, z, z))
    assert m["n_elem"] == 24 and len(m["ifaces"]) == 0
    one = np.array([[2]])
    m1 = build_mesh(one, one - 1, one)
    _same(m1, configs.amr_mesh(one, one - 1, one))
    assert m1["n_elem"] == 4 * 2 * 4


def test_native_builder_rejects_unbalanced_and_out_of_range_levels():
    ly = np.array([[0, 2]])
    z = np.zeros_like(ly)
    with pytest.raises(DrfError):
        build_mesh(z, ly, z)  # x neighbours two levels apart along their shared face
    with pytest.raises(DrfError):
        build_mesh(z, np.array([[0, 1]]), np.array([[1, 0]]))  # finer in y, coarser in z
    with pytest.raises(DrfError):
        build_mesh(np.array([[11]]), np.array([[0]]), np.array([[0]]))
    with pytest.raises(DrfError):
        build_mesh(np.array([[-1]]), np.array([[0]]), np.array([[0]]))


def test_native_builder_full_c3_size():
    lx, ly, lz = configs.c3_levels(256)
    m = build_mesh(lx, ly, lz)
    assert m["n_elem"] == 258624
    counts = {t: sum(1 for r in m["ifaces"] if r[0] == t) for t in (1, 2, 5)}
    assert counts == {1: 14710, 2: 2704, 5: 8092}
    assert len(m["conf"]) == 512081 and len(m["bnd"]) == 434880
