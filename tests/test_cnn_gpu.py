"""GPU kernels of the learned preconditioner against the CPU reference network, and what the
trained network gains inside CG. Tolerances: forward/gradient relative L2 error 2e-2 (both
sides round weights and activations to bfloat16 at the same points; the GPU accumulates in
FP32, the reference in FP64, so a value can round to a neighbouring bfloat16)."""
import numpy as np
import pytest

import pyoracle as O
from drifter_b200.cnn import CNN, from_superpixels, to_superpixels, train_preconditioner
from drifter_b200.bezier import BezierSmoother

pytestmark = pytest.mark.gpu


def rl2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _img(rng, B, H, W):
    X = np.zeros((B, H, W, 16))
    X[..., :9] = rng.standard_normal((B, H, W, 9))
    return X


def test_forward_matches_reference():
    rng = np.random.default_rng(0)
    net = CNN(seed=3)
    p = net.params()
    X = _img(rng, 2, 19, 37)  # ragged tiles (H % 8, W % 16 != 0)
    Y, _, _ = net.forward_backward(X)
    for b in range(2):
        Yo, _, _ = O.cnn_forward_backward(p, X[b])
        assert rl2(Y[b][..., :9], Yo[..., :9]) < 2e-2
        assert np.abs(Y[b][..., 9:]).max() == 0.0


def test_gradient_matches_reference():
    rng = np.random.default_rng(1)
    net = CNN(seed=4)
    p = net.params()
    X = _img(rng, 1, 13, 21)
    T = _img(rng, 1, 13, 21)
    _, g, loss = net.forward_backward(X, T)
    _, go, lo = O.cnn_forward_backward(p, X[0], T[0])
    assert abs(loss - lo) / lo < 1e-2
    assert rl2(g, go) < 2e-2


_TC_CHILD = """
import sys, numpy as np
from drifter_b200.cnn import CNN
rng = np.random.default_rng(5)
X = np.zeros((2, 19, 37, 16)); X[..., :9] = rng.standard_normal((2, 19, 37, 9))
T = np.zeros((2, 19, 37, 16)); T[..., :9] = rng.standard_normal((2, 19, 37, 9))
Y, g, loss = CNN(seed=6).forward_backward(X, T)
np.savez(sys.argv[1], Y=Y, g=g, loss=loss)
"""


def test_tcgen05_conv_equals_mma_sync_conv(tmp_path):
    """DRIFTER_B200_CNN_MMA=tcgen05 runs every conv of the network (forward and input-gradient)
    on the tcgen05 kernel: TMA halo copies, MMAs from shared-memory descriptors into TMEM,
    tcgen05.ld epilogue. Both kernels add the same FP32 products of each 16-channel step in the
    same tap order, so the forward output, the loss and the gradient are bit-identical to the
    mma.sync kernel's (ragged 19 x 37 images, batch 2). The choice is read once per process:
    each form runs in its own child process."""
    import os
    import subprocess
    import sys

    out = {}
    for form in ("sync", "tcgen05"):
        env = dict(os.environ, DRIFTER_B200_CNN_MMA=form)
        path = tmp_path / f"{form}.npz"
        subprocess.run([sys.executable, "-c", _TC_CHILD, str(path)], env=env, check=True, timeout=600)
        out[form] = np.load(path)
    a, b = out["sync"], out["tcgen05"]
    assert np.isfinite(a["Y"]).all() and np.abs(a["Y"]).max() > 0
    for k in ("Y", "g", "loss"):
        assert np.array_equal(a[k], b[k]), k


def test_superpixel_layout():
    # control point (gi, gj) -> superpixel (I, J) = (gi // 3, gj // 3), channel gi % 3 + 3 (gj % 3)
    # (the layout of the library's pack/unpack kernels)
    n = 7
    nd = 3 * n + 1
    f = np.random.default_rng(2).standard_normal(nd * nd)
    sp = to_superpixels(f, n)
    for gi, gj in ((0, 0), (4, 2), (2, 7), (21, 21), (13, 5)):
        assert sp[gj // 3, gi // 3, gi % 3 + 3 * (gj % 3)] == f[gi + nd * gj]
    assert np.array_equal(from_superpixels(sp, n), f)


def test_trained_preconditioner_gains_over_plain_cg():
    """Trained on multigrid (residual, error) pairs of a 32x32 grid, used in flexible CG on a
    different bathymetry: reaches the FP64 1e-10 residual in fewer iterations than CG without
    a preconditioner and than Jacobi-PCG, and gives the same solution."""
    net, info = train_preconditioner(n=32, steps=600, rhs_count=12, seed=5, crop=33, batch=8)
    assert np.isfinite(info["loss"])
    from drifter_b200 import configs
    n, L = 32, 3200.0
    s = BezierSmoother(n, n, L, L, configs.c4(n=n, L=L, seed=77)["d"])
    s.mg_setup(2)
    net.attach(s)
    x_cnn, i_cnn = s.solve("cnn", tol=1e-10, maxit=2000)
    assert np.isfinite(x_cnn).all()
    x_cg, i_cg = s.solve("none", tol=1e-10, maxit=5000)
    x_j, i_j = s.solve("jacobi", tol=1e-10, maxit=5000)
    x_mg, i_mg = s.solve("mg", tol=1e-10, maxit=200)
    assert i_cnn["relres"] <= 1e-10
    assert i_cnn["iters"] < i_cg["iters"]
    assert i_cnn["iters"] < i_j["iters"]
    assert np.abs(x_cnn - x_mg).max() / np.abs(x_mg).max() < 1e-8


def test_c4_learned_pcg_beats_multigrid_and_jacobi_pcg_in_wall_time():
    """C4 at full size (512 x 512, 2.36 M control points): the learned preconditioner (trained
    on a 64 x 64 grid with the same element operator) reaches the FP64 1e-10 residual in less
    device time than multigrid-preconditioned CG and than Jacobi-PCG, and the same solution as
    multigrid to 1e-6 (the solves
    timed by CUDA events inside the library, best of three after a warm-up)."""
    from drifter_b200 import configs
    c = configs.c4()
    net, _ = train_preconditioner(n=64, dx=c["L"] / c["n"], lam=c["lam"], eps=c["eps"], steps=10000,
                                  rhs_count=16, seed=1)
    s = BezierSmoother(c["n"], c["n"], c["L"], c["L"], c["d"], lam=c["lam"], ridge_epsilon=c["eps"])
    s.mg_setup(2)
    net.attach(s)

    def best(pc):
        s.solve(pc, tol=1e-10, maxit=5000)
        runs = [s.solve(pc, tol=1e-10, maxit=5000) for _ in range(3)]
        return min(runs, key=lambda t: t[1]["ms"])

    x_cnn, i_cnn = best("cnn")
    x_mg, i_mg = best("mg")
    _, i_j = best("jacobi")
    assert i_cnn["relres"] <= 1e-10 and i_mg["relres"] <= 1e-10
    assert i_cnn["ms"] < i_mg["ms"], (i_cnn, i_mg)
    assert i_cnn["ms"] < i_j["ms"], (i_cnn, i_j)
    # two solves to the same 1e-10 residual differ by the operator's conditioning times that
    assert np.abs(x_cnn - x_mg).max() / np.abs(x_mg).max() < 1e-6
    s.close()
    net.close()


def test_conv_form_autotuner_keeps_the_preconditioner_unchanged(monkeypatch):
    """Attaching a network to a smoother times both conv forms (mma.sync, tcgen05) of every
    layer at the smoother's size and keeps the faster; the forms are bit-identical, so the
    preconditioner's output equals the one with the form forced either way."""
    n = 48
    X, Y = O.gauss_points(n, n, 0, 0, 3000.0, 3000.0)
    s = BezierSmoother(n, n, 3000.0, 3000.0, 100.0 + 0.01 * X, lam=1.0, ridge_epsilon=1e-4)
    net = CNN(seed=3)
    net.attach(s)
    t = s.cnn_tuning()
    assert all(f in ("mma_sync", "tcgen05") for f in t["forms"])
    assert all(v > 0 for f in ("mma_sync", "tcgen05") for v in t["ms"][f])
    r = np.random.default_rng(4).standard_normal(s.ndof)
    z = s.precondition(r, "cnn")
    assert np.isfinite(z).all() and np.abs(z).max() > 0
    s.close()
    net.close()
