"""Learned preconditioner for the Bezier smoother's CG (no counterpart in the reference).

A 4-layer conv3x3 network (BF16 weights/activations, FP32 accumulation, hand-written tensor-
core kernels in libdrifter_b200.so) maps a residual to an approximate error on 3x3
superpixels of the control-point grid. It is trained on the GPU on (residual, error) pairs
that the smoother's own multigrid iterations produce (x_{k+1} = x_k + M(b - Q x_k), the
reference's repeated V-cycles of BezierMultigridPreconditioner::apply), and used as
preconditioner kind "cnn" of BezierSmoother.solve (flexible CG).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import check, dptr, lib
from .bezier import BezierSmoother


def _sigs():
    L = lib()
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    sigs = {
        "drf_cnn_create": ([C.c_uint64, C.POINTER(C.c_void_p)], C.c_int),
        "drf_cnn_destroy": ([vp], C.c_int),
        "drf_cnn_get_params": ([vp, dp], C.c_int),
        "drf_cnn_set_params": ([vp, dp], C.c_int),
        "drf_cnn_forward_backward": ([vp, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp], C.c_int),
        "drf_cnn_set_dataset": ([vp, C.c_int, C.c_int, C.c_int, dp, dp], C.c_int),
        "drf_cnn_train": ([vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64, dp], C.c_int),
        "drf_bz_set_cnn": ([vp, vp, C.c_double], C.c_int),
        "drf_cnn_nparams": ([], C.c_int64),
    }
    for k, (a, r) in sigs.items():
        getattr(L, k).argtypes = a
        getattr(L, k).restype = r
    return L


def to_superpixels(field: np.ndarray, n: int) -> np.ndarray:
    """(3n+1)^2 control-point field -> (n+1) x (n+1) x 16 (channel di + 3 dj, 9 used)."""
    nd = 3 * n + 1
    S = n + 1
    g = np.zeros((3 * S, 3 * S))
    g[:nd, :nd] = field.reshape(nd, nd)  # [gj][gi]
    sp = g.reshape(S, 3, S, 3).transpose(0, 2, 1, 3).reshape(S, S, 9)  # [J][I][di + 3 dj]
    out = np.zeros((S, S, 16))
    out[:, :, :9] = sp
    return out


def from_superpixels(sp: np.ndarray, n: int) -> np.ndarray:
    nd = 3 * n + 1
    S = n + 1
    g = sp[:, :, :9].reshape(S, S, 3, 3).transpose(0, 2, 1, 3).reshape(3 * S, 3 * S)
    return g[:nd, :nd].reshape(-1).copy()


class CNN:
    """The network handle: parameters, forward/backward, training on a device dataset."""

    def __init__(self, seed: int = 1):
        L = _sigs()
        h = C.c_void_p()
        check(L.drf_cnn_create(seed, C.byref(h)))
        self.h = h
        self.nparams = int(L.drf_cnn_nparams())
        self.out_scale = 1.0

    def close(self):
        if getattr(self, "h", None):
            lib().drf_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.empty(self.nparams)
        check(lib().drf_cnn_get_params(self.h, dptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        check(lib().drf_cnn_set_params(self.h, dptr(p)))

    def forward_backward(self, X, T=None):
        X = np.ascontiguousarray(X, dtype=np.float64)
        B, H, W, _ = X.shape
        Y = np.empty_like(X)
        grad = np.empty(self.nparams) if T is not None else None
        loss = C.c_double()
        Tc = np.ascontiguousarray(T, dtype=np.float64) if T is not None else None
        check(lib().drf_cnn_forward_backward(self.h, B, H, W, dptr(X), dptr(Tc) if Tc is not None else None,
                                             dptr(Y), dptr(grad) if grad is not None else None,
                                             C.byref(loss)))
        return Y, grad, loss.value

    def set_dataset(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        N, H, W, _ = X.shape
        check(lib().drf_cnn_set_dataset(self.h, N, H, W, dptr(X), dptr(T)))

    def train(self, steps, batch=16, crop=48, lr=1e-3, seed=0) -> float:
        loss = C.c_double()
        check(lib().drf_cnn_train(self.h, steps, batch, crop, lr, seed, C.byref(loss)))
        return loss.value

    def attach(self, smoother: BezierSmoother):
        check(lib().drf_bz_set_cnn(smoother.h, self.h, self.out_scale))


def multigrid_pairs(s: BezierSmoother, n: int, rhs_list, vcycles: int = 6):
    """(residual, error) pairs from the smoother's multigrid iteration x_{k+1} = x_k + M r_k
    for each right-hand side; the exact solution comes from an MG-PCG solve to 1e-12."""
    pairs = []
    for b in rhs_list:
        xs, _ = s.solve("mg", tol=1e-12, maxit=200, b=b)
        x = np.zeros_like(b)
        for _ in range(vcycles):
            r = b - s.apply_Q(x)
            pairs.append((r, xs - x))
            x = x + s.mg_apply(r)
    return pairs


def random_rhs(s: BezierSmoother, n: int, L: float, count: int, seed: int):
    """Right-hand sides of the smoother for random bathymetries (smooth fBm-like sums of
    Fourier modes plus rough noise), i.e. Q x for random control-point fields."""
    rng = np.random.default_rng(seed)
    nd = 3 * n + 1
    gi, gj = np.meshgrid(np.arange(nd), np.arange(nd))
    out = []
    for k in range(count):
        f = np.zeros((nd, nd))
        for _ in range(24):
            kx, ky = rng.normal(0, 6, 2)
            amp = 1.0 / (1.0 + kx * kx + ky * ky)
            f += amp * np.sin(2 * np.pi * (kx * gi + ky * gj) / nd + rng.uniform(0, 6.3))
        if k % 2:
            f += 0.05 * rng.standard_normal((nd, nd))
        out.append(s.apply_Q(f.reshape(-1)))
    return out


def build_dataset(pairs, n, s: BezierSmoother, scale=None):
    """Inputs r / rms(r); targets the error the Jacobi base leaves, (e - D^-1 r) / (rms(r) s)."""
    res = [(r, e - s.precondition(r, "jacobi")) for r, e in pairs]
    if scale is None:
        scale = float(np.median([np.sqrt(np.mean(c * c) / np.mean(r * r)) for r, c in res]))
    X, T = [], []
    for r, c in res:
        sr = np.sqrt(np.mean(r * r))
        X.append(to_superpixels(r / sr, n))
        T.append(to_superpixels(c / (sr * scale), n))
    return np.stack(X), np.stack(T), scale


def fcg_pairs(s: BezierSmoother, net: "CNN", rhs_list, iters: int = 8):
    """(residual, error) pairs along flexible CG with the current network (its own residual
    distribution), exact solutions from multigrid PCG."""
    net.attach(s)
    pairs = []
    for b in rhs_list:
        xs, _ = s.solve("mg", tol=1e-12, maxit=200, b=b)
        for k in range(1, iters + 1):
            x, _ = s.solve("cnn", tol=1e-30, maxit=k, b=b)
            pairs.append((b - s.apply_Q(x), xs - x))
    return pairs


def bathymetry_rhs(n: int, L: float, lam: float, eps: float, count: int, seed: int):
    """Right-hand sides lambda B^T W d of smoothing problems on seeded fBm bathymetries."""
    from . import configs
    out = []
    for k in range(count):
        d = configs.c4(n=n, L=L, seed=seed * 1000 + k, lam=lam, eps=eps)["d"]
        s = BezierSmoother(n, n, L, L, d, lam=lam, ridge_epsilon=eps)
        out.append(s.rhs())
        s.close()
    return out


def train_preconditioner(n=64, dx=100.0, lam=1.0, eps=1e-4, d=None, rhs_count=16, steps=10000,
                         seed=1, lr=2e-3, crop=48, batch=16, rounds=3, fcg_iters=14):
    """Trains a network on a training grid of n x n elements with element size dx (the same
    element operator as the target grid) and returns it with its output scale set. Training
    pairs come from the multigrid iterations of smoothing problems (bathymetry right-hand
    sides) and of random fields; each later round (rounds - 1 of them) adds the residuals the
    current network meets inside flexible CG on every right-hand side (fcg_iters iterations
    each) and trains on, for half the steps at half the rate."""
    L = n * dx
    if d is None:
        from . import configs
        d = configs.c4(n=n, L=L, seed=seed + 101)["d"]
    s = BezierSmoother(n, n, L, L, d, lam=lam, ridge_epsilon=eps)
    s.mg_setup(2)
    rhs = bathymetry_rhs(n, L, lam, eps, rhs_count, seed) + random_rhs(s, n, L, rhs_count // 2, seed)
    X, T, scale = build_dataset(multigrid_pairs(s, n, rhs), n, s)
    net = CNN(seed)
    net.set_dataset(X, T)
    loss = net.train(steps, batch=batch, crop=min(crop, n + 1), lr=lr, seed=seed)
    net.out_scale = scale
    for r in range(1, rounds):
        X2, T2, _ = build_dataset(fcg_pairs(s, net, rhs, iters=fcg_iters), n, s, scale)
        X, T = np.concatenate([X, X2]), np.concatenate([T, T2])
        net.set_dataset(X, T)
        loss = net.train(steps // 2, batch=batch, crop=min(crop, n + 1), lr=lr * 0.5, seed=seed + r)
    s.close()
    return net, dict(loss=loss, scale=scale, pairs=len(X))
