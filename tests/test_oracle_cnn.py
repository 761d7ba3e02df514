"""The preconditioner network's CPU reference: its backward pass against finite differences
(FP64, no bfloat16 rounding). Parity unpinned (no reference counterpart)."""
import numpy as np

import pyoracle as O


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    npar = O.cnn_nparams()
    assert npar == 32 * 9 * 16 + 32 + 2 * (32 * 9 * 32 + 32) + 16 * 9 * 32 + 16
    p = 0.2 * rng.standard_normal(npar)
    X = np.zeros((5, 6, 16))
    X[:, :, :9] = rng.standard_normal((5, 6, 9))
    T = np.zeros_like(X)
    T[:, :, :9] = rng.standard_normal((5, 6, 9))
    _, g, loss = O.cnn_forward_backward(p, X, T, round_bf16=False)
    for k in rng.choice(npar, 40, replace=False):
        e = np.zeros(npar)
        e[k] = 1e-6
        lp = O.cnn_forward_backward(p + e, X, T, round_bf16=False)[2]
        lm = O.cnn_forward_backward(p - e, X, T, round_bf16=False)[2]
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])
