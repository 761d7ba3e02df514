"""Seeded synthetic basins standing in for the reference's GeoTIFF/EMODnet inputs.

C1  plain FP64 DG, CPU-runnable: 100x100 km closed basin, 16x16x4 hexes, N=3, Gaussian
    seamount 50-500 m, uniform 0.1 N/m^2 wind stress, T/S constant, 20 barotropic subcycles.
C2  uniform large DG: 200x200 km, 128x128x16 hexes, N=4, depth 20 m + 32 random Gaussians
    clipped to [20, 2000] m, M2 tide (1 m, 44714 s) on the west boundary, linear T
    stratification (20 C surface to 4 C bottom), S = 35.
C5  uneven ensemble: 64 independent runs, N=3, meshes 16..64 x 16..64 x 4..8 hexes, per-member
    seeded bathymetry (Gaussian bumps over a sloping shelf) and wind stress 0-0.2 N/m^2, mixed
    precision.
Any config can be shrunk (nx, ny, nz overrides) for parity tests: the generator keeps the
physics and the seeded bathymetry law.
"""
from __future__ import annotations

import numpy as np

from .dg import DGConfig

SEED = 20261203


def lgl_nodes(order: int) -> np.ndarray:
    from numpy.polynomial import legendre as L
    if order == 1:
        return np.array([-1.0, 1.0])
    inner = np.sort(L.Legendre.basis(order).deriv().roots().real)
    return np.concatenate([[-1.0], inner, [1.0]])


def node_coords(cfg: DGConfig):
    """2D node coordinates x, y (size n2) and sigma of the 3D nodes (size n3)."""
    npn = cfg.order + 1
    xi = lgl_nodes(cfg.order)
    dx, dy, ds = cfg.Lx / cfg.nx, cfg.Ly / cfg.ny, 1.0 / cfg.nz
    ex = np.arange(cfg.nx)
    ey = np.arange(cfg.ny)
    # [ey, ex, j, i]
    X = (ex[None, :, None, None] + 0.5 * (xi[None, None, None, :] + 1.0)) * dx
    Y = (ey[:, None, None, None] + 0.5 * (xi[None, None, :, None] + 1.0)) * dy
    X = np.broadcast_to(X, (cfg.ny, cfg.nx, npn, npn)).reshape(-1).copy()
    Y = np.broadcast_to(Y, (cfg.ny, cfg.nx, npn, npn)).reshape(-1).copy()
    ez = np.arange(cfg.nz)
    # [col, ez, k, j, i]
    S = -1.0 + ds * (ez[:, None] + 0.5 * (xi[None, :] + 1.0))  # [ez, k]
    S = np.broadcast_to(S[None, :, :, None, None], (cfg.nx * cfg.ny, cfg.nz, npn, npn, npn))
    return X, Y, S.reshape(-1).copy()


def expand_2d_to_3d(cfg: DGConfig, a2: np.ndarray) -> np.ndarray:
    npn = cfg.order + 1
    a = a2.reshape(cfg.nx * cfg.ny, 1, 1, npn * npn)
    return np.broadcast_to(a, (cfg.nx * cfg.ny, cfg.nz, npn, npn * npn)).reshape(-1).copy()


def _cfl_dt(cfg: DGConfig, hmax: float, nsub: int, cfl: float = 0.3) -> float:
    xi = lgl_nodes(cfg.order)
    dmin = min(cfg.Lx / cfg.nx, cfg.Ly / cfg.ny) * 0.5 * (xi[1] - xi[0])
    c = np.sqrt(cfg.g * hmax) + 1.0
    return nsub * cfl * dmin / c


def c1(nx=16, ny=16, nz=4, order=3, precision="fp64", seed=SEED, flux2d="lf"):
    cfg = DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=100e3, Ly=100e3, precision=precision,
                   flux2d=flux2d)
    X, Y, Sg = node_coords(cfg)
    r2 = (X - 50e3) ** 2 + (Y - 50e3) ** 2
    h = 500.0 - 450.0 * np.exp(-r2 / (2 * 15e3 ** 2))
    f = np.full(cfg.n2, 1e-4)
    taux = np.full(cfg.n2, 0.1)
    tauy = np.zeros(cfg.n2)
    eta = np.zeros(cfg.n2)
    H3 = expand_2d_to_3d(cfg, h + eta)
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), 10.0 * H3, 35.0 * H3]
    nsub = 20
    dt = _cfl_dt(cfg, h.max(), nsub)
    return dict(cfg=cfg, h=h, f=f, taux=taux, tauy=tauy, q=q, eta=eta, dt=dt, nsub=nsub,
                steps=100, name=f"C1 {nx}x{ny}x{nz} N={order}")


def c2(nx=128, ny=128, nz=16, order=4, precision="mixed", seed=SEED, flux2d="lf", Lx=200e3):
    rng = np.random.default_rng(seed)
    cfg = DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=Lx, Ly=Lx, precision=precision,
                   flux2d=flux2d, bc=("tide", "wall", "wall", "wall"), tide_amp=1.0,
                   tide_period=44714.0)
    X, Y, Sg = node_coords(cfg)
    h = np.full(cfg.n2, 20.0)
    amp = rng.uniform(0.0, 1980.0, 32)
    wid = rng.uniform(5e3, 40e3, 32) * (Lx / 200e3)
    cx = rng.uniform(0.0, Lx, 32)
    cy = rng.uniform(0.0, Lx, 32)
    for a, w, x0, y0 in zip(amp, wid, cx, cy):
        h += a * np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * w * w))
    h = np.clip(h, 20.0, 2000.0)
    f = np.full(cfg.n2, 1e-4)
    taux = np.zeros(cfg.n2)
    tauy = np.zeros(cfg.n2)
    eta = np.zeros(cfg.n2)
    H3 = expand_2d_to_3d(cfg, h + eta)
    T = 4.0 + 16.0 * (1.0 + Sg)
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), T * H3, 35.0 * H3]
    nsub = 20
    dt = _cfl_dt(cfg, h.max(), nsub)
    return dict(cfg=cfg, h=h, f=f, taux=taux, tauy=tauy, q=q, eta=eta, dt=dt, nsub=nsub,
                steps=500, name=f"C2 {nx}x{ny}x{nz} N={order}")


def perturb(case: dict, seed: int = 7, amp_u: float = 0.05, amp_eta: float = 0.05) -> dict:
    """Adds a seeded smooth velocity and surface perturbation (to exercise every term)."""
    cfg = case["cfg"]
    rng = np.random.default_rng(seed)
    X, Y, Sg = node_coords(cfg)
    kx, ky = rng.uniform(1, 3, 2)
    ph = rng.uniform(0, 2 * np.pi, 4)
    eta = amp_eta * np.sin(2 * np.pi * kx * X / cfg.Lx + ph[0]) * np.cos(2 * np.pi * ky * Y / cfg.Ly + ph[1])
    H3 = expand_2d_to_3d(cfg, case["h"] + eta)
    X3, Y3 = expand_2d_to_3d(cfg, X), expand_2d_to_3d(cfg, Y)
    u = amp_u * np.sin(2 * np.pi * X3 / cfg.Lx + ph[2]) * (1.0 + 0.5 * Sg)
    v = amp_u * np.cos(2 * np.pi * Y3 / cfg.Ly + ph[3]) * (1.0 - 0.3 * Sg)
    q = [u * H3, v * H3, case["q"][2] / expand_2d_to_3d(cfg, case["h"] + case["eta"]) * H3,
         case["q"][3] / expand_2d_to_3d(cfg, case["h"] + case["eta"]) * H3]
    out = dict(case)
    out.update(q=q, eta=eta)
    return out


def gauss01_4() -> np.ndarray:
    a = np.sqrt(3 / 7 - 2 / 7 * np.sqrt(6 / 5))
    b = np.sqrt(3 / 7 + 2 / 7 * np.sqrt(6 / 5))
    return np.array([0.5 * (1 - b), 0.5 * (1 - a), 0.5 * (1 + a), 0.5 * (1 + b)])


def fbm_field(m: int, seed: int = SEED, beta: float = 2.0) -> np.ndarray:
    """Periodic fractional-Brownian surface on an m x m grid with power spectrum 1/f^beta."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(m)[None, :]
    ky = np.fft.fftfreq(m)[:, None]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-beta / 2.0)
    amp[0, 0] = 0.0
    ph = rng.uniform(0, 2 * np.pi, (m, m))
    return np.real(np.fft.ifft2(amp * np.exp(1j * ph)))


def c4(n: int = 512, L: float = 51200.0, seed: int = SEED, lam: float = 1.0, eps: float = 1e-4):
    """C4: cubic Bezier smoother on an n x n grid over seeded fBm bathymetry (1/f^2 spectrum)
    scaled to 0-4000 m, sampled at the 4x4 Gauss points of every element ([ey][ex][qj][qi])."""
    m = 4 * n
    f = fbm_field(m, seed)
    f = 4000.0 * (f - f.min()) / (f.max() - f.min())
    p = gauss01_4()
    dx = L / n
    ex = np.arange(n)
    X = (ex[None, :, None, None] + p[None, None, None, :]) * dx
    Y = (ex[:, None, None, None] + p[None, None, :, None]) * dx
    X = np.broadcast_to(X, (n, n, 4, 4)).reshape(-1)
    Y = np.broadcast_to(Y, (n, n, 4, 4)).reshape(-1)
    # bilinear sampling of the periodic grid field (cell-centred samples at (i + 0.5) L / m)
    u = X / L * m - 0.5
    v = Y / L * m - 0.5
    i0 = np.floor(u).astype(np.int64)
    j0 = np.floor(v).astype(np.int64)
    fu, fv = u - i0, v - j0
    i0 %= m
    j0 %= m
    i1, j1 = (i0 + 1) % m, (j0 + 1) % m
    d = ((1 - fu) * (1 - fv) * f[j0, i0] + fu * (1 - fv) * f[j0, i1] + (1 - fu) * fv * f[j1, i0]
         + fu * fv * f[j1, i1])
    return dict(n=n, L=L, lam=lam, eps=eps, d=d.copy(), name=f"C4 Bezier {n}x{n}")


def c5_member(i: int, nx: int, ny: int, nz: int, order: int = 3, precision: str = "mixed",
              seed: int = SEED) -> dict:
    """Member i of the C5 ensemble: a closed 2 km-per-element basin with its own seeded
    bathymetry (20-1000 m: a sloping shelf plus 8 Gaussian bumps) and uniform wind stress."""
    rng = np.random.default_rng(seed + 1000 + i)
    L = 2e3
    cfg = DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=nx * L, Ly=ny * L, precision=precision)
    X, Y, Sg = node_coords(cfg)
    h = 20.0 + 480.0 * X / cfg.Lx
    for _ in range(8):
        a, w = rng.uniform(0.0, 400.0), rng.uniform(0.03, 0.12) * min(cfg.Lx, cfg.Ly)
        x0, y0 = rng.uniform(0.0, cfg.Lx), rng.uniform(0.0, cfg.Ly)
        h += a * np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * w * w))
    h = np.clip(h, 20.0, 1000.0)
    tau = rng.uniform(0.0, 0.2)
    ang = rng.uniform(0.0, 2 * np.pi)
    f = np.full(cfg.n2, 1e-4)
    taux = np.full(cfg.n2, tau * np.cos(ang))
    tauy = np.full(cfg.n2, tau * np.sin(ang))
    eta = np.zeros(cfg.n2)
    H3 = expand_2d_to_3d(cfg, h + eta)
    T = 8.0 + 8.0 * (1.0 + Sg)
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), T * H3, 35.0 * H3]
    nsub = 20
    dt = _cfl_dt(cfg, h.max(), nsub)
    return dict(cfg=cfg, h=h, f=f, taux=taux, tauy=tauy, q=q, eta=eta, dt=dt, nsub=nsub,
                name=f"C5 member {i} {nx}x{ny}x{nz} N={order}")


def c5(members: int = 64, nmin: int = 16, nmax: int = 64, zmin: int = 4, zmax: int = 8,
       order: int = 3, precision: str = "mixed", seed: int = SEED) -> list:
    """C5: an uneven ensemble; member sizes uniform in {nmin..nmax}^2 x {zmin..zmax}."""
    rng = np.random.default_rng(seed + 5)
    sizes = [(int(rng.integers(nmin, nmax + 1)), int(rng.integers(nmin, nmax + 1)),
              int(rng.integers(zmin, zmax + 1))) for _ in range(members)]
    return [c5_member(i, nx, ny, nz, order, precision, seed) for i, (nx, ny, nz) in enumerate(sizes)]
