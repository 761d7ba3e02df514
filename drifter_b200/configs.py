"""Seeded synthetic basins standing in for the reference's GeoTIFF/EMODnet inputs.

C1  plain FP64 DG, CPU-runnable: 100x100 km closed basin, 16x16x4 hexes, N=3, Gaussian
    seamount 50-500 m, uniform 0.1 N/m^2 wind stress, T/S constant, 20 barotropic subcycles.
C2  uniform large DG: 200x200 km, 128x128x16 hexes, N=4, depth 20 m + 32 random Gaussians
    clipped to [20, 2000] m, M2 tide (1 m, 44714 s) on the west boundary, linear T
    stratification with level isotherms (20 C at the surface to 4 C at 2000 m), S = 35, passive
    unless the equation of state is switched on (c2(baroclinic=True)), whose pressure gradient
    is then taken against the same profile as reference stratification.
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
# C2's linear stratification: 20 C at the surface, 4 C at 2000 m depth
C2_T_SURFACE = 20.0
C2_T_DZ = 16.0 / 2000.0


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
    # T and S constant: no baroclinic pressure (the equation of state is off)
    cfg = DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=100e3, Ly=100e3, precision=precision,
                   flux2d=flux2d, alpha=0.0, beta=0.0)
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


def c2(nx=128, ny=128, nz=16, order=4, precision="mixed", seed=SEED, flux2d="lf", Lx=200e3,
       wscale=None, baroclinic=False):
    """wscale scales the seamount widths (default Lx / 200 km: a shrunk copy of the basin;
    1.0 keeps C2's 5-40 km widths, and so its slopes, in a smaller basin).

    baroclinic=True switches the equation of state on (the stratification's pressure gradient,
    against the same profile as reference stratification); by default the stratification is a
    passive tracer. On C2's seamount flanks (slopes to 0.19) the coupled baroclinic step grows
    within about a hundred steps, so the 500-step workload runs with the tracer passive."""
    rng = np.random.default_rng(seed)
    eos = {} if baroclinic else {"alpha": 0.0, "beta": 0.0}
    cfg = DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=Lx, Ly=Lx, precision=precision,
                   flux2d=flux2d, bc=("tide", "wall", "wall", "wall"), tide_amp=1.0,
                   tide_period=44714.0, Tref_s=C2_T_SURFACE, Tref_dz=C2_T_DZ, **eos)
    X, Y, Sg = node_coords(cfg)
    h = np.full(cfg.n2, 20.0)
    amp = rng.uniform(0.0, 1980.0, 32)
    wid = rng.uniform(5e3, 40e3, 32) * (Lx / 200e3 if wscale is None else wscale)
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
    T = C2_T_SURFACE + C2_T_DZ * (expand_2d_to_3d(cfg, eta) + Sg * H3)  # T(z), z = eta + sigma H
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
    bathymetry (20-1000 m: a sloping shelf plus 8 Gaussian bumps) and uniform wind stress;
    temperature and salinity uniform (10 C, 35), so the equation of state is off."""
    rng = np.random.default_rng(seed + 1000 + i)
    L = 2e3
    cfg = DGConfig(nx=nx, ny=ny, nz=nz, order=order, Lx=nx * L, Ly=ny * L, precision=precision,
                   alpha=0.0, beta=0.0)
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
    # T and S at the equation of state's reference values: a wind-driven, unstratified member
    q = [np.zeros(cfg.n3), np.zeros(cfg.n3), cfg.T0 * H3, cfg.S0 * H3]
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


# ----------------------------------------------------------------------------- C3 AMR mesh
FINE_TYPE = {(0, 0): 0, (1, 0): 1, (0, 1): 2, (1, 1): 5}  # (split t1, split t2) -> FaceConnectionType


def fbm_hurst(m: int, hurst: float, seed: int) -> np.ndarray:
    """Periodic fractional-Brownian surface with Hurst exponent H (spectrum 1/f^(2H+2))."""
    return fbm_field(m, seed, beta=2.0 * hurst + 2.0)


def c3_levels(nb: int = 256, hurst: float = 0.7, seed: int = SEED, lmax: int = 3):
    """Directional refinement levels (lx, ly, lz) per base column of an nb x nb grid, refined
    towards the zero line of a seeded fBm field (the coastline: wet columns, mean below the
    median, with a dry column across a face): level lmax on coastal columns,
    one less per column of Chebyshev distance; on the coast the direction along the coastline
    is refined one level less (anisotropy); 2:1 balance in every tangential direction; a
    vertical split where both horizontal levels are lmax."""
    sub = 4
    phi = fbm_hurst(nb * sub, hurst, seed)
    phi = phi - np.median(phi)
    pm = phi.reshape(nb, sub, nb, sub).mean(axis=(1, 3))  # [iy, ix] column means
    wet = pm < 0
    coast = np.zeros_like(wet)  # wet columns with a dry column across a face
    coast[:, :-1] |= wet[:, :-1] & ~wet[:, 1:]
    coast[:, 1:] |= wet[:, 1:] & ~wet[:, :-1]
    coast[:-1, :] |= wet[:-1, :] & ~wet[1:, :]
    coast[1:, :] |= wet[1:, :] & ~wet[:-1, :]
    # Chebyshev distance to the coast (in columns), capped at lmax + 1
    dist = np.where(coast, 0, lmax + 1).astype(np.int64)
    for d in range(1, lmax + 1):
        near = np.zeros_like(coast)
        src = dist == d - 1
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                near |= np.roll(np.roll(src, dy, 0), dx, 1)
        dist = np.where((dist > d) & near, d, dist)
    L = np.maximum(0, lmax - dist)
    gy, gx = np.gradient(pm)
    lx, ly = L.copy(), L.copy()
    along_y = coast & (np.abs(gx) >= 2.0 * np.abs(gy))  # coastline runs along y: refine x more
    along_x = coast & (np.abs(gy) >= 2.0 * np.abs(gx))
    ly[along_y] = np.maximum(0, ly[along_y] - 1)
    lx[along_x] = np.maximum(0, lx[along_x] - 1)
    # 2:1 balance of the tangential levels across faces (raise the coarser side)
    for _ in range(2 * lmax + 2):
        ly_n = np.maximum(np.roll(ly, 1, 1), np.roll(ly, -1, 1))  # x neighbours (periodic rolls
        lx_n = np.maximum(np.roll(lx, 1, 0), np.roll(lx, -1, 0))  # are harmless: only raise)
        ly2, lx2 = np.maximum(ly, ly_n - 1), np.maximum(lx, lx_n - 1)
        if (ly2 == ly).all() and (lx2 == lx).all():
            break
        ly, lx = ly2, lx2
    lz = ((lx == lmax) & (ly == lmax)).astype(np.int64)
    return lx, ly, lz


def amr_mesh(lx, ly, lz, L: float = 1.0):
    """Hexahedra and face connections of a column-wise directionally refined grid.

    Returns elements (grouped by level tuple), conforming face pairs, boundary faces and the
    non-conforming interfaces (type, coarse element and face, fine elements and faces in the
    sub-face order of MortarSpace::compute_subface_bounds, src/dg/mortar.cpp:27), sorted by
    connection type. Face f has its normal along axis f // 2, positive when f is odd; the
    tangential axes of a face are the other two in axis order (t1 < t2)."""
    ny, nx = lx.shape
    lv = np.stack([lx.ravel(), ly.ravel(), lz.ravel()], 1)  # column c = ix + nx * iy
    ncol = nx * ny
    order = np.lexsort((np.arange(ncol), lv[:, 2], lv[:, 1], lv[:, 0]))
    ncell = (1 << lv[:, 0]) * (1 << lv[:, 1]) * (1 << lv[:, 2])
    off = np.zeros(ncol, np.int64)
    off[order] = np.concatenate([[0], np.cumsum(ncell[order])[:-1]])
    n_elem = int(ncell.sum())

    def eid(c, sx, sy, sz):
        nxc, nyc = 1 << lv[c, 0], 1 << lv[c, 1]
        return off[c] + sx + nxc * (sy + nyc * sz)

    elem_level = np.zeros((n_elem, 3), np.int64)
    elem_box = np.zeros((n_elem, 6))
    conf, bnd, ifs = [], [], []
    dxb = L / nx
    for c in range(ncol):
        ix, iy = c % nx, c // nx
        nxc, nyc, nzc = 1 << lv[c, 0], 1 << lv[c, 1], 1 << lv[c, 2]
        for sz in range(nzc):
            for sy in range(nyc):
                for sx in range(nxc):
                    e = eid(c, sx, sy, sz)
                    elem_level[e] = lv[c]
                    elem_box[e] = [(ix + sx / nxc) * dxb, (iy + sy / nyc) * dxb, sz / nzc,
                                   (ix + (sx + 1) / nxc) * dxb, (iy + (sy + 1) / nyc) * dxb, (sz + 1) / nzc]
                    # faces inside the column, and the column's bottom/top/basin sides
                    if sx + 1 < nxc: conf.append((e, 1, eid(c, sx + 1, sy, sz), 0))
                    if sy + 1 < nyc: conf.append((e, 3, eid(c, sx, sy + 1, sz), 2))
                    if sz + 1 < nzc: conf.append((e, 5, eid(c, sx, sy, sz + 1), 4))
                    if sz == 0: bnd.append((e, 4))
                    if sz == nzc - 1: bnd.append((e, 5))
                    if sx == 0 and ix == 0: bnd.append((e, 0))
                    if sx == nxc - 1 and ix == nx - 1: bnd.append((e, 1))
                    if sy == 0 and iy == 0: bnd.append((e, 2))
                    if sy == nyc - 1 and iy == ny - 1: bnd.append((e, 3))
        # faces with the next column in x (normal axis 0: tangents y, z) and in y (axis 1: x, z)
        for axis, nbc in ((0, c + 1 if ix + 1 < nx else -1), (1, c + nx if iy + 1 < ny else -1)):
            if nbc < 0:
                continue
            t1 = 1 if axis == 0 else 0
            la, lb = lv[c], lv[nbc]
            da = (la[t1] - lb[t1], la[2] - lb[2])
            fa, fb = 2 * axis + 1, 2 * axis  # face of this column / of the neighbour
            if da[0] >= 0 and da[1] >= 0:
                coarse, fine, cf, ff, d = nbc, c, fb, fa, da
            else:
                coarse, fine, cf, ff, d = c, nbc, fa, fb, (-da[0], -da[1])
            assert d[0] in (0, 1) and d[1] in (0, 1), "2:1 balance violated"
            lc, lf = lv[coarse], lv[fine]
            n1c, nzc_ = 1 << lc[t1], 1 << lc[2]
            # the layer of cells of each column that touches the shared face
            def cell(col, lvl, a1, a2, at_max):
                nxc, nyc = 1 << lvl[0], 1 << lvl[1]
                s_norm = ((nxc if axis == 0 else nyc) - 1) if at_max else 0
                if axis == 0:
                    return eid(col, s_norm, a1, a2)
                return eid(col, a1, s_norm, a2)
            coarse_is_low = (coarse == c)  # the lower column holds the +normal face
            for p2 in range(nzc_):
                for p1 in range(n1c):
                    ce = cell(coarse, lc, p1, p2, coarse_is_low)
                    fines = []
                    for b2 in range(1 + d[1]):
                        for b1 in range(1 + d[0]):
                            fines.append(cell(fine, lf, p1 * (1 + d[0]) + b1, p2 * (1 + d[1]) + b2,
                                              not coarse_is_low))
                    t = FINE_TYPE[d]
                    if t == 0:
                        conf.append((ce, cf, fines[0], ff))
                    else:
                        ifs.append((t, ce, cf, fines, [ff] * len(fines)))
    ifs.sort(key=lambda r: r[0])  # interfaces grouped by connection type
    conf = np.array(conf, np.int64).reshape(-1, 4)
    bnd = np.array(bnd, np.int64).reshape(-1, 2)
    return dict(n_elem=n_elem, level=elem_level, box=elem_box, conf=conf, bnd=bnd, ifaces=ifs,
                col_levels=lv)


def c3(nb: int = 256, order: int = 3, seed: int = SEED, hurst: float = 0.7):
    """C3: directional AMR (4 levels per horizontal direction, 2 vertically) refined towards a
    seeded fBm (Hurst 0.7) coastline on an nb x nb base grid, N=3; a scalar field advected
    with a constant velocity (the scalar conservation law of DG3DIntegration::compute_rhs)."""
    from .amr import build_mesh  # the native builder; amr_mesh above is its Python statement

    lx, ly, lz = c3_levels(nb, hurst, seed)
    mesh = build_mesh(lx, ly, lz)
    npn = order + 1
    rng = np.random.default_rng(seed + 3)
    box = mesh["box"]
    x = lgl_nodes(order)
    # a smooth seeded field sampled at every element's nodes
    kx, ky, kz = rng.uniform(1, 4, 3)
    X = box[:, None, 0] + 0.5 * (x[None, :] + 1) * (box[:, None, 3] - box[:, None, 0])
    Y = box[:, None, 1] + 0.5 * (x[None, :] + 1) * (box[:, None, 4] - box[:, None, 1])
    Z = box[:, None, 2] + 0.5 * (x[None, :] + 1) * (box[:, None, 5] - box[:, None, 2])
    U = (np.sin(2 * np.pi * kx * X)[:, None, None, :] * np.cos(2 * np.pi * ky * Y)[:, None, :, None]
         * (1.0 + 0.5 * Z)[:, :, None, None]).reshape(mesh["n_elem"], npn ** 3)
    a = np.array([1.0, 0.6, 0.2])
    return dict(order=order, mesh=mesh, U=np.ascontiguousarray(U), a=a,
                name=f"C3 AMR {nb}x{nb} base, {mesh['n_elem']} hexes N={order}")
