"""ORACLE binding — test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
CPU-baseline leg). ctypes access to oracle/_build/liboracle.so, the FP64 CPU restatement of
the reference algorithms. Never imported by the drifter_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_dp = C.POINTER(C.c_double)
_lib = None


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_last_error.restype = C.c_char_p
        _lib.orc_phys_create.restype = C.c_void_p
        for name in ("orc_phys_destroy", "orc_phys_set_state", "orc_phys_get_state",
                     "orc_phys_rhs", "orc_phys_rhs2d", "orc_phys_split_steps",
                     "orc_phys_rk_steps", "orc_phys_diagnostics"):
            getattr(_lib, name).argtypes = None
        _lib.orc_phys_destroy.argtypes = [C.c_void_p]
    return _lib


def _p(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _pa(arrs):
    return (_dp * len(arrs))(*[_p(a) for a in arrs])


def _chk(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def basis(order: int, kind: str = "lgl"):
    np_ = order + 1
    x, w, D, S = np.empty(np_), np.empty(np_), np.empty(np_ * np_), np.empty(np_ * np_)
    _chk(lib().orc_basis(order, 0 if kind == "lgl" else 1, _p(x), _p(w), _p(D), _p(S)))
    return x, w, D.reshape(np_, np_), S.reshape(np_, np_)


def dense_3d(order: int):
    nd = (order + 1) ** 3
    a, b, c = (np.empty(nd * nd) for _ in range(3))
    _chk(lib().orc_dense_3d(order, _p(a), _p(b), _p(c)))
    return a.reshape(nd, nd), b.reshape(nd, nd), c.reshape(nd, nd)


FLUX = {"lf": 0, "hllc": 1, "roe": 2}


def sw_flux(kind, UL, UR, nx, ny, g=9.81):
    F = np.empty(3)
    _chk(lib().orc_sw_flux(FLUX[kind], _p(_c(UL)), _p(_c(UR)), C.c_double(nx), C.c_double(ny),
                           C.c_double(g), _p(F)))
    return F


def compat_params(p=None):
    d = dict(g=9.81, rho0=1025.0, alpha=2e-4, beta=7.6e-4, nu_h=1.0, nu_v=1e-4, kappa_v_T=1e-5,
             kappa_v_S=1e-5)
    d.update(p or {})
    return np.array([d[k] for k in ("g", "rho0", "alpha", "beta", "nu_h", "nu_v", "kappa_v_T",
                                    "kappa_v_S")])


def compat_rhs(order, states, h, f, params=None):
    ins = [_c(states[k]) for k in ("Hu", "Hv", "eta", "HT", "HS", "omega")]
    outs = [np.empty_like(ins[0]) for _ in range(5)]
    _chk(lib().orc_compat_rhs(order, ins[0].shape[0], _pa(ins), _p(_c(h)), _p(_c(f)),
                              _p(compat_params(params)), _pa(outs)))
    return dict(zip(("dHu_dt", "dHv_dt", "deta_dt", "dHT_dt", "dHS_dt"), outs))


STATE12 = ("Hu", "Hv", "eta", "HT", "HS", "H", "u", "v", "T", "S", "omega", "rho")


def compat_modesplit(order, dt, nsub, state, h, f, params=None):
    arrs = [_c(state[k]).copy() for k in STATE12]
    _chk(lib().orc_compat_modesplit(order, arrs[0].shape[0], C.c_double(dt), nsub, _pa(arrs),
                                    _p(_c(h)), _p(_c(f)), _p(compat_params(params))))
    return dict(zip(STATE12, arrs))


def compat_ssprk3(order, dt, state, h, f, params=None, nthreads=1):
    """SimulationDriver::step without mode splitting on nel elements (in place on copies)."""
    arrs = [_c(state[k]).copy() for k in ("Hu", "Hv", "eta", "HT", "HS", "omega")]
    _chk(lib().orc_compat_ssprk3(order, arrs[0].shape[0], C.c_double(dt), _pa(arrs), _p(_c(h)),
                                 _p(_c(f)), _p(compat_params(params)), nthreads))
    return dict(zip(("Hu", "Hv", "eta", "HT", "HS", "omega"), arrs))


BCS = {"wall": 0, "tide": 1}
RK = {"euler": 0, "midpoint": 1, "ssp3": 2, "rk4": 3, "lsrk45": 4, "dopri": 5}


class PhysOracle:
    """FP64 CPU model of the coupled DG scheme (same spec as the GPU OceanModel)."""

    def __init__(self, cfg, h, f, taux, tauy):
        self.cfg = cfg
        iv = np.array([cfg.nx, cfg.ny, cfg.nz, cfg.order, FLUX[cfg.flux2d]] +
                      [BCS[b] for b in cfg.bc], dtype=np.int32)
        dv = np.array([cfg.Lx, cfg.Ly, cfg.g, cfg.rho0, cfg.nu_h, cfg.nu_v, cfg.kappa_v_T,
                       cfg.kappa_v_S, cfg.cd, cfg.tide_amp, cfg.tide_period, cfg.alpha,
                       cfg.beta, cfg.T0, cfg.S0, cfg.Tref_s, cfg.Tref_dz])
        self._keep = [_c(h), _c(f), _c(taux), _c(tauy)]
        L = lib()
        L.orc_phys_create.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        self.h = L.orc_phys_create(iv.ctypes.data, _p(dv), *[_p(a) for a in self._keep])
        if not self.h:
            raise RuntimeError("oracle: " + L.orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_phys_destroy(C.c_void_p(self.h))
            self.h = None

    def set_state(self, q4, eta, t=0.0):
        qs = [_c(a) for a in q4]
        _chk(lib().orc_phys_set_state(C.c_void_p(self.h), _pa(qs), _p(_c(eta)), C.c_double(t)))

    def get_state(self):
        n3, n2 = self.cfg.n3, self.cfg.n2
        q = [np.empty(n3) for _ in range(4)]
        eta, HU, HV, eavg = (np.empty(n2) for _ in range(4))
        t = C.c_double()
        _chk(lib().orc_phys_get_state(C.c_void_p(self.h), _pa(q), _p(eta), _p(HU), _p(HV),
                                      _p(eavg), C.byref(t)))
        return dict(Hu=q[0], Hv=q[1], HT=q[2], HS=q[3], eta=eta, HU=HU, HV=HV, eta_avg=eavg,
                    t=t.value)

    def rhs(self, etab=None):
        """3D right-hand side at the current state; etab (optional) is the surface elevation
        of the baroclinic pressure gradient (default: the model's eta)."""
        n3, n2 = self.cfg.n3, self.cfg.n2
        r = [np.empty(n3) for _ in range(4)]
        om, de = np.empty(n3), np.empty(n2)
        eb = None if etab is None else _c(etab)
        _chk(lib().orc_phys_rhs(C.c_void_p(self.h), _pa(r), _p(om), _p(de),
                                None if eb is None else _p(eb)))
        return dict(dHu=r[0], dHv=r[1], dHT=r[2], dHS=r[3], omega=om, deta=de)

    def rhs2d(self, Fx, Fy, time):
        n2 = self.cfg.n2
        a, b, c = np.empty(n2), np.empty(n2), np.empty(n2)
        _chk(lib().orc_phys_rhs2d(C.c_void_p(self.h), _p(_c(Fx)), _p(_c(Fy)), C.c_double(time),
                                  _p(a), _p(b), _p(c)))
        return a, b, c

    def split_steps(self, dt, nsub, nsteps=1):
        _chk(lib().orc_phys_split_steps(C.c_void_p(self.h), C.c_double(dt), nsub, nsteps))

    def rk_steps(self, scheme, dt, nsteps=1):
        _chk(lib().orc_phys_rk_steps(C.c_void_p(self.h), RK[scheme], C.c_double(dt), nsteps))

    def diagnostics(self):
        out = np.empty(10)
        _chk(lib().orc_phys_diagnostics(C.c_void_p(self.h), _p(out)))
        keys = ("mass", "mass_unweighted", "energy", "heat", "salt", "max_speed", "max_eta",
                "min_eta", "max_T", "min_T")
        return dict(zip(keys, out.tolist()))


def rk_ode(scheme, lam, U0, T, nsteps):
    out = C.c_double()
    _chk(lib().orc_rk_ode(RK[scheme], C.c_double(lam), C.c_double(U0), C.c_double(T), nsteps,
                          C.byref(out)))
    return out.value


# ----------------------------------------------------------------------------- Bezier smoother
def gauss01_4():
    a = np.sqrt(3 / 7 - 2 / 7 * np.sqrt(6 / 5))
    b = np.sqrt(3 / 7 + 2 / 7 * np.sqrt(6 / 5))
    return np.array([0.5 * (1 - b), 0.5 * (1 - a), 0.5 * (1 + a), 0.5 * (1 + b)])


def gauss_points(nx, ny, x0, y0, Lx, Ly):
    """Physical coordinates of the 4x4 data Gauss points, layout [ey][ex][qj][qi]."""
    p = gauss01_4()
    dx, dy = Lx / nx, Ly / ny
    ex = np.arange(nx)[None, :, None, None]
    ey = np.arange(ny)[:, None, None, None]
    X = x0 + (ex + p[None, None, None, :]) * dx
    Y = y0 + (ey + p[None, None, :, None]) * dy
    X = np.broadcast_to(X, (ny, nx, 4, 4))
    Y = np.broadcast_to(Y, (ny, nx, 4, 4))
    return X.reshape(-1).copy(), Y.reshape(-1).copy()


class BezierOracle:
    """Uniform-grid cubic Bezier smoother system (Q, b, constraints, multigrid, PCG)."""

    def __init__(self, nx, ny, Lx, Ly, dgauss, lam=1.0, eps=1e-4, x0=0.0, y0=0.0):
        L = lib()
        L.orc_bz_build.restype = C.c_void_p
        L.orc_bz_build.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, _dp]
        L.orc_bz_destroy.argtypes = [C.c_void_p]
        for fn in ("orc_bz_nnz", "orc_bz_rows"):
            getattr(L, fn).restype = C.c_long
            getattr(L, fn).argtypes = [C.c_void_p, C.c_int]
        self.d = _c(dgauss)
        self.h = L.orc_bz_build(nx, ny, x0, y0, Lx, Ly, lam, eps, _p(self.d))
        if not self.h:
            raise RuntimeError("oracle: " + L.orc_last_error().decode())
        n, a, d = C.c_long(), C.c_double(), C.c_double()
        _chk(L.orc_bz_info(C.c_void_p(self.h), C.byref(n), C.byref(a), C.byref(d)))
        self.ndof, self.alpha, self.dTWd = n.value, a.value, d.value
        self.nx, self.ny = nx, ny

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bz_destroy(C.c_void_p(self.h))
            self.h = None

    def vec(self, which="b"):
        out = np.empty(self.ndof)
        _chk(lib().orc_bz_vec(C.c_void_p(self.h), 0 if which == "b" else 1, _p(out)))
        return out

    def csr(self, which):
        import scipy.sparse as sp
        w = {"H": 0, "BtWB": 1, "Q": 2, "A": 3}[which]
        L = lib()
        nnz, rows = L.orc_bz_nnz(C.c_void_p(self.h), w), L.orc_bz_rows(C.c_void_p(self.h), w)
        rp = np.empty(rows + 1, dtype=np.int64)
        ci = np.empty(nnz, dtype=np.int64)
        v = np.empty(nnz)
        _chk(L.orc_bz_csr(C.c_void_p(self.h), w, rp.ctypes.data_as(C.c_void_p),
                          ci.ctypes.data_as(C.c_void_p), _p(v)))
        return sp.csr_matrix((v, ci, rp), shape=(rows, self.ndof))

    def constraints(self, edge_ngauss=4):
        _chk(lib().orc_bz_constraints(C.c_void_p(self.h), edge_ngauss))
        return self.csr("A")

    def objective(self, x):
        parts, obj = np.empty(2), C.c_double()
        _chk(lib().orc_bz_objective(C.c_void_p(self.h), _p(_c(x)), _p(parts), C.byref(obj)))
        return obj.value, parts[0], parts[1]

    def mg_setup(self, coarsest_n=2):
        nl = C.c_int()
        _chk(lib().orc_bz_mg_setup(C.c_void_p(self.h), coarsest_n, C.byref(nl)))
        self.nlevels = nl.value
        return nl.value

    def level(self, l):
        n = C.c_int()
        K = np.empty(256)
        _chk(lib().orc_bz_level_info(C.c_void_p(self.h), l, C.byref(n), _p(K), None, None))
        nd = 3 * n.value + 1
        rho = np.empty(nd)
        binv = np.zeros(9 * 256)
        _chk(lib().orc_bz_level_info(C.c_void_p(self.h), l, C.byref(n), _p(K), _p(rho), _p(binv)))
        return dict(n=n.value, K=K.reshape(16, 16), rho=rho, binv=binv.reshape(9, 16, 16))

    def level_apply(self, l, x):
        y = np.empty_like(_c(x))
        _chk(lib().orc_bz_level_apply(C.c_void_p(self.h), l, _p(_c(x)), _p(y)))
        return y

    def vcycle(self, r):
        z = np.empty(self.ndof)
        _chk(lib().orc_bz_mg_vcycle(C.c_void_p(self.h), _p(_c(r)), _p(z)))
        return z

    def mg_apply_ref(self, b, tol=1e-6, max_cycles=100):
        """BezierMultigridPreconditioner::apply with the reference's V-cycle, repeated to tol."""
        x = np.empty(self.ndof)
        cyc = C.c_int()
        _chk(lib().orc_bz_mg_apply_ref(C.c_void_p(self.h), _p(_c(b)), _p(x), C.c_double(tol),
                                       max_cycles, C.byref(cyc)))
        return x, cyc.value

    def pcg(self, b=None, precond="mg", tol=1e-10, maxit=2000, x0=None):
        b = self.vec("b") if b is None else _c(b)
        x = np.zeros(self.ndof) if x0 is None else _c(x0).copy()
        it, rr = C.c_int(), C.c_double()
        _chk(lib().orc_bz_pcg(C.c_void_p(self.h), {"none": 0, "jacobi": 1, "mg": 2}[precond],
                              _p(b), _p(x), C.c_double(tol), maxit, C.byref(it), C.byref(rr)))
        return x, it.value, rr.value


# ----------------------------------------------------------------------------- learned preconditioner
def cnn_nparams():
    L = lib()
    L.orc_cnn_nparams.restype = C.c_long
    return int(L.orc_cnn_nparams())


def cnn_forward_backward(params, X, T=None, round_bf16=True):
    """CPU reference of the preconditioner network for one image X (H x W x 16)."""
    L = lib()
    L.orc_cnn_forward_backward.restype = C.c_double
    L.orc_cnn_forward_backward.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
    X = _c(X)
    H, W, _ = X.shape
    out = np.empty_like(X)
    grad = np.empty(cnn_nparams()) if T is not None else None
    loss = L.orc_cnn_forward_backward(_p(_c(params)), _p(X), H, W,
                                      _p(_c(T)) if T is not None else None, _p(out),
                                      _p(grad) if grad is not None else None, int(round_bf16))
    return out, grad, loss


# ----------------------------------------------------------------------------- mortars
MORTAR_NUM_FINE = {0: 1, 1: 2, 2: 2, 3: 3, 4: 3, 5: 4}  # FaceConnectionType 0..5


def mortar_ops(order, ctype):
    """Mortar operators of one connection type (MortarSpace, src/dg/mortar.cpp:80)."""
    L = lib()
    L.orc_mortar_ops.argtypes = [C.c_int, C.c_int] + [_dp] * 6
    nm = (order + 1) ** 2
    nfine = MORTAR_NUM_FINE[ctype]
    M, Minv, Pc, Lc = (np.empty((nm, nm)) for _ in range(4))
    Pf, Lf = np.empty((nfine, nm, nm)), np.empty((nfine, nm, nm))
    r = L.orc_mortar_ops(order, ctype, _p(M), _p(Minv), _p(Pc), _p(Lc), _p(Pf), _p(Lf))
    if r < 0:
        raise ValueError("oracle: bad mortar arguments")
    return dict(M=M, Minv=Minv, Pc=Pc, Lc=Lc, Pf=Pf, Lf=Lf)


def mortar_apply(order, ifaces, flux_kind, a, U, rhs=None):
    """rhs + the non-conforming face fluxes of the interfaces (list of (type, coarse_elem,
    coarse_face, [fine_elems], [fine_faces])) for the scalar field U (n_elem x (order+1)^3)."""
    L = lib()
    L.orc_mortar_apply.argtypes = [C.c_int, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_int, _dp, C.c_long, _dp, _dp]
    arr = mortar_arrays(ifaces)
    U = _c(U)
    out = np.zeros_like(U) if rhs is None else _c(rhs).copy()
    ptr = lambda x: x.ctypes.data_as(C.c_void_p)
    r = L.orc_mortar_apply(order, len(ifaces), ptr(arr["type"]), ptr(arr["ce"]), ptr(arr["cf"]),
                           ptr(arr["fe"]), ptr(arr["ff"]), flux_kind, _p(_c(a)), U.shape[0],
                           _p(U), _p(out))
    if r < 0:
        raise ValueError("oracle: bad mortar arguments")
    return out


def mortar_arrays(ifaces):
    """Flat arrays (type, coarse elem/face, 4 fine elems/faces per interface, -1 padded)."""
    n = len(ifaces)
    out = dict(type=np.zeros(n, np.int32), ce=np.zeros(n, np.int64), cf=np.zeros(n, np.int32),
               fe=-np.ones((n, 4), np.int64), ff=-np.ones((n, 4), np.int32))
    for i, (t, ce, cf, fe, ff) in enumerate(ifaces):
        out["type"][i], out["ce"][i], out["cf"][i] = t, ce, cf
        out["fe"][i, :len(fe)] = fe
        out["ff"][i, :len(ff)] = ff
    return out


# ----------------------------------------------------------------------------- AMR scalar DG
LSRK_A = (0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257)
LSRK_B = (0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488, 0.1530572479681)


def amr_rhs(order, mesh, mode, flux_kind, a, U):
    """DG3DIntegration::compute_rhs (src/dg/operators_3d.cpp:228) on an AMR mesh (the dict of
    configs.amr_mesh): mode 0 the reference's semantics, 1 with conforming and boundary faces."""
    L = lib()
    vp = C.c_void_p
    L.orc_amr_rhs.argtypes = [C.c_int, C.c_long, C.c_int, C.c_int, _dp, C.c_long, vp, C.c_long, vp,
                              C.c_long, vp, vp, vp, vp, vp, _dp, _dp]
    arr = mortar_arrays(mesh["ifaces"])
    U = _c(U)
    out = np.zeros_like(U)
    conf = np.ascontiguousarray(mesh["conf"], np.int64)
    bnd = np.ascontiguousarray(mesh["bnd"], np.int64)
    ptr = lambda x: x.ctypes.data_as(C.c_void_p)
    r = L.orc_amr_rhs(order, U.shape[0], mode, flux_kind, _p(_c(a)), len(conf), ptr(conf), len(bnd),
                      ptr(bnd), len(mesh["ifaces"]), ptr(arr["type"]), ptr(arr["ce"]), ptr(arr["cf"]),
                      ptr(arr["fe"]), ptr(arr["ff"]), _p(U), _p(out))
    if r < 0:
        raise ValueError("oracle: bad AMR arguments")
    return out


def amr_lsrk(order, mesh, mode, flux_kind, a, U, dt, nsteps):
    """nsteps of the five-stage low-storage RK45 (LSRK45::step, src/solver/time_stepper.cpp:126)
    on du/dt = -R(u), R = compute_rhs (the reference's right-hand side is the weak divergence
    of a u: its volume term carries -grad(phi) and its face terms +F)."""
    u = _c(U).copy()
    res = np.zeros_like(u)
    for _ in range(nsteps):
        for s in range(5):
            r = amr_rhs(order, mesh, mode, flux_kind, a, u)
            res = LSRK_A[s] * res + dt * (-r)
            u = u + LSRK_B[s] * res
    return u


# ----------------------------------------------------------------------------- AMR refinement
def amr_estimate(order, U, hchar, refine_threshold=0.1, coarsen_threshold=0.01, smoothness_factor=0.5):
    """GradientErrorEstimator::estimate with compute_directional_mask (src/amr/refinement.cpp:44-160):
    per element the normalised value, the RefineMask bits and the flags (1 refine, 2 coarsen)."""
    L = lib()
    vp = C.c_void_p
    L.orc_amr_estimate.argtypes = [C.c_int, C.c_long, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp,
                                   vp, vp]
    U = _c(U)
    ne = U.shape[0]
    val = np.zeros(ne)
    mask = np.zeros(ne, np.int32)
    flags = np.zeros(ne, np.int32)
    ptr = lambda x: x.ctypes.data_as(C.c_void_p)
    if L.orc_amr_estimate(order, ne, _p(U), _p(_c(hchar)), refine_threshold, coarsen_threshold,
                          smoothness_factor, _p(val), ptr(mask), ptr(flags)) < 0:
        raise ValueError("oracle: bad estimate arguments")
    return val, mask, flags


def amr_project_children(order, U_parent, mask):
    """SolutionProjection::project_to_children (src/amr/refinement.cpp:217)."""
    L = lib()
    L.orc_amr_project_children.argtypes = [C.c_int, _dp, C.c_int, _dp]
    nch = (2 if mask & 1 else 1) * (2 if mask & 2 else 1) * (2 if mask & 4 else 1)
    nd = (order + 1) ** 3
    out = np.zeros((nch, nd))
    if L.orc_amr_project_children(order, _p(_c(U_parent)), mask, _p(out)) < 0:
        raise ValueError("oracle: bad projection arguments")
    return out


def amr_project_parent(order, U_children, mask):
    """SolutionProjection::project_from_children (src/amr/refinement.cpp:278)."""
    L = lib()
    L.orc_amr_project_parent.argtypes = [C.c_int, _dp, C.c_int, _dp]
    out = np.zeros((order + 1) ** 3)
    if L.orc_amr_project_parent(order, _p(_c(U_children)), mask, _p(out)) < 0:
        raise ValueError("oracle: bad projection arguments")
    return out


def amr_transfer(order, old_levels, new_levels, U_old):
    """The column-wise remap of a solution between per-column levels ((ncol, 3) arrays over an
    nx x ny grid given as (ny, nx, 3)), each new node taking the old cell's value at its position."""
    L = lib()
    vp = C.c_void_p
    L.orc_amr_transfer.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, _dp, _dp]
    ol = np.ascontiguousarray(old_levels, np.int32)
    nl = np.ascontiguousarray(new_levels, np.int32)
    ny, nx = ol.shape[:2]
    ne = int(sum(1 << int(v) for v in nl.reshape(-1, 3).sum(1)))
    out = np.zeros((ne, (order + 1) ** 3))
    ptr = lambda x: x.ctypes.data_as(C.c_void_p)
    if L.orc_amr_transfer(order, nx, ny, ptr(ol), ptr(nl), _p(_c(U_old)), _p(out)) < 0:
        raise ValueError("oracle: bad transfer arguments")
    return out


def bz_mesh_element_errors(bounds, coeffs, zdata, ngauss):
    """compute_element_l2_error / estimate_element_error on a list of quadtree elements
    (bounds n x 4, coefficients n x 16, data n x ngauss^2): (l2, normalized)."""
    L = lib()
    L.orc_bz_mesh_element_errors.argtypes = [C.c_long, _dp, _dp, _dp, C.c_int, _dp, _dp]
    b = _c(bounds).reshape(-1, 4)
    n = len(b)
    l2, nrm = np.empty(n), np.empty(n)
    if L.orc_bz_mesh_element_errors(n, _p(b), _p(_c(coeffs)), _p(_c(zdata)), ngauss, _p(l2), _p(nrm)) < 0:
        raise ValueError("oracle: bad element-error arguments")
    return l2, nrm


def bz_mesh_data_fitting(bounds, zdata, ngauss, relax=None):
    """The element part of assemble_data_fitting_global on a list of quadtree elements:
    (BtWB n x 16 x 16, BtWd n x 16, dTWd n)."""
    L = lib()
    L.orc_bz_mesh_data_fitting.argtypes = [C.c_long, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp]
    b = _c(bounds).reshape(-1, 4)
    n = len(b)
    K, r, dd = np.empty((n, 16, 16)), np.empty((n, 16)), np.empty(n)
    rel = _p(_c(relax)) if relax is not None else None
    if L.orc_bz_mesh_data_fitting(n, _p(b), _p(_c(zdata)), rel, ngauss, _p(K), _p(r), _p(dd)) < 0:
        raise ValueError("oracle: bad data-fitting arguments")
    return K, r, dd


def bz_element_errors(nx, ny, Lx, Ly, ngauss, x, zdata, x0=0.0, y0=0.0):
    """Per-element L2 misfit and normalized error of the adaptive smoother's estimate
    (AdaptiveCGCubicBezierSmoother::compute_element_l2_error)."""
    L = lib()
    L.orc_bz_element_errors.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_int, _dp, _dp, _dp, _dp]
    l2, nrm = np.empty(nx * ny), np.empty(nx * ny)
    r = L.orc_bz_element_errors(nx, ny, x0, y0, Lx, Ly, ngauss, _p(_c(x)), _p(_c(zdata)), _p(l2), _p(nrm))
    if r < 0:
        raise ValueError("oracle: bad element-error arguments")
    return l2, nrm
