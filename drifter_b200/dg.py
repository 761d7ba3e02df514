"""Host-side mirror of DRIFTER's DG operator/solver interfaces over the C ABI.

Names and argument meaning follow the reference classes:
  * PrimitiveEquationsSolver.compute_rhs  (include/physics/primitive_equations.hpp:240)
  * ModeSplittingSolver.step              (include/physics/mode_splitting.hpp:241)
  * NumericalFluxFactory fluxes           (include/flux/numerical_flux.hpp:180-210)
  * OceanModel = SimulationDriver-like coupled model (include/solver/simulation_driver.hpp:92-127)
Errors raise DrfError (the reference throws std::invalid_argument / std::runtime_error).
All compute runs in libdrifter_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import check, dptr, dptr_array, lib

COMPAT_DEFAULTS = dict(g=9.81, rho0=1025.0, alpha=2e-4, beta=7.6e-4, nu_h=1.0, nu_v=1e-4,
                       kappa_v_T=1e-5, kappa_v_S=1e-5)


def _compat_params(p: dict | None) -> np.ndarray:
    d = dict(COMPAT_DEFAULTS)
    d.update(p or {})
    return np.array([d["g"], d["rho0"], d["alpha"], d["beta"], d["nu_h"], d["nu_v"],
                     d["kappa_v_T"], d["kappa_v_S"]], dtype=np.float64)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def numerical_flux(kind: str, UL, UR, normals, g: float = 9.81) -> np.ndarray:
    """F*(U_L, U_R, n) for batches of shallow-water states (h, hu, hv); kind in lf/hllc/roe."""
    UL, UR, nr = _c(UL).reshape(-1, 3), _c(UR).reshape(-1, 3), _c(normals).reshape(-1, 2)
    if not (len(UL) == len(UR) == len(nr)):
        raise ValueError("UL, UR and normals must have the same length")
    F = np.empty_like(UL)
    check(lib().drf_sw_flux_batch(_abi.FLUX[kind], len(UL), dptr(UL), dptr(UR), dptr(nr), g,
                                  dptr(F)))
    return F


class PrimitiveEquationsSolver:
    """Element-local primitive-equation tendencies with the reference's semantics.

    `compute_rhs(states)` takes a dict of [nel, (N+1)^3] arrays Hu, Hv, eta, HT, HS, omega and
    returns dHu_dt, dHv_dt, deta_dt, dHT_dt, dHS_dt (PrimitiveTendencies).
    """

    def __init__(self, order: int, bathymetry, coriolis, constants: dict | None = None):
        self.order = order
        self.h = _c(bathymetry)
        self.f = _c(coriolis)
        self.params = _compat_params(constants)

    def compute_rhs(self, states: dict) -> dict:
        ins = [_c(states[k]) for k in ("Hu", "Hv", "eta", "HT", "HS", "omega")]
        nel = ins[0].shape[0]
        outs = [np.empty_like(ins[0]) for _ in range(5)]
        check(lib().drf_compat_compute_rhs(self.order, nel, dptr_array(ins), dptr(self.h),
                                           dptr(self.f), dptr(self.params), dptr_array(outs)))
        return dict(zip(("dHu_dt", "dHv_dt", "deta_dt", "dHT_dt", "dHS_dt"), outs))

    def time_rhs(self, states: dict, nel: int, reps: int = 20) -> float:
        """Device milliseconds of one compute_rhs launch over nel elements: the given elements
        repeated to nel on the device (the bathymetry and Coriolis arrays with them)."""
        ins = [_c(states[k]) for k in ("Hu", "Hv", "eta", "HT", "HS", "omega")]
        ms = np.zeros(1)
        check(lib().drf_compat_time_rhs(self.order, ins[0].shape[0], dptr_array(ins),
                                        dptr(self.h), dptr(self.f), dptr(self.params), nel,
                                        reps, dptr(ms)))
        return float(ms[0])


STATE12 = ("Hu", "Hv", "eta", "HT", "HS", "H", "u", "v", "T", "S", "omega", "rho")


class ModeSplittingSolver:
    """Per-element barotropic/baroclinic split step with the reference's semantics."""

    def __init__(self, order: int, bathymetry, coriolis, subcycles: int = 30,
                 constants: dict | None = None):
        self.order = order
        self.h = _c(bathymetry)
        self.f = _c(coriolis)
        self.subcycles = subcycles
        self.params = _compat_params(constants)

    def step(self, dt_3d: float, full_state: dict) -> None:
        arrs = [np.ascontiguousarray(full_state[k], dtype=np.float64) for k in STATE12]
        nel = arrs[0].shape[0]
        check(lib().drf_compat_modesplit_step(self.order, nel, dt_3d, self.subcycles,
                                              dptr_array(arrs), dptr(self.h), dptr(self.f),
                                              dptr(self.params)))
        for k, a in zip(STATE12, arrs):
            full_state[k] = a


@dataclass
class DGConfig:
    nx: int
    ny: int
    nz: int
    order: int
    Lx: float
    Ly: float
    g: float = 9.81
    rho0: float = 1025.0
    nu_h: float = 1.0
    nu_v: float = 1e-4
    kappa_v_T: float = 1e-5
    kappa_v_S: float = 1e-5
    cd: float = 2.5e-3
    flux2d: str = "lf"
    precision: str = "mixed"
    bc: tuple = ("wall", "wall", "wall", "wall")
    tide_amp: float = 0.0
    tide_period: float = 44714.0
    # linear equation of state (EquationOfState include/physics/equation_of_state.hpp:35-40);
    # alpha = beta = 0 switches the baroclinic pressure gradient off
    alpha: float = 2e-4
    beta: float = 7.6e-4
    T0: float = 10.0
    S0: float = 35.0
    # reference stratification T_ref(z) = Tref_s + Tref_dz z subtracted before the pressure
    # integral (its own pressure has no horizontal gradient); (T0, 0) subtracts nothing
    Tref_s: float = 10.0
    Tref_dz: float = 0.0

    @property
    def np_(self) -> int:
        return self.order + 1

    @property
    def n3(self) -> int:
        return self.nx * self.ny * self.nz * self.np_ ** 3

    @property
    def n2(self) -> int:
        return self.nx * self.ny * self.np_ ** 2


def _mesh_params(cfg: DGConfig):
    mesh = _abi.MeshDesc(cfg.nx, cfg.ny, cfg.nz, cfg.order, cfg.Lx, cfg.Ly)
    prm = _abi.DGParams()
    prm.g, prm.rho0, prm.nu_h, prm.nu_v = cfg.g, cfg.rho0, cfg.nu_h, cfg.nu_v
    prm.kappa_v_T, prm.kappa_v_S, prm.cd = cfg.kappa_v_T, cfg.kappa_v_S, cfg.cd
    prm.alpha, prm.beta, prm.T0, prm.S0 = cfg.alpha, cfg.beta, cfg.T0, cfg.S0
    prm.Tref_s, prm.Tref_dz = cfg.Tref_s, cfg.Tref_dz
    prm.flux2d = _abi.FLUX[cfg.flux2d]
    prm.precision = _abi.PREC[cfg.precision]
    for s in range(4):
        prm.bc[s] = _abi.BC[cfg.bc[s]]
    prm.tide_amp, prm.tide_period = cfg.tide_amp, cfg.tide_period
    return mesh, prm


class OceanModel:
    """Coupled sigma-coordinate DG model resident on the GPU (one CUDA stream)."""

    def __init__(self, cfg: DGConfig, h, f, taux, tauy):
        self.cfg = cfg
        mesh, prm = _mesh_params(cfg)
        self._keep = [_c(h), _c(f), _c(taux), _c(tauy)]
        hd = C.c_void_p()
        check(lib().drf_dg_create(C.byref(mesh), C.byref(prm), *[dptr(a) for a in self._keep],
                                  C.byref(hd)))
        self.handle = hd
        self._owner = None

    @classmethod
    def _member(cls, cfg: DGConfig, handle, owner) -> "OceanModel":
        """A member of an Ensemble: shares the ensemble's memory and stream, stepped by it."""
        m = cls.__new__(cls)
        m.cfg, m.handle, m._owner = cfg, handle, owner
        return m

    def close(self):
        if getattr(self, "handle", None):
            if self._owner is None:
                lib().drf_dg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(lib().drf_dg_set_stream(self.handle, C.c_void_p(stream_ptr or 0)))

    def sync(self):
        check(lib().drf_dg_sync(self.handle))

    def upload_state(self, q4, eta, t: float = 0.0):
        qs = [_c(a) for a in q4]
        check(lib().drf_dg_upload_state(self.handle, dptr_array(qs), dptr(_c(eta)), float(t)))

    def download_state(self) -> dict:
        n3, n2 = self.cfg.n3, self.cfg.n2
        q = [np.empty(n3) for _ in range(4)]
        eta, HU, HV, eavg = (np.empty(n2) for _ in range(4))
        t = C.c_double()
        check(lib().drf_dg_download_state(self.handle, dptr_array(q), dptr(eta), dptr(HU),
                                          dptr(HV), dptr(eavg), C.byref(t)))
        return dict(Hu=q[0], Hv=q[1], HT=q[2], HS=q[3], eta=eta, HU=HU, HV=HV, eta_avg=eavg,
                    t=t.value)

    def output_stage(self, out: dict) -> None:
        """Snapshot the state and copy it to the host arrays of `out` (keys Hu, Hv, HT, HS, eta,
        HU, HV; float64, contiguous, ideally pinned) while later steps run; the arrays hold the
        snapshot after output_wait()."""
        q = [out.get(k) for k in ("Hu", "Hv", "HT", "HS")]
        q4 = dptr_array(q) if any(a is not None for a in q) else None
        self._staged = out  # kept alive until the copy is done
        check(lib().drf_dg_output_stage(self.handle, q4, *[dptr(out[k]) if out.get(k) is not None else None
                                                           for k in ("eta", "HU", "HV")]))

    def output_wait(self) -> float:
        """Waits for the staged copy; returns the snapshot's model time."""
        t = C.c_double()
        check(lib().drf_dg_output_wait(self.handle, C.byref(t)))
        self._staged = None
        return t.value

    def compute_rhs(self) -> dict:
        n3, n2 = self.cfg.n3, self.cfg.n2
        r = [np.empty(n3) for _ in range(4)]
        om, de = np.empty(n3), np.empty(n2)
        check(lib().drf_dg_compute_rhs(self.handle, dptr_array(r), dptr(om), dptr(de)))
        return dict(dHu=r[0], dHv=r[1], dHT=r[2], dHS=r[3], omega=om, deta=de)

    def compute_rhs2d(self, Fx, Fy, time: float) -> tuple:
        n2 = self.cfg.n2
        ke, ku, kv = np.empty(n2), np.empty(n2), np.empty(n2)
        check(lib().drf_dg_compute_rhs2d(self.handle, dptr(_c(Fx)), dptr(_c(Fy)), time,
                                         dptr(ke), dptr(ku), dptr(kv)))
        return ke, ku, kv

    def step(self, dt: float, nsub: int, nsteps: int = 1):
        """nsteps baroclinic steps, each one CUDA graph (ModeSplittingSolver::step)."""
        check(lib().drf_dg_step_modesplit(self.handle, dt, nsub, nsteps))

    def rk_step(self, scheme: str, dt: float, nsteps: int = 1):
        check(lib().drf_dg_rk_step(self.handle, _abi.RK[scheme], dt, nsteps))

    def set_forcing(self, taux, tauy):
        self._forcing = (_c(taux), _c(tauy))
        check(lib().drf_dg_set_forcing(self.handle, dptr(self._forcing[0]), dptr(self._forcing[1])))

    def download_surface(self, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(self.cfg.n2) if out is None else out
        check(lib().drf_dg_download_surface(self.handle, dptr(out)))
        return out

    def diagnostics(self) -> dict:
        out = np.empty(10)
        check(lib().drf_dg_diagnostics(self.handle, dptr(out)))
        keys = ("mass", "mass_unweighted", "energy", "heat", "salt", "max_speed", "max_eta",
                "min_eta", "max_T", "min_T")
        return dict(zip(keys, out.tolist()))

    def tuning(self) -> dict:
        """The autotuned launch shapes with each candidate's time (ms): the barotropic tile
        (columns per CTA) and the stage kernel's L2 prefetch distance (half waves of resident
        CTAs)."""
        cpb, ms = C.c_int(), np.zeros(4)
        check(lib().drf_dg_tuning(self.handle, C.byref(cpb), dptr(ms)))
        hw, cols, sms = C.c_int(), C.c_int(), np.zeros(3)
        check(lib().drf_dg_stage_tuning(self.handle, C.byref(hw), C.byref(cols), dptr(sms)))
        return dict(baro_cols_per_cta=cpb.value,
                    candidates_ms={str(c): round(float(t), 5) for c, t in zip((2, 4, 8, 16), ms)},
                    stage_prefetch_half_waves=hw.value, stage_prefetch_columns=cols.value,
                    stage_candidates_ms={str(w): round(float(t), 5) for w, t in enumerate(sms)})

    def time_copy(self, nrep: int = 20) -> dict:
        """The stage kernel's access structure as a pure copy: time per launch and bytes."""
        ms, b = C.c_double(), C.c_double()
        check(lib().drf_dg_time_copy(self.handle, nrep, C.byref(ms), C.byref(b)))
        return dict(ms=ms.value, bytes=b.value, gbs=b.value / (ms.value / 1e3) / 1e9)

    def time_stage(self, nrep: int = 20) -> dict:
        ms, ab, nd = C.c_double(), C.c_double(), C.c_double()
        check(lib().drf_dg_time_stage(self.handle, nrep, C.byref(ms), C.byref(ab), C.byref(nd)))
        return dict(ms=ms.value, alg_bytes=ab.value, ndof=nd.value)


class Ensemble:
    """Independent coupled DG runs stepped together (one launch per LSRK stage and layer count
    over all members' water columns, one launch per barotropic substep, one CUDA graph per
    baroclinic step).

    `members[i]` is an OceanModel view of member i (upload/download/diagnostics); the members
    are stepped only through `step`. Each member's result equals OceanModel.step on it alone.
    """

    def __init__(self, cases: list):
        """cases: dicts with cfg (DGConfig), h, f, taux, tauy (the configs generators' form)."""
        n = len(cases)
        meshes = (_abi.MeshDesc * n)()
        prms = (_abi.DGParams * n)()
        for i, c in enumerate(cases):
            meshes[i], prms[i] = _mesh_params(c["cfg"])
        self._keep = [[_c(c[k]) for c in cases] for k in ("h", "f", "taux", "tauy")]
        arrs = [dptr_array(a) for a in self._keep]
        hd = C.c_void_p()
        check(lib().drf_ens_create(n, meshes, prms, *arrs, C.byref(hd)))
        self.handle = hd
        self.members = []
        for i, c in enumerate(cases):
            mh = C.c_void_p()
            check(lib().drf_ens_member(self.handle, i, C.byref(mh)))
            self.members.append(OceanModel._member(c["cfg"], mh, self))

    def close(self):
        if getattr(self, "handle", None):
            for m in self.members:
                m.handle = None
            lib().drf_ens_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(lib().drf_ens_set_stream(self.handle, C.c_void_p(stream_ptr or 0)))

    def sync(self):
        check(lib().drf_ens_sync(self.handle))

    def step(self, dts, nsub: int, nsteps: int = 1):
        """nsteps baroclinic steps; member i advances by dts[i] per step."""
        d = _c(dts)
        if len(d) != len(self.members):
            raise ValueError("one step size per member")
        check(lib().drf_ens_step(self.handle, dptr(d), nsub, nsteps))

    def info(self) -> dict:
        n3, it, gr = C.c_int64(), C.c_int(), C.c_int()
        check(lib().drf_ens_info(self.handle, C.byref(n3), C.byref(it), C.byref(gr)))
        return dict(n3=n3.value, items=it.value, grid=gr.value)
