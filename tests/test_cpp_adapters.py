"""The C++ adapters of include/drifter_b200.hpp (the reference's class names and call shapes
over the C ABI): tests/cpp/adapter_check.cpp compiles against the header and the in-tree
library here; on a GPU it runs and its results equal the same computations through the Python
mirror (one library underneath, so to summation order)."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from drifter_b200 import configs
from drifter_b200.bezier import BezierSmoother
from drifter_b200.dg import DGConfig, ModeSplittingSolver, OceanModel, PrimitiveEquationsSolver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "drifter_b200")


def _compile(out_dir):
    exe = os.path.join(out_dir, "adapter_check")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp"), "-L", LIBDIR, "-ldrifter_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_adapters_compile_against_the_header_and_library(tmp_path):
    assert os.path.exists(_compile(str(tmp_path)))


def _close(a, b, rtol=1e-12):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) <= rtol * np.maximum(np.abs(b), 1e-300) + 1e-300)


@pytest.mark.gpu
def test_adapters_equal_the_python_mirror(tmp_path):
    exe = _compile(str(tmp_path))
    res = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)
    assert res["invalid_throws"] is True
    # reference-semantics DG, the same closed-form inputs
    nel, nd = 3, 64
    x = 0.1 * (np.arange(nd)[None, :] + 7 * np.arange(nel)[:, None])
    h = 50.0 + 10.0 * np.sin(x)
    f = np.full_like(h, 1e-4)
    eta = 0.01 * np.cos(x)
    H = h + eta
    st = dict(Hu=0.1 * H * np.sin(2 * x), Hv=0.05 * H * np.cos(3 * x), eta=eta,
              HT=(10.0 + np.sin(x)) * H, HS=35.0 * H, omega=1e-5 * np.sin(x))
    td = PrimitiveEquationsSolver(3, h, f).compute_rhs(st)
    sums = [td[k].sum() for k in ("dHu_dt", "dHv_dt", "deta_dt", "dHT_dt", "dHS_dt")]
    assert _close(res["compat_rhs"], sums, 1e-11)
    full = dict(st)
    full.update(H=H, u=st["Hu"] / H, v=st["Hv"] / H, T=st["HT"] / H, S=st["HS"] / H)
    full["rho"] = 1025.0 * (1.0 - 2e-4 * (full["T"] - 10.0) + 7.6e-4 * (full["S"] - 35.0))
    ModeSplittingSolver(3, h, f, subcycles=10).step(0.01, full)
    assert np.isfinite(full["eta"]).all()
    assert _close(res["compat_step"], [full["eta"].sum(), full["Hu"].sum()], 1e-11)
    # the coupled model
    cfg = DGConfig(nx=3, ny=2, nz=2, order=2, Lx=30e3, Ly=20e3, precision="fp64")
    n2, n3 = cfg.n2, cfg.n3
    h2 = 100.0 + 20.0 * np.sin(0.3 * np.arange(n2))
    n = np.arange(n3)
    Hn = h2[(n // 54) * 9 + n % 9]
    q = [np.zeros(n3), np.zeros(n3), (10.0 + 0.5 * np.sin(0.1 * n)) * Hn, 35.0 * Hn]
    m = OceanModel(cfg, h2, np.full(n2, 1e-4), np.full(n2, 0.1), np.zeros(n2))
    m.upload_state(q, np.zeros(n2))
    m.step(30.0, 5, 2)
    d = m.diagnostics()
    assert _close(res["coupled_diag"], [d["mass"], d["energy"], d["heat"], d["max_speed"], d["max_eta"]])
    m.close()
    # the smoother and the reference multigrid apply
    data = 500.0 + 100.0 * np.sin(0.05 * np.arange(8 * 8 * 16))
    s = BezierSmoother(8, 8, 2000.0, 2000.0, data, lam=1.0, ridge_epsilon=1e-4)
    s.mg_setup(2, 1, 1)
    r = np.cos(0.01 * np.arange(s.ndof))
    z, cycles, _ = s.mg_apply_reference(r)
    xs, info = s.solve("mg", tol=1e-10, maxit=500)
    assert res["mg"][0] == cycles and res["mg"][2] == info["iters"]
    assert _close([res["mg"][1], res["mg"][3]], [np.linalg.norm(z), np.linalg.norm(xs)], 1e-11)
    s.close()
