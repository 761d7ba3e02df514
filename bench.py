"""Benchmark of the DRIFTER operator path on B200.

Step = one baroclinic step of the coupled DG model on C2 (128x128x16 hexes, N=4, 200x200 km,
seeded 32-Gaussian bathymetry, M2 tide on the west boundary, linear T stratification):
5 LSRK45 3D stages (FP32 bulk) + 20 FP64 barotropic predictor-corrector subcycles, one CUDA
graph. Metric: 3D DOF-stage updates per second (DOF = node x 3D prognostic variable).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): independent replicas, one per GPU (the path is single-GPU by design; no
collective on the data path). Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-stage/s (mixed-precision DG step, C2)"
UNIT = "DOF-stage/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="C2 physics on a 32x32x16 mesh (quick)")
    ap.add_argument("--mid", action="store_true", help="C2 physics on a 64x64x16 mesh (profiling)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 GPU comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-cg", action="store_true", help="skip the C4 Bezier CG comparison")
    ap.add_argument("--no-ens", action="store_true", help="skip the C5 ensemble measurement")
    ap.add_argument("--no-amr", action="store_true", help="skip the C3 AMR measurement")
    ap.add_argument("--no-baroclinic", action="store_true",
                    help="skip the C2 measurement with the baroclinic pressure gradient on")
    ap.add_argument("--only", choices=["amr", "ens", "cg", "baro"], default=None,
                    help="run one workload section alone and print its JSON (profiling aid)")
    return ap.parse_args()


def dist_init(n):
    """One process per GPU (RANK / WORLD_SIZE / LOCAL_RANK from the launcher). The process group
    is NCCL; DRIFTER_B200_DIST_BACKEND=gloo selects gloo (the CPU tests of this logic). Its
    timeout is short, so ranks that wait for a rank that died end with an error."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = os.environ.get("DRIFTER_B200_DIST_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ms_local, world):
    """Whole-job throughput: the units all ranks processed over the slowest rank's device time
    (max over ranks). Returns (max ms, units per second)."""
    ms_max = max_over_ranks(ms_local, world)
    return ms_max, world * units_per_rank / (ms_max / 1e3)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        if not sm:
            return None
        maxsm = float(self.rows[-1][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9
                          for i, v in enumerate(r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": maxsm, "reasons": reasons,
                "samples": len(sm)}


def gpu_smi_id(local):
    """nvidia-smi --id for the CUDA device `local` (PCI bus id), or the ordinal."""
    try:
        import torch
        p = torch.cuda.get_device_properties(local)
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
    except Exception:
        return str(local)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>.md), or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":")[1])
            except ValueError:
                return None
    return None


def make_case(small, mid=False):
    from drifter_b200 import configs
    if mid:
        return configs.c2(nx=64, ny=64, nz=16, Lx=100e3)
    if small:
        return configs.c2(nx=32, ny=32, nz=16, Lx=50e3)
    return configs.c2()


def compat_sample(nel):
    """Seeded C2-shaped N=4 element states (500-550 m deep, random transports) for the
    reference-semantics element RHS."""
    nd = 125
    rng = np.random.default_rng(0)
    h = np.full((nel, nd), 500.0) + rng.uniform(0, 50, (nel, nd))
    f = np.full((nel, nd), 1e-4)
    H = h.copy()
    st = dict(Hu=H * 0.1 * rng.standard_normal((nel, nd)), Hv=H * 0.1 * rng.standard_normal((nel, nd)),
              eta=np.zeros((nel, nd)), HT=H * 10.0, HS=H * 35.0, omega=np.zeros((nel, nd)))
    return st, h, f


def cpu_baseline(seconds=12.0, threads=1):
    """Reference CPU path (SimulationDriver::step, non-split SSPRK3 over the dense-Kronecker
    element RHS, src/solver/simulation_driver.cpp:108) on C2-shaped N=4 elements."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    order, nd = 4, 125
    nel = 64 * max(1, threads)
    st, h, f = compat_sample(nel)
    done, t0 = 0, time.perf_counter()
    while True:
        st = O.compat_ssprk3(order, 1.0, st, h, f, nthreads=threads)
        done += 1
        el = time.perf_counter() - t0
        if el > seconds:
            break
    rate = nel * nd * 4 * 3 * done / el
    return rate, dict(sample=f"{done} SSPRK3 steps x {nel} N=4 elements ({nel*nd*4} DOFs), "
                      f"{el:.1f} s", threads=threads)


def same_algorithm(cpu_value, nel=128 * 128 * 16, reps=20):
    """The reference's element-local RHS (PrimitiveEquationsSolver::compute_rhs with its
    semantics, FP64) timed on the GPU over C2's element count, from the CPU sample's elements
    repeated: one algorithm on both sides, so the ratio compares hardware and implementation
    only. DOF-stages count the 4 transported variables per node and RHS evaluation, as the
    CPU baseline does."""
    from drifter_b200.dg import PrimitiveEquationsSolver
    st, h, f = compat_sample(64)
    pe = PrimitiveEquationsSolver(4, h, f)
    ms = pe.time_rhs(st, nel, reps)
    gpu = nel * 125 * 4 / (ms / 1e3)
    out = {"workload": f"reference element RHS (FP64), {nel} N=4 elements, device time per launch",
           "gpu_ms_per_rhs": ms, "gpu_value": gpu, "unit": UNIT}
    if cpu_value:
        out["cpu_value_1core"] = cpu_value
        out["ratio_gpu_over_cpu_1core"] = gpu / cpu_value
    return out


def run_cg(stream, reps=3):
    """C4 Bezier smoother: PCG time-to-1e-10 per preconditioner (device time of whole solves,
    CUDA events inside the library), the learned network trained on a 64x64 grid first."""
    from drifter_b200 import configs
    from drifter_b200.bezier import BezierSmoother
    from drifter_b200.cnn import train_preconditioner
    c = configs.c4()
    t0 = time.perf_counter()
    net, info = train_preconditioner(n=64, dx=c["L"] / c["n"], lam=c["lam"], eps=c["eps"],
                                     steps=10000, rhs_count=16, seed=1)
    train_s = time.perf_counter() - t0
    s = BezierSmoother(c["n"], c["n"], c["L"], c["L"], c["d"], lam=c["lam"], ridge_epsilon=c["eps"])
    s.set_stream(stream.cuda_stream)
    s.mg_setup(2)
    net.attach(s)
    out = {"workload": c["name"] + " cubic Bezier, lambda=1, eps=1e-4, FP64 PCG to 1e-10",
           "dofs": s.ndof, "train_s": round(train_s, 2), "train_loss": info["loss"],
           "cnn_conv_autotuned": s.cnn_tuning()}
    sols = {}
    import torch
    torch.cuda.synchronize()
    torch.cuda.profiler.start()  # the solves only (ncu --profile-from-start off), not the training
    for pc in ("mg", "cnn", "jacobi", "none"):
        s.solve(pc, tol=1e-10, maxit=5000)  # warm-up (graph capture)
        best = None
        for _ in range(reps):
            x, inf = s.solve(pc, tol=1e-10, maxit=5000)
            if best is None or inf["ms"] < best["ms"]:
                best = inf
        sols[pc] = x
        out[pc] = {"iters": best["iters"], "ms": round(best["ms"], 3), "relres": best["relres"]}
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    # the reference's multigrid apply (V-cycles to 1e-6 per apply) under flexible CG: host-driven
    # iterations, so one timed solve
    x, inf = s.solve("mg_reference", tol=1e-10, maxit=200)
    out["mg_reference"] = {"iters": inf["iters"], "ms": round(inf["ms"], 3), "relres": inf["relres"]}
    # roofline of the Jacobi and unpreconditioned solves: algorithmic bytes per control point and
    # iteration of their fused kernels (Q apply: x in, y out, 16 B; x/r update: p, q, x, r in and
    # x, r out, 48 B, plus d in and z out for Jacobi, 16 B; p update: z (or r) and p in, p out,
    # 24 B). The vectors (19 MB each) are largely L2-resident, so the fraction of HBM can pass 1.
    peak, _ = measured_peaks()
    out["roofline"] = {}
    for pc, bpd in (("jacobi", 104), ("none", 88)):
        gbs = bpd * s.ndof * out[pc]["iters"] / (out[pc]["ms"] / 1e3) / 1e9
        out["roofline"][pc] = {"bytes_per_dof_iter": bpd, "achieved_gbs": round(gbs, 1),
                               "frac_of_hbm_peak": round(gbs / peak, 3)}
    out["cnn_vs_mg_speedup"] = round(out["mg"]["ms"] / out["cnn"]["ms"], 3)
    out["cnn_vs_mg_solution_rel_diff"] = float(np.abs(sols["cnn"] - sols["mg"]).max() /
                                               np.abs(sols["mg"]).max())
    s.close()
    net.close()
    return out


def run_baroclinic(stream, steps=10, warmup=3):
    """C2 with the equation of state on (the baroclinic pressure gradient against the linear
    reference stratification): the cost of the pressure integral and gradient in the stage
    kernel, and the mixed-precision surface error against the FP64 GPU form over a short
    window (the coupled baroclinic step grows on C2's steep seamount flanks within about a
    hundred steps, so it is not run for the config's 500)."""
    import torch
    from drifter_b200 import configs
    from drifter_b200.dg import DGConfig, OceanModel
    case = configs.c2(baroclinic=True)
    cfg = case["cfg"]
    dt, nsub = case["dt"], case["nsub"]
    m = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    m.set_stream(stream.cuda_stream)
    m.upload_state(case["q"], case["eta"])
    m.step(dt, nsub, warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(dt, nsub, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    sm = m.download_state()
    st = m.time_stage(nrep=5 * steps)
    m.close()
    cfg64 = DGConfig(**{**cfg.__dict__, "precision": "fp64"})
    m64 = OceanModel(cfg64, case["h"], case["f"], case["taux"], case["tauy"])
    m64.set_stream(stream.cuda_stream)
    m64.upload_state(case["q"], case["eta"])
    m64.step(dt, nsub, warmup + steps)
    s64 = m64.download_state()
    vmax = m64.diagnostics()["max_speed"]
    m64.close()
    peak, _ = measured_peaks()
    ndof = 4 * cfg.n3
    gbs = st["alg_bytes"] / (st["ms"] / 1e3) / 1e9
    return {"workload": case["name"] + " with the baroclinic pressure gradient (linear EOS, "
                                       "reference stratification 20 C - 0.008 C/m)",
            "value": ndof * 5 / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "stage_kernel_ms": st["ms"], "stage_alg_bytes": st["alg_bytes"],
            "roofline_frac": gbs / peak, "achieved_gbs": gbs,
            "eta_rel_err_mixed_vs_fp64": float(np.linalg.norm(sm["eta"] - s64["eta"]) /
                                               np.linalg.norm(s64["eta"])),
            "steps_compared": warmup + steps, "max_speed_m_s": vmax}


def run_ensemble(stream, steps=5, warmup=3):
    """C5: 64 independent N=3 runs of uneven size stepped together (one stage launch per LSRK
    stage and layer count over all members' columns, one graph per baroclinic step), against the
    same members stepped one model after another on the same stream. Device time with CUDA
    events."""
    import torch
    from drifter_b200 import configs
    from drifter_b200.dg import Ensemble, OceanModel
    cases = configs.c5()
    nsub = cases[0]["nsub"]
    dts = [c["dt"] for c in cases]
    ndof = sum(4 * c["cfg"].n3 for c in cases)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ens = Ensemble(cases)
    ens.set_stream(stream.cuda_stream)
    for m, c in zip(ens.members, cases):
        m.upload_state(c["q"], c["eta"])
    ens.step(dts, nsub, warmup)
    torch.cuda.synchronize()
    e0.record(stream)
    ens.step(dts, nsub, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    info = ens.info()
    diag = ens.members[0].diagnostics()
    # algorithmic bytes of the five stage launches of one step, all members (each member's stage
    # as the single model's: per 3D DOF s (4 + 4 / (N + 1)) bytes, per 2D node 9 FP64 words)
    stage_bytes = 0.0
    for c in cases:
        cf = c["cfg"]
        s_b = 8.0 if cf.precision == "fp64" else 4.0
        stage_bytes += 5 * (4 * cf.n3 * s_b * (4 + 4.0 / cf.np_) + cf.n2 * 8.0 * 9)
    ens.close()
    del ens
    # the same members one after another (each model's own step graph)
    models = []
    for c in cases:
        m = OceanModel(c["cfg"], c["h"], c["f"], c["taux"], c["tauy"])
        m.set_stream(stream.cuda_stream)
        m.upload_state(c["q"], c["eta"])
        models.append(m)
    for m, c in zip(models, cases):
        m.step(c["dt"], nsub, warmup)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        for m, c in zip(models, cases):
            m.step(c["dt"], nsub, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1) / steps
    for m in models:
        m.close()
    return {"workload": f"C5 {len(cases)} members N=3, meshes 16..64 x 16..64 x 4..8, mixed precision, "
                        f"{nsub} barotropic subcycles",
            "dofs": ndof, "columns": info["items"], "stage_grid": info["grid"],
            "value": ndof * 5 / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "sequential_ms_per_step": ms_seq, "speedup_vs_sequential": ms_seq / ms,
            "member0_max_eta": diag["max_eta"],
            # the stages' algorithmic bytes over the whole step's time (barotropic included):
            # a lower bound of the stage launch's rate
            "roofline": {"stage_bytes_per_step": stage_bytes,
                         "step_gbs": stage_bytes / (ms / 1e3) / 1e9,
                         "frac_of_hbm_peak": stage_bytes / (ms / 1e3) / 1e9 / measured_peaks()[0]}}


def run_amr(stream, steps=5, warmup=3):
    """C3: DG3DIntegration::compute_rhs on the directionally refined mesh of the seeded fBm
    coastline (about 2.6e5 hexes, N=3), complete mode (conforming, boundary and mortar faces),
    LF flux: the right-hand side alone and the LSRK45 step (one graph per step), device time."""
    import torch
    from drifter_b200 import configs
    from drifter_b200.amr import DG3DIntegration
    c = configs.c3()
    m = c["mesh"]
    gpu = DG3DIntegration(c["order"], m)
    gpu.set_stream(stream.cuda_stream)
    gpu.upload(c["U"])
    rhs = gpu.time_rhs(c["a"], nrep=20, flux="lf", mode="complete")
    dt = 1e-4
    gpu.step(c["a"], dt, warmup, flux="lf", mode="complete")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    gpu.step(c["a"], dt, steps, flux="lf", mode="complete")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ndof = m["n_elem"] * (c["order"] + 1) ** 3
    adapt = run_amr_adapt(c, gpu)
    gpu.close()
    types = np.bincount([f[0] for f in m["ifaces"]], minlength=6)
    return {"workload": c["name"] + ", complete mode, LF flux, LSRK45",
            "hexes": int(m["n_elem"]), "dofs": int(ndof),
            "faces": {"conforming": int(len(m["conf"])), "boundary": int(len(m["bnd"])),
                      "mortar_2x1": int(types[1]), "mortar_1x2": int(types[2]), "mortar_2x2": int(types[5])},
            "value": ndof * 5 / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "rhs_ms": rhs["ms"], "rhs_gbs": rhs["alg_bytes"] / (rhs["ms"] / 1e3) / 1e9,
            "adapt": adapt}


def run_amr_adapt(c, gpu):
    """One AdaptiveMeshRefinement::adapt of the C3 state after its steps: the estimator and the
    transfer on the GPU, the column levels, face tables and mortar operators on the host
    (wall-clock milliseconds of each part, host calls that end with a synchronize)."""
    from drifter_b200.amr import AdaptiveMeshRefinement, DG3DIntegration, RefinementParams, build_mesh
    m = c["mesh"]
    nb = int(round(len(m["col_levels"]) ** 0.5))
    levels = tuple(np.ascontiguousarray(m["col_levels"][:, d].reshape(nb, nb)) for d in range(3))
    amr = AdaptiveMeshRefinement(c["order"], RefinementParams(max_level=4))
    amr.estimate(gpu, m)  # warm-up
    t = [time.perf_counter()]
    _, mask, flags = amr.estimate(gpu, m)
    t.append(time.perf_counter())
    new_levels, changed = amr.refine_levels(levels, mask, flags)
    t.append(time.perf_counter())
    m2 = build_mesh(*new_levels)
    t.append(time.perf_counter())
    g2 = DG3DIntegration(c["order"], m2)
    t.append(time.perf_counter())
    amr.transfer(gpu, g2, levels, new_levels)
    t.append(time.perf_counter())
    nd = (c["order"] + 1) ** 3
    out = {"columns_changed": int(changed), "hexes_before": int(m["n_elem"]), "hexes_after": int(m2["n_elem"]),
           "estimate_ms": round(1e3 * (t[1] - t[0]), 3), "refine_levels_ms": round(1e3 * (t[2] - t[1]), 3),
           "build_mesh_ms": round(1e3 * (t[3] - t[2]), 3), "create_ms": round(1e3 * (t[4] - t[3]), 3),
           "transfer_ms": round(1e3 * (t[5] - t[4]), 3),
           "transfer_bytes": int((m["n_elem"] + m2["n_elem"]) * nd * 8)}
    g2.close()
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(seconds=2.0, threads=threads)
    for _ in range(args.steps):
        v, meta = cpu_baseline(seconds=max(2.0, 60.0 / max(args.steps, 1)), threads=threads)
        vals.append(v)
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "reference non-split SSPRK3 DG step (dense Kronecker element RHS) "
                               "on C2-shaped N=4 elements", "threads": threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": meta["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_only(args, local):
    import torch
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    fn = {"amr": run_amr, "ens": run_ensemble, "cg": run_cg, "baro": run_baroclinic}[args.only]
    out = fn(stream, steps=args.steps, warmup=args.warmup) if args.only != "cg" else fn(stream)
    print(json.dumps({"only": args.only, **out}), flush=True)


def run_ours(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    from drifter_b200 import launch_count
    from drifter_b200.dg import OceanModel

    case = make_case(args.small, args.mid)
    cfg = case["cfg"]
    model = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
    stream = torch.cuda.Stream()  # a real (non-legacy) stream: graphs are captured on it
    model.set_stream(stream.cuda_stream)
    model.upload_state(case["q"], case["eta"])
    dt, nsub = case["dt"], case["nsub"]
    ndof = 4 * cfg.n3
    for _ in range(args.warmup):
        model.step(dt, nsub, 1)
    torch.cuda.synchronize()

    clocks = ClockSampler(gpu_smi_id(local))
    clocks.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    l0 = launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    model.step(dt, nsub, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    launches = launch_count() - l0
    ms = e0.elapsed_time(e1)
    ck = clocks.stop()
    ms_max, value = job_rate(ndof * 5 * args.steps, ms, world)
    ms_step = ms_max / args.steps

    tuning = model.tuning()  # autotuned barotropic tile (chosen at the first step)

    # dominant kernel: the fused 3D stage, timed alone with CUDA events on the model's stream
    st = model.time_stage(nrep=5 * args.steps)
    peak, peak_kind = measured_peaks()
    achieved = st["alg_bytes"] / (st["ms"] / 1e3) / 1e9
    traffic = profile_traffic("dg3d_stage_c2_mixed.md")
    copy = model.time_copy(nrep=5 * args.steps)  # the stage's access structure as a pure copy

    # end to end through the C ABI: per step upload the surface stress from pinned host memory,
    # run the step, read back the surface elevation and the diagnostics
    taux = torch.from_numpy(case["taux"]).pin_memory().numpy()
    tauy = torch.from_numpy(case["tauy"]).pin_memory().numpy()
    eta_out = torch.empty(cfg.n2, dtype=torch.float64).pin_memory().numpy()
    torch.cuda.synchronize()
    barrier(world)
    calls = {"set_forcing": 0.0, "step": 0.0, "download_surface": 0.0, "diagnostics": 0.0}
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ta = time.perf_counter()
        model.set_forcing(taux, tauy)
        tb = time.perf_counter()
        model.step(dt, nsub, 1)
        tc = time.perf_counter()
        model.download_surface(eta_out)
        td = time.perf_counter()
        model.diagnostics()
        te = time.perf_counter()
        calls["set_forcing"] += tb - ta
        calls["step"] += tc - tb
        calls["download_surface"] += td - tc
        calls["diagnostics"] += te - td
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = {"value": world * ndof * 5 * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": 2 * 8 * cfg.n2, "d2h_bytes_per_step": 8 * cfg.n2 + 80,
           "ms_per_step": 1e3 * e2e_s / args.steps,
           "host_ms_per_call": {k: round(1e3 * v / args.steps, 3) for k, v in calls.items()}}

    # FP64 GPU form of the same step, and the mixed-precision surface error against it over the
    # config's full length (both forms stepped from the initial state)
    fp64 = None
    if not args.no_fp64:
        del model
        torch.cuda.synchronize()
        nref = max(case["steps"], args.warmup + 2 * args.steps)
        from drifter_b200.dg import DGConfig
        cfg64 = DGConfig(**{**cfg.__dict__, "precision": "fp64"})
        m64 = OceanModel(cfg64, case["h"], case["f"], case["taux"], case["tauy"])
        m64.set_stream(stream.cuda_stream)
        m64.upload_state(case["q"], case["eta"])
        m64.step(dt, nsub, args.warmup)
        torch.cuda.synchronize()
        e0.record(stream)
        m64.step(dt, nsub, 2 * args.steps)
        e1.record(stream)
        m64.step(dt, nsub, nref - args.warmup - 2 * args.steps)
        torch.cuda.synchronize()
        ms64 = max_over_ranks(e0.elapsed_time(e1), world) / (2 * args.steps)
        s64 = m64.download_state()
        m64.close()
        mm = OceanModel(cfg, case["h"], case["f"], case["taux"], case["tauy"])
        mm.set_stream(stream.cuda_stream)
        mm.upload_state(case["q"], case["eta"])
        mm.step(dt, nsub, nref)
        sm = mm.download_state()
        mm.close()
        err = float(np.linalg.norm(sm["eta"] - s64["eta"]) / np.linalg.norm(s64["eta"]))
        fp64 = {"value": world * ndof * 5 / (ms64 / 1e3), "ms_per_step": ms64,
                "eta_rel_err_mixed_vs_fp64": err, "steps_compared": nref,
                "max_abs_eta_m": float(np.abs(s64["eta"]).max())}

    # Bezier smoother CG on C4 (512x512, 2.36 M control points): time to the FP64 1e-10 residual
    # with the multigrid and the learned preconditioner (plus Jacobi and none for reference)
    cg = None
    if not args.no_cg:
        cg = run_cg(stream)

    baro = None
    if not args.no_baroclinic:
        baro = run_baroclinic(stream)

    ens = None
    if not args.no_ens:
        ens = run_ensemble(stream)
    amr = None
    if not args.no_amr:
        amr = run_amr(stream)

    cpu = None
    if rank == 0 and not args.no_cpu:
        v, meta = cpu_baseline(seconds=12.0, threads=1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": meta["sample"]}
    same = None
    if rank == 0 and not args.no_cpu:
        same = same_algorithm(cpu["value"] if cpu else None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (3D bulk) + f64 (barotropic)",
            "data": "synthetic",
            "config": {"workload": case["name"] + " coupled DG baroclinic step (5 LSRK45 stages + "
                                                  f"{nsub} FP64 barotropic subcycles)",
                       "dofs": ndof, "dt_s": dt, "l2": "inputs > L2 (state 2.1 GB)",
                       "parallelism": f"replicas x{world}", "autotuned": tuning},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "dg3d_stage_kernel<float,5>", "kernel_ms": st["ms"],
                         "alg_bytes_per_launch": st["alg_bytes"],
                         "copy_ceiling_gbs": copy["gbs"], "copy_ceiling_frac": copy["gbs"] / peak,
                         "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs"},
            "cpu_baseline": cpu,
            "same_algorithm": same,
            "e2e": e2e,
            "fp64_gpu": fp64,
            "baroclinic": baro,
            "cg": cg,
            "ensemble": ens,
            "amr": amr,
            "gpu_launches": int(launches),
            "clocks": ck,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_init(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.only:
            run_only(args, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
