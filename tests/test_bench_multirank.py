"""The multi-rank logic of bench.py (one process per GPU; N > 1 runs replicas): the barrier, the
max-over-ranks device time and the whole-job rate, on two ranks of the gloo backend on CPU
(the same calls run on NCCL on GPUs); and the reference arm, which only rank 0 runs."""
import contextlib
import io
import json
import os
import socket
import subprocess
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = """
import json, sys
sys.path.insert(0, {root!r})
import bench
import torch.distributed as dist
rank, world, local = bench.dist_init(2)
bench.barrier(world)
ms_local = {{0: 10.0, 1: 25.0}}[rank]
ms_max, rate = bench.job_rate(1000.0, ms_local, world)
bench.barrier(world)
print(json.dumps({{"rank": rank, "world": world, "local": local, "ms_max": ms_max, "rate": rate}}))
dist.destroy_process_group()
"""


def _free_port():
    with contextlib.closing(socket.socket(socket.AF_INET, socket.SOCK_STREAM)) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_time_by_the_slowest_and_count_every_ranks_units():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), DRIFTER_B200_DIST_BACKEND="gloo")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            outs.append(p.communicate(timeout=180))
        finally:
            if p.poll() is None:
                p.kill()
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    res = sorted((json.loads(o.strip().splitlines()[-1]) for o, _ in outs), key=lambda d: d["rank"])
    assert [d["rank"] for d in res] == [0, 1] and all(d["world"] == 2 for d in res)
    for d in res:
        assert d["ms_max"] == 25.0  # the slower rank's time, on every rank
        assert d["rate"] == 2 * 1000.0 / 0.025  # both ranks' units over that time


def test_single_rank_rate_and_reference_arm_off_rank_zero():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.job_rate(500.0, 20.0, 1) == (20.0, 500.0 / 0.02)
    args = types.SimpleNamespace(gpus=2, steps=3, warmup=3)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, rank=1, world=2)  # ranks other than 0 exit without work
    assert buf.getvalue() == ""
