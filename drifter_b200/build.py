"""Builds libdrifter_b200.so in-tree with nvcc for sm_100a (no JIT, no torch extension)."""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdrifter_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    # a source is rebuilt when it, or any header it may include, is newer than its object
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))] + [
        os.path.join(HERE, "..", "include", "drifter_b200.h")]
    newest_header = max(os.path.getmtime(d) for d in headers)
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(newest_header, os.path.getmtime(src)):
            continue
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC, *FLAGS, "-x", "cu", *ARCH, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _wait(procs.pop(0))
    for p in procs:
        _wait(p)
    if (not os.path.exists(OUT)) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart", "-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return OUT


def _wait(item):
    src, p = item
    out, _ = p.communicate()
    text = out.decode(errors="replace")
    if p.returncode != 0:
        sys.stderr.write(text)
        raise RuntimeError(f"nvcc failed on {src}")
    # ptxas -warn-spills names each function that spills ("N bytes spill stores", N > 0)
    if re.search(r"\b[1-9][0-9]* bytes spill", text):
        sys.stderr.write(text)


if __name__ == "__main__":
    print(build(verbose=True))
