"""Build libsteps_b200.so in-tree with nvcc for sm_100a.

    python -m steps_b200.build [--force]

Device code of the window kernels (sg_solver.cu, sg_noalloc.cu) is compiled with
-fmad=false and host code with -ffp-contract=off, so that the samplers only contract
where the sources call fma() explicitly (bit-exact agreement with the CPU oracle).  The
EField solver (sg_efield.cu) has no bit-level contract with a CPU restatement (its
results are checked against an FP64 direct solve within a tolerance), so its device code
is compiled with fused multiply-adds.  Each source is compiled to its own object (in
parallel) and the objects are linked into the library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsteps_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-fopenmp",
]
# Sources whose device arithmetic must match the CPU oracle bit for bit.
NO_FMAD = {"sg_solver.cu", "sg_noalloc.cu"}
OBJ_DIR = os.path.join(HERE, "_build")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    jobs, objs = [], []
    for src in sources():
        name = os.path.basename(src)
        obj = os.path.join(OBJ_DIR, name + ".o")
        flags = NVCC_FLAGS + (["-fmad=false"] if name in NO_FMAD else [])
        cmd = [NVCC] + flags + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for cmd, pr in jobs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"nvcc failed ({pr.returncode}): {' '.join(cmd)}\n{out}\n{err}")
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + ["-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
