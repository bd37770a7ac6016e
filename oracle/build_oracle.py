"""TEST INFRASTRUCTURE ONLY — build recipe of the CPU oracle and of the pieces of the
reference that compile from their own sources here.

    python oracle/build_oracle.py [--force]

Outputs:
  oracle/_build/liboracle.so     the C restatement (opsplit_oracle.c), gcc, OpenMP
  oracle/_ref/libsteps_ref.so    the reference TetOpSplitP and Tetexact compiled from their
                                 own sources (build_ref_tetopsplit.py)
  oracle/_ref/ref_philox_kat     Philox known-answer generator compiled against the
                                 reference's vendored Random123 header, read where it lies
                                 in the reference tree ($STEPS_REFERENCE, default
                                 /root/reference; only when that tree is present)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
REFERENCE = os.environ.get("STEPS_REFERENCE", "/root/reference")
LIB = os.path.join(BUILD, "liboracle.so")

CFLAGS = ["-O2", "-ffp-contract=off", "-mfma", "-fopenmp", "-fPIC", "-std=c11", "-Wall"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)} failed:\n{r.stdout}\n{r.stderr}")


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "opsplit_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        _run(["gcc"] + CFLAGS + ["-shared", "-o", LIB, src, "-lm"])
    return LIB


def build_ref(force=False):
    """Reference-side pieces; skipped when the reference tree is absent: the
    Philox known-answer generator and the reference solvers (build_ref_tetopsplit)."""
    third = os.path.join(REFERENCE, "src", "third_party")
    if not os.path.isdir(third):
        return None
    try:
        from . import build_ref_tetopsplit
    except ImportError:  # run as a script
        import build_ref_tetopsplit

    build_ref_tetopsplit.build(force=force)
    try:
        build_ref_tetopsplit.build_cython(force=force)
    except RuntimeError as e:  # the binding module is optional test infrastructure
        print(f"reference Python binding not built: {e}", file=sys.stderr)
    os.makedirs(REF_OUT, exist_ok=True)
    exe = os.path.join(REF_OUT, "ref_philox_kat")
    src = os.path.join(HERE, "ref_philox_kat.c")
    if force or not os.path.exists(exe) or os.path.getmtime(exe) < os.path.getmtime(src):
        _run(["gcc", "-O2", "-I", third, "-o", exe, src])
    return exe


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_ref(force))
