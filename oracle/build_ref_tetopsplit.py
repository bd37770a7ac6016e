"""TEST INFRASTRUCTURE ONLY — build recipe of the reference solvers for the checker.

    python oracle/build_ref_tetopsplit.py [--force] [-j N]

Compiles the reference's own sources where they lie in the reference tree
($STEPS_REFERENCE, default /root/reference) — src/steps/{util, util/tracker, math, geom,
model, rng, solver, solver/efield (minus the PETSc and LAPACK back-ends), mpi,
mpi/tetopsplit, tetexact} — against the project-written stand-ins in oracle/ref_shim/
(single-rank MPI, easylogging++, the few Boost pieces used, METIS declarations), plus the
C driver oracle/ref_tetopsplit_harness.cpp, into oracle/_ref/libsteps_ref.so.  The
reference's CMake build is not used and no reference file is copied into this
repository.  Outputs go to oracle/_ref/ only (git-ignored, shipped with the tree).

It also compiles the drop-in steps_b200/steps_api/tetopsplit_b200.cpp (the
steps::solver::API subclass on the GPU solver) against the same reference headers and
links it, with the harness built for it, into oracle/_ref/libsteps_ref_b200.so, which
loads steps_b200/libsteps_b200.so: the library a STEPS build with the drop-in would be.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("STEPS_REFERENCE", "/root/reference")
SRC = os.path.join(REFERENCE, "src")
SHIM = os.path.join(HERE, "ref_shim")
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libsteps_ref.so")
HARNESS = os.path.join(HERE, "ref_tetopsplit_harness.cpp")
REPO = os.path.dirname(HERE)
DROPIN = os.path.join(REPO, "steps_b200", "steps_api", "tetopsplit_b200.cpp")
LIB_B200 = os.path.join(OUT, "libsteps_ref_b200.so")

DIRS = ["util", "util/tracker", "math", "geom", "model", "rng", "solver", "solver/efield", "mpi",
        "mpi/tetopsplit", "tetexact"]
EXCLUDE = ("petsc", "lapack")
FLAGS = ["-std=c++17", "-O2", "-fPIC", "-w", "-DENABLE_ASSERTLOG=1",
         "-I" + SHIM, "-I" + os.path.join(SRC, "steps"), "-I" + SRC, "-I" + os.path.join(SRC, "third_party"),
         "-I" + os.path.join(SRC, "third_party", "gsl-lite", "include"),
         "-I" + os.path.join(SRC, "third_party", "fau.de", "include")]


def sources():
    out = []
    for d in DIRS:
        for f in sorted(glob.glob(os.path.join(SRC, "steps", d, "*.cpp"))):
            if not any(x in os.path.basename(f) for x in EXCLUDE):
                out.append(f)
    return out


def shim_mtime():
    return max(os.path.getmtime(p) for p in glob.glob(os.path.join(SHIM, "**", "*"), recursive=True)
               if os.path.isfile(p))


def _compile(src, force, t_shim):
    rel = os.path.relpath(src, os.path.join(SRC, "steps")).replace(os.sep, "_")
    obj = os.path.join(OBJ, rel[:-4] + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), t_shim):
        return obj, None
    r = subprocess.run(["g++"] + FLAGS + ["-c", src, "-o", obj], capture_output=True, text=True)
    return obj, (None if r.returncode == 0 else f"{src}:\n{r.stderr[-2000:]}")


def available():
    return os.path.isdir(os.path.join(SRC, "steps", "mpi", "tetopsplit"))


def build(force=False, jobs=None):
    """Build oracle/_ref/libsteps_ref.so; returns its path, or None without the reference tree."""
    if not available():
        return None
    os.makedirs(OBJ, exist_ok=True)
    t_shim = max(shim_mtime(), os.path.getmtime(HARNESS))
    srcs = sources() + [HARNESS]
    jobs = jobs or os.cpu_count() or 4
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        res = list(ex.map(lambda s: _compile(s, force, t_shim), srcs))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("reference build failed:\n" + "\n".join(errs[:3]))
    objs = [o for o, _ in res]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        r = subprocess.run(["g++", "-shared", "-o", LIB] + objs, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference link failed:\n{r.stderr[-3000:]}")
    build_dropin(objs[:-1], force)
    return LIB


def build_dropin(ref_objs, force=False):
    """oracle/_ref/libsteps_ref_b200.so: the reference objects, the drop-in and the harness
    with its TetOpSplitB200 kind, linked to steps_b200/libsteps_b200.so."""
    inc = ["-I" + os.path.join(REPO, "steps_b200"), "-I" + os.path.join(REPO, "include")]
    hdr = os.path.join(REPO, "steps_b200", "steps_api", "tetopsplit_b200.hpp")
    t_src = max(os.path.getmtime(DROPIN), os.path.getmtime(hdr), os.path.getmtime(HARNESS), shim_mtime())
    objs = []
    for src, name, extra in ((DROPIN, "dropin_tetopsplit_b200.o", []),
                             (HARNESS, "harness_b200.o", ["-DSTEPS_WITH_B200_API"])):
        o = os.path.join(OBJ, name)
        if force or not os.path.exists(o) or os.path.getmtime(o) < t_src:
            r = subprocess.run(["g++"] + FLAGS + inc + extra + ["-c", src, "-o", o], capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"drop-in build failed ({src}):\n{r.stderr[-3000:]}")
        objs.append(o)
    lib_dir = os.path.join(REPO, "steps_b200")
    if not os.path.exists(os.path.join(lib_dir, "libsteps_b200.so")):
        return None
    if force or not os.path.exists(LIB_B200) or os.path.getmtime(LIB_B200) < max(
            [os.path.getmtime(o) for o in objs + ref_objs] + [os.path.getmtime(os.path.join(lib_dir, "libsteps_b200.so"))]):
        r = subprocess.run(["g++", "-shared", "-o", LIB_B200] + ref_objs + objs +
                           ["-L" + lib_dir, "-lsteps_b200", "-Wl,-rpath,$ORIGIN/../../steps_b200"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"drop-in link failed:\n{r.stderr[-3000:]}")
    return LIB_B200


if __name__ == "__main__":
    j = None
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    print(build(force="--force" in sys.argv, jobs=j))
