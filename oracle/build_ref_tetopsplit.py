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
        "mpi/tetopsplit", "tetexact", "wmdirect", "wmrk4", "wmrssa"]
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


PYSTEPS = os.path.join(os.path.dirname(SRC), "pysteps")
CYSRC = os.path.join(REPO, "steps_b200", "steps_api", "cysteps_b200.pyx")
CYPXD = os.path.join(REPO, "steps_b200", "steps_api", "steps_b200.pxd")
TETODE_STANDIN = os.path.join(SHIM, "tetode_standin.cpp")


def cython_module_path():
    import sysconfig

    return os.path.join(OUT, "cysteps_b200" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_cython(force=False):
    """oracle/_ref/cysteps_b200.<ext>: the reference's own Python binding (pysteps/cysteps.pyx,
    cythonized where it lies, with the compile-time settings of its CMake build for a
    build without PETSc, the distributed mesh or SUNDIALS) plus the drop-in's binding class
    steps_b200/steps_api/cysteps_b200.pyx, linked to libsteps_ref_b200.so.  TetODE, which
    needs SUNDIALS, is replaced by oracle/ref_shim/tetode_standin.cpp.  Returns the module
    path, or None without the reference tree, Cython or the drop-in library."""
    if not available() or not os.path.isdir(PYSTEPS) or not os.path.exists(LIB_B200):
        return None
    try:
        import Cython  # noqa: F401
    except ImportError:
        return None
    import sysconfig

    import numpy

    mod = cython_module_path()
    deps = [CYSRC, CYPXD, TETODE_STANDIN, LIB_B200, os.path.join(REPO, "steps_b200", "steps_api", "tetopsplit_b200.hpp")]
    if not force and os.path.exists(mod) and os.path.getmtime(mod) >= max(os.path.getmtime(p) for p in deps):
        return mod
    cydir = os.path.join(OUT, "cy")
    os.makedirs(cydir, exist_ok=True)
    cpp = os.path.join(cydir, "cysteps_b200.cpp")
    env = ["--compile-time-env", "USE_PETSC=False", "--compile-time-env", "STEPS_USE_DIST_MESH=False",
           "--compile-time-env", "STEPS_SUNDIALS_VERSION_MAJOR=6"]
    _run_checked([sys.executable, "-m", "cython", "-3", "--cplus", "-I", PYSTEPS, "-I", os.path.dirname(CYSRC)] + env +
                 ["-o", cpp, CYSRC], "cythonize")
    inc = ["-I" + os.path.join(REPO, "steps_b200"), "-I" + os.path.join(REPO, "include"), "-I" + PYSTEPS,
           "-I" + sysconfig.get_paths()["include"], "-I" + numpy.get_include()]
    objs = []
    for src, obj in ((cpp, os.path.join(cydir, "cysteps_b200.o")), (TETODE_STANDIN, os.path.join(cydir, "tetode_standin.o"))):
        flags = [f for f in FLAGS if f != "-O2"] + ["-O1"]
        _run_checked(["g++"] + flags + inc + ["-c", src, "-o", obj], "compile " + os.path.basename(src))
        objs.append(obj)
    _run_checked(["g++", "-shared", "-o", mod] + objs + ["-L" + OUT, "-lsteps_ref_b200", "-Wl,-rpath,$ORIGIN"],
                 "link the binding module")
    return mod


def _run_checked(cmd, what):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{what} failed:\n{r.stdout[-2000:]}\n{r.stderr[-3000:]}")


if __name__ == "__main__":
    j = None
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    print(build(force="--force" in sys.argv, jobs=j))
    print(build_cython(force="--force" in sys.argv))
