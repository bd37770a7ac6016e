"""TEST INFRASTRUCTURE ONLY — Python handle on the reference solvers built from the
reference's own sources (oracle/build_ref_tetopsplit.py -> oracle/_ref/libsteps_ref.so).

    sim = RefSim(mesh, model_tables, seed, kind="tetopsplit" | "tetexact")

``model_tables`` is the dict ``steps_b200.solver.flatten`` returns (species, reactions,
diffusion rules of one compartment); the reference receives the same mesh arrays, rate
constants and seed as the GPU solver and builds its own tables from them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libsteps_ref.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python oracle/build_ref_tetopsplit.py` "
                          "where the reference tree is present")
    lib = C.CDLL(LIB_PATH, mode=os.RTLD_NOW)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_create.restype = vp
    lib.ref_create.argtypes = [ip, ip, dp, ip, C.POINTER(C.c_int64), ip, dp, ip, C.POINTER(C.c_uint32),
                               C.POINTER(C.c_uint32), dp, C.c_uint64, ip]
    lib.ref_destroy.argtypes = [vp]
    for nm, args in (("ref_set_comp_count", [vp, ip, C.c_double]), ("ref_set_tet_counts", [vp, ip, dp]),
                     ("ref_get_tet_counts", [vp, ip, dp]), ("ref_get_comp_count", [vp, ip, dp]),
                     ("ref_run", [vp, C.c_double])):
        f = getattr(lib, nm)
        f.argtypes = args
        f.restype = C.c_int
    lib.ref_get_time.argtypes = [vp]
    lib.ref_get_time.restype = C.c_double
    lib.ref_upd_period.argtypes = [vp]
    lib.ref_upd_period.restype = C.c_double
    lib.ref_nsteps.argtypes = [vp]
    lib.ref_nsteps.restype = C.c_uint64
    _lib = lib
    return lib


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class RefSim:
    """One reference solver (TetOpSplitP or Tetexact) on one compartment of every tet."""

    def __init__(self, mesh, tables, seed, kind="tetopsplit", rng_buf=512):
        lib = load()
        self._lib = lib
        S = len(tables["spec_names"]) if "spec_names" in tables else int(tables["nspec"])
        R = len(tables["reacs"])
        dcst = np.zeros(S)
        for (_c, _d, s, d) in tables["diffs"]:
            dcst[s] = d
        lhs = np.zeros((max(R, 1), S), dtype=np.uint32)
        rhs = np.zeros((max(R, 1), S), dtype=np.uint32)
        kc = np.zeros(max(R, 1))
        for q, r in enumerate(tables["reacs"]):
            lhs[q] = r[2]
            rhs[q] = np.asarray(r[2], dtype=np.int64) + np.asarray(r[3], dtype=np.int64)
            kc[q] = r[4]
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        tets = np.ascontiguousarray(mesh.tets, dtype=np.int64)
        self.nspec, self.ntets = S, int(tets.shape[0])
        self._keep = (verts, tets, dcst, lhs, rhs, kc)
        h = lib.ref_create(0 if kind == "tetopsplit" else 1, verts.shape[0], _ptr(verts, C.c_double),
                           self.ntets, _ptr(tets, C.c_int64), S, _ptr(dcst, C.c_double), R,
                           _ptr(lhs, C.c_uint32), _ptr(rhs, C.c_uint32), _ptr(kc, C.c_double), int(seed),
                           int(rng_buf))
        if not h:
            raise RuntimeError("reference solver construction failed: " + lib.ref_last_error().decode())
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ref_destroy(self._h)
            self._h = None

    def _ok(self, st):
        if st != 0:
            raise RuntimeError(self._lib.ref_last_error().decode())

    def set_comp_count(self, s, n):
        self._ok(self._lib.ref_set_comp_count(self._h, int(s), float(n)))

    def set_tet_counts(self, s, counts):
        c = np.ascontiguousarray(counts, dtype=np.float64)
        self._ok(self._lib.ref_set_tet_counts(self._h, int(s), _ptr(c, C.c_double)))

    def get_tet_counts(self, s):
        out = np.zeros(self.ntets)
        self._ok(self._lib.ref_get_tet_counts(self._h, int(s), _ptr(out, C.c_double)))
        return out

    def get_comp_count(self, s):
        out = C.c_double()
        self._ok(self._lib.ref_get_comp_count(self._h, int(s), C.byref(out)))
        return out.value

    def run(self, t):
        self._ok(self._lib.ref_run(self._h, float(t)))

    def time(self):
        return self._lib.ref_get_time(self._h)

    def period(self):
        return self._lib.ref_upd_period(self._h)

    def nsteps(self):
        return int(self._lib.ref_nsteps(self._h))
