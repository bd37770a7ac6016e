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
# The same reference objects plus the drop-in TetOpSplitB200 (kind "b200"), linked to
# steps_b200/libsteps_b200.so.
LIB_B200_PATH = os.path.join(HERE, "_ref", "libsteps_ref_b200.so")
_libs = {}


def available(with_dropin=False):
    return os.path.exists(LIB_B200_PATH if with_dropin else LIB_PATH)


def load(with_dropin=False):
    path = LIB_B200_PATH if with_dropin else LIB_PATH
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python oracle/build_ref_tetopsplit.py` "
                          "where the reference tree is present")
    lib = C.CDLL(path, mode=os.RTLD_NOW)
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
    lib.ref_create_memb.restype = vp
    lib.ref_create_memb.argtypes = [ip, ip, dp, ip, C.POINTER(C.c_int64), ip, dp, dp, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_uint64, ip]
    i64, cs = C.c_int64, C.c_char_p
    for nm, args in (("ref_surf_tris", [vp, C.POINTER(i64), ip, C.POINTER(ip)]),
                     ("ref_tri_verts", [vp, i64, C.POINTER(i64)]),
                     ("ref_get_tet_count", [vp, i64, cs, dp]), ("ref_set_tet_count", [vp, i64, cs, C.c_double]),
                     ("ref_get_tri_count", [vp, i64, cs, dp]), ("ref_set_tri_count", [vp, i64, cs, C.c_double]),
                     ("ref_get_patch_count", [vp, cs, dp]), ("ref_set_patch_count", [vp, cs, C.c_double]),
                     ("ref_get_vert_v", [vp, i64, dp]), ("ref_set_vert_v", [vp, i64, C.c_double]),
                     ("ref_set_vert_iclamp", [vp, i64, C.c_double]),
                     ("ref_set_memb", [vp] + [C.c_double] * 6), ("ref_solver_name", [vp, C.c_char_p, ip]),
                     ("ref_get_comp_count_named", [vp, cs, cs, dp]),
                     ("ref_set_comp_count_named", [vp, cs, cs, C.c_double])):
        f = getattr(lib, nm)
        f.argtypes = args
        f.restype = C.c_int
    lib.ref_create_outer.restype = vp
    lib.ref_create_outer.argtypes = [ip, ip, dp, ip, C.POINTER(C.c_int64), C.POINTER(C.c_int32), dp, C.c_uint64]
    _libs[path] = lib
    return lib


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


_KINDS = {"tetopsplit": 0, "tetexact": 1, "b200": 2}


class RefSim:
    """One reference solver on one compartment of every tet: the reference TetOpSplitP,
    Tetexact, or ("b200") the drop-in TetOpSplitB200 on the same reference objects."""

    def __init__(self, mesh, tables, seed, kind="tetopsplit", rng_buf=512):
        lib = load(with_dropin=(kind == "b200"))
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
        h = lib.ref_create(_KINDS[kind], verts.shape[0], _ptr(verts, C.c_double),
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

    # ---- through the reference API's public methods (api.hpp) ----
    def get_tet_count(self, tet, name):
        out = C.c_double()
        self._ok(self._lib.ref_get_tet_count(self._h, int(tet), name.encode(), C.byref(out)))
        return out.value

    def set_tet_count(self, tet, name, n):
        self._ok(self._lib.ref_set_tet_count(self._h, int(tet), name.encode(), float(n)))

    def solver_name(self):
        buf = C.create_string_buffer(128)
        self._ok(self._lib.ref_solver_name(self._h, buf, 128))
        return buf.value.decode()


class RefMemb(RefSim):
    """The membrane model of ref_create_memb: every surface triangle a patch with channel
    states C and O (k(V) tables kopen / kclose at vmin + i dv), an ohmic current through O
    (g per channel, erev) and one membrane; kind "tetopsplit" or "b200"; efopt the
    reference's EField option (0 = none, 1 = EF_DEFAULT)."""

    def __init__(self, mesh, seed, kopen, kclose, vmin, vmax, dv, g, erev, kind="tetopsplit", efopt=1):
        lib = load(with_dropin=(kind == "b200"))
        self._lib = lib
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        tets = np.ascontiguousarray(mesh.tets, dtype=np.int64)
        ko = np.ascontiguousarray(kopen, dtype=np.float64)
        kc = np.ascontiguousarray(kclose, dtype=np.float64)
        self._keep = (verts, tets, ko, kc)
        self.ntets = int(tets.shape[0])
        self.nspec = 0
        h = lib.ref_create_memb(_KINDS[kind], verts.shape[0], _ptr(verts, C.c_double), self.ntets,
                                _ptr(tets, C.c_int64), ko.size, _ptr(ko, C.c_double), _ptr(kc, C.c_double),
                                vmin, vmax, dv, g, erev, int(seed), int(efopt))
        if not h:
            raise RuntimeError("reference membrane model construction failed: " + lib.ref_last_error().decode())
        self._h = h

    def surf_tris(self):
        n = C.c_int()
        self._ok(self._lib.ref_surf_tris(self._h, None, 0, C.byref(n)))
        out = np.zeros(n.value, dtype=np.int64)
        self._ok(self._lib.ref_surf_tris(self._h, _ptr(out, C.c_int64), n.value, C.byref(n)))
        return out

    def tri_verts(self, tri):
        out = np.zeros(3, dtype=np.int64)
        self._ok(self._lib.ref_tri_verts(self._h, int(tri), _ptr(out, C.c_int64)))
        return out

    def get_tri_count(self, tri, name):
        out = C.c_double()
        self._ok(self._lib.ref_get_tri_count(self._h, int(tri), name.encode(), C.byref(out)))
        return out.value

    def set_tri_count(self, tri, name, n):
        self._ok(self._lib.ref_set_tri_count(self._h, int(tri), name.encode(), float(n)))

    def get_patch_count(self, name):
        out = C.c_double()
        self._ok(self._lib.ref_get_patch_count(self._h, name.encode(), C.byref(out)))
        return out.value

    def set_patch_count(self, name, n):
        self._ok(self._lib.ref_set_patch_count(self._h, name.encode(), float(n)))

    def get_vert_v(self, v):
        out = C.c_double()
        self._ok(self._lib.ref_get_vert_v(self._h, int(v), C.byref(out)))
        return out.value

    def set_vert_v(self, v, x):
        self._ok(self._lib.ref_set_vert_v(self._h, int(v), float(x)))

    def set_vert_iclamp(self, v, amps):
        self._ok(self._lib.ref_set_vert_iclamp(self._h, int(v), float(amps)))

    def set_memb(self, v0, cm, ra, ro, vrev, efdt):
        """setMembPotential, setMembCapac, setMembVolRes, setMembRes, setEfieldDT."""
        self._ok(self._lib.ref_set_memb(self._h, v0, cm, ra, ro, vrev, efdt))


class RefOuter(RefMemb):
    """The two-compartment membrane of ref_create_outer: tets with is_outer = 0 in "cyto",
    the rest in "ecs", the triangles between them the patch "memb" with pump and channel
    surface reactions that reach both volumes; k the ten constants (D_Ca inner, D_B,
    bind, unbind, D_Ca outer, pin, pout, open, close, back); kind "tetopsplit", "tetexact"
    or "b200"."""

    def __init__(self, mesh, is_outer, k, seed, kind="tetopsplit"):
        lib = load(with_dropin=(kind == "b200"))
        self._lib = lib
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        tets = np.ascontiguousarray(mesh.tets, dtype=np.int64)
        flag = np.ascontiguousarray(is_outer, dtype=np.int32)
        kk = np.ascontiguousarray(k, dtype=np.float64)
        self._keep = (verts, tets, flag, kk)
        self.ntets = int(tets.shape[0])
        self.nspec = 0
        h = lib.ref_create_outer(_KINDS[kind], verts.shape[0], _ptr(verts, C.c_double), self.ntets,
                                 _ptr(tets, C.c_int64), _ptr(flag, C.c_int32), _ptr(kk, C.c_double), int(seed))
        if not h:
            raise RuntimeError("reference outer-membrane model construction failed: "
                               + lib.ref_last_error().decode())
        self._h = h

    def get_comp(self, comp, spec):
        out = C.c_double()
        self._ok(self._lib.ref_get_comp_count_named(self._h, comp.encode(), spec.encode(), C.byref(out)))
        return out.value

    def set_comp(self, comp, spec, n):
        self._ok(self._lib.ref_set_comp_count_named(self._h, comp.encode(), spec.encode(), float(n)))
