"""TEST INFRASTRUCTURE ONLY — ctypes wrapper of the CPU oracle (liboracle.so).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference arms.
The product (steps_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build_oracle

_lib = None


def load():
    global _lib
    if _lib is None:
        path = build_oracle.build_oracle()
        lib = C.CDLL(path)
        P = C.c_void_p
        pf, pi, pu = (C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_uint32))
        lib.or_create.restype = P
        lib.or_create.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, pf, pi, pf, pf, pi, C.c_int, pi]
        lib.or_destroy.argtypes = [P]
        lib.or_add_reac.argtypes = [P, C.c_int, pu, pi, C.c_double]
        lib.or_add_reac.restype = C.c_int
        lib.or_add_diff.argtypes = [P, C.c_int, C.c_int, C.c_double]
        lib.or_set_reac_k.argtypes = [P, C.c_int, C.c_int, C.c_double]
        lib.or_setup.argtypes = [P]
        lib.or_setup.restype = C.c_int
        lib.or_set_counts.argtypes = [P, C.c_int, pu]
        lib.or_get_counts.argtypes = [P, C.c_int, pu]
        lib.or_set_clamped.argtypes = [P, C.c_int, C.c_int, C.c_int]
        lib.or_set_time.argtypes = [P, C.c_int, C.c_double, C.c_uint64]
        lib.or_get_time.argtypes = [P, C.c_int]
        lib.or_get_time.restype = C.c_double
        lib.or_get_window.argtypes = [P, C.c_int]
        lib.or_get_window.restype = C.c_uint64
        lib.or_get_period.argtypes = [P, C.c_int]
        lib.or_get_period.restype = C.c_double
        lib.or_get_reac_extent.argtypes = [P, C.c_int]
        lib.or_get_reac_extent.restype = C.c_uint64
        lib.or_get_diff_extent.argtypes = [P]
        lib.or_get_diff_extent.restype = C.c_uint64
        lib.or_run.argtypes = [P, C.c_double]
        lib.or_run.restype = C.c_uint64
        lib.or_philox4x32_r.argtypes = [C.c_int, pu, pu, pu]
        lib.or_log_export.argtypes = [C.c_double]
        lib.or_log_export.restype = C.c_double
        lib.or_binom_many.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_uint32, pu]
        lib.or_leave_many.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_uint32, pu]
        lib.or_set_boundaries.argtypes = [P, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        lib.or_set_btab.argtypes = [P, C.POINTER(C.c_double)]
        lib.or_distribute.argtypes = [C.c_uint64, C.c_uint64, C.c_int, pf, C.c_double, pu]
        lib.or_distribute.restype = C.c_int
        lib.or_set_surface.argtypes = [P, C.c_int, C.c_int, pi, pi, pf, C.c_int]
        lib.or_add_sreac.argtypes = [P, C.c_int, pu, pu, pi, pi, C.c_double, C.c_double, C.c_double, C.c_int, pf]
        lib.or_add_sreac.restype = C.c_int
        lib.or_add_ghk.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_int]
        lib.or_set_temp.argtypes = [P, C.c_double]
        lib.or_set_tri_outer.argtypes = [P, pi]
        lib.or_set_sreac_outer.argtypes = [P, C.c_int, pu, pi]
        lib.or_set_tri_neighbours.argtypes = [P, pi, pi, pf, pf]
        lib.or_add_sdiff.argtypes = [P, C.c_int, C.c_int, C.c_double]
        lib.or_set_tri_counts.argtypes = [P, C.c_int, pu]
        lib.or_get_tri_counts.argtypes = [P, C.c_int, pu]
        lib.or_set_tri_v.argtypes = [P, pf]
        lib.or_get_surf_ext.argtypes = [P]
        lib.or_get_surf_ext.restype = C.c_uint64
        lib.or_get_echarge.argtypes = [P, C.POINTER(C.c_int64)]
        lib.or_exp_export.argtypes = [C.c_double]
        lib.or_exp_export.restype = C.c_double
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def distribute(seed, call, weights, x):
    """Counts of a compartment placement of x molecules over tets of the given weights
    (util/distribute.hpp:102-193), drawn from the solver's stream of its setter call
    number ``call``."""
    L = load()
    w = np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros(w.size, dtype=np.uint32)
    st = L.or_distribute(C.c_uint64(seed), C.c_uint64(call), w.size, _p(w, C.c_double), float(x),
                         _p(out, C.c_uint32))
    if st != 0:
        raise ValueError(f"distribute failed ({st})")
    return out


class Oracle:
    """CPU oracle over tables from steps_b200.solver.flatten (same species/reaction order).

    The number of OpenMP threads is taken from OMP_NUM_THREADS at library load."""

    def __init__(self, tables, seed, realizations=None):
        self.L = load()
        F = tables
        self.F = F
        self.ntets = int(F["vol"].size)
        self.nspec = len(F["spec_names"])
        off = np.ascontiguousarray(realizations if realizations is not None else [0, self.ntets],
                                   dtype=np.int32)
        self._keep = [F["vol"], F["neighb"], F["area"], F["dist"], F["tet_comp"], off]
        self.off = off
        self.nreal = len(off) - 1
        self.h = self.L.or_create(C.c_uint64(seed), self.ntets, self.nspec, max(len(F["comp_names"]), 1),
                                  _p(F["vol"], C.c_double), _p(F["neighb"], C.c_int32),
                                  _p(F["area"], C.c_double), _p(F["dist"], C.c_double),
                                  _p(F["tet_comp"], C.c_int32), self.nreal, _p(off, C.c_int32))
        if not self.h:
            raise ValueError("oracle supports at most 32 species")
        for (ci, _rid, lhs, upd, k) in F["reacs"]:
            self.L.or_add_reac(self.h, ci, _p(lhs, C.c_uint32), _p(upd, C.c_int32), k)
        for (ci, _did, s, d) in F["diffs"]:
            self.L.or_add_diff(self.h, ci, s, d)
        sf = F.get("surf")
        self.ntris = 0
        if sf is not None:
            # Membrane triangles, surface reactions (k(V) tables), GHK currents and surface
            # diffusion, from the same tables the GPU solver receives.
            tri_inner = np.ascontiguousarray(sf["tri_inner"], dtype=np.int32)
            tri_patch = np.ascontiguousarray(sf["tri_patch"], dtype=np.int32)
            self.ntris, self.nsspec = len(sf["tris"]), sf["nsspec"]
            self._keep += [tri_inner, tri_patch, sf["tri_area"], sf["tri_nbr"], sf["tri_nbr_edge"], sf["tri_len"],
                           sf["tri_dist"]]
            self.L.or_set_surface(self.h, sf["nsspec"], self.ntris, _p(tri_inner, C.c_int32),
                                  _p(tri_patch, C.c_int32), _p(sf["tri_area"], C.c_double),
                                  len(sf["patch_names"]))
            if sf.get("tri_outer") is not None:
                tri_outer = np.ascontiguousarray(sf["tri_outer"], dtype=np.int32)
                self._keep.append(tri_outer)
                self.L.or_set_tri_outer(self.h, _p(tri_outer, C.c_int32))
            outer_rows = sf.get("sreac_outer") or [None] * len(sf["sreacs"])
            for (pi, _rid, (slhs, ilhs, supd, iupd), k, vdep), orow in zip(sf["sreacs"], outer_rows):
                args = (self.h, pi, _p(slhs, C.c_uint32), _p(ilhs, C.c_uint32), _p(supd, C.c_int32),
                        _p(iupd, C.c_int32))
                if vdep is None:
                    idx = self.L.or_add_sreac(*args, k, 0.0, 0.0, 0, None)
                else:
                    vmin, dv, tab = vdep
                    tab = np.ascontiguousarray(tab, dtype=np.float64)
                    idx = self.L.or_add_sreac(*args, 0.0, vmin, dv, tab.size, _p(tab, C.c_double))
                if orow is not None:
                    olhs = np.ascontiguousarray(orow[0], dtype=np.uint32)
                    oupd = np.ascontiguousarray(orow[1], dtype=np.int32)
                    self.L.or_set_sreac_outer(self.h, idx, _p(olhs, C.c_uint32), _p(oupd, C.c_int32))
            for (pi, _gid, ss, ion, z, perm, vshift, voconc, flux) in sf["ghks"]:
                self.L.or_add_ghk(self.h, pi, ss, ion, int(z), float(perm), float(vshift), float(voconc),
                                  1 if flux else 0)
            if sf["sdiffs"]:
                self.L.or_set_tri_neighbours(self.h, _p(sf["tri_nbr"], C.c_int32), _p(sf["tri_nbr_edge"], C.c_int32),
                                             _p(sf["tri_len"], C.c_double), _p(sf["tri_dist"], C.c_double))
                for (pi, _did, ss, d) in sf["sdiffs"]:
                    self.L.or_add_sdiff(self.h, pi, ss, float(d))
        self.nbnd = len(F.get("diffbound_names", []))
        if self.nbnd:
            self._keep += [F["face_bnd"], F["bnd_comps"]]
            self.L.or_set_boundaries(self.h, self.nbnd, _p(F["face_bnd"], C.c_int32), _p(F["bnd_comps"], C.c_int32))
            self.bact = np.zeros((self.nbnd, self.nspec, 2), dtype=bool)
            self.bdcst = np.full((self.nbnd, self.nspec, 2), -1.0)
        if self.L.or_setup(self.h) != 0:
            raise ValueError("neighbour table is not symmetric")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_destroy(self.h)
            self.h = None

    def _push_btab(self):
        tab = np.where(self.bact, np.where(self.bdcst >= 0.0, self.bdcst, -2.0), -1.0)
        self._btab = np.ascontiguousarray(tab.reshape(-1), dtype=np.float64)
        self.L.or_set_btab(self.h, _p(self._btab, C.c_double))

    def set_bnd_active(self, b, s, on):
        """Same rule as the solver's setDiffBoundarySpecDiffusionActive."""
        self.bact[b, s, :] = on
        self._push_btab()

    def set_bnd_dcst(self, b, s, d, direction_comp=-1):
        """Same rule as the solver's setDiffBoundarySpecDcst (direction_comp index, -1 both)."""
        comps = self.F["bnd_comps"].reshape(-1, 2)[b]
        for side in range(2):
            if direction_comp >= 0 and comps[side] == direction_comp:
                continue
            self.bact[b, s, side] = True
            self.bdcst[b, s, side] = d
        self._push_btab()

    def set_counts(self, s, row):
        a = np.ascontiguousarray(row, dtype=np.uint32)
        self.L.or_set_counts(self.h, s, _p(a, C.c_uint32))

    def get_counts(self, s):
        a = np.empty(self.ntets, dtype=np.uint32)
        self.L.or_get_counts(self.h, s, _p(a, C.c_uint32))
        return a

    def set_tri_counts(self, ss, row):
        a = np.ascontiguousarray(row, dtype=np.uint32)
        self.L.or_set_tri_counts(self.h, ss, _p(a, C.c_uint32))

    def get_tri_counts(self, ss):
        a = np.empty(self.ntris, dtype=np.uint32)
        self.L.or_get_tri_counts(self.h, ss, _p(a, C.c_uint32))
        return a

    def set_temp(self, kelvin):
        self.L.or_set_temp(self.h, float(kelvin))

    def surf_extent(self):
        return self.L.or_get_surf_ext(self.h)

    def echarge(self):
        a = np.empty(self.ntris, dtype=np.int64)
        self.L.or_get_echarge(self.h, a.ctypes.data_as(C.POINTER(C.c_int64)))
        return a

    def set_reac_k(self, reac, real, k):
        self.L.or_set_reac_k(self.h, reac, real, k)

    def set_clamped(self, tet, s, on):
        self.L.or_set_clamped(self.h, tet, s, 1 if on else 0)

    def set_time(self, real, t, window):
        self.L.or_set_time(self.h, real, t, window)

    def time(self, real=0):
        return self.L.or_get_time(self.h, real)

    def window(self, real=0):
        return self.L.or_get_window(self.h, real)

    def period(self, real=0):
        return self.L.or_get_period(self.h, real)

    def reac_extent(self, reac):
        return self.L.or_get_reac_extent(self.h, reac)

    def diff_extent(self):
        return self.L.or_get_diff_extent(self.h)

    def run(self, endtime):
        return self.L.or_run(self.h, endtime)


def philox(ctr, key, rounds=8):
    """One Philox4x32 block; the streams use 8 rounds (the reference's R123)."""
    L = load()
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.empty(4, dtype=np.uint32)
    L.or_philox4x32_r(int(rounds), _p(c, C.c_uint32), _p(k, C.c_uint32), _p(o, C.c_uint32))
    return [int(x) for x in o]


def log(x):
    return load().or_log_export(float(x))


def leave_many(seed, unit, n, t1, c, count):
    """count per-molecule leaves of n molecules (leave probability t1, conditional face
    selectors c): [count][4] molecules per face."""
    out = np.empty(count * 4, dtype=np.uint32)
    load().or_leave_many(seed, unit, n, float(t1), float(c[0]), float(c[1]), float(c[2]), count,
                         _p(out, C.c_uint32))
    return out.reshape(count, 4)


def binom_many(seed, unit, n, p, count):
    out = np.empty(count, dtype=np.uint32)
    load().or_binom_many(seed, unit, n, p, count, _p(out, C.c_uint32))
    return out
