"""Python mirror of the reference's TetOpSplit solver class.

Same constructor arguments and method names as the Cython binding
``_py_TetOpSplitP`` (pysteps/cysteps_mpi.pyx:74-200 and the get/set methods at
:2593-2609, :3728-3742, :4831) and its API_1 aliases (getTetCount, setCompCount, ...).
The model and mesh are flattened here and handed to the C ABI of libsteps_b200.so;
every call below goes to the GPU solver.  Host lists (tet_hosts, tri_hosts,
wm_hosts) are accepted and ignored: the whole mesh lives on one GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import ArgErr, check, ptr

EF_NONE = 0
EF_DEFAULT = 1
EF_DV_BDSYS = 2
EF_DV_PETSC = 3
# GPU membrane-potential solvers: two-level preconditioned CG in FP64, or FP32 CG inside an
# FP64 residual-refinement loop.  The reference's direct/PETSc choices map to FP64 CG.
EF_DV_CG_FP64 = 10
EF_DV_CG_MIXED = 11
_EF_METHOD = {EF_DEFAULT: 0, EF_DV_BDSYS: 0, EF_DV_PETSC: 0, EF_DV_CG_FP64: 0, EF_DV_CG_MIXED: 1}

AVOGADRO = 6.02214179e23  # src/steps/math/constants.hpp:45


def flatten(model, geom):
    """Model x mesh -> index tables (the role of the reference Statedef / Compdef,
    src/steps/solver/statedef.hpp:40, compdef.hpp:252-266): volume species in model
    order, compartments in mesh order, per compartment its reactions (dense lhs/upd rows)
    in model order and its diffusion rules."""
    from .model import ChanState

    spec_names = [n for n, s in model.specs.items() if not isinstance(s, ChanState)]
    if not spec_names:
        spec_names = ["__inert__"]  # membrane-only models: one species that never changes
    spec_index = {n: i for i, n in enumerate(spec_names)}
    comp_names = list(geom.comps.keys())
    comp_index = {n: i for i, n in enumerate(comp_names)}
    S = len(spec_names)

    def sidx(name):
        try:
            return spec_index[name]
        except KeyError:
            raise ArgErr(f"unknown species '{name}'") from None

    tet_comp = np.full(geom.ntets, -1, dtype=np.int32)
    for ci, name in enumerate(comp_names):
        tet_comp[geom.comps[name].tets] = ci
    reacs, diffs = [], []
    for ci, cname in enumerate(comp_names):
        for vsname in geom.comps[cname].volsys:
            vs = model.volsys[vsname]
            for rid, r in vs.reacs.items():
                lhs = np.zeros(S, dtype=np.uint32)
                upd = np.zeros(S, dtype=np.int32)
                for s in r.lhs:
                    lhs[sidx(s)] += 1
                    upd[sidx(s)] -= 1
                for s in r.rhs:
                    upd[sidx(s)] += 1
                reacs.append((ci, rid, lhs, upd, r.kcst))
            for did, d in vs.diffs.items():
                diffs.append((ci, did, sidx(d.lig), d.dcst))
    surf = flatten_surface(model, geom, spec_index, comp_index, tet_comp)
    # Diffusion boundaries: the boundary of every tet face (-1 none) and the boundary's
    # two compartments (diffboundary.cpp).
    dbs = list(getattr(geom, "diffbounds", {}).values())
    face_bnd = np.full((geom.ntets, 4), -1, dtype=np.int32)
    bnd_comps = np.zeros((len(dbs), 2), dtype=np.int32)
    for bi, db in enumerate(dbs):
        bnd_comps[bi] = [comp_index[db.comps[0]], comp_index[db.comps[1]]]
        for tri in db.tris:
            for tet in geom.tri_tets[tri]:
                f = int(np.nonzero(geom.tet_tri[tet] == tri)[0][0])
                face_bnd[tet, f] = bi
    return {
        "diffbound_names": [db.id for db in dbs], "face_bnd": np.ascontiguousarray(face_bnd.reshape(-1)),
        "bnd_comps": np.ascontiguousarray(bnd_comps.reshape(-1)),
        "spec_names": spec_names, "spec_index": spec_index,
        "comp_names": comp_names, "comp_index": comp_index,
        "tet_comp": tet_comp, "reacs": reacs, "diffs": diffs, "surf": surf,
        "vol": np.ascontiguousarray(geom.tet_vol, dtype=np.float64),
        "neighb": np.ascontiguousarray(geom.tet_neighb, dtype=np.int32),
        "area": np.ascontiguousarray(geom.tet_area, dtype=np.float64),
        "dist": np.ascontiguousarray(geom.tet_dist, dtype=np.float64),
    }


def flatten_surface(model, geom, spec_index, comp_index, tet_comp):
    """Patches -> membrane triangle tables (the role of Patchdef, src/steps/solver/patchdef.hpp):
    the sorted union of all patch triangles, each with its inner tet (the tet on the side of
    the patch's inner compartment), its outer tet (on the side of the outer compartment, -1
    none), patch and area; the surface species; the surface reactions (dense slhs/ilhs/supd/
    iupd rows, and olhs/oupd rows of their outer-volume terms), k(V) tables of
    voltage-dependent ones, and the ohmic currents.  None when the mesh has no patch with a
    surface system."""
    patches = [p for p in getattr(geom, "patches", {}).values() if p.surfsys]
    if not patches:
        return None
    tris = np.unique(np.concatenate([p.tris for p in patches]))
    tri_index = {int(t): i for i, t in enumerate(tris)}
    tri_patch = np.full(len(tris), -1, dtype=np.int32)
    inner = np.full(len(tris), -1, dtype=np.int32)
    outer = np.full(len(tris), -1, dtype=np.int32)
    for pi, p in enumerate(patches):
        ci = comp_index[p.icomp.id] if p.icomp is not None else -1
        co = comp_index[p.ocomp.id] if getattr(p, "ocomp", None) is not None else -2
        for t in p.tris:
            m = tri_index[int(t)]
            if tri_patch[m] >= 0:
                raise ArgErr("a triangle belongs to two patches")
            tri_patch[m] = pi
            a, b = geom.tri_tets[t]
            inner[m] = a if (a >= 0 and tet_comp[a] == ci) else b
            if inner[m] < 0 or tet_comp[inner[m]] != ci:
                raise ArgErr(f"triangle {t} has no tet in the inner compartment of patch {p.id}")
            o = b if inner[m] == a else a
            if o >= 0 and tet_comp[o] == co:
                outer[m] = o
    sspecs = []

    def sid(name):
        if name not in sspecs:
            sspecs.append(name)
        return sspecs.index(name)

    for p in patches:
        for ssn in p.surfsys:
            ss = model.surfsys[ssn]
            for r in list(ss.sreacs.values()) + list(ss.vdepsreacs.values()):
                if r.olhs and r.ilhs:
                    raise ArgErr(f"surface reaction '{r.id}' has reactants in both volumes")
                if (r.olhs or r.orhs) and getattr(p, "ocomp", None) is None:
                    raise ArgErr(f"surface reaction '{r.id}' reaches the outer volume of patch {p.id}, "
                                 "which has no outer compartment")
                for s in r.slhs + r.srhs:
                    sid(s)
            for oc in ss.ohmiccurrs.values():
                sid(oc.chanstate)
            for gh in ss.ghkcurrs.values():
                sid(gh.chanstate)
    S, SS = len(spec_index), max(len(sspecs), 1)

    def rows(r):
        slhs = np.zeros(SS, np.uint32)
        ilhs = np.zeros(S, np.uint32)
        supd = np.zeros(SS, np.int32)
        iupd = np.zeros(S, np.int32)
        for s in r.slhs:
            slhs[sid(s)] += 1
            supd[sid(s)] -= 1
        for s in r.srhs:
            supd[sid(s)] += 1
        for s in r.ilhs:
            ilhs[spec_index[s]] += 1
            iupd[spec_index[s]] -= 1
        for s in r.irhs:
            iupd[spec_index[s]] += 1
        return slhs, ilhs, supd, iupd

    def outer_rows(r):
        if not (r.olhs or r.orhs):
            return None
        olhs = np.zeros(S, np.uint32)
        oupd = np.zeros(S, np.int32)
        for s in r.olhs:
            olhs[spec_index[s]] += 1
            oupd[spec_index[s]] -= 1
        for s in r.orhs:
            oupd[spec_index[s]] += 1
        return olhs, oupd

    sreacs, ohmics, sdiffs, ghks, sreac_outer = [], [], [], [], []
    for pi, p in enumerate(patches):
        for ssn in p.surfsys:
            ss = model.surfsys[ssn]
            for did, d in ss.diffs.items():
                sdiffs.append((pi, did, sid(d.lig), d.dcst))
            for rid, r in ss.sreacs.items():
                sreacs.append((pi, rid, rows(r), r.kcst, None))
                sreac_outer.append(outer_rows(r))
            for rid, r in ss.vdepsreacs.items():
                vmin, vmax, dv = r.vrange
                n = int(round((vmax - vmin) / dv)) + 1
                tab = np.array([r.kfunc(vmin + i * dv) for i in range(n)], dtype=np.float64)
                sreacs.append((pi, rid, rows(r), 0.0, (vmin, dv, tab)))
                sreac_outer.append(outer_rows(r))
            for oid, oc in ss.ohmiccurrs.items():
                ohmics.append((pi, oid, sid(oc.chanstate), oc.g, oc.erev))
            for gid, gh in ss.ghkcurrs.items():
                if gh.perm is None:
                    raise ArgErr(f"GHK current '{gid}' has no permeability (setP or setPInfo)")
                if gh.voconc < 0.0 and getattr(p, "ocomp", None) is None:
                    raise ArgErr(f"GHK current '{gid}' has no virtual outer concentration and patch {p.id} "
                                 "has no outer compartment")
                ghks.append((pi, gid, sid(gh.chanstate), spec_index[gh.ion], gh.valence, gh.perm, gh.vshift,
                             gh.voconc, gh.computeflux))
    # Edge neighbours of every membrane triangle (sdiff.cpp:62-83, TOS:585-630): across edge j
    # = (v_j, v_j+1) the other membrane triangle on that edge, its edge index, the edge length
    # and the distance between the two barycentres.
    tv = np.asarray(geom.tris)[tris]                       # (M, 3) vertex ids
    M = len(tris)
    e = np.stack([tv, np.roll(tv, -1, axis=1)], axis=2)   # (M, 3, 2)
    ek = np.sort(e, axis=2).reshape(-1, 2)
    order = np.lexsort((ek[:, 1], ek[:, 0]))
    eks = ek[order]
    same = np.all(eks[1:] == eks[:-1], axis=1)
    tri_nbr = np.full(M * 3, -1, dtype=np.int32)
    tri_nbr_edge = np.full(M * 3, -1, dtype=np.int32)
    for i in np.nonzero(same)[0]:
        a, b = order[i], order[i + 1]
        if i + 2 < len(order) and same[i + 1]:
            continue  # an edge of three membrane triangles: no surface diffusion across it
        if i > 0 and same[i - 1]:
            continue
        tri_nbr[a], tri_nbr_edge[a] = b // 3, b % 3
        tri_nbr[b], tri_nbr_edge[b] = a // 3, a % 3
    pv = np.asarray(geom.verts)
    tri_len = np.linalg.norm(pv[e[:, :, 1]] - pv[e[:, :, 0]], axis=2).reshape(-1)
    bary = pv[tv].mean(axis=1)
    nb = np.where(tri_nbr >= 0, tri_nbr, 0)
    tri_dist = np.where(tri_nbr >= 0, np.linalg.norm(bary[nb] - np.repeat(bary, 3, axis=0), axis=1), 0.0)
    return {
        "sdiffs": sdiffs, "ghks": ghks, "tri_nbr": tri_nbr, "tri_nbr_edge": tri_nbr_edge,
        "tri_len": np.ascontiguousarray(tri_len, dtype=np.float64),
        "tri_dist": np.ascontiguousarray(tri_dist, dtype=np.float64),
        "patch_names": [p.id for p in patches], "tris": tris, "tri_index": tri_index,
        "tri_patch": tri_patch, "tri_inner": inner,
        "tri_outer": outer if (outer >= 0).any() else None, "sreac_outer": sreac_outer,
        "tri_area": np.ascontiguousarray(geom.tri_area[tris], dtype=np.float64),
        "sspec_names": sspecs, "sspec_index": {n: i for i, n in enumerate(sspecs)},
        "sreacs": sreacs, "ohmics": ohmics, "nsspec": SS,
    }


class TetOpSplit:
    def __init__(self, model, geom, rng, calcMembPot=EF_NONE, tet_hosts=None, tri_hosts=None,
                 wm_hosts=None, device=0, realizations=None, block=128):
        self._h = None
        self._L = _lib.load()
        self.model, self.geom, self.rng = model, geom, rng
        if calcMembPot not in _EF_METHOD and calcMembPot != EF_NONE:
            raise ArgErr(f"unknown calcMembPot {calcMembPot}")
        h = C.c_void_p()
        check(self._L.sg_create(C.byref(h), C.c_uint64(rng.seed), device))
        self._h = h
        try:
            self._flatten(model, geom, realizations)
            check(self._L.sg_set_launch(self._h, block, 0))
            check(self._L.sg_setup(self._h))
            if calcMembPot != EF_NONE:
                self._setup_efield(geom, _EF_METHOD[calcMembPot])
        except Exception:
            self._L.sg_destroy(self._h)
            self._h = None
            raise

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.sg_destroy(h)
            self._h = None

    # ------------------------------------------------------------------ tables
    def _flatten(self, model, geom, realizations):
        F = flatten(model, geom)
        self.tables = F
        self.spec_names, self.spec_index = F["spec_names"], F["spec_index"]
        self.comp_names, self.comp_index = F["comp_names"], F["comp_index"]
        self.tet_comp = F["tet_comp"]
        L, h = self._L, self._h
        check(L.sg_set_nspecs(h, len(self.spec_names)))
        check(L.sg_set_mesh(h, geom.ntets, ptr(F["vol"], C.c_double), ptr(F["neighb"], C.c_int32),
                            ptr(F["area"], C.c_double), ptr(F["dist"], C.c_double),
                            ptr(F["tet_comp"], C.c_int32), max(len(self.comp_names), 1)))
        self.diffbound_index = {n: i for i, n in enumerate(F["diffbound_names"])}
        if F["diffbound_names"]:
            check(L.sg_set_diff_boundaries(h, len(F["diffbound_names"]), ptr(F["face_bnd"], C.c_int32),
                                           ptr(F["bnd_comps"], C.c_int32)))
        self.reac_index = {}   # (comp, reac id) -> ABI reaction index
        self.diff_index = {}   # (comp, diff id) -> species index
        for (ci, rid, lhs, upd, k) in F["reacs"]:
            out = C.c_int32()
            check(L.sg_add_reac(h, ci, ptr(lhs, C.c_uint32), ptr(upd, C.c_int32), k, C.byref(out)))
            self.reac_index[(self.comp_names[ci], rid)] = out.value
        for (ci, did, s, d) in F["diffs"]:
            out = C.c_int32()
            check(L.sg_add_diff(h, ci, s, d, C.byref(out)))
            self.diff_index[(self.comp_names[ci], did)] = s
        self.surf = F["surf"]
        if self.surf is not None:
            sf = self.surf
            tri_inner = np.ascontiguousarray(sf["tri_inner"], dtype=np.int32)
            tri_patch = np.ascontiguousarray(sf["tri_patch"], dtype=np.int32)
            check(L.sg_set_surface(h, sf["nsspec"], len(sf["tris"]), ptr(tri_inner, C.c_int32),
                                   ptr(tri_patch, C.c_int32), ptr(sf["tri_area"], C.c_double),
                                   len(sf["patch_names"])))
            if sf["tri_outer"] is not None:
                tri_outer = np.ascontiguousarray(sf["tri_outer"], dtype=np.int32)
                check(L.sg_set_tri_outer(h, ptr(tri_outer, C.c_int32)))
            self.sreac_index = {}
            for (pi, rid, (slhs, ilhs, supd, iupd), k, vdep), orow in zip(sf["sreacs"], sf["sreac_outer"]):
                out = C.c_int32()
                args = (h, pi, ptr(slhs, C.c_uint32), ptr(ilhs, C.c_uint32), ptr(supd, C.c_int32),
                        ptr(iupd, C.c_int32))
                if vdep is None:
                    check(L.sg_add_sreac(*args, k, C.byref(out)))
                else:
                    vmin, dv, tab = vdep
                    check(L.sg_add_vdep_sreac(*args, vmin, dv, len(tab), ptr(tab, C.c_double), C.byref(out)))
                if orow is not None:
                    check(L.sg_set_sreac_outer(h, out.value, ptr(orow[0], C.c_uint32), ptr(orow[1], C.c_int32)))
                self.sreac_index[(sf["patch_names"][pi], rid)] = out.value
            for (pi, oid, ss, g, erev) in sf["ohmics"]:
                out = C.c_int32()
                check(L.sg_add_ohmic(h, pi, ss, g, erev, C.byref(out)))
            self.ghk_index = {}
            for (pi, gid, ss, ion, z, perm, vshift, voconc, flux) in sf["ghks"]:
                out = C.c_int32()
                check(L.sg_add_ghk(h, pi, ss, ion, int(z), float(perm), float(vshift), float(voconc),
                                   1 if flux else 0, C.byref(out)))
                self.ghk_index[(sf["patch_names"][pi], gid)] = out.value
            if sf["sdiffs"]:
                check(L.sg_set_tri_neighbours(h, ptr(sf["tri_nbr"], C.c_int32), ptr(sf["tri_nbr_edge"], C.c_int32),
                                              ptr(sf["tri_len"], C.c_double), ptr(sf["tri_dist"], C.c_double)))
                self.sdiff_index = {}
                for (pi, did, ss, d) in sf["sdiffs"]:
                    out = C.c_int32()
                    check(L.sg_add_sdiff(h, pi, ss, float(d), C.byref(out)))
                    self.sdiff_index[(sf["patch_names"][pi], did)] = out.value
        if realizations is not None:
            off = np.ascontiguousarray(realizations, dtype=np.int32)
            self.nreal = len(off) - 1
            check(L.sg_set_realizations(h, self.nreal, ptr(off, C.c_int32)))
            self.real_offsets = off
        else:
            self.nreal = 1
            self.real_offsets = np.array([0, geom.ntets], dtype=np.int32)

    def _setup_efield(self, geom, method):
        membs = getattr(geom, "membs", {})
        if len(membs) != 1:
            raise ArgErr("the membrane potential needs exactly one Memb on the mesh")
        memb = next(iter(membs.values()))
        if self.surf is not None and not np.array_equal(memb.tris, self.surf["tris"]):
            raise ArgErr("the membrane must consist of exactly the patches with surface systems")
        self.memb_tris = memb.tris
        self.memb_index = {int(t): i for i, t in enumerate(memb.tris)}
        verts = np.ascontiguousarray(geom.verts, dtype=np.float64)
        tets = np.ascontiguousarray(geom.tets, dtype=np.int32)
        tris = np.ascontiguousarray(geom.tris[memb.tris], dtype=np.int32)
        check(self._L.sg_set_efield_mesh(self._h, geom.nverts, ptr(verts, C.c_double), ptr(tets, C.c_int32),
                                         len(memb.tris), ptr(tris, C.c_int32), method))

    def _spec(self, name):
        try:
            return self.spec_index[name]
        except KeyError:
            raise ArgErr(f"unknown species '{name}'") from None

    def _comp(self, name):
        try:
            return self.comp_index[name]
        except KeyError:
            raise ArgErr(f"unknown compartment '{name}'") from None

    def _reac(self, c, r):
        try:
            return self.reac_index[(c, r)]
        except KeyError:
            raise ArgErr(f"reaction '{r}' undefined in compartment '{c}'") from None

    # ------------------------------------------------------------ solver info
    def getSolverName(self):
        return "TetOpSplitB200"

    def getSolverDesc(self):
        return "Operator-split spatial SSA on one B200 GPU (Philox counter streams)"

    def getSolverAuthors(self):
        return "steps_b200 developers"

    def getSolverEmail(self):
        return ""

    # --------------------------------------------------------------- control
    def reset(self):
        check(self._L.sg_reset(self._h))

    def run(self, endtime):
        check(self._L.sg_run(self._h, float(endtime)))

    def advance(self, adv):
        check(self._L.sg_advance(self._h, float(adv)))

    def checkpoint(self, file_name):
        """Write the complete simulation state to file_name (API::checkpoint)."""
        check(self._L.sg_checkpoint(self._h, os.fsencode(file_name)))

    def restore(self, file_name):
        """Load a state written by checkpoint() of a solver on the same mesh and model
        (API::restore); the run continues exactly as the checkpointed one would have."""
        check(self._L.sg_restore(self._h, os.fsencode(file_name)))

    def step(self):
        raise _lib.NotImplErr("step() is not implemented for operator-split solvers")

    def getTime(self):
        t = C.c_double()
        check(self._L.sg_get_time(self._h, C.byref(t)))
        return t.value

    def getUpdPeriod(self, realization=0):
        p = C.c_double()
        check(self._L.sg_get_update_period(self._h, realization, C.byref(p)))
        return p.value

    def getNSteps(self):
        n = C.c_uint64()
        check(self._L.sg_get_nsteps(self._h, C.byref(n)))
        return n.value

    def getNIteration(self):
        n = C.c_uint64()
        check(self._L.sg_get_niteration(self._h, C.byref(n)))
        return n.value

    def getDiffExtent(self):
        n = C.c_uint64()
        check(self._L.sg_get_diff_extent(self._h, C.byref(n)))
        return n.value

    def getCompReacExtent(self, c, r):
        n = C.c_uint64()
        check(self._L.sg_get_reac_extent(self._h, self._reac(c, r), C.byref(n)))
        return n.value

    def setDiffApplyThreshold(self, threshold):
        check(self._L.sg_set_diff_apply_threshold(self._h, int(threshold)))

    # ---------------------------------------------------------------- counts
    def getTetSpecCount(self, idx, s):
        n = C.c_double()
        check(self._L.sg_get_tet_count(self._h, int(idx), self._spec(s), C.byref(n)))
        return n.value

    def setTetSpecCount(self, idx, s, n):
        check(self._L.sg_set_tet_count(self._h, int(idx), self._spec(s), float(n)))

    def getCompSpecCount(self, c, s, realization=-1):
        n = C.c_double()
        check(self._L.sg_get_comp_count(self._h, self._comp(c), self._spec(s), int(realization),
                                        C.byref(n)))
        return n.value

    def setCompSpecCount(self, c, s, n, realization=-1):
        check(self._L.sg_set_comp_count(self._h, self._comp(c), self._spec(s), int(realization),
                                        float(n)))

    def _comp_vol(self, c, realization=-1):
        tets = self.geom.comps[c].tets
        if realization >= 0:
            b, e = self.real_offsets[realization], self.real_offsets[realization + 1]
            tets = tets[(tets >= b) & (tets < e)]
        return float(self.geom.tet_vol[tets].sum())

    def getTetSpecConc(self, idx, s):
        return self.getTetSpecCount(idx, s) / (AVOGADRO * self.geom.tet_vol[idx] * 1.0e3)

    def setTetSpecConc(self, idx, s, c):
        self.setTetSpecCount(idx, s, c * AVOGADRO * self.geom.tet_vol[idx] * 1.0e3)

    def getCompSpecConc(self, c, s, realization=-1):
        v = self._comp_vol(c, realization)
        return self.getCompSpecCount(c, s, realization) / (AVOGADRO * v * 1.0e3)

    def setCompSpecConc(self, c, s, conc, realization=-1):
        if realization >= 0:
            self.setCompSpecCount(c, s, conc * AVOGADRO * self._comp_vol(c, realization) * 1.0e3,
                                  realization)
        else:
            for r in range(self.nreal):
                self.setCompSpecCount(c, s, conc * AVOGADRO * self._comp_vol(c, r) * 1.0e3, r)

    def setTetSpecClamped(self, idx, s, clamped):
        check(self._L.sg_set_tet_clamped(self._h, int(idx), self._spec(s), 1 if clamped else 0))

    def getSpecCounts(self, s, out=None):
        """All tets' counts of species s as uint32 (device -> host of one row)."""
        if out is None:
            out = np.empty(self.geom.ntets, dtype=np.uint32)
        check(self._L.sg_get_spec_counts(self._h, self._spec(s), ptr(out, C.c_uint32)))
        return out

    def setSpecCounts(self, s, counts):
        a = np.ascontiguousarray(counts, dtype=np.uint32)
        if a.size != self.geom.ntets:
            raise ArgErr("need one count per tet")
        check(self._L.sg_set_spec_counts(self._h, self._spec(s), ptr(a, C.c_uint32)))

    def getAllSpecCounts(self, out=None):
        """Every species row at once, [species][tet] uint32 in spec_names order (one
        device -> host copy)."""
        n = len(self.spec_names) * self.geom.ntets
        if out is None:
            out = np.empty((len(self.spec_names), self.geom.ntets), dtype=np.uint32)
        if out.dtype != np.uint32 or out.size != n or not out.flags.c_contiguous:
            raise ArgErr("need a contiguous uint32 array of species x tets")
        check(self._L.sg_get_all_counts(self._h, ptr(out, C.c_uint32)))
        return out

    def setAllSpecCounts(self, counts):
        """Set every species row at once from a [species][tet] array (one host -> device copy)."""
        a = np.ascontiguousarray(counts, dtype=np.uint32)
        if a.size != len(self.spec_names) * self.geom.ntets:
            raise ArgErr("need species x tets counts")
        check(self._L.sg_set_all_counts(self._h, ptr(a, C.c_uint32)))

    def getBatchTetSpecCountsNP(self, tets, s, counts):
        """Reference getBatchTetSpecCountsNP (TOS:5715): counts[i] = count of s in tets[i],
        gathered on the device."""
        idx = np.ascontiguousarray(tets, dtype=np.int32)
        out = np.empty(len(idx), dtype=np.float64)
        check(self._L.sg_get_batch_tet_counts(self._h, self._spec(s), ptr(idx, C.c_int32), len(idx),
                                               ptr(out, C.c_double)))
        counts[:] = out

    def getBatchTetSpecConcsNP(self, tets, s, concs):
        """Reference getBatchTetSpecConcsNP: molar concentrations of s in tets[i]."""
        idx = np.ascontiguousarray(tets, dtype=np.int64)
        c = np.empty(len(idx), dtype=np.float64)
        self.getBatchTetSpecCountsNP(idx, s, c)
        concs[:] = c / (AVOGADRO * self.geom.tet_vol[idx] * 1.0e3)

    def getBatchTetSpecCounts(self, tets, s):
        out = np.empty(len(tets), dtype=np.float64)
        self.getBatchTetSpecCountsNP(tets, s, out)
        return list(out)

    # ------------------------------------------------------------- constants
    # ------------------------------------------------- diffusion boundaries
    def _db(self, db):
        try:
            return self.diffbound_index[db]
        except KeyError:
            raise ArgErr(f"unknown diffusion boundary '{db}'") from None

    def setDiffBoundarySpecDiffusionActive(self, db, s, act):
        """Open (or close) diffusion of s across the boundary in both directions at each
        side's own constant (TOS:2745-2800)."""
        check(self._L.sg_set_diff_boundary_active(self._h, self._db(db), self._spec(s), 1 if act else 0))

    def getDiffBoundarySpecDiffusionActive(self, db, s):
        x = C.c_int32()
        check(self._L.sg_get_diff_boundary_active(self._h, self._db(db), self._spec(s), C.byref(x)))
        return bool(x.value)

    def setDiffBoundarySpecDcst(self, db, s, dcst, direction_comp=None):
        """Diffusion constant across the boundary (TOS:2865-2930); with direction_comp only
        the diffusion into that compartment takes it.  Opens the direction(s)."""
        dc = -1 if direction_comp is None else self.comp_index[direction_comp]
        check(self._L.sg_set_diff_boundary_dcst(self._h, self._db(db), self._spec(s), float(dcst), dc))

    setDiffBoundaryDiffusionActive = setDiffBoundarySpecDiffusionActive
    getDiffBoundaryDiffusionActive = getDiffBoundarySpecDiffusionActive
    setDiffBoundaryDcst = setDiffBoundarySpecDcst

    def setCompReacK(self, c, r, k, realization=-1):
        check(self._L.sg_set_reac_k(self._h, self._reac(c, r), int(realization), float(k)))

    def getCompReacK(self, c, r, realization=0):
        k = C.c_double()
        check(self._L.sg_get_reac_k(self._h, self._reac(c, r), int(realization), C.byref(k)))
        return k.value

    def setCompDiffD(self, c, d, dcst, realization=-1):
        try:
            s = self.diff_index[(c, d)]
        except KeyError:
            raise ArgErr(f"diffusion '{d}' undefined in compartment '{c}'") from None
        check(self._L.sg_set_diff_d(self._h, self._comp(c), s, int(realization), float(dcst)))

    # ------------------------------------------------------ triangles / patches
    def _tri(self, tidx):
        try:
            return self.surf["tri_index"][int(tidx)]
        except (TypeError, KeyError):
            raise ArgErr(f"triangle {tidx} is not in a patch") from None

    def _sspec(self, name):
        try:
            return self.surf["sspec_index"][name]
        except (TypeError, KeyError):
            raise ArgErr(f"unknown surface species '{name}'") from None

    def _patch(self, name):
        try:
            return self.surf["patch_names"].index(name)
        except (TypeError, ValueError):
            raise ArgErr(f"unknown patch '{name}'") from None

    def getTriSpecCount(self, tidx, s):
        n = C.c_double()
        check(self._L.sg_get_tri_count(self._h, self._tri(tidx), self._sspec(s), C.byref(n)))
        return n.value

    def setTriSpecCount(self, tidx, s, n):
        check(self._L.sg_set_tri_count(self._h, self._tri(tidx), self._sspec(s), float(n)))

    def getPatchSpecCount(self, p, s, realization=-1):
        n = C.c_double()
        check(self._L.sg_get_patch_count(self._h, self._patch(p), self._sspec(s), int(realization), C.byref(n)))
        return n.value

    def setPatchSpecCount(self, p, s, n, realization=-1):
        """Distribute n molecules over the patch's triangles by area (of one realization, or
        of all with realization=-1)."""
        check(self._L.sg_set_patch_count(self._h, self._patch(p), self._sspec(s), int(realization), float(n)))

    def getTriGHKI(self, tidx, ghk=None):
        """GHK current (A, outward positive) of the triangle over the last EField step."""
        x = C.c_double()
        check(self._L.sg_get_tri_ghk_i(self._h, self._tri(tidx), C.byref(x)))
        return x.value

    def setTemp(self, kelvin):
        check(self._L.sg_set_temp(self._h, float(kelvin)))

    def getTemp(self):
        x = C.c_double()
        check(self._L.sg_get_temp(self._h, C.byref(x)))
        return x.value

    def getTriOhmicI(self, tidx, oc=None):
        x = C.c_double()
        check(self._L.sg_get_tri_ohmic_i(self._h, self._tri(tidx), C.byref(x)))
        return x.value

    getTriCount = getTriSpecCount
    setTriCount = setTriSpecCount
    getPatchCount = getPatchSpecCount
    setPatchCount = setPatchSpecCount

    # ------------------------------------------------ membrane potential (EField)
    def setEfieldDT(self, dt):
        check(self._L.sg_set_efield_dt(self._h, float(dt)))

    def getEfieldDT(self):
        x = C.c_double()
        check(self._L.sg_get_efield_dt(self._h, C.byref(x)))
        return x.value

    def setEfieldTolerance(self, rel_tol, inner_rel_tol=1e-4, max_iter=20000):
        check(self._L.sg_set_efield_tolerance(self._h, float(rel_tol), float(inner_rel_tol), int(max_iter)))

    def setMembPotential(self, memb, v):
        check(self._L.sg_set_memb_potential(self._h, float(v)))

    def setMembCapac(self, memb, cm):
        check(self._L.sg_set_memb_capac(self._h, float(cm)))

    def setMembVolRes(self, memb, ra):
        check(self._L.sg_set_memb_vol_res(self._h, float(ra)))

    def setMembRes(self, memb, ro, vrev):
        check(self._L.sg_set_memb_res(self._h, float(ro), float(vrev)))

    def getVertV(self, vidx):
        x = C.c_double()
        check(self._L.sg_get_vert_v(self._h, int(vidx), C.byref(x)))
        return x.value

    def setVertV(self, vidx, v):
        check(self._L.sg_set_vert_v(self._h, int(vidx), float(v)))

    def setVertVClamped(self, vidx, cl):
        check(self._L.sg_set_vert_v_clamped(self._h, int(vidx), 1 if cl else 0))

    def setVertIClamp(self, vidx, cur):
        check(self._L.sg_set_vert_iclamp(self._h, int(vidx), float(cur)))

    def getTriV(self, tidx):
        try:
            m = self.memb_index[int(tidx)]
        except (AttributeError, KeyError):
            raise ArgErr(f"triangle {tidx} is not on the membrane") from None
        x = C.c_double()
        check(self._L.sg_get_tri_v(self._h, m, C.byref(x)))
        return x.value

    def getEfieldStats(self):
        """(EField steps, CG iterations, device ms in the solves, last relative residual)."""
        s, it, ms, rr = C.c_uint64(), C.c_uint64(), C.c_double(), C.c_double()
        check(self._L.sg_get_efield_stats(self._h, C.byref(s), C.byref(it), C.byref(ms), C.byref(rr)))
        return s.value, it.value, ms.value, rr.value

    def setEfieldCheck(self, on, rel_tol=1e-12):
        """EField (either method): after every step also solve the same system in FP64 to
        rel_tol (not timed) and record the largest per-vertex relative voltage difference."""
        check(self._L.sg_set_efield_check(self._h, 1 if on else 0, float(rel_tol)))

    def setEfieldPersistent(self, on):
        """Run each EField solve as one cooperative launch (True) or as three kernel
        launches per CG iteration (False)."""
        check(self._L.sg_set_efield_persistent(self._h, 1 if on else 0))

    def setEfieldBarrierLimit(self, polls):
        """Polls (about 100 ns each) of a grid-barrier wait after which the persistent EField
        solve gives up and the step raises DeviceError; default 2**22 (about 0.5 s)."""
        check(self._L.sg_set_efield_barrier_limit(self._h, int(polls)))

    def setEfieldReliableUpdates(self, on, delta=0.1):
        """Mixed method, persistent solve: one FP32 CG whose residual is replaced by the
        FP64 one whenever it has fallen by `delta` (True, default), or restarted FP32
        inner solves inside an FP64 refinement loop (False)."""
        check(self._L.sg_set_efield_reliable_updates(self._h, 1 if on else 0, float(delta)))

    def getEfieldCheck(self):
        """(checked steps, max over steps of max_v |V_mixed - V_fp64| / |V_fp64|, last step's)."""
        s, mx, last = C.c_uint64(), C.c_double(), C.c_double()
        check(self._L.sg_get_efield_check(self._h, C.byref(s), C.byref(mx), C.byref(last)))
        return s.value, mx.value, last.value

    # --------------------------------------------------------- device knobs
    def setLaunch(self, block, grid=0):
        check(self._L.sg_set_launch(self._h, int(block), int(grid)))

    def setSplit(self, on):
        """Run each window as two kernels (reactions per tet, diffusion per (species, tet));
        results are identical to the fused kernel."""
        check(self._L.sg_set_split(self._h, 1 if on else 0))

    def getSplit(self):
        x = C.c_int32()
        check(self._L.sg_get_split(self._h, C.byref(x)))
        return bool(x.value)

    def setPersistent(self, on, tets_per_lane=1):
        """Run the windows of every realization in one persistent launch per run() call (up
        to 64 windows each), warps taking chunks of 32 * tets_per_lane tets (1, 2, 4 or 8 per
        lane); the same results as the window launches.  Only for models without membrane triangles whose
        realizations take the same windows (otherwise the window launches run)."""
        check(self._L.sg_set_persistent(self._h, 1 if on else 0, int(tets_per_lane)))

    def getPersistent(self):
        on, tpl = C.c_int32(), C.c_int32()
        check(self._L.sg_get_persistent(self._h, C.byref(on), C.byref(tpl)))
        return bool(on.value), tpl.value

    def setWindowWaitLimit(self, polls):
        """Polls a persistent launch's wait on a realization makes before it gives up (and
        run() fails)."""
        check(self._L.sg_set_window_wait_limit(self._h, int(polls)))

    def getCarveout(self):
        """Preferred shared-memory carveout (percent) of the window kernels."""
        x = C.c_int32()
        check(self._L.sg_get_carveout(self._h, C.byref(x)))
        return x.value

    def getLaunch(self):
        """(block, grid) of the window kernel; grid 0 = occupancy-sized, -1 = one tet per
        thread."""
        b, g = C.c_int32(), C.c_int32()
        check(self._L.sg_get_launch(self._h, C.byref(b), C.byref(g)))
        return b.value, g.value

    def setAutotune(self, on=True):
        """Time 20 windows of the next run (after one untimed window) under ten launch
        shapes, two windows each in a palindromic order, and keep the fastest (results do
        not depend on the shape)."""
        check(self._L.sg_set_autotune(self._h, 1 if on else 0))

    def getAutotuneTimes(self):
        """ms of the two timed windows of each candidate: block 64, 128, 256 x grid
        {occupancy-sized, one tet per thread}; block 256 one tet per thread at carveouts 75%
        and 50%; split at block 128 and 256; empty before tuning."""
        buf = (C.c_float * 16)()
        n = C.c_int32()
        check(self._L.sg_get_autotune_ms(self._h, buf, 16, C.byref(n)))
        return list(buf)[: n.value]

    def setConservationCheck(self, on):
        check(self._L.sg_set_conservation_check(self._h, 1 if on else 0))

    def setGraphs(self, on):
        check(self._L.sg_set_graphs(self._h, 1 if on else 0))

    def getStream(self):
        """The cudaStream_t (as an int) all kernels of this solver run on."""
        p = C.c_void_p()
        check(self._L.sg_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def setProfiling(self, on):
        check(self._L.sg_set_profiling(self._h, 1 if on else 0))

    def getProfile(self):
        """(device ms in window launches, windows timed, kernels launched since creation)."""
        ms, w, n = C.c_double(), C.c_uint64(), C.c_uint64()
        check(self._L.sg_get_profile(self._h, C.byref(ms), C.byref(w), C.byref(n)))
        return ms.value, w.value, n.value

    def getStatus(self):
        s = C.c_uint32()
        check(self._L.sg_get_status(self._h, C.byref(s)))
        return s.value

    # ----------------------------------------------------------- API_1 names
    getTetCount = getTetSpecCount
    setTetCount = setTetSpecCount
    getCompCount = getCompSpecCount
    setCompCount = setCompSpecCount
    getTetConc = getTetSpecConc
    setTetConc = setTetSpecConc
    getCompConc = getCompSpecConc
    setCompConc = setCompSpecConc
    setTetClamped = setTetSpecClamped
