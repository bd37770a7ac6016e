"""Batched realizations with membrane triangles and EField: realizations are disjoint
copies of one mesh (geom.replicate); their vertex systems are independent blocks of one
solve, surface counts can be set per realization, and a realization behaves like a
single-realization solver of the same mesh."""
import math

import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import EF_DV_CG_FP64, EF_DV_CG_MIXED, TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu


def passive(mesh, method, realizations=None):
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(21), method, realizations=realizations)
    sim.setEfieldTolerance(1e-12, 1e-5)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    return sim


@pytest.mark.parametrize("method", [EF_DV_CG_FP64, EF_DV_CG_MIXED])
def test_realization_blocks_are_independent(steps_lib, method):
    base = sgeom.kuhn_box(3, 3, 6, W.H)
    zmin = [v for v in range(base.nverts) if base.verts[v, 2] <= 1e-12]
    single = passive(sgeom.kuhn_box(3, 3, 6, W.H), method)
    for v in zmin:
        single.setVertIClamp(v, 2e-12)
    rep = sgeom.replicate(base, 3)
    batched = passive(rep, method, realizations=rep.offsets)
    for v in zmin:
        batched.setVertIClamp(base.nverts + v, 2e-12)  # realization 1 only
    single.run(20e-6)
    batched.run(20e-6)
    vs = np.array([single.getVertV(v) for v in range(base.nverts)])
    vb = np.array([batched.getVertV(v) for v in range(rep.nverts)]).reshape(3, base.nverts)
    assert np.max(np.abs(vb[1] - vs) / np.abs(vs)) < 1e-8
    assert np.max(np.abs(vb[0] + 0.065)) < 1e-12 and np.max(np.abs(vb[2] + 0.065)) < 1e-12
    assert np.ptp(vs) > 1e-6


def test_patch_counts_per_realization_and_channels(steps_lib):
    base = sgeom.kuhn_box(3, 3, 6, W.H)
    rep = sgeom.replicate(base, 3)
    cyto = sgeom.TmComp("cyto", rep, np.arange(rep.ntets))
    cyto.addVolsys("vsys")
    patch = sgeom.TmPatch("memb", rep, rep.getSurfTris(), cyto)
    patch.addSurfsys("ssys")
    sgeom.Memb("membrane", rep, [patch])
    mdl = smodel.Model()
    ca = smodel.Spec("Ca", mdl)
    smodel.Volsys("vsys", mdl)
    ss = smodel.Surfsys("ssys", mdl)
    ch = smodel.Chan("K", mdl)
    c, o = smodel.ChanState("Kc", mdl, ch), smodel.ChanState("Ko", mdl, ch)
    smodel.VDepSReac("open", ss, slhs=[c], srhs=[o], k=lambda v: 2000.0 * math.exp(v / 0.025))
    smodel.VDepSReac("close", ss, slhs=[o], srhs=[c], k=lambda v: 2000.0 * math.exp(-v / 0.025))
    smodel.SReac("emit", ss, slhs=[o], srhs=[o], irhs=[ca], kcst=3000.0)
    smodel.OhmicCurr("I_K", ss, chanstate=o, g=20e-12, erev=0.05)
    sim = TetOpSplit(mdl, rep, make_rng(22), EF_DV_CG_MIXED, realizations=rep.offsets)
    sim.setEfieldDT(2e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    sim.setPatchSpecCount("memb", "Kc", 500, realization=1)
    assert sim.getPatchSpecCount("memb", "Kc", 1) == 500
    assert sim.getPatchSpecCount("memb", "Kc", 0) == 0 and sim.getPatchSpecCount("memb", "Kc", 2) == 0
    assert sim.getPatchSpecCount("memb", "Kc") == 500
    sim.run(200e-6)
    assert sim.getPatchSpecCount("memb", "Kc", 1) + sim.getPatchSpecCount("memb", "Ko", 1) == 500
    assert sim.getPatchSpecCount("memb", "Ko", 0) == 0
    assert sim.getPatchSpecCount("memb", "Ko", 1) > 0
    assert sim.getCompSpecCount("cyto", "Ca", 1) > 0
    assert sim.getCompSpecCount("cyto", "Ca", 0) == 0 and sim.getCompSpecCount("cyto", "Ca", 2) == 0


@pytest.mark.parametrize("batched", [False, True])
def test_split_window_equals_fused_with_membrane(steps_lib, batched):
    """Membrane models run the split window by default (volume SSA for the other tets,
    SURF SSA over the membrane tet list, diffusion leave per species); the fused SURF
    kernel gives bit-identical counts, channel states and potentials."""
    def build(split):
        base = sgeom.kuhn_box(4, 4, 6, W.H)
        mesh = sgeom.replicate(base, 2) if batched else base
        cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
        cyto.addVolsys("vsys")
        patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), cyto)
        patch.addSurfsys("ssys")
        sgeom.Memb("membrane", mesh, [patch])
        mdl = smodel.Model()
        ca, cb, cacb = smodel.Spec("Ca", mdl), smodel.Spec("CB", mdl), smodel.Spec("CaCB", mdl)
        vs = smodel.Volsys("vsys", mdl)
        smodel.Reac("bind", vs, lhs=[ca, cb], rhs=[cacb], kcst=1e8)
        smodel.Reac("unbind", vs, lhs=[cacb], rhs=[ca, cb], kcst=100.0)
        smodel.Diff("dCa", vs, ca, 2.2e-10)
        smodel.Diff("dCB", vs, cb, 2e-11)
        ss = smodel.Surfsys("ssys", mdl)
        ch = smodel.Chan("CaCh", mdl)
        c, o = smodel.ChanState("C", mdl, ch), smodel.ChanState("O", mdl, ch)
        smodel.VDepSReac("open", ss, slhs=[c], srhs=[o], k=lambda v: 3000.0 * math.exp(v / 0.025))
        smodel.VDepSReac("close", ss, slhs=[o], srhs=[c], k=lambda v: 3000.0 * math.exp(-v / 0.025))
        smodel.SReac("flux", ss, slhs=[o], srhs=[o], irhs=[ca], kcst=2e6)
        smodel.OhmicCurr("I", ss, chanstate=o, g=20e-12, erev=0.05)
        sim = TetOpSplit(mdl, mesh, make_rng(31), EF_DV_CG_FP64,
                         realizations=mesh.offsets if batched else None)
        sim.setSplit(split)
        sim.setEfieldDT(2e-6)
        sim.setMembPotential("membrane", -0.065)
        sim.setMembCapac("membrane", 0.01)
        sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
        sim.setCompSpecConc("cyto", "CB", 50e-6)
        # 50 channels of 20 pS: the explicit channel current stays stable at dt = 2 us
        # (membrane time constant C / g ~ 13 us on this 1.28 um^2 box).  Five start open,
        # so Ca is emitted on every sample path (at -65 mV a closed channel opens about
        # once per 4.5 ms, so from all-closed no channel may open in 100 us).
        sim.setPatchSpecCount("memb", "C", 45)
        sim.setPatchSpecCount("memb", "O", 5)
        sim.setVertIClamp(0, 5e-12)
        return mesh, patch, sim

    mesh, patch, fused = build(False)
    _, _, split = build(True)
    assert split.getSplit() and not fused.getSplit()
    for k in range(1, 6):
        fused.run(k * 20e-6)
        split.run(k * 20e-6)
        for s in ("Ca", "CB", "CaCB"):
            assert np.array_equal(fused.getSpecCounts(s), split.getSpecCounts(s)), (k, s)
        for s in ("C", "O"):
            assert fused.getPatchSpecCount("memb", s) == split.getPatchSpecCount("memb", s), (k, s)
    vf = np.array([fused.getVertV(v) for v in range(mesh.nverts)])
    vsp = np.array([split.getVertV(v) for v in range(mesh.nverts)])
    assert np.array_equal(vf, vsp)
    assert fused.getCompSpecCount("cyto", "Ca") > 0
