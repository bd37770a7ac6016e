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
