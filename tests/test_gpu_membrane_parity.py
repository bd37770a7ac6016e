"""Membrane chemistry on the GPU against the CPU oracle, bit for bit.

The oracle (oracle/opsplit_oracle.c) restates the SSA unit of a tet and its membrane
triangles (sreac.cpp:305-520 propensities and applies with surface and inner-volume
terms, vdepsreac.cpp / vdepsreacdef.cpp:194-218 k(V) tables, ghkcurr.cpp:168-280 GHK
events with ion flux, tri.cpp:486-561 surface occupancy) and surface diffusion
(sdiff.cpp:438-560, TOS:1716-1793) on the same Philox streams.  Without an EField every
triangle sits at 0 mV on both sides, so every count of every tet and triangle must agree
after every run().  With surface diffusion the solver runs the split window kernels, without
it the fused membrane kernel.
"""
import math

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu


def membrane_model(sdiff):
    mdl = smodel.Model()
    a = smodel.Spec("A", mdl)
    ca = smodel.Spec("Ca", mdl, valence=2)
    rc = smodel.Spec("R", mdl)
    ar = smodel.Spec("AR", mdl)
    vs = smodel.Volsys("vsys", mdl)
    smodel.Diff("dA", vs, a, 1.0e-12)
    smodel.Diff("dCa", vs, ca, 5.0e-13)
    smodel.Reac("deg", vs, lhs=[ca], rhs=[], kcst=3.0)
    ss = smodel.Surfsys("ssys", mdl)
    ch = smodel.Chan("K", mdl)
    kc = smodel.ChanState("Kc", mdl, ch)
    ko = smodel.ChanState("Ko", mdl, ch)
    vr = (-0.1, 0.05, 1e-4)
    smodel.VDepSReac("open", ss, slhs=[kc], srhs=[ko], k=lambda v: 200.0 * math.exp(v / 0.025), vrange=vr)
    smodel.VDepSReac("close", ss, slhs=[ko], srhs=[kc], k=lambda v: 150.0 * math.exp(-v / 0.025), vrange=vr)
    smodel.SReac("bind", ss, ilhs=[a], slhs=[rc], srhs=[ar], kcst=2.0e8)
    smodel.SReac("unbind", ss, slhs=[ar], srhs=[rc], irhs=[a], kcst=20.0)
    smodel.SReac("emit", ss, slhs=[ko], srhs=[ko], irhs=[ca], kcst=30.0)
    smodel.SReac("flip", ss, slhs=[rc, rc], srhs=[ar, rc], kcst=1.0e-3)
    g = smodel.GHKcurr("ICa", ss, ko, ca, computeflux=True, virtual_oconc=2e-3)
    g.setPInfo(g=20e-12, V=-0.065, T=293.15, oconc=2e-3, iconc=1e-4)
    if sdiff:
        smodel.Diff("dR", ss, rc, 2.0e-13)
    return mdl


def build(sdiff, seed):
    mesh = sgeom.kuhn_box(4, 4, 4, W.H)
    cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    cyto.addVolsys("vsys")
    patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), cyto)
    patch.addSurfsys("ssys")
    mdl = membrane_model(sdiff)
    sim = TetOpSplit(mdl, mesh, make_rng(seed))
    sim.setCompSpecCount("cyto", "A", 3000)
    sim.setCompSpecCount("cyto", "Ca", 800)
    sim.setPatchSpecCount("memb", "R", 1500)
    sim.setPatchSpecCount("memb", "Kc", 400)
    ora = Oracle(sim.tables, seed=seed)
    return mesh, sim, ora


def sync(sim, ora):
    for i, s in enumerate(sim.spec_names):
        ora.set_counts(i, sim.getSpecCounts(s))
    sf = sim.tables["surf"]
    for k, name in enumerate(sf["sspec_names"]):
        ora.set_tri_counts(k, np.array([sim.getTriSpecCount(int(t), name) for t in sf["tris"]], dtype=np.uint32))


def check(sim, ora, where):
    for i, s in enumerate(sim.spec_names):
        g, o = sim.getSpecCounts(s), ora.get_counts(i)
        assert np.array_equal(g, o), f"{where}: volume species {s} differs in {int(np.sum(g != o))} tets"
    sf = sim.tables["surf"]
    for k, name in enumerate(sf["sspec_names"]):
        g = np.array([sim.getTriSpecCount(int(t), name) for t in sf["tris"]], dtype=np.uint32)
        o = ora.get_tri_counts(k)
        assert np.array_equal(g, o), f"{where}: surface species {name} differs in {int(np.sum(g != o))} triangles"


@pytest.mark.parametrize("sdiff", [False, True])
def test_membrane_chemistry_matches_oracle(steps_lib, sdiff):
    mesh, sim, ora = build(sdiff, seed=29)
    sync(sim, ora)
    assert sim.getUpdPeriod() == ora.period()
    sf = sim.tables["surf"]
    ca = sim.spec_names.index("Ca")
    ca0 = int(sim.getSpecCounts("Ca").sum())
    for k in range(1, 7):
        t = k * 0.5e-3
        sim.run(t)
        ora.run(t)
        check(sim, ora, f"t={t} sdiff={sdiff}")
    assert sim.getNIteration() == ora.window()
    # Every reaction class fired, and the channels stayed a closed system.
    kc = sf["sspec_names"].index("Kc")
    ko = sf["sspec_names"].index("Ko")
    assert int(ora.get_tri_counts(kc).sum() + ora.get_tri_counts(ko).sum()) == 400
    assert ora.get_tri_counts(ko).sum() > 0
    assert ora.surf_extent() > 0
    assert int(ora.get_counts(ca).sum()) != ca0
    if sdiff:
        assert ora.diff_extent() > 0


def test_membrane_split_and_fused_kernels_agree(steps_lib):
    """Without surface diffusion the membrane model may run fused or split; both give the
    same counts (each unit draws from its own streams)."""
    _, a, ora = build(False, seed=31)
    _, b, _ = build(False, seed=31)
    b.setSplit(True)
    for k in range(1, 5):
        t = k * 0.5e-3
        a.run(t)
        b.run(t)
        for s in a.spec_names:
            assert np.array_equal(a.getSpecCounts(s), b.getSpecCounts(s)), (t, s)
