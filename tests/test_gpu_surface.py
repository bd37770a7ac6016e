"""Surface reactions on membrane triangles (SReac, VDepSReac, OhmicCurr) on the GPU.

Statistical checks against closed forms: a two-state channel relaxes to kf/(kf+kb) open,
a voltage-gated one to alpha(V)/(alpha(V)+beta(V)) at a clamped potential, the ohmic
current is g * n_open * (V - E), and emission into the inner tet follows k * n * t.
"""
import math

import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import EF_DV_CG_FP64, TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu


def membrane_box(n=4, nz=6):
    mesh = sgeom.kuhn_box(n, n, nz, W.H)
    cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    cyto.addVolsys("vsys")
    patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), cyto)
    patch.addSurfsys("ssys")
    return mesh, patch


def channel_model(kf, kb, vdep=False, emit=0.0):
    mdl = smodel.Model()
    ca = smodel.Spec("Ca", mdl)
    ch = smodel.Chan("K", mdl)
    c = smodel.ChanState("Kc", mdl, ch)
    o = smodel.ChanState("Ko", mdl, ch)
    smodel.Volsys("vsys", mdl)
    ss = smodel.Surfsys("ssys", mdl)
    if vdep:
        smodel.VDepSReac("open", ss, slhs=[c], srhs=[o], k=kf)
        smodel.VDepSReac("close", ss, slhs=[o], srhs=[c], k=kb)
    else:
        smodel.SReac("open", ss, slhs=[c], srhs=[o], kcst=kf)
        smodel.SReac("close", ss, slhs=[o], srhs=[c], kcst=kb)
    if emit > 0.0:
        smodel.SReac("emit", ss, slhs=[o], srhs=[o], irhs=[ca], kcst=emit)
    smodel.OhmicCurr("I_K", ss, chanstate=o, g=20e-12, erev=0.05)
    return mdl


def test_two_state_channel_equilibrium(steps_lib):
    mesh, patch = membrane_box()
    sim = TetOpSplit(channel_model(300.0, 100.0), mesh, make_rng(5))
    N = 50 * len(patch.tris)
    sim.setPatchSpecCount("memb", "Kc", N)
    assert sim.getPatchSpecCount("memb", "Kc") == N
    opens = []
    for k in range(1, 41):
        sim.run(0.01 + k * 0.005)
        opens.append(sim.getPatchSpecCount("memb", "Ko"))
        assert sim.getPatchSpecCount("memb", "Kc") + opens[-1] == N
    p = 300.0 / 400.0
    mean = np.mean(opens)
    sd = math.sqrt(N * p * (1 - p))
    assert abs(mean - N * p) < 5 * sd / math.sqrt(len(opens)) + 1e-9 + 2 * sd / 10


def test_vdep_channel_at_clamped_potential(steps_lib):
    mesh, patch = membrane_box()
    alpha = lambda v: 100.0 * math.exp(v / 0.025)   # /s, V in volts
    beta = lambda v: 100.0 * math.exp(-v / 0.025)
    sgeom.Memb("membrane", mesh, [patch])
    sim = TetOpSplit(channel_model(alpha, beta, vdep=True), mesh, make_rng(6), EF_DV_CG_FP64)
    v0 = -0.020
    sim.setMembPotential("membrane", v0)
    for v in range(mesh.nverts):
        sim.setVertVClamped(v, True)
    sim.setEfieldDT(1e-4)
    N = 40 * len(patch.tris)
    sim.setPatchSpecCount("memb", "Kc", N)
    opens = []
    for k in range(1, 31):
        sim.run(0.02 + k * 0.004)
        opens.append(sim.getPatchSpecCount("memb", "Ko"))
    p = alpha(v0) / (alpha(v0) + beta(v0))
    assert abs(np.mean(opens) / N - p) < 0.02, (np.mean(opens) / N, p)
    assert abs(sim.getTriV(int(patch.tris[0])) - v0) < 1e-12


def test_ohmic_current_of_open_channels(steps_lib):
    mesh, patch = membrane_box()
    sgeom.Memb("membrane", mesh, [patch])
    sim = TetOpSplit(channel_model(0.0, 0.0), mesh, make_rng(7), EF_DV_CG_FP64)
    v0 = -0.030
    sim.setMembPotential("membrane", v0)
    for v in range(mesh.nverts):
        sim.setVertVClamped(v, True)
    t0 = int(patch.tris[3])
    sim.setTriSpecCount(t0, "Ko", 7)
    sim.setEfieldDT(1e-5)
    sim.run(3e-5)
    assert sim.getTriSpecCount(t0, "Ko") == 7
    assert math.isclose(sim.getTriOhmicI(t0), 7 * 20e-12 * (v0 - 0.05), rel_tol=1e-9)
    assert sim.getTriOhmicI(int(patch.tris[4])) == 0.0


def test_emission_into_inner_tet(steps_lib):
    mesh, patch = membrane_box()
    sim = TetOpSplit(channel_model(0.0, 0.0, emit=50.0), mesh, make_rng(8))
    for t in patch.tris:
        sim.setTriSpecCount(int(t), "Ko", 2)
    T = 0.2
    sim.run(T)
    total = sim.getCompSpecCount("cyto", "Ca")
    lam = 50.0 * 2 * len(patch.tris) * T
    assert abs(total - lam) < 5 * math.sqrt(lam)
