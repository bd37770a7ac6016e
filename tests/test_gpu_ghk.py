"""GHK currents (ghkcurr.cpp:168-280, math/ghk.cpp:71-90) on the GPU: at a clamped
potential with a fixed channel count the mean triangle current equals n times the GHK
single-channel current; with computeflux every elementary charge moved is an ion leaving
or entering the inner tets."""
import math

import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import EF_DV_CG_FP64, TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu

F, R, E = 96485.3399, 8.314472, 1.602176487e-19


def ghk_i(P, v, z, T, ci, co):
    nu = z * v * F / (R * T)
    return P * z * F * nu * (ci - co * math.exp(-nu)) / (1.0 - math.exp(-nu))


def build(flux):
    mesh = sgeom.kuhn_box(4, 4, 4, W.H)
    cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    cyto.addVolsys("vsys")
    patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), cyto)
    patch.addSurfsys("ssys")
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    ca = smodel.Spec("Ca", mdl, valence=2)
    smodel.Volsys("vsys", mdl)
    ss = smodel.Surfsys("ssys", mdl)
    ch = smodel.Chan("CaCh", mdl)
    o = smodel.ChanState("O", mdl, ch)
    g = smodel.GHKcurr("ICa", ss, o, ca, computeflux=flux, virtual_oconc=2e-3)
    g.setPInfo(g=20e-12, V=-0.065, T=293.15, oconc=2e-3, iconc=1e-4)
    sim = TetOpSplit(mdl, mesh, make_rng(51), EF_DV_CG_FP64)
    sim.setEfieldDT(1e-5)
    sim.setMembPotential("membrane", -0.03)
    for v in range(mesh.nverts):
        sim.setVertVClamped(v, True)
    return mesh, patch, sim, g


def test_mean_current_matches_ghk_equation(steps_lib):
    mesh, patch, sim, g = build(flux=True)
    c0 = 5
    for t in range(mesh.ntets):
        sim.setTetSpecCount(t, "Ca", c0)
        sim.setTetSpecClamped(t, "Ca", True)
    for m in patch.tris:
        sim.setTriSpecCount(int(m), "O", 2)
    vol = mesh.tet_vol[0]
    ci = c0 / (6.02214179e23 * vol * 1e3) * 1e3
    i1 = ghk_i(g.getP(), -0.03, 2, 293.15, ci, 2e-3 * 1e3)
    expect = 2 * len(patch.tris) * i1
    tot = []
    for k in range(1, 41):
        sim.run(k * 1e-5)
        tot.append(sum(sim.getTriGHKI(int(m)) for m in patch.tris))
    mean = float(np.mean(tot))
    ions_per_step = abs(expect) * 1e-5 / (2 * E)
    sd = abs(expect) / math.sqrt(ions_per_step * len(tot))
    assert abs(mean - expect) < 5 * sd + 1e-6 * abs(expect), (mean, expect, sd)
    assert sim.getCompSpecCount("cyto", "Ca") == c0 * mesh.ntets  # clamped


def test_flux_moves_the_ions(steps_lib):
    mesh, patch, sim, g = build(flux=True)
    for m in patch.tris:
        sim.setTriSpecCount(int(m), "O", 3)
    before = sim.getCompSpecCount("cyto", "Ca")
    charge = 0.0
    for k in range(1, 21):
        sim.run(k * 1e-5)
        charge += sum(sim.getTriGHKI(int(m)) for m in patch.tris) * 1e-5 / E
    after = sim.getCompSpecCount("cyto", "Ca")
    assert after > before  # influx at -30 mV with 2 mM outside
    assert round(charge) == -2 * (after - before)
