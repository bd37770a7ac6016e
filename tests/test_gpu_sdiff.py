"""Surface diffusion (SDiff, the reference's sdiff.cpp and TOS:1716-1793) on the GPU.

Molecules released on one triangle of a planar patch spread with mean squared displacement
4 D t; they stay on their patch, the patch total is conserved, and the update period
follows the fastest surface rule (TOS:5373-5411 takes the max over volume and surface).
"""
import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu


def planar(n, D, two_patches=False):
    mesh = sgeom.kuhn_box(n, n, 1, W.H)
    cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    cyto.addVolsys("vsys")
    surf = mesh.getSurfTris()
    bot = np.array([t for t in surf if np.all(mesh.verts[mesh.tris[t]][:, 2] <= 1e-12)])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    ss = smodel.Surfsys("ssys", mdl)
    x = smodel.Spec("X", mdl)
    smodel.SReac("idle", ss, slhs=[x], srhs=[x], kcst=0.0)
    smodel.Diff("dX", ss, x, D)
    if two_patches:
        cx = mesh.tri_bary[bot, 0]
        left, right = bot[cx < 0.5 * n * W.H], bot[cx >= 0.5 * n * W.H]
        pl = sgeom.TmPatch("left", mesh, left, cyto)
        pr = sgeom.TmPatch("right", mesh, right, cyto)
        pl.addSurfsys("ssys")
        pr.addSurfsys("ssys")
        return mesh, mdl, (pl, pr)
    p = sgeom.TmPatch("memb", mesh, bot, cyto)
    p.addSurfsys("ssys")
    return mesh, mdl, (p,)


def test_msd_grows_as_4dt(steps_lib):
    D = 1e-12
    mesh, mdl, (patch,) = planar(40, D)
    sim = TetOpSplit(mdl, mesh, make_rng(41))
    c = np.array([0.5 * 40 * W.H, 0.5 * 40 * W.H])
    d2 = np.sum((mesh.tri_bary[patch.tris, :2] - c) ** 2, axis=1)
    t0 = int(patch.tris[np.argmin(d2)])
    N = 20000
    sim.setTriSpecCount(t0, "X", N)
    per = sim.getUpdPeriod()
    assert 0.0 < per < 1e-2
    x0 = mesh.tri_bary[t0, :2]
    for t in (0.02, 0.05):
        sim.run(t)
        n = np.array([sim.getTriSpecCount(int(m), "X") for m in patch.tris])
        assert n.sum() == N
        r = mesh.tri_bary[patch.tris, :2] - x0
        msd = float(np.sum(n * np.sum(r * r, axis=1)) / N)
        assert abs(msd / (4 * D * t) - 1.0) < 0.15, (t, msd, 4 * D * t)
        vx = float(np.sum(n * r[:, 0] ** 2) / N)
        vy = float(np.sum(n * r[:, 1] ** 2) / N)
        assert abs(vx / vy - 1.0) < 0.15
    assert sim.getDiffExtent() > 0


def test_confined_to_its_patch(steps_lib):
    mesh, mdl, (pl, pr) = planar(12, 2e-12, two_patches=True)
    sim = TetOpSplit(mdl, mesh, make_rng(42))
    sim.setPatchSpecCount("left", "X", 3000)
    sim.run(0.02)
    assert sim.getPatchSpecCount("left", "X") == 3000
    assert sim.getPatchSpecCount("right", "X") == 0
    n = np.array([sim.getTriSpecCount(int(m), "X") for m in pl.tris])
    assert (n > 0).sum() > 0.8 * len(pl.tris)  # spread over the patch
