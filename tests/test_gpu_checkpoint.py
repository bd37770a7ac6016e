"""checkpoint/restore (the reference's API::checkpoint / restore, TOS:217-451): a solver
restored from a checkpoint continues bit-identically to the uninterrupted run, for the
plain, batched and membrane (EField) forms; a checkpoint of another mesh is refused."""
import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200._lib import ArgErr
from steps_b200.solver import EF_DV_CG_FP64, TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu


def counts(sim):
    return np.stack([sim.getSpecCounts(s) for s in sim.spec_names])


def test_plain_resume_is_exact(steps_lib, tmp_path):
    mesh = W.cube_mesh(8)
    mdl = W.random_network(2)
    a = TetOpSplit(mdl, mesh, make_rng(9))
    rows = W.poisson_counts(mesh.ntets, 40.0, 9, nspec=8)
    for i, s in enumerate(a.spec_names):
        a.setSpecCounts(s, rows[i])
    a.setTetSpecClamped(5, a.spec_names[1], True)
    a.run(1.0e-3)
    f = str(tmp_path / "plain.ckpt")
    a.checkpoint(f)
    a.run(3.0e-3)
    ref = counts(a)
    b = TetOpSplit(mdl, mesh, make_rng(9))
    b.restore(f)
    assert b.getTime() == 1.0e-3
    b.run(3.0e-3)
    assert np.array_equal(counts(b), ref)
    assert b.getNIteration() == a.getNIteration()
    assert b.getTime() == a.getTime()
    for q in range(12):
        assert b.getCompReacExtent("comp", f"r{q}") == a.getCompReacExtent("comp", f"r{q}")
    assert b.getDiffExtent() == a.getDiffExtent()


def test_batched_resume_is_exact(steps_lib, tmp_path):
    sizes = [5, 7, 6]
    mesh = W.batched_mesh(sizes)
    mdl = W.random_network(4)

    def make():
        sim = TetOpSplit(mdl, mesh, make_rng(11), realizations=mesh.offsets)
        sim.setCompReacK("comp", "r3", 2.5 * sim.getCompReacK("comp", "r3", 0), realization=1)
        return sim

    a = make()
    rows = W.poisson_counts(mesh.ntets, 25.0, 11, nspec=8)
    for i, s in enumerate(a.spec_names):
        a.setSpecCounts(s, rows[i])
    a.run(0.5e-3)
    f = str(tmp_path / "batched.ckpt")
    a.checkpoint(f)
    a.run(2.0e-3)
    b = TetOpSplit(mdl, mesh, make_rng(11), realizations=mesh.offsets)
    b.restore(f)
    assert b.getCompReacK("comp", "r3", 1) == a.getCompReacK("comp", "r3", 1)
    b.run(2.0e-3)
    assert np.array_equal(counts(b), counts(a))


def test_membrane_resume_is_exact(steps_lib, tmp_path):
    import math

    def build():
        mesh = sgeom.kuhn_box(4, 4, 8, W.H)
        cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
        cyto.addVolsys("vsys")
        patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), cyto)
        patch.addSurfsys("ssys")
        sgeom.Memb("membrane", mesh, [patch])
        mdl = smodel.Model()
        smodel.Volsys("vsys", mdl)
        ss = smodel.Surfsys("ssys", mdl)
        ch = smodel.Chan("K", mdl)
        c = smodel.ChanState("Kc", mdl, ch)
        o = smodel.ChanState("Ko", mdl, ch)
        smodel.VDepSReac("open", ss, slhs=[c], srhs=[o], k=lambda v: 300.0 * math.exp(v / 0.025))
        smodel.VDepSReac("close", ss, slhs=[o], srhs=[c], k=lambda v: 300.0 * math.exp(-v / 0.025))
        smodel.OhmicCurr("I_K", ss, chanstate=o, g=20e-12, erev=0.05)
        sim = TetOpSplit(mdl, mesh, make_rng(12), EF_DV_CG_FP64)
        sim.setEfieldDT(2e-6)
        return mesh, patch, sim

    mesh, patch, a = build()
    a.setMembPotential("membrane", -0.065)
    a.setMembCapac("membrane", 0.01)
    a.setMembRes("membrane", 1.0 / 0.3, -0.065)
    a.setPatchSpecCount("memb", "Kc", 30 * len(patch.tris))
    a.setVertIClamp(0, 2e-12)
    a.run(40e-6)
    f = str(tmp_path / "memb.ckpt")
    a.checkpoint(f)
    a.run(100e-6)
    va = np.array([a.getVertV(v) for v in range(mesh.nverts)])
    _, _, b = build()
    b.restore(f)
    b.run(100e-6)
    vb = np.array([b.getVertV(v) for v in range(mesh.nverts)])
    assert np.array_equal(va, vb)
    assert b.getPatchSpecCount("memb", "Ko") == a.getPatchSpecCount("memb", "Ko")
    assert np.ptp(va) > 0.0


def test_restore_refuses_other_mesh(steps_lib, tmp_path):
    mdl = W.ab_c_model()
    a = TetOpSplit(mdl, W.cube_mesh(4), make_rng(1))
    f = str(tmp_path / "a.ckpt")
    a.checkpoint(f)
    b = TetOpSplit(mdl, W.cube_mesh(5), make_rng(1))
    with pytest.raises(ArgErr):
        b.restore(f)
