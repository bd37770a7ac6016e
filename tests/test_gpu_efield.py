"""EField on the GPU against the reference's golden data and an FP64 direct solve.

Rallpack1 (passive cable, 1000 um x 0.866 um, 1978 tets) as the reference's
test/validation/API_1/validation_efield/rallpack1_membres.py sets it up: membrane on the
lateral surface, R_A = 1 ohm m, R_M = 4 ohm m^2, C_M = 0.01 F/m^2 (both corrected by the
mesh's area factor), E_M = -65 mV, 0.1 nA injected over the z-min vertices, EField dt
10 us.  V(t) at the radial extrema of both ends must match the reference's
rallpack1_correct/{v0,vx} curves with RMS error below 1 mV (test_rallpack1_membres.py:45).
"""
import os

import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200.solver import EF_DV_CG_FP64, EF_DV_CG_MIXED, TetOpSplit
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))

P = dict(R_A=1.0, R_M=4.0, C_M=0.01, E_M=-0.065, Iinj=0.1e-9, diameter=1.0e-6, length=1.0e-3,
         sim_end=0.25, EF_dt=1.0e-5)


def rallpack1_sim(method):
    d = np.load(os.path.join(HERE, "golden", "rallpack1.npz"))
    mesh = sgeom.Tetmesh(d["verts"], d["tets"])
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    minz, maxz = mesh.getBoundMin()[2], mesh.getBoundMax()[2]
    zeps = (maxz - minz) / mesh.ntets
    surf = mesh.getSurfTris()
    z = mesh.verts[mesh.tris[surf]][:, :, 2]
    zmin = surf[np.all(z <= minz + zeps, axis=1)]
    zmax = surf[np.all(z >= maxz - zeps, axis=1)]
    memb_tris = np.setdiff1d(surf, np.concatenate([zmin, zmax]))
    patch = sgeom.TmPatch("memb", mesh, memb_tris, mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    zmin_v = np.unique(mesh.tris[zmin])
    zmax_v = np.unique(mesh.tris[zmax])

    def extrema(vs):
        r2 = (mesh.verts[vs, :2] ** 2).sum(axis=1)
        return [int(vs[np.argmin(r2)]), int(vs[np.argmax(r2)])]

    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(1), method)
    area_cyl = np.pi * P["diameter"] * P["length"]
    factor = patch.getArea() / area_cyl
    sim.setEfieldDT(P["EF_dt"])
    sim.setMembPotential("membrane", P["E_M"])
    sim.setMembVolRes("membrane", P["R_A"])
    sim.setMembCapac("membrane", P["C_M"] / factor)
    sim.setMembRes("membrane", P["R_M"] * factor, P["E_M"])
    for v in zmin_v:
        sim.setVertIClamp(int(v), P["Iinj"] / len(zmin_v))
    return sim, extrema(zmin_v), extrema(zmax_v), d["v0"], d["vx"]


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("method,rtol", [(EF_DV_CG_FP64, 1e-9), (EF_DV_CG_MIXED, 1e-7)])
def test_efield_steps_match_fp64_direct_solve(steps_lib, method, rtol, persistent):
    """20 EField steps on a 4x4x10 Kuhn box (membrane = every boundary triangle, leak,
    a current clamp, one voltage-clamped vertex) against the FP64 direct-solve oracle."""
    from oracle.efield_oracle import EFieldOracle

    mesh = sgeom.kuhn_box(4, 4, 10, 1e-7)
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    surf = mesh.getSurfTris()
    patch = sgeom.TmPatch("memb", mesh, surf, mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(3), method)
    sim.setEfieldPersistent(persistent)
    sim.setEfieldTolerance(1e-12, 1e-4)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembVolRes("membrane", 1.0)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    ora = EFieldOracle(mesh.verts, mesh.tets, mesh.tris[surf])
    ora.cm, ora.sigma, ora.g, ora.vext = 0.01, 1.0e3, 0.3e-3, -65.0
    zmin = np.unique(mesh.tris[surf][np.all(mesh.verts[mesh.tris[surf]][:, :, 2] <= 1e-12, axis=1)])
    for v in zmin:
        sim.setVertIClamp(int(v), 1e-9 / len(zmin))
        ora.iclamp[v] = 1e-9 / len(zmin) * 1e12
    top = int(np.argmax(mesh.verts[:, 2]))
    sim.setVertV(top, -0.070)
    sim.setVertVClamped(top, True)
    ora.V[top] = -70.0
    ora.clamped[top] = True
    for k in range(1, 21):
        sim.run(k * 1e-6)
        ora.advance(1e-3)
    got = np.array([sim.getVertV(v) for v in range(mesh.nverts)]) * 1e3
    assert got[top] == -70.0
    assert np.max(np.abs(got - ora.V) / np.abs(ora.V)) < rtol
    assert np.ptp(got) > 1e-3  # the clamp and the injection actually moved V


def test_step_length_changes_match_direct_solve(steps_lib):
    """Runs whose end is not a whole number of EField steps end on a short step; the next
    run resumes at the regular length (the previous length's matrices are swapped back in).
    Every step still equals the FP64 direct solve of its own length."""
    from oracle.efield_oracle import EFieldOracle

    mesh = sgeom.kuhn_box(4, 4, 8, 1e-7)
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    surf = mesh.getSurfTris()
    patch = sgeom.TmPatch("memb", mesh, surf, mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(9), EF_DV_CG_FP64)
    sim.setEfieldTolerance(1e-12, 1e-4)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    ora = EFieldOracle(mesh.verts, mesh.tets, mesh.tris[surf])
    ora.cm, ora.sigma, ora.g, ora.vext = 0.01, 1.0e3, 0.3e-3, -65.0
    zmin = np.unique(mesh.tris[surf][np.all(mesh.verts[mesh.tris[surf]][:, :, 2] <= 1e-12, axis=1)])
    for v in zmin:
        sim.setVertIClamp(int(v), 1e-9 / len(zmin))
        ora.iclamp[v] = 1e-9 / len(zmin) * 1e12
    t = 0.0
    for ends, steps in ((3.4e-6, [1e-3, 1e-3, 1e-3, 0.4e-3]), (6.4e-6, [1e-3, 1e-3, 1e-3]),
                        (7.0e-6, [0.6e-3])):
        sim.run(ends)
        for dt in steps:
            ora.advance(dt)
    got = np.array([sim.getVertV(v) for v in range(mesh.nverts)]) * 1e3
    assert np.max(np.abs(got - ora.V) / np.abs(ora.V)) < 1e-9
    assert sim.getEfieldStats()[0] == 8


@pytest.mark.parametrize("method", [EF_DV_CG_FP64, EF_DV_CG_MIXED])
def test_rallpack1_membres(steps_lib, method):
    sim, v0s, vxs, ref0, refx = rallpack1_sim(method)
    sim.setEfieldTolerance(1e-10)
    dt = 5.0e-5
    n = int(np.ceil(P["sim_end"] / dt)) + 1
    out0, outx = np.zeros(n), np.zeros(n)
    for k in range(n):
        sim.run(k * dt)
        out0[k] = np.mean([sim.getVertV(v) for v in v0s])
        outx[k] = np.mean([sim.getVertV(v) for v in vxs])
    npt = min(n, len(ref0))
    rms0 = np.linalg.norm(ref0[:npt, 1] - out0[:npt]) / np.sqrt(npt)
    rmsx = np.linalg.norm(refx[:npt, 1] - outx[:npt]) / np.sqrt(npt)
    steps, iters, ms, rr = sim.getEfieldStats()
    assert steps == 25000
    assert rms0 < 1.0e-3 and rmsx < 1.0e-3, (rms0, rmsx, iters / steps)


@pytest.mark.parametrize("persistent,reliable", [(False, False), (True, False), (True, True)])
def test_mixed_step_check_against_fp64(steps_lib, persistent, reliable):
    """The mixed method's per-step check: every step's V from the FP32 solve (restarted
    inner solves, or one solve with reliable updates) is within 1e-6 relative of an FP64
    solve of the same system."""
    mesh = sgeom.kuhn_box(6, 6, 30, 1e-7)
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    surf = mesh.getSurfTris()
    patch = sgeom.TmPatch("memb", mesh, surf, mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(4), EF_DV_CG_MIXED)
    sim.setEfieldPersistent(persistent)
    sim.setEfieldReliableUpdates(reliable)
    sim.setEfieldTolerance(1e-10, 1e-4)
    sim.setEfieldCheck(True, 1e-12)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    zmin = np.unique(mesh.tris[surf][np.all(mesh.verts[mesh.tris[surf]][:, :, 2] <= 1e-12, axis=1)])
    for v in zmin:
        sim.setVertIClamp(int(v), 1e-10 / len(zmin))
    sim.run(50e-6)
    n, mx, last = sim.getEfieldCheck()
    assert n == 50
    assert 0.0 < mx < 1e-6, mx
    assert last <= mx
    v = np.array([sim.getVertV(i) for i in range(mesh.nverts)])
    assert np.ptp(v) > 1e-6  # the injection moved V


def test_persistent_barrier_wait_runs_out(steps_lib):
    """A grid-barrier wait of the persistent EField solve that runs out ends the launch with
    an error status instead of waiting on: with a poll limit of 0 every block that is not
    the last to arrive gives up at once, the step raises DeviceError, and with the default
    limit restored the same solver steps on (the device is still usable)."""
    from steps_b200._lib import DeviceError

    mesh = sgeom.kuhn_box(8, 8, 40, 1e-7)  # 3321 vertices: several blocks in the solve
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(5), EF_DV_CG_FP64)
    sim.setEfieldPersistent(True)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    sim.setVertIClamp(0, 1e-12)
    sim.setEfieldBarrierLimit(0)
    with pytest.raises(DeviceError, match="timed out"):
        sim.run(3e-6)
    sim.setEfieldBarrierLimit(1 << 22)
    sim.run(sim.getTime() + 5e-6)
    v = np.array([sim.getVertV(i) for i in range(0, mesh.nverts, 11)])
    assert np.all(np.isfinite(v)) and np.all(np.abs(v + 0.065) < 0.01)
