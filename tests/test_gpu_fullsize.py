"""Parity at the benchmark configurations' full sizes.

  * plain 384k (40^3 Kuhn cubes, 8 species, 12 reactions, Poisson(50) species 0-3):
    5 windows from the initial state, every count of every tet against the CPU oracle;
  * batched: all 512 realizations (n^3 Kuhn cubes, n uniform in 8..30, 28.5 M tets) with
    per-realization rate jitter, 2 windows, bit for bit against the oracle;
  * EField: 20x20x200 Kuhn cubes (88,641 vertices, every boundary triangle membrane),
    capacitance, leak and 1 nA into the z = 0 face: 20 steps of 1 us of the FP64 and the
    mixed-precision solve against the FP64 direct solve of the reference's vertex
    coupling (oracle/efield_oracle.py), relative error per vertex below 1e-8 (FP64 CG) and
    1e-6 (mixed), the bound the mixed method is held to.
"""
import os

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import EF_DV_CG_FP64, EF_DV_CG_MIXED, TetOpSplit
from tests.helpers import assert_same, make_rng

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _threads():
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)


def test_plain_384k_five_windows(steps_lib):
    mesh = W.cube_mesh(40)
    mdl = W.random_network(1)
    rows = W.poisson_counts(mesh.ntets, 50.0, 1, nspec=8)
    sim = TetOpSplit(mdl, mesh, make_rng(1))
    ora = Oracle(sim.tables, seed=1)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
        ora.set_counts(i, rows[i])
    per = sim.getUpdPeriod()
    assert per == ora.period()
    t = 5 * per
    sim.run(t)
    ora.run(t)
    assert sim.getNIteration() == ora.window() == 5
    assert_same(sim, ora, "plain 384k after 5 windows")


def test_batched_512_realizations_two_windows(steps_lib):
    sizes = W.batched_sizes(512, 1)
    mesh = W.batched_mesh(sizes)
    mdl = W.random_network(1)
    sim = TetOpSplit(mdl, mesh, make_rng(1), realizations=mesh.offsets)
    ora = Oracle(sim.tables, seed=1, realizations=mesh.offsets)
    jit = W.rate_jitter(512, 12, 1)
    for q in range(12):
        base = sim.getCompReacK("comp", f"r{q}", 0)
        idx = sim.reac_index[("comp", f"r{q}")]
        for r in range(512):
            sim.setCompReacK("comp", f"r{q}", base * jit[r, q], realization=r)
            ora.set_reac_k(idx, r, base * jit[r, q])
    rows = W.poisson_counts(mesh.ntets, 50.0, 1, nspec=8)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
        ora.set_counts(i, rows[i])
    per = sim.getUpdPeriod(0)
    assert all(sim.getUpdPeriod(r) == per for r in (1, 100, 511))
    t = 2 * per
    sim.run(t)
    ora.run(t)
    assert sim.getNIteration() == 2 and ora.window(511) == 2
    assert_same(sim, ora, "512 realizations after 2 windows")


@pytest.mark.parametrize("method,tol,rtol", [(EF_DV_CG_FP64, 1e-12, 1e-8), (EF_DV_CG_MIXED, 1e-11, 1e-6)])
def test_efield_88k_vertices_twenty_steps(steps_lib, method, tol, rtol):
    """The mixed method stops on the true FP64 residual b - A x, which cannot fall much
    below 1.3e-12 of |b| on this system (the rounding of that product), so it is held to
    1e-11; FP64 CG stops on its recurrence residual and is run to 1e-12."""
    from oracle.efield_oracle import EFieldOracle

    mesh = sgeom.kuhn_box(20, 20, 200, 1e-7)
    sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    surf = mesh.getSurfTris()
    patch = sgeom.TmPatch("memb", mesh, surf, mesh.comps["cyto"])
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    sim = TetOpSplit(mdl, mesh, make_rng(2), method)
    sim.setEfieldTolerance(tol, 1e-4)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembVolRes("membrane", 1.0)
    sim.setMembRes("membrane", 1.0 / 3e-5 * 1e-4, -0.065)  # 3e-5 S/cm^2 = 0.3 S/m^2
    ora = EFieldOracle(mesh.verts, mesh.tets, mesh.tris[surf], fast=True)
    ora.cm, ora.sigma, ora.g, ora.vext = 0.01, 1.0e3, 0.3e-3, -65.0
    zmin = np.unique(mesh.tris[surf][np.all(mesh.verts[mesh.tris[surf]][:, :, 2] <= 1e-12, axis=1)])
    for v in zmin:
        sim.setVertIClamp(int(v), 1e-9 / len(zmin))
        ora.iclamp[v] = 1e-9 / len(zmin) * 1e12
    worst = 0.0
    for k in range(1, 21):
        sim.run(k * 1e-6)
        ora.advance(1e-3)
        got = np.array([sim.getVertV(v) for v in range(0, mesh.nverts, 7)]) * 1e3
        ref = ora.V[::7]
        worst = max(worst, float(np.max(np.abs(got - ref) / np.abs(ref))))
    assert worst < rtol, worst
    got = np.array([sim.getVertV(v) for v in range(mesh.nverts)]) * 1e3
    assert np.max(np.abs(got - ora.V) / np.abs(ora.V)) < rtol
    assert np.ptp(got) > 1e-2  # the injection moved V
