"""GPU split windows vs the CPU oracle, bit for bit, through the C ABI.

The oracle restates TetOpSplitP's window (src/steps/mpi/tetopsplit/tetopsplit.cpp:1528-1839)
with the same Philox counters; every count of every tet must agree after every run().
"""
import numpy as np
import pytest

from steps_b200 import workloads as W
from tests.helpers import assert_same, pair, sync_counts, two_comp_mesh, two_comp_model

pytestmark = pytest.mark.gpu


def test_plain_small_ab_c(steps_lib):
    """A + B <-> C with diffusion on 10^3 Kuhn cubes, recorded every 1 ms (4 windows/ms)."""
    sim, ora = pair(W.ab_c_model(), W.cube_mesh(10), seed=1)
    sim.setCompSpecCount("comp", "A", 10000)
    sim.setCompSpecCount("comp", "B", 10000)
    assert sim.getCompSpecCount("comp", "A") == 10000
    sync_counts(sim, ora)
    assert sim.getUpdPeriod() == ora.period()
    for k in range(1, 21):
        t = k * 1.0e-3
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"t={t}")
        assert sim.getTime() == t
    assert sim.getNIteration() == ora.window() == 80
    assert sim.getCompSpecCount("comp", "A") + sim.getCompSpecCount("comp", "C") == 10000
    for r, name in enumerate(["fwd", "bwd"]):
        assert sim.getCompReacExtent("comp", name) == ora.reac_extent(r)
    assert sim.getDiffExtent() == ora.diff_extent()
    assert sim.getStatus() == 0


def test_diffusion_only_large_counts(steps_lib):
    """Pure diffusion with counts in the BTRD regime (n p >= 10)."""
    mdl = W.ab_c_model(kf=0.0, kb=0.0)
    sim, ora = pair(mdl, W.cube_mesh(5), seed=99)
    row = np.zeros(sim.geom.ntets, dtype=np.uint32)
    row[::7] = 200000
    row[3] = 4000000000
    sim.setSpecCounts("A", row)
    sim.setSpecCounts("B", np.full(sim.geom.ntets, 3, dtype=np.uint32))
    sync_counts(sim, ora)
    total = int(row.sum(dtype=np.uint64))
    for k in range(1, 6):
        t = k * 3.0 * sim.getUpdPeriod()
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"window {k}")
        assert int(sim.getSpecCounts("A").sum(dtype=np.uint64)) == total


@pytest.mark.parametrize("split", [False, True])
def test_random_network_poisson(steps_lib, split):
    """8 species, 12 reactions (zeroth, first, second order) on 6^3 cubes, Poisson(50) counts;
    fused and split windows."""
    mdl = W.random_network(2025)
    sim, ora = pair(mdl, W.cube_mesh(6), seed=2025)
    sim.setSplit(split)
    rows = W.poisson_counts(sim.geom.ntets, 50.0, 2025)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    sync_counts(sim, ora)
    per = sim.getUpdPeriod()
    for k in range(1, 9):
        t = k * 2.5 * per
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"t={t}")
    for r in range(12):
        assert sim.getCompReacExtent("comp", f"r{r}") == ora.reac_extent(r)


@pytest.mark.parametrize("split", [False, True])
def test_two_compartments(steps_lib, split):
    """Different reactions and diffusion rules per compartment; no diffusion across."""
    sim, ora = pair(two_comp_model(), two_comp_mesh(6), seed=5)
    sim.setSplit(split)
    for c in ("left", "right"):
        for s in ("A", "B"):
            sim.setCompSpecCount(c, s, 2500.5)
    sync_counts(sim, ora)
    for k in range(1, 7):
        t = k * 1.7e-4
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"t={t}")


@pytest.mark.parametrize("split", [False, True])
def test_clamped_species(steps_lib, split):
    sim, ora = pair(W.ab_c_model(), W.cube_mesh(5), seed=11)
    sim.setSplit(split)
    sim.setCompSpecCount("comp", "A", 5000)
    sim.setCompSpecCount("comp", "B", 5000)
    for t in (0, 17, 400):
        sim.setTetSpecClamped(t, "A", True)
        ora.set_clamped(t, 0, True)
    sync_counts(sim, ora)
    clamped_before = [sim.getTetSpecCount(t, "A") for t in (0, 17, 400)]
    for k in range(1, 6):
        t = k * 1.0e-3
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"t={t}")
    assert [sim.getTetSpecCount(t, "A") for t in (0, 17, 400)] == clamped_before


@pytest.mark.parametrize("split", [False, True])
def test_batched_realizations_with_jitter(steps_lib, split):
    """Realizations of different sizes in one launch, per-realization rate constants."""
    sizes = [3, 5, 4, 6]
    mesh = W.batched_mesh(sizes)
    mdl = W.random_network(7)
    sim, ora = pair(mdl, mesh, seed=3, realizations=mesh.offsets)
    sim.setSplit(split)
    jit = W.rate_jitter(len(sizes), 12, 3)
    for r in range(len(sizes)):
        for q in range(12):
            k = sim.getCompReacK("comp", f"r{q}", r) * jit[r, q]
            sim.setCompReacK("comp", f"r{q}", k, realization=r)
            ora.set_reac_k(q, r, k)
    rows = W.poisson_counts(mesh.ntets, 20.0, 3)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    sync_counts(sim, ora)
    per = sim.getUpdPeriod()
    for k in range(1, 5):
        t = k * 3.0 * per
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"t={t}")


@pytest.mark.parametrize("graphs", [True, False])
def test_long_runs_graph_replay(steps_lib, graphs):
    """run() calls of 40+ windows replay a captured graph of 16 windows; the result must
    not depend on it."""
    sim, ora = pair(W.random_network(11), W.cube_mesh(6), seed=12)
    sim.setGraphs(graphs)
    rows = W.poisson_counts(sim.geom.ntets, 30.0, 12)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    sync_counts(sim, ora)
    per = sim.getUpdPeriod()
    for k in (1, 2):
        t = k * 41.5 * per
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"graphs={graphs} call {k}")
    assert sim.getNIteration() == ora.window() >= 80


@pytest.mark.parametrize("block,split", [(64, False), (256, False), (128, True), (256, True)])
def test_launch_shapes_agree(steps_lib, block, split):
    """The result does not depend on the block size or on the split window (counter-based
    streams)."""
    sim, ora = pair(W.ab_c_model(), W.cube_mesh(7), seed=4, block=block)
    sim.setSplit(split)
    sim.setCompSpecCount("comp", "A", 7000)
    sim.setCompSpecCount("comp", "B", 3000)
    sync_counts(sim, ora)
    for k in range(1, 4):
        sim.run(k * 1.0e-3)
        ora.run(k * 1.0e-3)
        assert_same(sim, ora, f"block {block} step {k}")


def test_autotuned_run_matches_oracle(steps_lib):
    """Autotuning times 24 windows (after an untimed one) under twelve launch shapes; the
    counts after the run still equal the oracle's, and the kept shape is a candidate."""
    mesh = W.cube_mesh(9)
    sim, ora = pair(W.random_network(3), mesh, seed=6)
    rows = W.poisson_counts(mesh.ntets, 30.0, 6, nspec=8)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    sync_counts(sim, ora)
    sim.setAutotune(True)
    t = 50 * sim.getUpdPeriod()
    sim.run(t)
    ora.run(t)
    assert_same(sim, ora, "autotuned run")
    times = sim.getAutotuneTimes()
    assert len(times) == 12 and all(x > 0.0 for x in times)
    assert sim.getCarveout() in (100, 75, 50)
    block, grid = sim.getLaunch()
    assert block in (64, 128, 256) and grid in (0, -1)
    sim.run(2 * t)
    ora.run(2 * t)
    assert_same(sim, ora, "after tuning")


def test_batch_tet_counts_gather(steps_lib):
    """getBatchTetSpecCountsNP gathers on the device: the values equal the full row at the
    requested tets (after the pending inflow is applied), concentrations follow, and an
    index outside the mesh is an ArgErr."""
    from steps_b200._lib import ArgErr

    mesh = W.cube_mesh(6)
    sim, ora = pair(W.ab_c_model(), mesh, seed=8)
    sim.setCompSpecCount("comp", "A", 9000)
    sim.setCompSpecCount("comp", "B", 9000)
    sim.run(2e-3)
    rng = np.random.default_rng(3)
    tets = rng.integers(0, mesh.ntets, size=777)
    got = np.empty(len(tets))
    sim.getBatchTetSpecCountsNP(tets, "A", got)
    assert np.array_equal(got, sim.getSpecCounts("A")[tets].astype(np.float64))
    conc = np.empty(len(tets))
    sim.getBatchTetSpecConcsNP(tets, "A", conc)
    assert np.allclose(conc, got / (6.02214179e23 * mesh.tet_vol[tets] * 1e3), rtol=1e-15)
    with pytest.raises(ArgErr):
        sim.getBatchTetSpecCountsNP(np.array([0, mesh.ntets]), "A", np.empty(2))


@pytest.mark.parametrize("split", [False, True])
def test_diffusion_boundary_matches_oracle(steps_lib, split):
    """A diffusion boundary between two compartments (diffboundary.cpp): closed, opened in
    both directions, then one direction with its own constant; every count equals the
    oracle's after every run, and molecules are conserved."""
    from steps_b200 import geom as sgeom
    from steps_b200 import model as smodel
    from steps_b200.solver import TetOpSplit
    from oracle.pyoracle import Oracle
    from tests.helpers import make_rng

    n = 6
    mesh = sgeom.kuhn_box(n, n, n, W.H)
    x = mesh.tet_bary[:, 0]
    left = np.nonzero(x < 0.5 * n * W.H)[0]
    right = np.nonzero(x >= 0.5 * n * W.H)[0]
    sgeom.TmComp("left", mesh, left).addVolsys("vl")
    sgeom.TmComp("right", mesh, right).addVolsys("vr")
    tt = mesh.tri_tets
    side = np.zeros(mesh.ntets, dtype=int)
    side[right] = 1
    both = (tt[:, 0] >= 0) & (tt[:, 1] >= 0)
    btris = np.nonzero(both & (side[np.maximum(tt[:, 0], 0)] != side[np.maximum(tt[:, 1], 0)]))[0]
    sgeom.DiffBoundary("db", mesh, btris)
    mdl = smodel.Model()
    A, B = smodel.Spec("A", mdl), smodel.Spec("B", mdl)
    vl, vr = smodel.Volsys("vl", mdl), smodel.Volsys("vr", mdl)
    smodel.Reac("conv", vr, lhs=[A], rhs=[B], kcst=20.0)
    smodel.Diff("dAl", vl, A, 2e-12)
    smodel.Diff("dAr", vr, A, 1e-12)
    smodel.Diff("dBr", vr, B, 1e-12)
    sim = TetOpSplit(mdl, mesh, make_rng(13))
    sim.setSplit(split)
    ora = Oracle(sim.tables, seed=13)
    sim.setCompSpecCount("left", "A", 20000)
    sync_counts(sim, ora)
    per = sim.getUpdPeriod()
    t = 0.0
    for phase in range(3):
        if phase == 1:
            sim.setDiffBoundarySpecDiffusionActive("db", "A", True)
            ora.set_bnd_active(0, 0, True)
            assert sim.getDiffBoundarySpecDiffusionActive("db", "A")
        if phase == 2:
            sim.setDiffBoundarySpecDiffusionActive("db", "A", False)
            sim.setDiffBoundarySpecDcst("db", "A", 5e-13, direction_comp="left")
            ora.set_bnd_active(0, 0, False)
            ora.set_bnd_dcst(0, 0, 5e-13, direction_comp=0)
        assert sim.getUpdPeriod() == ora.period()
        for k in range(4):
            t += 7.0 * sim.getUpdPeriod()
            sim.run(t)
            ora.run(t)
            assert_same(sim, ora, f"phase {phase} t={t}")
        if phase == 0:
            assert sim.getCompSpecCount("right", "A") == 0
        if phase == 1:
            assert sim.getCompSpecCount("right", "A") > 0
    total = sim.getCompSpecCount("left", "A") + sim.getCompSpecCount("right", "A") + sim.getCompSpecCount("right", "B")
    assert total == 20000


def test_placement_matches_oracle_restatement(steps_lib):
    """setCompSpecCount places molecules by the reference's rule (util/distribute.hpp:102-193:
    volume-weighted floors, then adjusted Pareto order sampling of the remainder); the
    solver's placement equals the oracle's restatement bit for bit, the n-th setter call
    drawing from setup stream n.  The sphere mesh of the reference's validation has tets
    of unequal volume; the batched case places each realization with its own call."""
    import os

    from oracle.pyoracle import distribute
    from steps_b200 import geom as sgeom
    from steps_b200.solver import TetOpSplit
    from tests.helpers import make_rng

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sphere_rad1_37tets.npz"))
    mesh = sgeom.Tetmesh(d["verts"], d["tets"])
    sgeom.TmComp("comp", mesh, np.arange(mesh.ntets)).addVolsys("vsys")
    seed = 77
    sim = TetOpSplit(W.ab_c_model(), mesh, make_rng(seed))
    vol = sim.tables["vol"]
    sim.setCompSpecCount("comp", "A", 1000.5)
    assert np.array_equal(sim.getSpecCounts("A"), distribute(seed, 0, vol, 1000.5))
    sim.setCompSpecCount("comp", "B", 37.25)
    assert np.array_equal(sim.getSpecCounts("B"), distribute(seed, 1, vol, 37.25))
    sim.setCompSpecCount("comp", "A", 0.0)
    assert not sim.getSpecCounts("A").any()

    base = W.cube_mesh(3)
    rep = sgeom.replicate(base, 3)
    sgeom.TmComp("comp", rep, np.arange(rep.ntets)).addVolsys("vsys")
    bs = TetOpSplit(W.ab_c_model(), rep, make_rng(seed), realizations=rep.offsets)
    bs.setCompSpecCount("comp", "C", 55.5)
    got = bs.getSpecCounts("C")
    T = base.ntets
    for r in range(3):
        want = distribute(seed, r, bs.tables["vol"][r * T:(r + 1) * T], 55.5)
        assert np.array_equal(got[r * T:(r + 1) * T], want), r


def test_all_species_rows_at_once(steps_lib):
    """getAllSpecCounts / setAllSpecCounts move every species row in one copy; the values
    equal the per-species rows, and a run from rows set that way matches the oracle."""
    mesh = W.cube_mesh(5)
    sim, ora = pair(W.random_network(5), mesh, seed=8)
    rows = W.poisson_counts(mesh.ntets, 12.0, 8, nspec=8)
    sim.setAllSpecCounts(np.stack(rows))
    for i, s in enumerate(sim.spec_names):
        assert np.array_equal(sim.getSpecCounts(s), rows[i])
    sync_counts(sim, ora)
    t = 7 * sim.getUpdPeriod()
    sim.run(t)
    ora.run(t)
    allc = sim.getAllSpecCounts()
    for i, s in enumerate(sim.spec_names):
        assert np.array_equal(allc[i], sim.getSpecCounts(s))
        assert np.array_equal(allc[i], ora.get_counts(i))
