"""The persistent form of the window loop on the GPU against the CPU oracle, bit for bit.

One cooperative launch runs up to 64 windows of every batched realization
(persistent_window_kernel): warps take (window, chunk) items in window order and wait,
bounded, until the chunk's realization has finished the previous window.  Every tet draws
from its own Philox streams, so the counts equal the oracle's (TOS:1528-1839 restated)
whatever the order the chunks ran in.  A wait limit of zero polls makes the waits run out:
run() reports it and the GPU stays usable.
"""
import numpy as np
import pytest

from steps_b200 import workloads as W
from steps_b200._lib import DeviceError
from tests.helpers import assert_same, pair, sync_counts, two_comp_mesh, two_comp_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("block,tpl", [(128, 1), (256, 2), (256, 4), (128, 8)])
def test_persistent_batched_matches_oracle(steps_lib, block, tpl):
    """Realizations of different sizes with per-realization rate constants; run() calls of
    a few windows, of 70 windows (two launches) and one ending off the window grid."""
    sizes = [3, 5, 4, 6, 2]
    mesh = W.batched_mesh(sizes)
    mdl = W.random_network(7)
    sim, ora = pair(mdl, mesh, seed=3, realizations=mesh.offsets, block=block)
    sim.setPersistent(True, tpl)
    assert sim.getPersistent() == (True, tpl)
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
    for t in (3.0 * per, 73.0 * per, 80.5 * per):
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"t={t} block={block} tets per lane={tpl}")
    assert sim.getNIteration() == ora.window()
    for q in range(12):
        assert sim.getCompReacExtent("comp", f"r{q}") == ora.reac_extent(q)
    assert sim.getDiffExtent() == ora.diff_extent()


def test_persistent_clamps_and_compartments_match_oracle(steps_lib):
    """Two compartments and a clamped species, one realization, then the window launches
    again after the persistent ones (the same stream of windows)."""
    mesh = two_comp_mesh(6)
    sim, ora = pair(two_comp_model(), mesh, seed=17)
    sim.setCompSpecCount("left", "A", 4000)
    sim.setCompSpecCount("right", "B", 3000)
    sim.setTetSpecClamped(5, "A", True)
    sync_counts(sim, ora)
    ora.set_clamped(5, 0, True)
    sim.setPersistent(True, 1)
    per = sim.getUpdPeriod()
    for k in range(1, 4):
        t = k * 20.0 * per
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"persistent t={t}")
    sim.setPersistent(False)
    for k in range(4, 6):
        t = k * 20.0 * per
        sim.run(t)
        ora.run(t)
        assert_same(sim, ora, f"window launches t={t}")


def test_persistent_wait_limit_runs_out(steps_lib):
    """With a wait limit of zero polls the first wait on an unfinished window gives up: the
    launch stops, run() raises, and the GPU takes the next solver's run as usual."""
    sim, _ = pair(W.ab_c_model(), W.cube_mesh(8), seed=2)
    sim.setCompSpecCount("comp", "A", 20000)
    sim.setCompSpecCount("comp", "B", 20000)
    sim.setPersistent(True, 1)
    sim.setWindowWaitLimit(0)
    with pytest.raises(DeviceError, match="gave up waiting"):
        sim.run(30 * sim.getUpdPeriod())
    del sim
    sim2, ora2 = pair(W.ab_c_model(), W.cube_mesh(6), seed=2)
    sim2.setCompSpecCount("comp", "A", 3000)
    sync_counts(sim2, ora2)
    sim2.setPersistent(True, 1)
    t = 10 * sim2.getUpdPeriod()
    sim2.run(t)
    ora2.run(t)
    assert_same(sim2, ora2, "after a run that gave up")
