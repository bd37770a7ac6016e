"""Merged SSA units on the GPU against the CPU oracle, bit for bit.

A patch between an inner and an outer compartment whose surface reactions take reactants
from either volume and put products into either (sreac.cpp:305-520 with the outer terms of
sreac.cpp:40-68, 431-520) and whose GHK current reads the outer tet's concentration and
moves ions between the tets (ghkcurr.cpp:168-280): every tet linked through the patch joins
one SSA unit (sreac.cpp:200-300 keeps them in one rank's SSA), run by unit_ssa_kernel on the
GPU and by or_unit_ssa in the oracle on the same Philox streams.  Every count of every tet
and triangle must agree after every run(), and calcium is conserved.
"""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from steps_b200.solver import TetOpSplit
from tests.helpers import make_rng
from tests.outer_membrane import INITIAL, outer_mesh, outer_model

pytestmark = pytest.mark.gpu


def _build(seed, ghk=True, realizations=None, sdiff=False):
    mesh = outer_mesh()
    sim = TetOpSplit(outer_model(ghk, sdiff), mesh, make_rng(seed))
    sim.setCompSpecCount("cyto", "Ca", INITIAL["Ca_in"])
    sim.setCompSpecCount("ecs", "Ca", INITIAL["Ca_out"])
    sim.setCompSpecCount("cyto", "B", INITIAL["B"])
    sim.setPatchSpecCount("memb", "P", INITIAL["P"])
    sim.setPatchSpecCount("memb", "Kc", INITIAL["Kc"])
    ora = Oracle(sim.tables, seed=seed)
    for i, s in enumerate(sim.spec_names):
        ora.set_counts(i, sim.getSpecCounts(s))
    sf = sim.tables["surf"]
    for k, name in enumerate(sf["sspec_names"]):
        ora.set_tri_counts(k, np.array([sim.getTriSpecCount(int(t), name) for t in sf["tris"]], dtype=np.uint32))
    return mesh, sim, ora


def _check(sim, ora, where):
    for i, s in enumerate(sim.spec_names):
        g, o = sim.getSpecCounts(s), ora.get_counts(i)
        assert np.array_equal(g, o), f"{where}: volume species {s} differs in {int(np.sum(g != o))} tets"
    sf = sim.tables["surf"]
    for k, name in enumerate(sf["sspec_names"]):
        g = np.array([sim.getTriSpecCount(int(t), name) for t in sf["tris"]], dtype=np.uint32)
        o = ora.get_tri_counts(k)
        assert np.array_equal(g, o), f"{where}: surface species {name} differs in {int(np.sum(g != o))} triangles"


def _ca_total(sim):
    sf = sim.tables["surf"]
    pc = sum(sim.getTriSpecCount(int(t), "PCa") for t in sf["tris"])
    return int(sim.getSpecCounts("Ca").sum()) + int(sim.getSpecCounts("CaB").sum()) + int(pc)


@pytest.mark.parametrize("ghk,sdiff", [(False, False), (True, False), (True, True)])
def test_outer_membrane_matches_oracle(steps_lib, ghk, sdiff):
    """With sdiff the pumps also diffuse on the patch (surface diffusion of merged units'
    triangles, sdiff.cpp:438-560)."""
    mesh, sim, ora = _build(41, ghk, sdiff=sdiff)
    assert sim.getUpdPeriod() == ora.period()
    total = _ca_total(sim)
    outer = np.unique(sim.tables["surf"]["tri_outer"])
    ca_out0 = int(sim.getSpecCounts("Ca")[outer].sum())
    for k in range(1, 9):
        t = k * 0.5e-3
        sim.run(t)
        ora.run(t)
        _check(sim, ora, f"t={t} ghk={ghk} sdiff={sdiff}")
        assert _ca_total(sim) == total
    assert sim.getNIteration() == ora.window()
    assert ora.surf_extent() > 0
    assert int(sim.getSpecCounts("Ca")[outer].sum()) != ca_out0
    if ghk:
        assert np.any(ora.echarge() != 0)
    if sdiff:
        assert ora.diff_extent() > 0


def test_outer_membrane_split_setting_is_ignored(steps_lib):
    """Merged units need the split window; asking for the fused kernel changes nothing."""
    _, a, ora = _build(43)
    _, b, _ = _build(43)
    b.setSplit(False)
    for k in range(1, 4):
        t = k * 0.4e-3
        a.run(t)
        b.run(t)
        ora.run(t)
        _check(a, ora, f"t={t}")
        for s in a.spec_names:
            assert np.array_equal(a.getSpecCounts(s), b.getSpecCounts(s))


def test_outer_membrane_ensemble_matches_reference_tetopsplit(steps_lib):
    """200 batched realizations (one merged unit each) against 200 seeds of the reference
    TetOpSplitP on the same configuration (tests/golden/ref_ensemble_outer.npz): Ca in each
    volume, CaB, PCa and open channels every 0.5 ms to 10 ms, family-wise 3 sigma on mean
    and variance and KS p > 0.01 (tests/ensemble_stats.py)."""
    import os
    import sys

    from steps_b200 import geom as sgeom
    from steps_b200 import workloads as W
    from tests.ensemble_stats import compare
    from tests.outer_membrane import outer_split

    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, gold)
    import make_ref_ensembles as MR

    fx = np.load(os.path.join(gold, "ref_ensemble_outer.npz"))
    n = fx["tos"].shape[0]
    base = sgeom.kuhn_box(6, 4, 4, W.H)
    inner, outer, _ = outer_split(base)
    mesh = outer_mesh(replicas=n)
    sim = TetOpSplit(outer_model(ghk=False), mesh, make_rng(5), realizations=mesh.offsets)
    sim.setCompSpecCount("cyto", "Ca", INITIAL["Ca_in"])
    sim.setCompSpecCount("ecs", "Ca", INITIAL["Ca_out"])
    sim.setCompSpecCount("cyto", "B", INITIAL["B"])
    for r in range(n):
        sim.setPatchSpecCount("memb", "P", INITIAL["P"], realization=r)
        sim.setPatchSpecCount("memb", "Kc", INITIAL["Kc"], realization=r)
    T = base.ntets
    out = np.zeros((n, len(MR.OUTER_RECORDS), 5))
    for i, t in enumerate(MR.OUTER_RECORDS):
        if t > 0:
            sim.run(t)
        ca = sim.getSpecCounts("Ca").astype(np.int64).reshape(n, T)
        cab = sim.getSpecCounts("CaB").astype(np.int64).reshape(n, T)
        out[:, i, 0] = ca[:, inner].sum(axis=1)
        out[:, i, 1] = ca[:, outer].sum(axis=1)
        out[:, i, 2] = cab.sum(axis=1)
        out[:, i, 3] = [sim.getPatchSpecCount("memb", "PCa", r) for r in range(n)]
        out[:, i, 4] = [sim.getPatchSpecCount("memb", "Ko", r) for r in range(n)]
    assert np.all(out[:, :, 0] + out[:, :, 1] + out[:, :, 2] + out[:, :, 3] ==
                  INITIAL["Ca_in"] + INITIAL["Ca_out"])
    rep = compare(out, fx["tos"])
    assert rep["ok"], rep
