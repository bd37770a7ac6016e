"""The oracle's law against the reference solvers themselves (CPU).

The fixtures tests/golden/ref_ensemble_*.npz and ref_placement.npz hold ensembles of the
reference TetOpSplitP and Tetexact, compiled from the reference's own sources
(tests/golden/make_ref_ensembles.py).  The oracle is the CPU restatement the GPU kernels
are checked against bit for bit, so these tests pin the oracle's statistical law to the
reference's: ensemble mean, variance and distribution per record, family-wise 3 sigma
and KS p > 0.01 (tests/ensemble_stats.py).
"""
import os
import sys
import warnings

import numpy as np
import pytest

from oracle.pyoracle import Oracle, distribute
from steps_b200 import workloads as W
from steps_b200.solver import flatten
from tests.ensemble_stats import compare

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import make_ref_ensembles as M  # noqa: E402


@pytest.fixture(autouse=True)
def _quiet():
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # KS on integer data falls back to the asymptotic form
        yield


def test_placement_law_matches_reference():
    """setCompSpecCount's placement (util/distribute.hpp:102-193) on the reference's sphere
    mesh, whose tets have unequal volumes: per-tet count distributions over 4000 draws."""
    fx = np.load(os.path.join(GOLD, "ref_placement.npz"))
    ref = fx["counts"].astype(np.int64)
    mesh, F = M.sphere_case()
    vol = F["vol"]
    n = ref.shape[0]
    ora = np.stack([distribute(9000 + k, 0, vol, float(fx["x"])) for k in range(n)]).astype(np.int64)
    # x = 1000.5: every draw places 1000 or 1001, each half of the time.
    assert set(np.unique(ora.sum(axis=1))) <= {1000, 1001}
    assert abs((ora.sum(axis=1) == 1001).mean() - 0.5) < 0.03
    rep = compare(ora[:, None, :], ref[:, None, :])
    assert rep["ok"], rep
    # The expected count of tet i is x v_i / V.
    assert np.allclose(ora.mean(axis=0), 1000.5 * vol / vol.sum(), atol=0.05)


def test_diffusion_spread_matches_reference_tetopsplit():
    fx = np.load(os.path.join(GOLD, "ref_ensemble_spread.npz"))
    times = fx["times"]
    mesh, F = M.c0_case()
    a0, slab = M.spread_initial(mesh)
    n = fx["tos"].shape[0]
    out = np.zeros((n, len(times), M.NSLAB))
    for k in range(n):
        o = Oracle(F, seed=7000 + k)
        o.set_counts(0, a0.astype(np.uint32))
        for i, t in enumerate(times):
            if t > 0:
                o.run(t)
            out[k, i] = np.bincount(slab, weights=o.get_counts(0).astype(np.float64), minlength=M.NSLAB)
    assert np.all(out.sum(axis=2) == 6000)
    rep = compare(out, fx["tos"])
    assert rep["ok"], rep


def test_plain_small_matches_reference_tetopsplit_and_tetexact():
    """The plain small configuration over its first 40 ms (100 oracle members)."""
    fx = np.load(os.path.join(GOLD, "ref_ensemble_c0.npz"))
    nrec = 41
    times = fx["times"][:nrec]
    mesh, F = M.c0_case()
    n = 100
    out = np.zeros((n, nrec, 3))
    for k in range(n):
        o = Oracle(F, seed=8000 + k)
        o.set_counts(0, distribute(8000 + k, 0, F["vol"], 10000))
        o.set_counts(1, distribute(8000 + k, 1, F["vol"], 10000))
        for i, t in enumerate(times):
            if t > 0:
                o.run(t)
            out[k, i] = [o.get_counts(s).sum() for s in range(3)]
    for arm in ("tos", "tetexact"):
        rep = compare(out, fx[arm][:, :nrec], cols=[0, 2])
        assert rep["ok"], (arm, rep)


def _oracle_outer(n, seed0):
    """The outer-membrane configuration of make_ref_ensembles (same records and columns)
    run by the oracle, with the reference's placement law for the compartment and patch
    counts (util/distribute.hpp:102-193 over tet volumes and triangle areas)."""
    from tests.outer_membrane import INITIAL, outer_mesh, outer_model

    mesh = outer_mesh()
    F = flatten(outer_model(ghk=False), mesh)
    S = F["spec_index"]
    sf = F["surf"]
    ss = sf["sspec_index"]
    comp = F["tet_comp"]
    ci, co = F["comp_index"]["cyto"], F["comp_index"]["ecs"]
    inner, outer = np.nonzero(comp == ci)[0], np.nonzero(comp == co)[0]
    times = M.OUTER_RECORDS
    out = np.zeros((n, len(times), len(M.OUTER_COLUMNS)))
    for k in range(n):
        seed = seed0 + k
        o = Oracle(F, seed=seed)

        def place(call, tets, x):
            row = np.zeros(mesh.ntets, dtype=np.uint32)
            row[tets] = distribute(seed, call, F["vol"][tets], x)
            return row

        o.set_counts(S["Ca"], place(0, inner, INITIAL["Ca_in"]) + place(1, outer, INITIAL["Ca_out"]))
        o.set_counts(S["B"], place(2, inner, INITIAL["B"]))
        for call, name in ((3, "P"), (4, "Kc")):
            o.set_tri_counts(ss[name], distribute(seed, call, sf["tri_area"], INITIAL[name]))
        for i, t in enumerate(times):
            if t > 0:
                o.run(t)
            ca = o.get_counts(S["Ca"])
            out[k, i] = [ca[inner].sum(), ca[outer].sum(), o.get_counts(S["CaB"]).sum(),
                         o.get_tri_counts(ss["PCa"]).sum(), o.get_tri_counts(ss["Ko"]).sum()]
    return out


def test_outer_membrane_matches_reference_tetopsplit():
    """Merged SSA units (a patch whose surface reactions take reactants from and put products
    into both volumes, sreac.cpp:305-520): the oracle's ensemble against the reference
    TetOpSplitP's, five columns every 0.5 ms to 10 ms."""
    fx = np.load(os.path.join(GOLD, "ref_ensemble_outer.npz"))
    out = _oracle_outer(200, 9000)
    rep = compare(out, fx["tos"])
    assert rep["ok"], rep
