"""The reference's analytic TetOpSplit kinetics validation on the GPU solver.

Every reference iteration becomes one realization of a batched solver (the 37-tet sphere
mesh repeated niter times), with the reference's seed, iteration counts, sampling times
and tolerances (validation_rd_mpi/parallel_spatial_tetopsplit.py).
"""
import numpy as np
import pytest

from steps_b200.solver import TetOpSplit
from tests.helpers import make_rng
from tests.kinetics import CASES, TPNTS, batch_mesh, check, initial_count, model_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(CASES))
def test_reference_kinetics(steps_lib, name):
    _reacs, _diffs, init, niter, _tol = CASES[name]
    mesh, one = batch_mesh(niter)
    vol = one.getMeshVolume()
    sim = TetOpSplit(model_for(name), mesh, make_rng(100), realizations=mesh.offsets)
    for s, (kind, v) in init.items():
        sim.setCompSpecCount("comp1", s, initial_count(kind, v, vol))
    counts = {s: np.zeros((len(TPNTS), niter)) for s in sim.spec_names}
    for i, t in enumerate(TPNTS):
        sim.run(t)
        for s in sim.spec_names:
            row = sim.getSpecCounts(s).astype(np.int64)
            counts[s][i] = np.add.reduceat(row, mesh.offsets[:-1])
    fails = check(name, TPNTS, counts, vol)
    assert not fails, fails[:5]
