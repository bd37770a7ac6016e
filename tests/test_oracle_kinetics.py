"""The reference's analytic TetOpSplit kinetics validation on the CPU oracle: this pins
the oracle's statistics (and, through bit-exact parity, the GPU's) to the analytic
solutions the reference itself is validated against."""
import os

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from steps_b200.solver import flatten
from tests.kinetics import CASES, TPNTS, batch_mesh, check, initial_count, model_for


def distribute(x, weights, nreal, rng):
    """util::distribute_quantity (src/steps/util/distribute.hpp:102-193) for nreal copies
    of the same compartment: floor of the volume-weighted share, then the remainder placed
    by adjusted Pareto order sampling (src/steps/math/sample.hpp:59-200)."""
    w = np.asarray(weights, dtype=np.float64)
    out = np.zeros((nreal, w.size), dtype=np.uint32)
    fl = np.floor(x)
    xs = np.where(rng.random(nreal) < x - fl, fl + 1.0, fl)
    for r in range(nreal):
        xi = xs[r] / w.sum() * w
        base = np.floor(xi)
        pi = xi - base
        out[r] = base.astype(np.uint32)
        rem = int(xs[r] - base.sum())
        if rem <= 0:
            continue
        p = np.minimum(pi * (rem / pi.sum()), 1.0)
        d = np.sum(p * (1 - p))
        ood2 = 1.0 if d == 0 else 1.0 / (d * d)
        nz = np.nonzero(p > 0)[0]
        q = p[nz]
        loga = q * (1 - q) * (q - 0.5) * ood2
        qc = (1 - q) / q * (1 + loga + 0.5 * loga * loga)
        u = rng.random(nz.size)
        keys = qc * u / (1 - u)
        pick = nz[np.argpartition(keys, rem - 1)[:rem]]
        out[r, pick] += 1
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_reference_kinetics_oracle(name):
    _reacs, _diffs, init, niter, _tol = CASES[name]
    mesh, one = batch_mesh(niter)
    vol = one.getMeshVolume()
    F = flatten(model_for(name), mesh)
    ora = Oracle(F, seed=100, realizations=mesh.offsets)
    rng = np.random.default_rng(100)
    for s, (kind, v) in init.items():
        rows = distribute(initial_count(kind, v, vol), one.tet_vol, niter, rng)
        ora.set_counts(F["spec_index"][s], rows.reshape(-1))
    counts = {s: np.zeros((len(TPNTS), niter)) for s in F["spec_names"]}
    for i, t in enumerate(TPNTS):
        ora.run(t)
        for s in F["spec_names"]:
            row = ora.get_counts(F["spec_index"][s]).astype(np.int64)
            counts[s][i] = np.add.reduceat(row, mesh.offsets[:-1])
    fails = check(name, TPNTS, counts, vol)
    assert not fails, fails[:5]
