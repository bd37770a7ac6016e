"""The EField oracle (CPU): the reference's flux-integration coupling
(tetcoupler.cpp fluxCoeficients, restated in oracle/efield_oracle.py) equals the
linear-FEM stiffness the GPU library computes, and the direct solve charges a membrane
patch as C dV/dt = I predicts."""
import os

import numpy as np

from oracle.efield_oracle import EFieldOracle, couple
from steps_b200 import geom as sgeom

HERE = os.path.dirname(os.path.abspath(__file__))


def fem_coupling(X, tets):
    acc = {}
    for tet in tets:
        J = (X[tet[1:]] - X[tet[0]]).T
        inv = np.linalg.inv(J)
        gr = np.vstack([-inv.sum(axis=0), inv])
        vol = abs(np.linalg.det(J)) / 6.0
        for i in range(4):
            for j in range(4):
                if i != j:
                    acc[(int(tet[i]), int(tet[j]))] = acc.get((int(tet[i]), int(tet[j])), 0.0) - vol * gr[i] @ gr[j]
    return acc


def test_flux_coupling_equals_fem_stiffness_kuhn():
    m = sgeom.kuhn_box(2, 2, 3, 1e-7)
    X = m.verts * 1e6
    a, b = couple(X, m.tets), fem_coupling(X, m.tets)
    assert a.keys() == b.keys()
    assert max(abs(a[k] - b[k]) for k in a) < 1e-14
    # symmetric, and Kuhn tets are non-obtuse: no negative couplings
    assert all(abs(a[(i, j)] - a[(j, i)]) < 1e-15 for (i, j) in a)
    assert min(a.values()) > -1e-15


def test_flux_coupling_equals_fem_stiffness_rallpack_mesh():
    d = np.load(os.path.join(HERE, "golden", "rallpack1.npz"))
    X, tets = d["verts"] * 1e6, d["tets"][:300]
    a, b = couple(X, tets), fem_coupling(X, tets)
    assert max(abs(a[k] - b[k]) / max(abs(b[k]), 1e-12) for k in a) < 1e-9


def test_oracle_charges_membrane():
    m = sgeom.kuhn_box(2, 2, 2, 1e-7)
    surf = m.getSurfTris()
    ora = EFieldOracle(m.verts, m.tets, m.tris[surf])
    ora.iclamp[:] = 0.0
    ora.iclamp[0] = 1.0  # pA
    total_c = ora.cm * ora.area.sum()
    v0 = ora.V.mean()
    for _ in range(20):
        ora.advance(1e-3)
    # all vertices are membrane vertices here; charge conservation: sum C dV = I t
    dq = (ora.cm * ora.area * (ora.V - (-65.0))).sum()
    assert abs(dq - 1.0 * 20e-3) < 1e-9
    assert ora.V.mean() > v0 and total_c > 0


def test_vectorised_coupling_equals_the_loop():
    """couple_fast (batched over every tet and vertex) gives the coupling of couple()."""
    from oracle.efield_oracle import couple, couple_fast
    from steps_b200 import geom as sgeom

    mesh = sgeom.kuhn_box(3, 2, 4, 1e-7)
    X = mesh.verts * 1e6
    cc = couple(X, mesh.tets)
    fast = couple_fast(X, mesh.tets).tocoo()
    got = {(int(i), int(j)): float(v) for i, j, v in zip(fast.row, fast.col, fast.data)}
    assert set(got) == set(cc)
    for k, v in cc.items():
        assert abs(got[k] - v) <= 1e-12 * max(1.0, abs(v)), k
