"""Kuhn-cube meshes and the derived geometry the solver consumes (CPU only)."""
import os

import numpy as np
import pytest

from steps_b200 import geom as sgeom
from steps_b200 import workloads as W
from steps_b200.solver import flatten

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("n", [1, 3, 10])
def test_kuhn_box_counts_and_volumes(n):
    m = sgeom.kuhn_box(n, n, n, W.H)
    assert m.ntets == 6 * n ** 3
    assert m.nverts == (n + 1) ** 3
    assert np.allclose(m.tet_vol, W.H ** 3 / 6, rtol=1e-12)
    assert np.isclose(m.getMeshVolume(), (n * W.H) ** 3, rtol=1e-12)
    # boundary triangles: 2 per cube face on the box surface
    assert len(m.getSurfTris()) == 6 * 2 * n * n


def test_neighbours_symmetric_and_interior_scaled_dcst():
    m = sgeom.kuhn_box(6, 6, 6, W.H)
    nb = m.tet_neighb
    for t in range(m.ntets):
        for n in nb[t]:
            if n >= 0:
                assert t in nb[n]
    g = m.tet_area / (m.tet_vol[:, None] * np.where(m.tet_dist > 0, m.tet_dist, np.inf))
    interior = (nb >= 0).all(axis=1)
    G = g[interior].sum(axis=1)
    # sum_f A_f / (V d_f) of an interior Kuhn tet with h = 0.1 um
    assert np.allclose(G, 3.3798e15, rtol=1e-4)


def test_uneven_box_and_tris():
    m = sgeom.kuhn_box(2, 3, 4, W.H)
    assert m.ntets == 6 * 24
    inner = m.tri_tets[:, 1] >= 0
    assert m.ntris == inner.sum() + len(m.getSurfTris())
    assert np.isclose(m.tri_area[m.getSurfTris()].sum(), 2 * (6 + 8 + 12) * W.H ** 2)


def test_reference_sphere_fixture_geometry():
    d = np.load(os.path.join(HERE, "golden", "sphere_rad1_37tets.npz"))
    m = sgeom.Tetmesh(d["verts"], d["tets"])
    assert m.ntets == 37
    assert (m.tet_vol > 0).all()
    assert 2.0e-18 < m.getMeshVolume() < 4.2e-18


def test_flatten_tables():
    m = W.cube_mesh(3)
    F = flatten(W.ab_c_model(), m)
    assert F["spec_names"] == ["A", "B", "C"]
    assert len(F["reacs"]) == 2 and len(F["diffs"]) == 3
    ci, rid, lhs, upd, k = F["reacs"][0]
    assert rid == "fwd" and list(lhs) == [1, 1, 0] and list(upd) == [-1, -1, 1] and k == 1e6


def test_two_compartments_exclusive():
    m = sgeom.kuhn_box(2, 2, 2, W.H)
    sgeom.TmComp("a", m, range(10))
    with pytest.raises(ValueError):
        sgeom.TmComp("b", m, range(5, 20))


def test_replicate_matches_full_construction():
    """geom.replicate tiles a mesh's derived arrays; they equal a Tetmesh built from the
    concatenated vertices and tets."""
    import numpy as np

    from steps_b200 import geom as G

    m = G.kuhn_box(3, 2, 4, 1e-7)
    r = G.replicate(m, 3)
    t = G.Tetmesh(r.verts, r.tets)
    for k in ["tet_vol", "tet_area", "tet_neighb", "tet_dist", "tris", "tet_tri", "tri_tets", "tri_area",
              "tri_bary", "tet_bary"]:
        a, b = getattr(r, k), getattr(t, k)
        assert a.shape == b.shape and np.allclose(a, b), k
    assert list(r.offsets) == [0, m.ntets, 2 * m.ntets, 3 * m.ntets]
    assert len(r.getSurfTris()) == 3 * len(m.getSurfTris())
