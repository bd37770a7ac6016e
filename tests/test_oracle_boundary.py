"""Diffusion boundaries in the CPU oracle (diffboundary.cpp; Diff::setDiffBndActive and
setDirectionDcst, diff.cpp:307-398): closed boundaries pass nothing, open ones let the
species equilibrate across at the compartments' constants, a direction constant only
acts into its compartment, and molecules are conserved."""
import numpy as np

from oracle.pyoracle import Oracle
from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W
from steps_b200.solver import flatten


def setup(n=6):
    mesh = sgeom.kuhn_box(n, n, n, W.H)
    x = mesh.tet_bary[:, 0]
    left = np.nonzero(x < 0.5 * n * W.H)[0]
    right = np.nonzero(x >= 0.5 * n * W.H)[0]
    a = sgeom.TmComp("left", mesh, left)
    b = sgeom.TmComp("right", mesh, right)
    a.addVolsys("vs")
    b.addVolsys("vs")
    tt = mesh.tri_tets
    side = np.zeros(mesh.ntets, dtype=int)
    side[right] = 1
    both = (tt[:, 0] >= 0) & (tt[:, 1] >= 0)
    btris = np.nonzero(both & (side[np.maximum(tt[:, 0], 0)] != side[np.maximum(tt[:, 1], 0)]))[0]
    sgeom.DiffBoundary("db", mesh, btris)
    mdl = smodel.Model()
    A = smodel.Spec("A", mdl)
    vs = smodel.Volsys("vs", mdl)
    smodel.Diff("dA", vs, A, 2e-12)
    F = flatten(mdl, mesh)
    return mesh, F, left, right


def test_boundary_tables():
    mesh, F, left, right = setup()
    fb = F["face_bnd"].reshape(-1, 4)
    assert (fb >= 0).sum() == 2 * 2 * 6 * 6  # 72 boundary triangles, seen from both sides
    assert set(F["bnd_comps"]) == {0, 1}


def test_closed_open_and_direction():
    mesh, F, left, right = setup()
    ora = Oracle(F, seed=3)
    row = np.zeros(mesh.ntets, dtype=np.uint32)
    row[left] = 40
    ora.set_counts(0, row)
    total = int(row.sum())
    per = ora.period()
    ora.run(20 * per)
    c = ora.get_counts(0)
    assert c[right].sum() == 0 and c.sum() == total
    ora.set_bnd_active(0, 0, True)
    ora.run(ora.time() + 1500 * ora.period())
    c = ora.get_counts(0).astype(np.int64)
    assert c.sum() == total
    assert abs(c[right].sum() / c[left].sum() - len(right) / len(left)) < 0.05
    # Only into "left" (compartment 0): everything ends up there.
    ora.set_bnd_active(0, 0, False)
    ora.set_bnd_dcst(0, 0, 2e-12, direction_comp=0)
    ora.run(ora.time() + 2000 * ora.period())
    c = ora.get_counts(0).astype(np.int64)
    assert c.sum() == total
    assert c[right].sum() < 0.05 * total
