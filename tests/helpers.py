"""Shared builders for the parity tests: a GPU solver and the CPU oracle on the same
tables, seeded identically, started from the same counts."""
from __future__ import annotations

import numpy as np

from oracle.pyoracle import Oracle
from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import rng as srng
from steps_b200 import workloads as W
from steps_b200.solver import TetOpSplit


def make_rng(seed):
    r = srng.create("r123", 512)
    r.initialize(seed)
    return r


def pair(mdl, mesh, seed, realizations=None, block=128):
    """(GPU solver, oracle) over the same model and mesh."""
    sim = TetOpSplit(mdl, mesh, make_rng(seed), realizations=realizations, block=block)
    ora = Oracle(sim.tables, seed=seed, realizations=realizations)
    return sim, ora


def sync_counts(sim, ora):
    for i, s in enumerate(sim.spec_names):
        ora.set_counts(i, sim.getSpecCounts(s))


def assert_same(sim, ora, where=""):
    for i, s in enumerate(sim.spec_names):
        g = sim.getSpecCounts(s)
        o = ora.get_counts(i)
        if not np.array_equal(g, o):
            idx = np.nonzero(g != o)[0]
            raise AssertionError(
                f"{where}: species {s} differs in {idx.size} tets, first {idx[:5].tolist()}: "
                f"gpu {g[idx[:5]].tolist()} oracle {o[idx[:5]].tolist()}")


def two_comp_mesh(n=6):
    """n^3 Kuhn box split into two compartments at the x mid-plane."""
    mesh = sgeom.kuhn_box(n, n, n, W.H)
    x = mesh.tet_bary[:, 0]
    left = np.nonzero(x < 0.5 * n * W.H)[0]
    right = np.nonzero(x >= 0.5 * n * W.H)[0]
    a = sgeom.TmComp("left", mesh, left)
    b = sgeom.TmComp("right", mesh, right)
    a.addVolsys("vl")
    b.addVolsys("vr")
    return mesh


def two_comp_model():
    mdl = smodel.Model()
    A, B, C = smodel.Spec("A", mdl), smodel.Spec("B", mdl), smodel.Spec("C", mdl)
    vl = smodel.Volsys("vl", mdl)
    vr = smodel.Volsys("vr", mdl)
    smodel.Reac("f", vl, lhs=[A, B], rhs=[C], kcst=2.0e6)
    smodel.Reac("b", vl, lhs=[C], rhs=[A, B], kcst=5.0)
    smodel.Reac("dec", vr, lhs=[A], rhs=[], kcst=3.0)
    smodel.Reac("pro", vr, lhs=[], rhs=[B], kcst=50.0)
    smodel.Diff("dAl", vl, A, 1.0e-12)
    smodel.Diff("dBl", vl, B, 2.0e-12)
    smodel.Diff("dAr", vr, A, 4.0e-12)
    smodel.Diff("dCr", vr, C, 1.0e-12)
    return mdl
