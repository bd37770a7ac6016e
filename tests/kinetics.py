"""Analytic kinetics cases of the reference's TetOpSplit validation
(test/validation/API_1/validation_rd_mpi/parallel_spatial_tetopsplit.py): model,
initial state, iteration count, tolerance and the analytic check of each case, on the
reference's 37-tet sphere mesh (tests/golden/sphere_rad1_37tets.npz).

Each case is run as a batch of independent realizations (one per reference iteration):
``run_case`` returns the per-realization compartment counts at the sampling times.
"""
from __future__ import annotations

import math
import os

import numpy as np

from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
NA_REF = 6.0221415e26          # the value the reference test uses for N_A * 1e3
AVOGADRO = 6.02214179e23        # src/steps/math/constants.hpp:45
TPNTS = np.arange(0.0, 1.1, 0.1)


def tolerable(a, b, tol):
    """validation_rd_mpi/tol_funcs.py: relative difference to the mean."""
    return abs(2.0 * (a - b) / (a + b)) <= tol


def sphere():
    d = np.load(os.path.join(HERE, "golden", "sphere_rad1_37tets.npz"))
    return sgeom.Tetmesh(d["verts"], d["tets"])


# name: (reactions [(lhs, rhs, k)], diffusion {spec: D}, initial {spec: ("count"|"conc", v)}, niter, tol)
CASES = {
    "foi": ([(["A"], [], 5.0)], {"A": 0.01e-12}, {"A": ("count", 50.0)}, 100000, 0.02),
    "for": ([(["A"], ["B"], 10.0), (["B"], ["A"], 2.0)], {"A": 0.01e-12, "B": 0.01e-12},
            {"A": ("count", 100000.0)}, 10, 0.01),
    "soA2": ([(["A", "A"], ["C"], 10.0e6)], {"A": 1e-12}, {"A": ("conc", 10.0e-6)}, 1000, 0.03),
    "soAA": ([(["A", "B"], ["C"], 5.0e6)], {"A": 0.2e-12, "B": 0.2e-12},
             {"A": ("conc", 20.0e-6), "B": ("conc", 20.0e-6)}, 1000, 0.02),
    "soAB": ([(["A", "B"], ["C"], 5.0e6)], {"A": 0.1e-12, "B": 0.1e-12},
             {"A": ("conc", 1.0e-6), "B": ("conc", 0.5e-6)}, 1000, 0.01),
    "toA3": ([(["A", "A", "A"], ["C"], 1.0e12)], {"A": 0.2e-12}, {"A": ("conc", 10.0e-6)}, 1000, 0.03),
    "toA2B": ([(["A", "A", "B"], ["C"], 0.1e12)], {"A": 0.1e-12, "B": 0.1e-12},
              {"A": ("conc", 30.0e-6), "B": ("conc", 20.0e-6)}, 1000, 0.01),
}


def model_for(name):
    reacs, diffs, _init, _n, _tol = CASES[name]
    mdl = smodel.Model()
    names = sorted({s for r in reacs for s in r[0] + r[1]} | set(diffs))
    sp = {s: smodel.Spec(s, mdl) for s in names}
    vs = smodel.Volsys("vsys", mdl)
    for i, (l, r, k) in enumerate(reacs):
        smodel.Reac(f"R{i}", vs, lhs=[sp[s] for s in l], rhs=[sp[s] for s in r], kcst=k)
    for s, d in diffs.items():
        smodel.Diff(f"D{s}", vs, sp[s], d)
    return mdl


def batch_mesh(nreal):
    m = sphere()
    mesh = W.ConcatMesh([m] * nreal)
    comp = sgeom.TmComp("comp1", mesh, np.arange(mesh.ntets))
    comp.addVolsys("vsys")
    return mesh, m


def initial_count(kind, v, vol):
    return v if kind == "count" else v * 1.0e3 * vol * AVOGADRO


def check(name, t, counts, vol):
    """Analytic check of the reference test; counts[spec] = array [ntimes][nreal].
    Returns a list of failure messages (empty = pass)."""
    reacs, _d, init, _n, tol = CASES[name]
    fails = []
    conc = {s: c / (1.0e3 * vol * AVOGADRO) for s, c in counts.items()}
    mean = {s: c.mean(axis=1) for s, c in conc.items()}
    k = reacs[0][2]
    for i in range(len(t)):
        ti = t[i]
        if name == "foi":
            if i == 0:
                continue
            n0 = init["A"][1]
            analy = n0 * math.exp(-k * ti)
            std = math.sqrt(n0 * math.exp(-k * ti) * (1 - math.exp(-k * ti)))
            m, s = counts["A"][i].mean(), counts["A"][i].std()
            if not tolerable(analy, m, tol):
                fails.append(f"foi mean t={ti:.1f}: {m} vs {analy}")
            if not tolerable(std, s, tol):
                fails.append(f"foi std t={ti:.1f}: {s} vs {std}")
        elif name == "for":
            if i < 7:
                continue
            c0 = init["A"][1]
            kb = reacs[1][2]
            aeq = c0 * (kb / k) / (1 + kb / k) / (vol * NA_REF) * 1e6
            beq = (c0 / (vol * NA_REF)) * 1e6 - aeq
            for s, eq in (("A", aeq), ("B", beq)):
                if not tolerable(mean[s][i] * 1e6, eq, tol):
                    fails.append(f"for {s} t={ti:.1f}: {mean[s][i] * 1e6} vs {eq}")
        elif name == "soA2":
            a0 = init["A"][1]
            if not tolerable(1.0 / mean["A"][i], 1.0 / a0 + ti * 2 * k, tol):
                fails.append(f"soA2 t={ti:.1f}")
        elif name == "soAA":
            a0 = init["A"][1]
            for s in ("A", "B"):
                if not tolerable(1.0 / mean[s][i], 1.0 / a0 + ti * k, tol):
                    fails.append(f"soAA {s} t={ti:.1f}")
        elif name == "soAB":
            a0, b0 = init["A"][1], init["B"][1]
            lhs = math.log(mean["B"][i] / mean["A"][i])
            rhs = math.log(b0 / a0) - (a0 - b0) * k * ti
            if not tolerable(lhs, rhs, tol):
                fails.append(f"soAB t={ti:.1f}: {lhs} vs {rhs}")
        elif name == "toA3":
            a0 = init["A"][1]
            if not tolerable(1.0 / mean["A"][i] ** 2, 1.0 / a0 ** 2 + ti * 6 * k, tol):
                fails.append(f"toA3 t={ti:.1f}")
        elif name == "toA2B":
            if i == 0:
                continue
            a0, b0 = init["A"][1], init["B"][1]
            dab, dba = a0 - 2 * b0, 2 * b0 - a0
            a, b = mean["A"][i], mean["B"][i]
            line = (-1.0 / dab) * ((-1.0 / dba) * math.log((b / a) / (b0 / a0)) + 1.0 / a - 1.0 / a0)
            if not tolerable(ti * k, line, tol):
                fails.append(f"toA2B t={ti:.1f}: {line} vs {ti * k}")
    return fails
