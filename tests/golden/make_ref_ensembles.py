"""Regenerate the reference ensemble fixtures (run where the reference tree is present).

    python tests/golden/make_ref_ensembles.py [--seeds N] [-j JOBS]

Runs the reference solvers themselves — TetOpSplitP and Tetexact compiled from the
reference's sources by oracle/build_ref_tetopsplit.py and driven through
oracle/refsim.py — and stores their trajectories:

  ref_ensemble_c0.npz      plain small configuration: 10^3 Kuhn cubes of 0.1 um (6,000
                           tets), A + B <-> C (kf 1e6 /M/s, kb 1 /s), D_A = D_B = 1e-12,
                           D_C = 5e-13 m^2/s, A = B = 10,000 placed by the reference's
                           setCompSpecCount, C = 0; compartment counts of A, B, C every
                           1 ms from 0 to 100 ms.  Arrays tos / tetexact [seed][record][species].
  ref_ensemble_spread.npz  pure diffusion of A (same mesh and model, B = C = 0): 10 A in
                           each tet of the first layer of cubes (barycentre x < 0.1 um,
                           6,000 molecules); counts of A in the 10 slabs of 0.1 um along x
                           every 2 ms from 0 to 40 ms.  Arrays tos / tetexact
                           [seed][record][slab].

  ref_ensemble_outer.npz   a membrane between two compartments (tests/outer_membrane.py:
                           6x4x4 Kuhn cubes cut at the middle plane into cyto and ecs, the
                           triangles between them the patch memb; pump and channel surface
                           reactions with inner- and outer-volume reactants and products);
                           Ca in cyto, Ca in ecs, CaB, PCa and Ko every 0.5 ms from 0 to
                           10 ms.  Arrays tos / tetexact [seed][record][column].

  ref_placement.npz        placement law of setCompSpecCount on the reference's 37-tet
                           sphere mesh (tets of unequal volume): 1000.5 molecules of A
                           placed by TetOpSplitP; per-tet counts [seed][tet] for seeds
                           1..PLACEMENT_SEEDS.

Seeds are 1..N for both solvers (each solver's own r123 stream).  Trajectory parity of
the GPU solver with the reference is statistical: the tests compare ensemble means,
variances and distributions against these.
"""
from __future__ import annotations

import argparse
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

C0_RECORDS = np.arange(0, 101) * 1e-3
SPREAD_RECORDS = np.arange(0, 21) * 2e-3
NSLAB = 10
H = 1e-7
PLACEMENT_SEEDS = 4000
PLACEMENT_X = 1000.5


def c0_case():
    from steps_b200 import workloads as W
    from steps_b200.solver import flatten

    mesh = W.cube_mesh(10)
    return mesh, flatten(W.ab_c_model(), mesh)


def spread_initial(mesh):
    """Per-tet initial A of the spread case and each tet's slab index along x."""
    bary = mesh.verts[mesh.tets].mean(axis=1)
    slab = np.clip((bary[:, 0] / H).astype(np.int64), 0, NSLAB - 1)
    a0 = np.where(slab == 0, 10.0, 0.0)
    return a0, slab


def sphere_case():
    from steps_b200 import geom as sgeom
    from steps_b200 import workloads as W
    from steps_b200.solver import flatten

    d = np.load(os.path.join(HERE, "sphere_rad1_37tets.npz"))
    mesh = sgeom.Tetmesh(d["verts"], d["tets"])
    comp = sgeom.TmComp("comp", mesh, np.arange(mesh.ntets))
    comp.addVolsys("vsys")
    return mesh, flatten(W.ab_c_model(), mesh)


def _place_one(seed):
    from oracle.refsim import RefSim

    mesh, F = sphere_case()
    sim = RefSim(mesh, F, seed, kind="tetopsplit")
    sim.set_comp_count(0, PLACEMENT_X)
    return sim.get_tet_counts(0).astype(np.uint16)


OUTER_RECORDS = np.arange(0, 21) * 0.5e-3
OUTER_K = (2.0e-12, 5.0e-13, 5.0e7, 40.0, 1.0e-12, 1.0e8, 60.0, 120.0, 90.0, 2.0e7)
OUTER_COLUMNS = (("cyto", "Ca"), ("ecs", "Ca"), ("cyto", "CaB"), ("memb", "PCa"), ("memb", "Ko"))


def _run_outer(kind, seed):
    from oracle.refsim import RefOuter
    from steps_b200 import geom as sgeom
    from steps_b200 import workloads as W
    from tests.outer_membrane import INITIAL, outer_split

    base = sgeom.kuhn_box(6, 4, 4, W.H)
    _, outer, _ = outer_split(base)
    flag = np.zeros(base.ntets, np.int32)
    flag[outer] = 1
    sim = RefOuter(base, flag, OUTER_K, seed, kind=kind)
    sim.set_comp("cyto", "Ca", INITIAL["Ca_in"])
    sim.set_comp("ecs", "Ca", INITIAL["Ca_out"])
    sim.set_comp("cyto", "B", INITIAL["B"])
    sim.set_patch_count("P", INITIAL["P"])
    sim.set_patch_count("Kc", INITIAL["Kc"])
    out = np.zeros((len(OUTER_RECORDS), len(OUTER_COLUMNS)), dtype=np.uint16)
    for i, t in enumerate(OUTER_RECORDS):
        if t > 0:
            sim.run(t)
        out[i] = [sim.get_patch_count(sp) if c == "memb" else sim.get_comp(c, sp) for c, sp in OUTER_COLUMNS]
    return out


def _run_one(args):
    kind, case, seed = args
    from oracle.refsim import RefSim

    if case == "outer":
        return _run_outer(kind, seed)

    mesh, F = c0_case()
    sim = RefSim(mesh, F, seed, kind=kind)
    if case == "c0":
        sim.set_comp_count(0, 10000)
        sim.set_comp_count(1, 10000)
        out = np.zeros((len(C0_RECORDS), 3), dtype=np.uint16)
        for i, t in enumerate(C0_RECORDS):
            if t > 0:
                sim.run(t)
            out[i] = [sim.get_comp_count(s) for s in range(3)]
        return out
    a0, slab = spread_initial(mesh)
    sim.set_tet_counts(0, a0)
    out = np.zeros((len(SPREAD_RECORDS), NSLAB), dtype=np.uint16)
    for i, t in enumerate(SPREAD_RECORDS):
        if t > 0:
            sim.run(t)
        c = sim.get_tet_counts(0)
        out[i] = np.bincount(slab, weights=c, minlength=NSLAB).astype(np.uint16)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=200)
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--placement-only", action="store_true")
    ap.add_argument("--cases", default="placement,c0,spread,outer", help="comma-separated cases to regenerate")
    a = ap.parse_args()
    from oracle import build_ref_tetopsplit

    if build_ref_tetopsplit.build() is None:
        raise SystemExit("the reference tree is absent")
    ctx = mp.get_context("spawn")
    cases = a.cases.split(",")
    if "placement" in cases:
        with ctx.Pool(a.j) as pool:
            pl = np.stack(pool.map(_place_one, range(1, PLACEMENT_SEEDS + 1)))
        np.savez_compressed(os.path.join(HERE, "ref_placement.npz"), counts=pl, x=PLACEMENT_X,
                            seeds=np.arange(1, PLACEMENT_SEEDS + 1))
        print("placement", pl.shape, flush=True)
    if a.placement_only:
        return
    seeds = list(range(1, a.seeds + 1))
    for case, recs in (("c0", C0_RECORDS), ("spread", SPREAD_RECORDS), ("outer", OUTER_RECORDS)):
        if case not in cases:
            continue
        res = {}
        for kind in ("tetopsplit", "tetexact"):
            with ctx.Pool(a.j) as pool:
                res["tos" if kind == "tetopsplit" else kind] = np.stack(
                    pool.map(_run_one, [(kind, case, s) for s in seeds]))
            print(case, kind, res["tos" if kind == "tetopsplit" else kind].shape, flush=True)
        np.savez_compressed(os.path.join(HERE, f"ref_ensemble_{case}.npz"), times=recs, seeds=np.array(seeds),
                            **res)


if __name__ == "__main__":
    main()
