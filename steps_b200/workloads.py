"""Synthetic Kuhn-cube workloads of the benchmark configurations.

All meshes are n_x * n_y * n_z cubes of side h = 0.1 um, 6 tets per cube.

plain_small   : 10^3 cubes (6,000 tets), A + B <-> C (kf 1e6 /M/s, kb 1 /s),
                D_A = D_B = 1e-12, D_C = 5e-13 m^2/s, A = B = 10,000 placed over the
                compartment by the reference's distribution rule, C = 0.
plain_384k    : 40^3 cubes (384,000 tets), 8 species and 12 reactions drawn from the
                seed (draw order in ``random_network``), species 0-3 Poisson(50) per tet.
batched       : realizations of n^3 cubes, n uniform in {8..30}, the plain_384k network with
                log-normal (sigma 0.2) jitter of every rate constant per realization.
"""
from __future__ import annotations

import numpy as np

from . import geom as sgeom
from . import model as smodel

H = 1.0e-7


def ab_c_model(kf=1.0e6, kb=1.0, dA=1.0e-12, dB=1.0e-12, dC=5.0e-13):
    mdl = smodel.Model()
    A, B, C = smodel.Spec("A", mdl), smodel.Spec("B", mdl), smodel.Spec("C", mdl)
    vs = smodel.Volsys("vsys", mdl)
    smodel.Reac("fwd", vs, lhs=[A, B], rhs=[C], kcst=kf)
    smodel.Reac("bwd", vs, lhs=[C], rhs=[A, B], kcst=kb)
    smodel.Diff("dA", vs, A, dA)
    smodel.Diff("dB", vs, B, dB)
    smodel.Diff("dC", vs, C, dC)
    return mdl


def random_network(seed, nspec=8, n_low=4, n_second=8):
    """8-species / 12-reaction network.  Draw order from numpy PCG64(seed):
      1. D_s = 10**U(-13, -11) for s = 0..7
      2. reaction r0 (zeroth order): product X = int[0, 8), k = 10**U(-2, 2) (M/s)
      3. reactions r1..r3 (first order): X = int[0, 8), Y = int[0, 8) redrawn until Y != X,
         X -> Y, k = 10**U(-2, 2) (/s)
      4. reactions r4..r11 (second order): X, Y, Z = int[0, 8) each, X + Y -> Z,
         k = 10**U(5, 8) (/M/s)
    """
    g = np.random.Generator(np.random.PCG64(seed))
    mdl = smodel.Model()
    sp = [smodel.Spec(f"S{i}", mdl) for i in range(nspec)]
    vs = smodel.Volsys("vsys", mdl)
    D = 10.0 ** g.uniform(-13.0, -11.0, size=nspec)
    for i in range(nspec):
        smodel.Diff(f"d{i}", vs, sp[i], float(D[i]))
    x = int(g.integers(0, nspec))
    smodel.Reac("r0", vs, lhs=[], rhs=[sp[x]], kcst=float(10.0 ** g.uniform(-2.0, 2.0)))
    for r in range(1, n_low):
        x = int(g.integers(0, nspec))
        y = int(g.integers(0, nspec))
        while y == x:
            y = int(g.integers(0, nspec))
        smodel.Reac(f"r{r}", vs, lhs=[sp[x]], rhs=[sp[y]], kcst=float(10.0 ** g.uniform(-2.0, 2.0)))
    for r in range(n_low, n_low + n_second):
        x, y, z = (int(v) for v in g.integers(0, nspec, size=3))
        smodel.Reac(f"r{r}", vs, lhs=[sp[x], sp[y]], rhs=[sp[z]], kcst=float(10.0 ** g.uniform(5.0, 8.0)))
    return mdl


def cube_mesh(nx, ny=None, nz=None, volsys="vsys"):
    mesh = sgeom.kuhn_box(nx, ny or nx, nz or nx, H)
    comp = sgeom.TmComp("comp", mesh, np.arange(mesh.ntets))
    comp.addVolsys(volsys)
    return mesh


def poisson_counts(ntets, mean, seed, nspec=8, nfilled=4):
    """Per-tet Poisson(mean) counts for species 0..nfilled-1, zero for the rest."""
    g = np.random.Generator(np.random.PCG64(seed + 7919))
    rows = np.zeros((nspec, ntets), dtype=np.uint32)
    for s in range(nfilled):
        rows[s] = g.poisson(mean, size=ntets).astype(np.uint32)
    return rows


class ConcatMesh:
    """Several independent meshes laid end to end (batched realizations).  Carries the
    per-tet arrays the solver reads (tet_vol, tet_neighb, tet_area, tet_dist) with
    neighbour indices shifted into the concatenated numbering."""

    def __init__(self, meshes):
        self.parts = meshes
        off = [0]
        for m in meshes:
            off.append(off[-1] + m.ntets)
        self.offsets = np.asarray(off, dtype=np.int32)
        self.ntets = int(off[-1])
        self.tet_vol = np.concatenate([m.tet_vol for m in meshes])
        self.tet_area = np.concatenate([m.tet_area for m in meshes])
        self.tet_dist = np.concatenate([m.tet_dist for m in meshes])
        nb = []
        for m, o in zip(meshes, off[:-1]):
            nb.append(np.where(m.tet_neighb >= 0, m.tet_neighb + o, -1))
        self.tet_neighb = np.concatenate(nb)
        self.comps = {}
        self.patches = {}


def batched_sizes(nreal, seed, lo=8, hi=30):
    g = np.random.Generator(np.random.PCG64(seed + 104729))
    return [int(v) for v in g.integers(lo, hi + 1, size=nreal)]


def batched_mesh(sizes):
    """Concatenate n^3 Kuhn meshes (geometry computed once per distinct n)."""
    cache = {}
    parts = []
    for n in sizes:
        if n not in cache:
            cache[n] = sgeom.kuhn_box(n, n, n, H)
        parts.append(cache[n])
    mesh = ConcatMesh(parts)
    comp = sgeom.TmComp("comp", mesh, np.arange(mesh.ntets))
    comp.addVolsys("vsys")
    return mesh


def rate_jitter(nreal, nreac, seed, sigma=0.2):
    """Per-realization multiplicative log-normal(0, sigma) factors [nreal][nreac]."""
    g = np.random.Generator(np.random.PCG64(seed + 15485863))
    return np.exp(g.normal(0.0, sigma, size=(nreal, nreac)))
