"""TEST INFRASTRUCTURE ONLY — FP64 CPU oracle of the EField step.

Restates, with numpy/scipy, the reference's membrane-potential update:
  * vertex coupling by integrating the linear field's flux through the vertex dual
    cells, tet by tet (src/steps/solver/efield/tetcoupler.cpp:48-300, fluxCoeficients:
    rows to the 3 other vertices, orientation swap on negative determinant, the
    1/12, 2/12, 1/12 weights, the left product with the inverse, the 1/2 of the cross
    product), summed per edge;
  * vertex membrane area = 1/3 of each adjacent membrane triangle (tetmesh.cpp:231-262);
  * the backward-Euler system of dVsolver.hpp:126-180 and its exact (direct) solve.
Units: um, ms, mV, pA, pF, nS.  Only tests and bench.py call it.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def flux_coefficients(ve, ves):
    """Coefficients of the three neighbour potentials in the flux out of ve's dual cell
    inside one tet (tetcoupler.cpp fluxCoeficients)."""
    m = np.array([ves[i] - ve for i in range(3)], dtype=np.float64)
    swap = False
    if np.linalg.det(m) < 0.0:
        m[[1, 2]] = m[[2, 1]]
        swap = True
    vmi = np.linalg.inv(m)
    ret = np.zeros(3)
    f, g = 1.0 / 12.0, 2.0 / 12.0
    for ivert in range(3):
        ip, iq, ir = ivert, (ivert + 1) % 3, (ivert + 2) % 3
        c1 = np.cross(m[ip], m[iq])
        c2 = np.cross(m[iq], m[ir])
        c3 = np.cross(m[ir], m[ip])
        vec = f * c1 + g * c2 + f * c3
        wk = vec @ vmi  # left vector product (matrix.cpp lvprod)
        ret += 0.5 * wk
    if swap:
        ret[1], ret[2] = ret[2], ret[1]
    return ret


def couple(verts_um, tets):
    """Symmetric geometric coupling {(i, j): w} (um) summed over the tets of each edge."""
    acc = {}
    for tet in tets:
        for a in range(4):
            others = [tet[b] for b in range(4) if b != a]
            facs = flux_coefficients(verts_um[tet[a]], [verts_um[o] for o in others])
            for o, w in zip(others, facs):
                acc[(int(tet[a]), int(o))] = acc.get((int(tet[a]), int(o)), 0.0) + w
    return acc


class EFieldOracle:
    def __init__(self, verts_m, tets, memb_tri_verts):
        self.X = np.asarray(verts_m, dtype=np.float64) * 1.0e6
        self.n = len(self.X)
        cc = couple(self.X, np.asarray(tets))
        rows, cols, vals = zip(*[(i, j, w) for (i, j), w in cc.items()])
        self.CC = sp.csr_matrix((vals, (rows, cols)), shape=(self.n, self.n))
        self.area = np.zeros(self.n)
        for t in np.asarray(memb_tri_verts):
            p = self.X[t]
            a = 0.5 * np.linalg.norm(np.cross(p[1] - p[0], p[2] - p[0]))
            self.area[t] += a / 3.0
        self.cm, self.sigma, self.g, self.vext = 0.01, 1.0e3, 0.0, 0.0
        self.V = np.full(self.n, -65.0)
        self.iclamp = np.zeros(self.n)
        self.clamped = np.zeros(self.n, dtype=bool)

    def advance(self, dt_ms):
        C = self.cm * self.area
        G = self.g * self.area
        K = self.CC * self.sigma
        ksum = np.asarray(K.sum(axis=1)).ravel()
        b = self.iclamp + G * (self.vext - self.V) + (K @ self.V - ksum * self.V)
        A = sp.diags(C / dt_ms + G + ksum) - K
        free = ~self.clamped
        dv = np.zeros(self.n)
        Af = A[free][:, free].tocsc()
        dv[free] = spla.spsolve(Af, b[free])
        self.V = self.V + dv
        return dv
