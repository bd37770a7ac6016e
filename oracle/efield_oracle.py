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


def couple_fast(verts_um, tets):
    """The coupling of couple() for every (tet, vertex) pair at once with batched numpy
    linear algebra (the same flux integration), as a CSR matrix (um)."""
    X = np.asarray(verts_um, dtype=np.float64)
    T = np.asarray(tets, dtype=np.int64)
    others = np.array([[b for b in range(4) if b != a] for a in range(4)])   # (4, 3)
    ve = X[T]                                      # (T, 4, 3)
    own = np.repeat(np.arange(4)[None, :], len(T), axis=0)                   # (T, 4)
    nb = T[:, others]                              # (T, 4, 3) vertex ids of the other three
    m = X[nb] - ve[:, :, None, :]                  # (T, 4, 3 rows, 3)
    m = m.reshape(-1, 3, 3)
    swap = np.linalg.det(m) < 0.0
    m[swap] = m[swap][:, [0, 2, 1]]
    vmi = np.linalg.inv(m)
    f, g = 1.0 / 12.0, 2.0 / 12.0
    ret = np.zeros((m.shape[0], 3))
    for ivert in range(3):
        ip, iq, ir = ivert, (ivert + 1) % 3, (ivert + 2) % 3
        c1 = np.cross(m[:, ip], m[:, iq])
        c2 = np.cross(m[:, iq], m[:, ir])
        c3 = np.cross(m[:, ir], m[:, ip])
        vec = f * c1 + g * c2 + f * c3
        ret += 0.5 * np.einsum("ni,nij->nj", vec, vmi)
    ret[swap] = ret[swap][:, [0, 2, 1]]
    rows = np.repeat(T[np.arange(len(T))[:, None], own].reshape(-1), 3)
    cols = nb.reshape(-1)
    n = len(X)
    return sp.coo_matrix((ret.reshape(-1), (rows, cols)), shape=(n, n)).tocsr()


class EFieldOracle:
    def __init__(self, verts_m, tets, memb_tri_verts, fast=False):
        self.X = np.asarray(verts_m, dtype=np.float64) * 1.0e6
        self.n = len(self.X)
        if fast:
            self.CC = couple_fast(self.X, tets)
        else:
            cc = couple(self.X, np.asarray(tets))
            rows, cols, vals = zip(*[(i, j, w) for (i, j), w in cc.items()])
            self.CC = sp.csr_matrix((vals, (rows, cols)), shape=(self.n, self.n))
        self._lu = {}
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
        # One factorisation per step length, clamp pattern and membrane parameters.
        key = (dt_ms, self.clamped.tobytes(), self.cm, self.g, self.sigma)
        lu = self._lu.get(key)
        if lu is None:
            lu = spla.splu(A[free][:, free].tocsc())
            self._lu = {key: lu}
        dv[free] = lu.solve(b[free])
        self.V = self.V + dv
        return dv
