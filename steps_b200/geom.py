"""Tetrahedral mesh geometry for the solver boundary.

Mirrors what the reference's ``steps.geom.Tetmesh`` provides to TetOpSplitP
(src/steps/geom/tetmesh.hpp:113, constructor from vertex/tet arrays at :151):
tet volumes, the four face areas, the four face neighbours and the
barycentre-to-barycentre distances (src/steps/mpi/tetopsplit/tetopsplit.cpp:644-681),
plus the triangles and compartments/patches built on it
(src/steps/geom/tmcomp.hpp, tmpatch.hpp).

Face ``f`` of a tet is the face opposite its vertex ``f``.
"""
from __future__ import annotations

import numpy as np

UNKNOWN_TET = -1

_FACE_VERTS = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]], dtype=np.int64)


class Tetmesh:
    """Vertices (m) and tetrahedra (vertex indices), with derived geometry."""

    def __init__(self, verts, tets):
        self.verts = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 3))
        self.tets = np.ascontiguousarray(np.asarray(tets, dtype=np.int64).reshape(-1, 4))
        self.ntets = int(self.tets.shape[0])
        self.nverts = int(self.verts.shape[0])
        if self.ntets == 0:
            raise ValueError("mesh has no tetrahedra")
        if self.tets.min() < 0 or self.tets.max() >= self.nverts:
            raise ValueError("tet vertex index out of range")
        self.comps = {}
        self.patches = {}
        self._compute_geometry()
        self._build_tris()

    # -- geometry -----------------------------------------------------------
    def _compute_geometry(self):
        v = self.verts[self.tets]                       # (T, 4, 3)
        e1, e2, e3 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]
        self.tet_vol = np.abs(np.einsum("ij,ij->i", e1, np.cross(e2, e3))) / 6.0
        self.tet_bary = v.mean(axis=1)
        fv = self.tets[:, _FACE_VERTS]                  # (T, 4, 3) vertex ids per face
        p = self.verts[fv]                              # (T, 4, 3, 3)
        cr = np.cross(p[:, :, 1] - p[:, :, 0], p[:, :, 2] - p[:, :, 0])
        self.tet_area = 0.5 * np.linalg.norm(cr, axis=2)  # (T, 4)
        # Face neighbours by matching sorted vertex triples.
        key = np.sort(fv.reshape(-1, 3), axis=1)
        order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
        ks = key[order]
        same = np.all(ks[1:] == ks[:-1], axis=1)
        if np.any(same[1:] & same[:-1]):
            raise ValueError("a face is shared by more than two tetrahedra")
        neighb = np.full(self.ntets * 4, UNKNOWN_TET, dtype=np.int64)
        i = np.nonzero(same)[0]
        a, b = order[i], order[i + 1]
        neighb[a] = b // 4
        neighb[b] = a // 4
        self.tet_neighb = neighb.reshape(self.ntets, 4)
        self.face_key = key.reshape(self.ntets, 4, 3)
        dist = np.zeros((self.ntets, 4))
        has = self.tet_neighb >= 0
        tn = np.where(has, self.tet_neighb, 0)
        d = np.linalg.norm(self.tet_bary[tn] - self.tet_bary[:, None, :], axis=2)
        dist[has] = d[has]
        self.tet_dist = dist

    def _build_tris(self):
        """Unique triangles of the mesh with their (up to two) tets."""
        key = self.face_key.reshape(-1, 3)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        self.tris = uniq
        self.ntris = int(uniq.shape[0])
        self.tet_tri = inv.reshape(self.ntets, 4)
        tri_tets = np.full((self.ntris, 2), UNKNOWN_TET, dtype=np.int64)
        owner = np.arange(self.ntets * 4) // 4
        order = np.argsort(inv, kind="stable")
        sinv = inv[order]
        starts = np.r_[0, np.nonzero(np.diff(sinv))[0] + 1]
        tri_tets[sinv[starts], 0] = owner[order[starts]]
        second = starts + 1
        ok = second < len(sinv)
        ok[ok] = sinv[second[ok]] == sinv[starts[ok]]
        tri_tets[sinv[starts[ok]], 1] = owner[order[second[ok]]]
        self.tri_tets = tri_tets
        p = self.verts[self.tris]
        self.tri_area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)
        self.tri_bary = p.mean(axis=1)

    # -- reference-style accessors (tetmesh.hpp) ------------------------------
    def getTetVol(self, t):
        return float(self.tet_vol[t])

    def getTetTetNeighb(self, t):
        return [int(x) for x in self.tet_neighb[t]]

    def getTetTriNeighb(self, t):
        return [int(x) for x in self.tet_tri[t]]

    def getTetBarycenter(self, t):
        return [float(x) for x in self.tet_bary[t]]

    def getTriArea(self, tri):
        return float(self.tri_area[tri])

    def getTriTetNeighb(self, tri):
        return [int(x) for x in self.tri_tets[tri]]

    def getTriVerts(self, tri):
        return [int(x) for x in self.tris[tri]]

    def getBoundMin(self):
        return [float(x) for x in self.verts.min(axis=0)]

    def getBoundMax(self):
        return [float(x) for x in self.verts.max(axis=0)]

    def getMeshVolume(self):
        return float(self.tet_vol.sum())

    def getSurfTris(self):
        return np.nonzero(self.tri_tets[:, 1] == UNKNOWN_TET)[0]


class TmComp:
    """A compartment: a set of tets with volume systems (src/steps/geom/tmcomp.hpp)."""

    def __init__(self, id, mesh, tets):
        self.id = id
        self.mesh = mesh
        self.tets = np.unique(np.asarray(list(tets) if not isinstance(tets, np.ndarray) else tets,
                                         dtype=np.int64))
        if self.tets.size == 0:
            raise ValueError("compartment has no tetrahedra")
        if self.tets[0] < 0 or self.tets[-1] >= mesh.ntets:
            raise ValueError("compartment tet index out of range")
        for other in mesh.comps.values():
            if np.intersect1d(other.tets, self.tets).size:
                raise ValueError("a tetrahedron belongs to two compartments")
        self.volsys = []
        mesh.comps[id] = self

    def addVolsys(self, name):
        if name not in self.volsys:
            self.volsys.append(name)

    def getVol(self):
        return float(self.mesh.tet_vol[self.tets].sum())


class TmPatch:
    """A patch: a set of triangles with surface systems (src/steps/geom/tmpatch.hpp)."""

    def __init__(self, id, mesh, tris, icomp, ocomp=None):
        self.id = id
        self.mesh = mesh
        self.tris = np.unique(np.asarray(tris, dtype=np.int64))
        self.icomp = icomp
        self.ocomp = ocomp
        self.surfsys = []
        mesh.patches[id] = self

    def addSurfsys(self, name):
        if name not in self.surfsys:
            self.surfsys.append(name)

    def getArea(self):
        return float(self.mesh.tri_area[self.tris].sum())


class Memb:
    """A membrane for the EField: the triangles of its patches (src/steps/geom/memb.hpp:49).
    The conducting volume is every tet of every compartment."""

    def __init__(self, id, mesh, patches, supplementary_comps=None, opt_method=1, search_percent=100.0,
                 opt_file_name=""):
        self.id = id
        self.mesh = mesh
        self.patches = list(patches)
        tris = np.unique(np.concatenate([p.tris for p in self.patches])) if self.patches else np.zeros(0, int)
        self.tris = tris.astype(np.int64)
        if not hasattr(mesh, "membs"):
            mesh.membs = {}
        mesh.membs[id] = self


class DiffBoundary:
    """Triangles between two compartments across which chosen species may diffuse
    (src/steps/geom/diffboundary.hpp; activated per species on the solver)."""

    def __init__(self, id, mesh, tris):
        self.id = id
        self.mesh = mesh
        self.tris = np.asarray(tris, dtype=np.int64)
        owner = {}
        for name, c in mesh.comps.items():
            for t in c.tets:
                owner[int(t)] = name
        comps = set()
        for t in self.tris:
            a, b = mesh.tri_tets[t]
            if a < 0 or b < 0:
                raise ValueError(f"diffusion boundary triangle {t} is on the mesh surface")
            ca = owner.get(int(a))
            cb = owner.get(int(b))
            if ca is None or cb is None or ca == cb:
                raise ValueError(f"diffusion boundary triangle {t} does not join two compartments")
            comps.add(tuple(sorted((ca, cb))))
        if len(comps) != 1:
            raise ValueError("a diffusion boundary joins exactly two compartments")
        self.comps = next(iter(comps))
        if not hasattr(mesh, "diffbounds"):
            mesh.diffbounds = {}
        mesh.diffbounds[id] = self


def replicate(mesh, n, gap=None):
    """n disjoint copies of mesh in one Tetmesh (batched realizations of one geometry): copy r
    is shifted along x by r * (extent + gap) and owns tets [r T, (r + 1) T); every derived
    array is tiled from the original instead of recomputed.  offsets holds the
    realization tet ranges."""
    T, V, M = mesh.ntets, mesh.nverts, mesh.ntris
    lo, hi = mesh.verts.min(axis=0), mesh.verts.max(axis=0)
    step = (hi[0] - lo[0]) + (gap if gap is not None else 0.25 * (hi[0] - lo[0]))
    shift = np.zeros((n, 1, 3))
    shift[:, 0, 0] = step * np.arange(n)

    def tile_idx(a, per):
        r = np.arange(n).reshape((n,) + (1,) * a.ndim) * per
        out = np.where(a[None] >= 0, a[None] + r, a[None])
        return out.reshape((-1,) + a.shape[1:])

    m = object.__new__(Tetmesh)
    m.verts = np.ascontiguousarray((mesh.verts[None] + shift).reshape(-1, 3))
    m.tets = np.ascontiguousarray(tile_idx(mesh.tets, V))
    m.ntets, m.nverts = n * T, n * V
    m.comps, m.patches = {}, {}
    m.tet_vol = np.tile(mesh.tet_vol, n)
    m.tet_bary = (mesh.tet_bary[None] + shift).reshape(-1, 3)
    m.tet_area = np.tile(mesh.tet_area, (n, 1))
    m.tet_neighb = tile_idx(mesh.tet_neighb, T)
    m.face_key = tile_idx(mesh.face_key, V)
    m.tet_dist = np.tile(mesh.tet_dist, (n, 1))
    m.tris = tile_idx(mesh.tris, V)
    m.ntris = n * M
    m.tet_tri = tile_idx(mesh.tet_tri, M)
    m.tri_tets = tile_idx(mesh.tri_tets, T)
    m.tri_area = np.tile(mesh.tri_area, n)
    m.tri_bary = (mesh.tri_bary[None] + shift).reshape(-1, 3)
    m.offsets = np.arange(n + 1, dtype=np.int32) * T
    return m


def kuhn_box(nx, ny, nz, h=1.0e-7, origin=(0.0, 0.0, 0.0)):
    """Box of nx*ny*nz cubes of side h, each cut into 6 tets along its main diagonal
    (Kuhn / Freudenthal triangulation; conforming across cubes).

    Tets are numbered cube-major (x fastest), 6 per cube.  Returns a Tetmesh."""
    ix, iy, iz = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    verts = np.stack([ix.ravel(order="F"), iy.ravel(order="F"), iz.ravel(order="F")], axis=1)
    verts = verts.astype(np.float64) * h + np.asarray(origin, dtype=np.float64)

    def vid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    cz, cy, cx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cx, cy, cz = cx.ravel(), cy.ravel(), cz.ravel()
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = np.empty((cx.size, 6, 4), dtype=np.int64)
    for p, perm in enumerate(perms):
        cur = [cx.copy(), cy.copy(), cz.copy()]
        tets[:, p, 0] = vid(*cur)
        for s in range(3):
            cur[perm[s]] = cur[perm[s]] + 1
            tets[:, p, s + 1] = vid(*cur)
    return Tetmesh(verts, tets.reshape(-1, 4))
