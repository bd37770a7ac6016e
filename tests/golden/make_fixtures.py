"""Regenerate the golden fixtures from the reference tree (run in the build container only).

    python tests/golden/make_fixtures.py

  sphere_rad1_37tets.npz  vertices (m, scale 1e-6 as the reference test imports them) and
                          tets of test/validation/API_1/validation_rd_mpi/meshes/
                          sphere_rad1_37tets.inp, the mesh of the reference's analytic
                          TetOpSplit kinetics validation (parallel_spatial_tetopsplit.py).
  philox_kat.json         Philox4x32 known answers (8 and 10 rounds) from the reference's vendored Random123
                          (oracle/ref_philox_kat.c, built by oracle/build_oracle.py).
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("STEPS_REFERENCE", "/root/reference")


def read_abaqus(path, scale):
    """Nodes and C3D4 elements of an Abaqus .inp file (1-based ids in the file)."""
    nodes, elems, mode = {}, [], None
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("**"):
                continue
            if s.startswith("*"):
                u = s.upper()
                mode = "node" if u.startswith("*NODE") else ("elem" if u.startswith("*ELEMENT") else None)
                continue
            parts = [p for p in s.replace(",", " ").split()]
            if mode == "node":
                nodes[int(parts[0])] = [float(x) * scale for x in parts[1:4]]
            elif mode == "elem":
                elems.append([int(x) for x in parts[1:5]])
    ids = sorted(nodes)
    remap = {nid: i for i, nid in enumerate(ids)}
    verts = np.array([nodes[i] for i in ids])
    tets = np.array([[remap[n] for n in e] for e in elems], dtype=np.int64)
    return verts, tets


def read_steps_xml(path):
    """Vertices and tets of a STEPS XML mesh (<nodes><node><coords>, <tetrahedrons><tet><nodes>)."""
    import re

    txt = open(path).read()
    nodes = re.search(r"<nodes size\s*=\s*\"\d+\">(.*?)</nodes>\s*<triangles", txt, re.S).group(1)
    verts = np.array([[float(x) for x in m.split(",")] for m in re.findall(r"<coords>(.*?)</coords>", nodes)])
    tets_blk = re.search(r"<tetrahedrons.*?</tetrahedrons>", txt, re.S).group(0)
    tets = np.array([[int(x) for x in m.split(",")] for m in re.findall(r"<nodes>(.*?)</nodes>", tets_blk)],
                    dtype=np.int64)
    return verts, tets


def main():
    inp = os.path.join(REF, "test/validation/API_1/validation_rd_mpi/meshes/sphere_rad1_37tets.inp")
    v, t = read_abaqus(inp, 1.0e-6)
    np.savez(os.path.join(HERE, "sphere_rad1_37tets.npz"), verts=v, tets=t)
    print("sphere:", v.shape, t.shape)
    # Rallpack1 passive cable: mesh and the reference V(t) at 0 um and 1000 um
    # (test/validation/API_1/validation_efield/, used by test_rallpack1_membres.py).
    ef = os.path.join(REF, "test/validation/API_1/validation_efield")
    v, t = read_steps_xml(os.path.join(ef, "meshes/axon_cube_L1000um_D866nm_1978tets.xml"))
    v0 = np.loadtxt(os.path.join(ef, "data/rallpack1_correct/v0"))
    vx = np.loadtxt(os.path.join(ef, "data/rallpack1_correct/vx"))
    np.savez_compressed(os.path.join(HERE, "rallpack1.npz"), verts=v, tets=t, v0=v0, vx=vx)
    print("rallpack1:", v.shape, t.shape, v0.shape, vx.shape)
    sys.path.insert(0, ROOT)
    from oracle import build_oracle

    exe = build_oracle.build_ref(force=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        f.write(out)
    print("philox_kat.json written")


if __name__ == "__main__":
    main()
