"""The drop-in TetOpSplitB200 (a steps::solver::API subclass compiled against the reference,
steps_b200/steps_api/tetopsplit_b200.cpp) on the GPU, called through the reference API's
own public methods on the reference's Model / Tetmesh / RNG objects:

  * volume model: run, get/setTetSpecCount, get/setCompSpecCount and
    getBatchTetSpecCountsNP give the same counts, bit for bit, as the Python solver on the
    same mesh, model and seed (same tables, same Philox streams);
  * membrane model: get/setTriSpecCount, get/setPatchSpecCount, get/setVertV, the
    membrane setters and run with the EField;
  * the EField of a passive membrane (channels closed; leak, capacitance, current clamp)
    matches the reference TetOpSplitP's own EField solve (banded direct solver,
    src/steps/solver/efield/dVsolver.hpp:126-180) at every vertex after every step.
"""
import math
import os

import numpy as np
import pytest

from oracle import refsim
from steps_b200 import geom as sgeom
from steps_b200 import model as smodel
from steps_b200.solver import TetOpSplit, flatten
from tests.helpers import make_rng

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not refsim.available(with_dropin=True),
                                                  reason="drop-in library not built")]


def volume_model():
    mdl = smodel.Model()
    sp = [smodel.Spec(f"S{i}", mdl) for i in range(3)]
    vs = smodel.Volsys("vsys", mdl)
    smodel.Reac("R0", vs, lhs=[sp[0], sp[1]], rhs=[sp[2]], kcst=1.0e6)
    smodel.Reac("R1", vs, lhs=[sp[2]], rhs=[sp[0], sp[1]], kcst=2.0)
    for i, d in enumerate((1e-12, 7e-13, 4e-13)):
        smodel.Diff(f"D{i}", vs, sp[i], d)
    return mdl


def test_dropin_volume_model_matches_python_solver(steps_lib):
    mesh = sgeom.kuhn_box(8, 8, 8, 1e-7)
    sgeom.TmComp("comp", mesh, np.arange(mesh.ntets)).addVolsys("vsys")
    mdl = volume_model()
    seed = 11
    py = TetOpSplit(mdl, mesh, make_rng(seed))
    dr = refsim.RefSim(mesh, flatten(mdl, mesh), seed, kind="b200")
    assert dr.solver_name() == "TetOpSplitB200"
    py.setCompSpecCount("comp", "S0", 5000.5)
    dr.set_comp_count(0, 5000.5)
    py.setCompSpecCount("comp", "S1", 3000)
    dr.set_comp_count(1, 3000)
    py.setTetSpecCount(17, "S2", 40)
    dr.set_tet_count(17, "S2", 40)
    assert dr.get_tet_count(17, "S2") == 40
    for k in range(1, 6):
        t = k * 1e-3
        py.run(t)
        dr.run(t)
        assert dr.time() == t
        for i in range(3):
            got = dr.get_tet_counts(i)  # getBatchTetSpecCountsNP through the API
            assert np.array_equal(got, py.getSpecCounts(f"S{i}").astype(np.float64)), (t, i)
            assert dr.get_comp_count(i) == py.getCompSpecCount("comp", f"S{i}")
    # S0 + S2 is conserved: 5000.5 placed (5000 or 5001) plus the 40 S2 set in tet 17.
    assert dr.get_comp_count(0) + dr.get_comp_count(2) in (5040, 5041)


def _tables(vmin, vmax, dv, fopen, fclose):
    n = math.floor((vmax - vmin) / dv) + 1
    v = vmin + dv * np.arange(n)
    return np.array([fopen(x) for x in v]), np.array([fclose(x) for x in v])


def test_dropin_membrane_calls(steps_lib):
    mesh = sgeom.kuhn_box(4, 4, 10, 1e-7)
    vmin, vmax, dv = -0.15, 0.2, 1e-4
    ko, kc = _tables(vmin, vmax, dv, lambda v: 100.0 * math.exp(v / 0.025), lambda v: 100.0 * math.exp(-v / 0.025))
    dr = refsim.RefMemb(mesh, 5, ko, kc, vmin, vmax, dv, 20e-12, 0.05, kind="b200", efopt=1)
    dr.set_memb(-0.065, 0.01, 1.0, 1.0 / 0.3, -0.065, 1e-6)
    surf = dr.surf_tris()
    dr.set_patch_count("C", 2000)
    assert dr.get_patch_count("C") == 2000
    t0 = int(surf[3])
    dr.set_tri_count(t0, "O", 7)
    assert dr.get_tri_count(t0, "O") == 7
    assert dr.get_patch_count("O") == 7
    v0 = int(dr.tri_verts(t0)[0])
    dr.set_vert_v(v0, -0.060)
    assert dr.get_vert_v(v0) == pytest.approx(-0.060, abs=1e-15)
    for v in dr.tri_verts(int(surf[0])):
        dr.set_vert_iclamp(int(v), 1e-12)
    dr.run(2e-4)
    assert dr.time() == pytest.approx(2e-4)
    assert dr.get_patch_count("C") + dr.get_patch_count("O") == 2007
    vs = np.array([dr.get_vert_v(v) for v in range(mesh.nverts)])
    assert np.all(np.isfinite(vs)) and np.ptp(vs) > 0


def test_dropin_passive_efield_matches_reference_efield(steps_lib):
    """Channels stay closed (k_open = 0), so the membrane is passive and the EField
    deterministic: leak, capacitance, a current clamp on one corner's vertices.  The
    drop-in's two-level PCG (FP64, relative residual 1e-10) against TetOpSplitP's banded
    direct solve, every EField step, every vertex."""
    mesh = sgeom.kuhn_box(4, 4, 10, 1e-7)
    vmin, vmax, dv = -0.15, 0.2, 1e-4
    ko, kc = _tables(vmin, vmax, dv, lambda v: 0.0, lambda v: 100.0)
    sims = [refsim.RefMemb(mesh, 3, ko, kc, vmin, vmax, dv, 20e-12, 0.05, kind=k, efopt=1)
            for k in ("tetopsplit", "b200")]
    zmin = np.unique(mesh.tris[mesh.getSurfTris()][np.all(mesh.verts[mesh.tris[mesh.getSurfTris()]][:, :, 2] <= 1e-12,
                                                           axis=1)])
    for s in sims:
        s.set_memb(-0.065, 0.01, 1.0, 1.0 / 0.3, -0.065, 1e-6)
        for v in zmin:
            s.set_vert_iclamp(int(v), 2e-12 / len(zmin))
    worst = 0.0
    for k in range(1, 21):
        t = k * 1e-6
        vv = []
        for s in sims:
            s.run(t)
            vv.append(np.array([s.get_vert_v(v) for v in range(mesh.nverts)]))
        dv_ref = vv[0] + 0.065
        assert np.max(np.abs(dv_ref)) > 0  # the clamp moves the potential
        worst = max(worst, float(np.max(np.abs(vv[1] - vv[0]) / np.abs(vv[0]))))
    assert worst < 1e-8, worst


def test_dropin_outer_membrane_matches_python_solver(steps_lib):
    """A patch between two compartments whose surface reactions reach both volumes (merged
    SSA units), built by the reference's own model classes (SReac with outer-volume
    reactants and products, model/sreac.hpp:67) and run by the drop-in: every tet's counts
    and the patch totals equal the Python solver's on the same model, bit for bit."""
    import sys

    from tests.outer_membrane import INITIAL, outer_mesh, outer_model, outer_split

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_ref_ensembles as MR

    seed = 23
    mesh = outer_mesh()
    _, outer, _ = outer_split(mesh)
    flag = np.zeros(mesh.ntets, np.int32)
    flag[outer] = 1
    dr = refsim.RefOuter(mesh, flag, MR.OUTER_K, seed, kind="b200")
    py = TetOpSplit(outer_model(ghk=False), mesh, make_rng(seed))
    for c, s, n in (("cyto", "Ca", INITIAL["Ca_in"]), ("ecs", "Ca", INITIAL["Ca_out"]), ("cyto", "B", INITIAL["B"])):
        py.setCompSpecCount(c, s, n)
        dr.set_comp(c, s, n)
    for s in ("P", "Kc"):
        py.setPatchSpecCount("memb", s, INITIAL[s])
        dr.set_patch_count(s, INITIAL[s])
    for k in range(1, 7):
        t = k * 0.5e-3
        py.run(t)
        dr.run(t)
        for s in ("B", "Ca", "CaB"):
            g = py.getSpecCounts(s)
            d = np.array([dr.get_tet_count(i, s) for i in range(mesh.ntets)])
            assert np.array_equal(g, d), (t, s)
        for s in ("P", "PCa", "Kc", "Ko"):
            assert py.getPatchSpecCount("memb", s) == dr.get_patch_count(s), (t, s)
    assert py.getCompSpecCount("ecs", "Ca") != INITIAL["Ca_out"]


def test_reference_python_binding_drives_the_gpu_solver(steps_lib):
    """The reference's own Python classes (pysteps/cysteps.pyx: _py_Model, _py_Tetmesh,
    _py_TmComp, the r123 RNG) with the drop-in's binding class _py_TetOpSplitB200
    (steps_b200/steps_api/cysteps_b200.pyx), as a STEPS script would call it: the counts
    equal the Python solver's bit for bit."""
    from tests.test_cysteps_b200 import _module, build_reference_objects

    S = _module()
    mesh = sgeom.kuhn_box(8, 8, 8, 1e-7)
    sgeom.TmComp("comp", mesh, np.arange(mesh.ntets)).addVolsys("vsys")
    seed = 19
    mdl, tm, comp, rng = build_reference_objects(S, mesh, seed)
    dr = S._py_TetOpSplitB200(mdl, tm, rng, 0)
    assert dr.getSolverName() in (b"TetOpSplitB200", "TetOpSplitB200")
    py = TetOpSplit(volume_model(), mesh, make_rng(seed))
    for s, n in (("S0", 5000.5), ("S1", 3000)):
        py.setCompSpecCount("comp", s, n)
        dr.setCompSpecCount("comp", s, n)
    py.setTetSpecCount(17, "S2", 40)
    dr.setTetSpecCount(17, "S2", 40)
    idx = np.arange(mesh.ntets, dtype=np.uint32)
    out = np.zeros(mesh.ntets)
    for k in range(1, 5):
        t = k * 1e-3
        py.run(t)
        dr.run(t)
        assert dr.getTime() == t
        for s in ("S0", "S1", "S2"):
            dr.getBatchTetSpecCountsNP(idx, s, out)
            assert np.array_equal(out, py.getSpecCounts(s).astype(np.float64)), (t, s)
    assert dr.getCompSpecCount("comp", "S0") == py.getCompSpecCount("comp", "S0")
    assert dr.getNSteps() == py.getNSteps()
