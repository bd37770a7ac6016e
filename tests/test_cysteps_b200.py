"""The drop-in's Python binding class inside the reference's own Python binding (CPU).

oracle/build_ref_tetopsplit.py cythonizes steps_b200/steps_api/cysteps_b200.pyx, which
includes the reference's pysteps/cysteps.pyx (model, geometry, RNG and solver classes)
and adds _py_TetOpSplitB200 with _py_TetOpSplitP's constructor (pysteps/cysteps_mpi.pyx:74),
and links it to the reference library and the drop-in (oracle/_ref/cysteps_b200.*).  Here:
the module loads, the reference's Python classes build a model and mesh and run the
reference Tetexact, and the drop-in class carries the whole _py_TetAPI surface.  The GPU run
through it is in tests/test_gpu_dropin_api.py.
"""
import importlib
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref")


def _module():
    import sysconfig

    path = os.path.join(REF, "cysteps_b200" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not os.path.exists(path):
        pytest.skip("binding module not built (needs the reference tree and Cython)")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    return importlib.import_module("cysteps_b200")


def build_reference_objects(S, mesh, seed):
    """A + B <-> C with diffusion of A on mesh, through the reference's own Python classes."""
    mdl = S._py_Model()
    a, b, c = S._py_Spec("S0", mdl), S._py_Spec("S1", mdl), S._py_Spec("S2", mdl)
    vs = S._py_Volsys("vsys", mdl)
    S._py_Reac("R0", vs, [a, b], [c], 1.0e6)
    S._py_Reac("R1", vs, [c], [a, b], 2.0)
    S._py_Diff("D0", vs, a, 1.0e-12)
    S._py_Diff("D1", vs, b, 7.0e-13)
    S._py_Diff("D2", vs, c, 4.0e-13)
    tm = S._py_Tetmesh(mesh.verts.reshape(-1).tolist(), mesh.tets.reshape(-1).tolist())
    comp = S._py_TmComp("comp", tm, list(range(mesh.ntets)))
    comp.addVolsys("vsys")
    rng = S._py_rng_create("r123", 512)
    rng.initialize(seed)
    return mdl, tm, comp, rng


def test_binding_module_runs_the_reference_tetexact():
    from steps_b200 import geom as sgeom

    S = _module()
    mesh = sgeom.kuhn_box(4, 4, 4, 1e-7)
    mdl, tm, comp, rng = build_reference_objects(S, mesh, 3)
    sim = S._py_Tetexact(mdl, tm, rng, 0)
    sim.setCompSpecCount("comp", "S0", 1000)
    sim.setCompSpecCount("comp", "S1", 800)
    sim.run(1e-3)
    a, c = sim.getCompSpecCount("comp", "S0"), sim.getCompSpecCount("comp", "S2")
    assert a + c == 1000 and c > 0


def test_dropin_class_has_the_solver_api():
    S = _module()
    cls = S._py_TetOpSplitB200
    assert issubclass(cls, S._py_TetAPI)
    for name in ("run", "advance", "reset", "getTime", "getTetSpecCount", "setTetSpecCount", "getCompSpecCount",
                 "setCompSpecCount", "getTriSpecCount", "setTriSpecCount", "getPatchSpecCount", "getVertV",
                 "setVertV", "getBatchTetSpecCountsNP", "checkpoint", "restore", "getSolverName", "getNSteps",
                 "setEfieldDT", "getTemp"):
        assert hasattr(cls, name), name


def test_tetode_standin_raises():
    """TetODE needs SUNDIALS, which is absent: its stand-in raises instead."""
    from steps_b200 import geom as sgeom

    S = _module()
    mesh = sgeom.kuhn_box(2, 2, 2, 1e-7)
    mdl, tm, comp, rng = build_reference_objects(S, mesh, 1)
    with pytest.raises(RuntimeError, match="SUNDIALS"):
        S._py_TetODE(mdl, tm, rng)
    assert np.isfinite(tm.getMeshVolume())
