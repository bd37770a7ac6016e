"""The compiled drop-in TetOpSplitB200 (steps_b200/steps_api/tetopsplit_b200.cpp), a
subclass of the reference's steps::solver::API (src/steps/solver/api.hpp:58), built against
the reference's own headers and objects (oracle/build_ref_tetopsplit.py ->
oracle/_ref/libsteps_ref_b200.so).  CPU checks: it links, defines every pure virtual of
the API and every override the drop-in contract lists, and without a GPU its constructor
raises the reference's own exception."""
import os
import subprocess

import pytest

from oracle import refsim

pytestmark = pytest.mark.skipif(not refsim.available(with_dropin=True),
                                reason="the drop-in library needs the reference tree at build time")

# api.hpp's pure virtual methods and the overrides the drop-in boundary must provide.
REQUIRED = [
    "getSolverName", "getSolverDesc", "getSolverAuthors", "getSolverEmail", "checkpoint", "restore", "reset",
    "run", "advance", "getTime", "getNSteps", "setTemp", "getTemp", "setEfieldDT", "getEfieldDT",
    "getBatchTetSpecCountsNP",
    "_getCompVol", "_getCompSpecCount", "_setCompSpecCount", "_getCompSpecAmount", "_setCompSpecAmount",
    "_getCompSpecConc", "_setCompSpecConc", "_getCompSpecClamped", "_setCompSpecClamped", "_getCompReacK",
    "_setCompReacK", "_getCompReacActive", "_setCompReacActive",
    "_getPatchArea", "_getPatchSpecCount", "_setPatchSpecCount", "_getPatchSpecAmount", "_setPatchSpecAmount",
    "_getPatchSpecClamped", "_setPatchSpecClamped", "_getPatchSReacK", "_setPatchSReacK",
    "_getPatchSReacActive", "_setPatchSReacActive",
    "_getTetVol", "_getTetSpecCount", "_setTetSpecCount", "_getTriArea", "_getTriSpecCount", "_setTriSpecCount",
    "_getVertV", "_setVertV", "_getVertVClamped", "_setVertVClamped", "_setVertIClamp",
    "_setMembPotential", "_setMembCapac", "_setMembVolRes", "_setMembRes",
]


def test_dropin_defines_every_required_override():
    out = subprocess.run(["nm", "-C", "--defined-only", refsim.LIB_B200_PATH], capture_output=True, text=True,
                         check=True).stdout
    defined = set()
    for ln in out.splitlines():
        if "steps::b200::TetOpSplitB200::" in ln:
            name = ln.split("steps::b200::TetOpSplitB200::", 1)[1].split("(", 1)[0].split("[", 1)[0]
            defined.add(name)
    missing = [m for m in REQUIRED if m not in defined]
    assert not missing, missing
    assert "TetOpSplitB200" in defined  # the constructor
    # The vtable of the drop-in is emitted in the library (the class is concrete).
    assert "vtable for steps::b200::TetOpSplitB200" in out


def test_dropin_without_gpu_raises_the_reference_exception():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from steps_b200 import workloads as W
    from steps_b200.solver import flatten

    mesh = W.cube_mesh(3)
    with pytest.raises(RuntimeError) as e:
        refsim.RefSim(mesh, flatten(W.ab_c_model(), mesh), 1, kind="b200")
    msg = str(e.value)
    assert "ProgErr" in msg and "cuda" in msg.lower(), msg
