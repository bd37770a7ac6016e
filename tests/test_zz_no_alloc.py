"""The allocation-free entry point sg_run_noalloc against the solver object.

sg_run_noalloc exists for callers that cannot call cudaMalloc (hosts that hand out device
memory only from their own pool allocator, loops that must not pay an allocation's
device-wide synchronisation on every call).  This
test is that kind of caller: it owns every device buffer (made here with torch), calls
the entry point twice in a row through the C ABI, and checks that the counts match the
ones the ordinary solver (sg_create / sg_setup / sg_run) produces for the same seed and
times, bit for bit (integer counts, as in every parity test).

It sits in its own file named to be collected last, so that a run stopping at the first
failure has already run every other test; it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

from steps_b200 import workloads as W
from steps_b200.solver import TetOpSplit, flatten
from tests.helpers import make_rng

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.sg_run_noalloc
    f.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_double,
                  C.c_double, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


def test_noalloc_matches_solver_on_two_calls(steps_lib):
    import torch

    run_noalloc = _bind(steps_lib)
    seed = 21
    mesh = W.cube_mesh(8)
    mdl = W.ab_c_model()
    sim = TetOpSplit(mdl, mesh, make_rng(seed))
    sim.setCompSpecCount("comp", "A", 6000)
    sim.setCompSpecCount("comp", "B", 4000)
    S, T = len(sim.spec_names), mesh.ntets
    rows = np.stack([sim.getSpecCounts(s) for s in sim.spec_names])

    F = flatten(mdl, mesh)
    R = len(F["reacs"])
    lhs = np.ascontiguousarray(np.stack([r[2] for r in F["reacs"]]), dtype=np.uint32)
    upd = np.ascontiguousarray(np.stack([r[3] for r in F["reacs"]]), dtype=np.int32)
    kcst = np.ascontiguousarray([r[4] for r in F["reacs"]], dtype=np.float64)
    dcst = np.zeros(S, dtype=np.float64)
    for (_c, _d, s, d) in F["diffs"]:
        dcst[s] = d

    dev = torch.device("cuda", 0)
    counts = torch.from_numpy(rows.view(np.int32).copy()).to(dev)
    vol = torch.from_numpy(F["vol"]).to(dev)
    neighb = torch.from_numpy(F["neighb"]).to(dev)
    area = torch.from_numpy(F["area"]).to(dev)
    dist = torch.from_numpy(F["dist"]).to(dev)
    torch.cuda.synchronize()

    def call(t0, t1, w0):
        nwin, per = C.c_uint64(), C.c_double()
        st = run_noalloc(T, S, R, counts.data_ptr(), vol.data_ptr(), neighb.data_ptr(), area.data_ptr(),
                         dist.data_ptr(), lhs.ctypes.data, upd.ctypes.data, kcst.ctypes.data,
                         dcst.ctypes.data, seed, t0, t1, w0, None, C.byref(nwin), C.byref(per))
        assert st == 0, steps_lib.sg_last_error().decode()
        return nwin.value, per.value

    w = 0
    t = 0.0
    for t_next in (1.0e-3, 2.5e-3):
        n, per = call(t, t_next, w)
        sim.run(t_next)
        assert per == sim.getUpdPeriod()
        w += n
        assert w == sim.getNIteration()
        got = counts.cpu().numpy().view(np.uint32)
        for i, s in enumerate(sim.spec_names):
            assert np.array_equal(got[i], sim.getSpecCounts(s)), f"species {s} at t={t_next}"
        t = t_next
    assert int(got[0].sum()) + int(got[2].sum()) == 6000


def test_noalloc_rejects_oversize(steps_lib):
    run_noalloc = _bind(steps_lib)
    nwin = C.c_uint64()
    st = run_noalloc(70000, 3, 0, 1, 1, 1, 1, 1, None, None, None, 1, 0, 0.0, 1.0, 0, None,
                     C.byref(nwin), None)
    assert st == 1
    assert "ntets" in steps_lib.sg_last_error().decode()


def test_noalloc_rejects_face_open_on_one_side(steps_lib):
    """A face whose barycentre distance is positive on one side only would send molecules
    into a slot the other side never gathers; the table build reports it as an argument
    error before any window runs."""
    import torch

    run_noalloc = _bind(steps_lib)
    mesh = W.cube_mesh(4)
    mdl = W.ab_c_model()
    F = flatten(mdl, mesh)
    S, T = 3, mesh.ntets
    R = len(F["reacs"])
    lhs = np.ascontiguousarray(np.stack([r[2] for r in F["reacs"]]), dtype=np.uint32)
    upd = np.ascontiguousarray(np.stack([r[3] for r in F["reacs"]]), dtype=np.int32)
    kcst = np.ascontiguousarray([r[4] for r in F["reacs"]], dtype=np.float64)
    dcst = np.array([1e-12, 1e-12, 5e-13])
    dist = F["dist"].copy()
    t0 = int(np.nonzero((F["neighb"] >= 0).all(axis=1))[0][0])
    dist[t0, 0] = 0.0  # closed from tet t0's side only
    dev = torch.device("cuda", 0)
    counts = torch.zeros(S * T, dtype=torch.int32, device=dev)
    vol = torch.from_numpy(F["vol"]).to(dev)
    neighb = torch.from_numpy(F["neighb"]).to(dev)
    area = torch.from_numpy(F["area"]).to(dev)
    d_dist = torch.from_numpy(dist).to(dev)
    torch.cuda.synchronize()
    st = run_noalloc(T, S, R, counts.data_ptr(), vol.data_ptr(), neighb.data_ptr(), area.data_ptr(),
                     d_dist.data_ptr(), lhs.ctypes.data, upd.ctypes.data, kcst.ctypes.data,
                     dcst.ctypes.data, 1, 0.0, 1e-3, 0, None, None, None)
    assert st == 1
    assert "face open on one side" in steps_lib.sg_last_error().decode()
