"""Benchmark: operator-split spatial SSA throughput (tet-species updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): 40^3 Kuhn cubes of 0.1 um (384,000 tets), the seeded 8-species /
12-reaction network, species 0-3 Poisson(50) per tet, run at the update period the
solver derives from the largest scaled diffusion constant.  One step advances 1 ms of
simulated time (all split windows in it); K = 10 steps cover the configuration's 10 ms.

value: updates = tets x species x windows over the timed steps, divided by the device
time of the steps (CUDA events on the solver's stream, L2 flushed between steps).
e2e:   the same metric through the C ABI with host buffers: each step uploads every
species row from pinned host memory, runs 1 ms and downloads every row.
parity: after the timed steps the GPU state is copied into the CPU oracle and both run 5
more windows; every count of every tet must agree bit for bit.
extra: the batched ensemble (512 realizations) against the same realizations run one at
a time, the EField configuration (FP64 and mixed-precision solves, per-step error against
an FP64 solve) and the full coupled batched configuration (16 realizations of 1.2 M tets
with membrane channels and the mixed-precision EField, 0.03 ms after 0.01 ms), all at
reduced step counts.
cpu_baseline: the reference TetOpSplitP itself (compiled from its sources, oracle/_ref),
one window from the GPU's final state on one host core.
--impl reference: the reference TetOpSplitP on every host core (independent single-rank
replicas, as `mpirun -n 1` each), from the state the oracle reaches after the warm-up.
N > 1: independent replicas, one per GPU (the path is not sharded).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STEP_SIM_S = 1.0e-3
SEED = 1
NCUBE = 40
NSPEC = 8
BYTES_PER_TET_SPEC = 40    # count r/w 8 B + 4 face outflows written 16 B + 4 inflows read 16 B
BYTES_PER_TET = 32         # neighbour table 16 B + face coefficients 16 B
L2_FLUSH_BYTES = 256 << 20


def workload():
    from steps_b200 import workloads as W

    mesh = W.cube_mesh(NCUBE)
    mdl = W.random_network(SEED)
    rows = W.poisson_counts(mesh.ntets, 50.0, SEED, nspec=NSPEC)
    return mdl, mesh, rows


def config_dict(mesh):
    return {
        "workload": "plain_384k: 40^3 Kuhn cubes (0.1 um), 384,000 tets, 8 species, 12 reactions, "
                    "Poisson(50) species 0-3, 10 ms",
        "tets": int(mesh.ntets), "species": NSPEC, "reactions": 12,
        "sim_ms_per_step": STEP_SIM_S * 1e3,
        "network_seed": SEED,
        "l2": "flushed between timed steps (256 MiB device write)",
    }


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "20",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(mdl, mesh, state):
    """The reference TetOpSplitP (oracle/_ref, compiled from its sources) on one host
    core: one split window from the given counts (the GPU's state after the timed steps),
    after one untimed window.  Without that library, the CPU oracle on all host threads."""
    from steps_b200.solver import flatten

    F = flatten(mdl, mesh)
    try:
        from oracle import refsim

        have_ref = refsim.available()
    except ImportError:
        have_ref = False
    if have_ref:
        c0 = time.perf_counter()
        sim = refsim.RefSim(mesh, F, SEED)
        for i in range(NSPEC):
            sim.set_tet_counts(i, state[i].astype(np.float64))
        build_s = time.perf_counter() - c0
        sim.run(1e-12)
        per = sim.period()
        sim.run(sim.time() + per)
        n0 = sim.nsteps()
        t0 = time.perf_counter()
        sim.run(sim.time() + per)
        dt = time.perf_counter() - t0
        n = sim.nsteps() - n0
        del sim
        return {"value": mesh.ntets * NSPEC * n / dt, "unit": "tet-species updates/s", "cores": 1,
                "kind": "reference",
                "sample": f"{n} split window of the same workload from the GPU's final state, {dt:.2f} s on one "
                          f"host core (reference TetOpSplitP built from its sources; construction {build_s:.1f} s "
                          f"and one warm-up window not timed)"}
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle.pyoracle import Oracle

    ora = Oracle(F, seed=SEED)
    for i in range(NSPEC):
        ora.set_counts(i, state[i])
    per = ora.period()
    ora.run(per)
    t0 = time.perf_counter()
    n = ora.run(per * 5)
    dt = time.perf_counter() - t0
    return {"value": mesh.ntets * NSPEC * n / dt, "unit": "tet-species updates/s", "cores": threads, "kind": "port",
            "sample": f"{n} split windows of the same workload, {dt:.2f} s on {threads} host threads "
                      "(the reference library is absent, so its CPU restatement ran)"}


def parity_leg(sim, mdl, mesh, windows=5):
    """Copy the GPU state into the CPU oracle, run `windows` more windows on both and
    compare every count of every tet (not timed)."""
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
    from oracle.pyoracle import Oracle

    ora = Oracle(sim.tables, seed=SEED)
    for i, s in enumerate(sim.spec_names):
        ora.set_counts(i, sim.getSpecCounts(s))
    ora.set_time(0, sim.getTime(), sim.getNIteration())
    per = sim.getUpdPeriod()
    t_end = sim.getTime() + windows * per
    w0 = sim.getNIteration()
    sim.run(t_end)
    ora.run(t_end)
    ok = sim.getNIteration() - w0 == windows and ora.window() == sim.getNIteration()
    diff = 0
    for i, s in enumerate(sim.spec_names):
        diff += int(np.count_nonzero(sim.getSpecCounts(s) != ora.get_counts(i)))
    return {"config": "plain_384k", "windows": int(sim.getNIteration() - w0), "tets": int(mesh.ntets),
            "species": NSPEC, "bit_exact": bool(ok and diff == 0), "differing_counts": diff,
            "checker": "CPU oracle (oracle/opsplit_oracle.c) from the GPU state after the timed steps"}


def replica_totals(dist, device, total_ms, updates, e2e_s, e2e_upd):
    """Whole-job figures of N independent replicas: the slowest rank's device time and
    end-to-end time (max over ranks) against the updates of all ranks (sum)."""
    if dist is None:
        return total_ms, float(updates), e2e_upd / e2e_s
    import torch

    t = torch.tensor([total_ms, e2e_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([float(updates), float(e2e_upd)], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t[0].item()), float(u[0].item()), float(u[1].item()) / float(t[1].item())


def _ref_replica_run(job):
    state_path, seed, wps, steps = job
    import time as _t

    from oracle.refsim import RefSim
    from steps_b200.solver import flatten

    mdl, mesh, _ = workload()
    c0 = _t.time()
    sim = RefSim(mesh, flatten(mdl, mesh), seed)
    rows = np.load(state_path)
    for i in range(NSPEC):
        sim.set_tet_counts(i, rows[i].astype(np.float64))
    build_s = _t.time() - c0
    # The update period is computed on the first run(); a negligible first window fixes
    # it, then one full untimed window.
    sim.run(1e-12)
    per = sim.period()
    t = sim.time() + per
    sim.run(t)
    n0 = sim.nsteps()
    w0 = _t.time()
    for _ in range(steps):
        t += wps * per
        sim.run(t)
    w1 = _t.time()
    return sim.nsteps() - n0, w0, w1, build_s


def reference_state(args):
    """Counts after the warm-up steps, from the CPU oracle (law-equal to the GPU and the
    reference; fast on all host threads)."""
    from oracle.pyoracle import Oracle
    from steps_b200.solver import flatten

    mdl, mesh, rows = workload()
    os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
    ora = Oracle(flatten(mdl, mesh), seed=SEED)
    for i in range(NSPEC):
        ora.set_counts(i, rows[i])
    ora.run(args.warmup * STEP_SIM_S)
    return mesh, np.stack([ora.get_counts(i) for i in range(NSPEC)])


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    import tempfile

    from oracle import refsim

    if not refsim.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsteps_ref.so (the reference "
                          "TetOpSplitP built from its sources by oracle/build_ref_tetopsplit.py) is missing"}),
              flush=True)
        return 0
    mesh, state = reference_state(args)
    cores = os.cpu_count() or 1
    # Each replica holds about 5 GB; keep a margin of host memory.
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
        nproc = max(1, min(cores, int(avail // (6 << 30))))
    except (ValueError, OSError):
        nproc = cores
    wps = args.ref_windows
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "state.npy")
        np.save(path, state)
        ctx = mp.get_context("spawn")
        with ctx.Pool(nproc) as pool:
            res = pool.map(_ref_replica_run, [(path, SEED + k, wps, args.steps) for k in range(nproc)])
    wins = sum(r[0] for r in res)
    span = max(r[2] for r in res) - min(r[1] for r in res)
    upd = mesh.ntets * NSPEC * wins
    v = upd / span
    sample = (f"{nproc} independent single-rank TetOpSplitP replicas (one per host core, as mpirun -n 1 each; "
              f"no MPI on this host) from the state at t = {args.warmup} ms; {args.steps} steps of {wps} split "
              f"window(s) each; {wins} windows in {span:.1f} s of wall time across the replicas; "
              f"construction {max(r[3] for r in res):.1f} s not timed")
    line = {
        "metric": "tet-species updates/s", "value": v, "unit": "tet-species updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * span / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32+f64", "data": "synthetic",
        "config": dict(config_dict(mesh), step=f"{wps} split window(s) per step (bounded CPU sample of the 1 ms step)",
                       parallelism=f"{nproc} single-rank replicas"),
        "cpu_baseline": {"value": v, "unit": "tet-species updates/s", "cores": nproc, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": v, "unit": "tet-species updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from steps_b200 import rng as srng
    from steps_b200.solver import TetOpSplit

    mdl, mesh, rows = workload()
    r = srng.create("r123", 512)
    r.initialize(SEED + rank)
    sim = TetOpSplit(mdl, mesh, r, device=local)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    ext = torch.cuda.ExternalStream(sim.getStream(), device=local)
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    t_sim = 0.0
    for i in range(args.warmup):
        # The last warm-up step picks the launch shape (results unchanged): by then the
        # counts are past the initial transient the timed steps no longer see.
        if i == args.warmup - 1:
            sim.setAutotune(True)
        t_sim += STEP_SIM_S
        sim.run(t_sim)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    clocks = Clocks(local)
    barrier()
    clocks.start()
    sim.setProfiling(True)
    _, _, launches0 = sim.getProfile()
    it0 = sim.getNIteration()
    total_ms = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(ext):
            flush_buf.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
        t_sim += STEP_SIM_S
        sim.run(t_sim)
        with torch.cuda.stream(ext):
            e1.record(ext)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    barrier()
    clk = clocks.stop()
    win_ms, nwin, launches1 = sim.getProfile()
    windows = sim.getNIteration() - it0
    sim.setProfiling(False)
    updates = mesh.ntets * NSPEC * windows

    # End-to-end through the C ABI with a pinned host buffer of every species row: each step
    # uploads all rows, runs 1 ms and downloads all rows.
    host = torch.empty((NSPEC, mesh.ntets), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    sim.getAllSpecCounts(host)
    barrier()
    e2e_s, e2e_upd = 0.0, 0
    for _ in range(args.steps):
        it_a = sim.getNIteration()
        t0 = time.perf_counter()
        sim.setAllSpecCounts(host)
        t_sim += STEP_SIM_S
        sim.run(t_sim)
        sim.getAllSpecCounts(host)
        e2e_s += time.perf_counter() - t0
        e2e_upd += mesh.ntets * NSPEC * (sim.getNIteration() - it_a)
    t_max, upd_all, e2e_val = replica_totals(dist, f"cuda:{local}", total_ms, updates, e2e_s, e2e_upd)
    value = upd_all / (t_max * 1e-3)

    peak, peak_kind = peaks()
    bytes_per_window = mesh.ntets * (BYTES_PER_TET_SPEC * NSPEC + BYTES_PER_TET)
    avg_win_s = (win_ms * 1e-3) / max(nwin, 1)
    achieved = bytes_per_window / avg_win_s / 1e9
    # DRAM bytes per window of the kernels the run used, from the committed ncu summary
    # (profiles/split_window_plain_384k.md: one capture of each split kernel).
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "split_window_plain_384k.md")
    if os.path.exists(prof_path) and sim.getSplit():
        with open(prof_path) as f:
            for ln in f:
                if ln.startswith("dram_bytes_per_window:"):
                    traffic = int(ln.split(":")[1])

    parity = None
    extra = None
    cpu = None
    if rank == 0 and world == 1:
        state = np.stack([sim.getSpecCounts(s) for s in sim.spec_names])
        parity = parity_leg(sim, mdl, mesh)
        cpu = cpu_baseline(mdl, mesh, state)
    if rank == 0:
        line = {
            "metric": "tet-species updates/s", "value": value, "unit": "tet-species updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32+f64", "data": "synthetic",
            "config": dict(config_dict(mesh), parallelism=f"replicas{world}",
                           launch={"block": sim.getLaunch()[0], "grid": sim.getLaunch()[1],
                                   "smem_carveout_pct": sim.getCarveout(), "split": sim.getSplit(),
                                   "persistent": sim.getPersistent()[0],
                                   "autotune_ms": sim.getAutotuneTimes()}),
            "sim_ms_per_wall_s": (STEP_SIM_S * 1e3 * args.steps) / (t_max * 1e-3),
            "windows_per_step": windows / args.steps,
            "e2e": {"value": e2e_val, "unit": "tet-species updates/s",
                    "h2d_bytes_per_step": NSPEC * mesh.ntets * 4, "d2h_bytes_per_step": NSPEC * mesh.ntets * 4},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "kernel": (f"sg::persistent_window_kernel<{256 if sim.getLaunch()[0] >= 256 else 128}, "
                                    f"{sim.getPersistent()[1]}>" if sim.getPersistent()[0] else
                                    f"sg::window_kernel<{sim.getLaunch()[0]}, split> + sg::leave_kernel<256>"
                                    if sim.getSplit() else f"sg::window_kernel<{sim.getLaunch()[0]}>"),
                         "algorithmic_bytes_per_launch": bytes_per_window,
                         "avg_launch_us": avg_win_s * 1e6},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(launches1 - launches0),
            "parity": parity,
        }
        if world == 1 and not args.no_extra:
            del sim
            line["extra"] = {"batched": batched_extra(args), "efield": efield_extra(args),
                             "coupled": coupled_extra(argparse.Namespace(**dict(vars(args), cp_ms=args.cpx_ms,
                                                                                cp_warmup_ms=0.01)))}
            sim = None
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    del sim
    return 0


def batched_extra(args):
    """Batched ensemble: 512 realizations of n^3 Kuhn cubes (n uniform in 8..30) with the
    8-species network and per-realization log-normal (0.2) rate jitter, in one launch per
    window; against the same realizations run one after another with the plain path."""
    import torch

    from steps_b200 import rng as srng
    from steps_b200 import workloads as W
    from steps_b200.solver import TetOpSplit

    nreal = args.nreal
    sizes = W.batched_sizes(nreal, SEED)
    t0 = time.perf_counter()
    mesh = W.batched_mesh(sizes)
    mdl = W.random_network(SEED)
    r = srng.create("r123", 512)
    r.initialize(SEED)
    sim = TetOpSplit(mdl, mesh, r, realizations=mesh.offsets)
    jit = W.rate_jitter(nreal, 12, SEED)
    names = [f"r{q}" for q in range(12)]
    base = [sim.getCompReacK("comp", n, 0) for n in names]
    for rr in range(nreal):
        for q, n in enumerate(names):
            sim.setCompReacK("comp", n, base[q] * jit[rr, q], realization=rr)
    rows = W.poisson_counts(mesh.ntets, 50.0, SEED, nspec=NSPEC)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    setup_s = time.perf_counter() - t0
    ext = torch.cuda.ExternalStream(sim.getStream())
    t_sim = 0.0
    for i in range(args.bx_warmup):
        if i == args.bx_warmup - 1:
            sim.setAutotune(True)  # tuned on the last warm-up step
        t_sim += STEP_SIM_S
        sim.run(t_sim)
    torch.cuda.synchronize()
    launch = sim.getLaunch()
    sim_split = sim.getSplit()
    sim_persist = sim.getPersistent()
    tune_ms = sim.getAutotuneTimes()
    it0 = sim.getNIteration()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(args.bx_steps):
        t_sim += STEP_SIM_S
        sim.run(t_sim)
    e1.record(ext)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    windows = sim.getNIteration() - it0
    batched = mesh.ntets * NSPEC * windows / (ms * 1e-3)
    del sim
    # The same realizations with the plain path, one solver per realization (bounded sample).
    sample = sizes[: args.plain_sample]
    upd, plain_ms = 0, 0.0
    for k, n in enumerate(sample):
        m = W.cube_mesh(n)
        rk = srng.create("r123", 512)
        rk.initialize(SEED + k)
        ps = TetOpSplit(mdl, m, rk)
        for q, nm in enumerate(names):
            ps.setCompReacK("comp", nm, base[q] * jit[k, q])
        pr = W.poisson_counts(m.ntets, 50.0, SEED + k, nspec=NSPEC)
        for i, s in enumerate(ps.spec_names):
            ps.setSpecCounts(s, pr[i])
        es = torch.cuda.ExternalStream(ps.getStream())
        ps.run((args.bx_warmup - 1) * STEP_SIM_S)
        ps.setAutotune(True)  # tuned on the last warm-up step, as the batched solver
        ps.run(args.bx_warmup * STEP_SIM_S)
        i0 = ps.getNIteration()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(es)
        ps.run((args.bx_warmup + args.bx_steps) * STEP_SIM_S)
        a1.record(es)
        a1.synchronize()
        plain_ms += a0.elapsed_time(a1)
        upd += m.ntets * NSPEC * (ps.getNIteration() - i0)
        del ps
    plain = upd / (plain_ms * 1e-3)
    return {
        "metric": "tet-species updates/s", "value": batched, "unit": "tet-species updates/s",
        "config": {"workload": f"batched: {nreal} realizations of n^3 Kuhn cubes, n in 8..30, "
                               f"{mesh.ntets} tets, 8 species, 12 reactions, rate jitter 0.2",
                   "sim_ms_per_step": 1.0, "steps": args.bx_steps, "warmup": args.bx_warmup,
                   "launch": {"block": launch[0], "grid": launch[1], "split": sim_split,
                              "persistent": sim_persist[0], "tets_per_lane": sim_persist[1],
                              "autotune_ms": tune_ms}},
        "windows": windows, "ms": ms, "setup_s": setup_s,
        "plain_sequential": {"value": plain, "realizations_sampled": len(sample), "ms": plain_ms},
        "batched_over_plain": batched / plain,
    }


def run_batched(args):
    print(json.dumps(batched_extra(args)), flush=True)
    return 0


def efield_extra(args):
    """EField configuration: 20x20x200 Kuhn cubes (480,000 tets), every boundary triangle
    membrane, Cm 1 uF/cm^2, leak 3e-5 S/cm^2 at -65 mV, a two-state voltage-gated channel
    at 10/um^2 (alpha = 0.1 exp(V/25 mV)/ms, beta = 0.1 exp(-V/25 mV)/ms, 20 pS, +50 mV),
    1 nA on the z = 0 face, EField dt 1 us; FP64 CG against FP32 CG + FP64 refinement."""
    import math

    from steps_b200 import geom as sgeom
    from steps_b200 import model as smodel
    from steps_b200 import rng as srng
    from steps_b200.solver import EF_DV_CG_FP64, EF_DV_CG_MIXED, TetOpSplit

    nx, ny, nz = args.ef_dims
    mesh = sgeom.kuhn_box(nx, ny, nz, 1e-7)
    cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    cyto.addVolsys("vsys")
    surf = mesh.getSurfTris()
    patch = sgeom.TmPatch("memb", mesh, surf, cyto)
    patch.addSurfsys("ssys")
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    smodel.Volsys("vsys", mdl)
    ss = smodel.Surfsys("ssys", mdl)
    ch = smodel.Chan("Na", mdl)
    c = smodel.ChanState("C", mdl, ch)
    o = smodel.ChanState("O", mdl, ch)
    # 1 nA into 168 um^2 of membrane drives V to about +110 mV before the channels clamp it
    # near +80 mV, above the default 100 mV table top, so the rate tables reach +200 mV.
    vr = (-150.0e-3, 200.0e-3, 1.0e-4)
    smodel.VDepSReac("open", ss, slhs=[c], srhs=[o], k=lambda v: 100.0 * math.exp(v / 0.025), vrange=vr)
    smodel.VDepSReac("close", ss, slhs=[o], srhs=[c], k=lambda v: 100.0 * math.exp(-v / 0.025), vrange=vr)
    smodel.OhmicCurr("I", ss, chanstate=o, g=20e-12, erev=0.05)
    zmin = np.unique(mesh.tris[surf][np.all(mesh.verts[mesh.tris[surf]][:, :, 2] <= 1e-12, axis=1)])
    out = {}
    finals = {}
    for name, method in (("fp64", EF_DV_CG_FP64), ("mixed", EF_DV_CG_MIXED)):
        r = srng.create("r123", 512)
        r.initialize(SEED)
        sim = TetOpSplit(mdl, mesh, r, method)
        sim.setEfieldTolerance(args.ef_tol, args.ef_inner_tol)
        sim.setEfieldPersistent(bool(args.ef_persistent))
        sim.setEfieldCheck(True, 1e-12)  # untimed FP64 solve of every step's system to 1e-12
        if method == EF_DV_CG_MIXED:
            sim.setEfieldReliableUpdates(bool(args.ef_reliable), args.ef_ru_delta)
        sim.setEfieldDT(1e-6)
        sim.setMembPotential("membrane", -0.065)
        sim.setMembCapac("membrane", 0.01)
        sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
        sim.setPatchSpecCount("memb", "C", 10.0 * patch.getArea() * 1e12)
        for v in zmin:
            sim.setVertIClamp(int(v), 1e-9 / len(zmin))
        t_end = args.ef_steps * 1e-6
        w0 = time.perf_counter()
        sim.run(t_end)
        wall = time.perf_counter() - w0
        steps, iters, solve_ms, rr = sim.getEfieldStats()
        chk = sim.getEfieldCheck()
        finals[name] = np.array([sim.getVertV(v) for v in range(0, mesh.nverts, 97)])
        out[name] = {"steps": steps, "cg_iterations_per_step": iters / max(steps, 1),
                     "solve_ms_per_step": solve_ms / max(steps, 1), "wall_s": wall,
                     "sim_ms_per_wall_s": t_end * 1e3 / wall}
        if chk:
            out[name]["check_vs_fp64_solve"] = {"steps": chk[0], "max_rel_v_err": chk[1], "tol_fp64": 1e-12,
                                                "note": "wall_s includes the check solves; solve_ms does not"}
        del sim
    err = float(np.max(np.abs(finals["mixed"] - finals["fp64"]) / np.abs(finals["fp64"])))
    return {
        "metric": "EField solve ms per step", "config": {"mesh": f"{nx}x{ny}x{nz} Kuhn cubes",
                                                         "tets": mesh.ntets, "verts": mesh.nverts,
                                                         "steps": args.ef_steps, "tol": args.ef_tol,
                                                         "persistent_solve": bool(args.ef_persistent),
                                                         "mixed_reliable_updates": bool(args.ef_reliable),
                                                         "reliable_update_delta": args.ef_ru_delta},
        "fp64": out["fp64"], "mixed": out["mixed"],
        "mixed_speedup": out["fp64"]["solve_ms_per_step"] / out["mixed"]["solve_ms_per_step"],
        "max_rel_v_err_per_step": out["mixed"]["check_vs_fp64_solve"]["max_rel_v_err"],
        "fp64_cg_max_rel_v_err_per_step": out["fp64"]["check_vs_fp64_solve"]["max_rel_v_err"],
        "max_rel_v_diff_end_of_run": err,
    }


def run_efield(args):
    print(json.dumps(efield_extra(args)), flush=True)
    return 0


def run_windows(args):
    """Profiling mode: the plain 384k workload with a fixed launch (block 256, one tet per
    thread, split or fused by --split), run to the warm-up time (--warmup ms), then
    --windows more windows; prints the mean window time.  The ncu summaries under
    profiles/ capture the kernels of these last windows."""
    import torch

    from steps_b200 import rng as srng
    from steps_b200.solver import TetOpSplit

    mdl, mesh, rows = workload()
    r = srng.create("r123", 512)
    r.initialize(SEED)
    sim = TetOpSplit(mdl, mesh, r, device=0)
    for i, s in enumerate(sim.spec_names):
        sim.setSpecCounts(s, rows[i])
    sim.setLaunch(256, -1)
    sim.setSplit(bool(args.split))
    sim.run(args.warmup * STEP_SIM_S)
    torch.cuda.synchronize()
    per = sim.getUpdPeriod()
    sim.setProfiling(True)
    sim.run(sim.getTime() + args.windows * per * 0.999999)
    wms, nw, _ = sim.getProfile()
    print(json.dumps({"mode": "windows", "split": bool(args.split), "warmup_ms": args.warmup, "windows": nw,
                      "ms_per_window": wms / max(nw, 1)}), flush=True)
    return 0


def coupled_extra(args):
    """Full coupled batched configuration: 16 realizations of a 5x5x8 um box (50x50x80 Kuhn
    cubes, 1.2 M tets each) in one launch per window.  Volume: Ca + CB <-> CaCB (kf 1e8 /M/s,
    kb 100 /s), D_Ca 2.2e-10, D_CB = D_CaCB = 2e-11 m^2/s, CB 50 uM, Ca 50 nM.  Membrane (every
    boundary triangle): Cm 1 uF/cm^2, leak 3e-5 S/cm^2 at -65 mV, the two-state channel of the
    EField configuration (10/um^2, 20 pS, +50 mV) and a voltage-gated Ca channel (3/um^2, the
    same kinetics with the exponent's sign flipped) whose open state emits Ca into its tet at
    0.1 pA per channel (0.1e-12 / 2e per second).  Mixed-precision EField, dt 1 us; the split
    window is shorter than the EField step only when D_Ca G < 1e6 /s, so each EField step runs
    one truncated window."""
    import math

    from steps_b200 import geom as sgeom
    from steps_b200 import model as smodel
    from steps_b200 import rng as srng
    from steps_b200.solver import EF_DV_CG_FP64, EF_DV_CG_MIXED, TetOpSplit

    t0 = time.perf_counter()
    nx, ny, nz = args.cp_dims
    base = sgeom.kuhn_box(nx, ny, nz, 1e-7)
    mesh = sgeom.replicate(base, args.cp_nreal)
    cyto = sgeom.TmComp("cyto", mesh, np.arange(mesh.ntets))
    cyto.addVolsys("vsys")
    patch = sgeom.TmPatch("memb", mesh, mesh.getSurfTris(), cyto)
    patch.addSurfsys("ssys")
    sgeom.Memb("membrane", mesh, [patch])
    mdl = smodel.Model()
    ca, cb, cacb = smodel.Spec("Ca", mdl), smodel.Spec("CB", mdl), smodel.Spec("CaCB", mdl)
    vs = smodel.Volsys("vsys", mdl)
    smodel.Reac("bind", vs, lhs=[ca, cb], rhs=[cacb], kcst=1e8)
    smodel.Reac("unbind", vs, lhs=[cacb], rhs=[ca, cb], kcst=100.0)
    smodel.Diff("dCa", vs, ca, 2.2e-10)
    smodel.Diff("dCB", vs, cb, 2e-11)
    smodel.Diff("dCaCB", vs, cacb, 2e-11)
    ss = smodel.Surfsys("ssys", mdl)
    vr = (-150.0e-3, 200.0e-3, 1.0e-4)
    na = smodel.Chan("Na", mdl)
    c, o = smodel.ChanState("C", mdl, na), smodel.ChanState("O", mdl, na)
    smodel.VDepSReac("open", ss, slhs=[c], srhs=[o], k=lambda v: 100.0 * math.exp(v / 0.025), vrange=vr)
    smodel.VDepSReac("close", ss, slhs=[o], srhs=[c], k=lambda v: 100.0 * math.exp(-v / 0.025), vrange=vr)
    smodel.OhmicCurr("I", ss, chanstate=o, g=20e-12, erev=0.05)
    cach = smodel.Chan("CaCh", mdl)
    cc, co = smodel.ChanState("CaC", mdl, cach), smodel.ChanState("CaO", mdl, cach)
    smodel.VDepSReac("caopen", ss, slhs=[cc], srhs=[co], k=lambda v: 100.0 * math.exp(-v / 0.025), vrange=vr)
    smodel.VDepSReac("caclose", ss, slhs=[co], srhs=[cc], k=lambda v: 100.0 * math.exp(v / 0.025), vrange=vr)
    smodel.SReac("caflux", ss, slhs=[co], srhs=[co], irhs=[ca], kcst=0.1e-12 / (2.0 * 1.602176487e-19))
    method = EF_DV_CG_MIXED if args.cp_method == "mixed" else EF_DV_CG_FP64
    r = srng.create("r123", 512)
    r.initialize(SEED)
    sim = TetOpSplit(mdl, mesh, r, method, realizations=mesh.offsets)
    sim.setEfieldDT(1e-6)
    sim.setMembPotential("membrane", -0.065)
    sim.setMembCapac("membrane", 0.01)
    sim.setMembRes("membrane", 1.0 / 0.3, -0.065)
    sim.setCompSpecConc("cyto", "CB", 50e-6)
    sim.setCompSpecConc("cyto", "Ca", 50e-9)
    area_r = patch.getArea() / args.cp_nreal * 1e12  # um^2 per realization
    for q in range(args.cp_nreal):
        sim.setPatchSpecCount("memb", "C", 10.0 * area_r, realization=q)
        sim.setPatchSpecCount("memb", "CaC", 3.0 * area_r, realization=q)
    setup_s = time.perf_counter() - t0
    import torch

    ext = torch.cuda.ExternalStream(sim.getStream())
    sim.run(args.cp_warmup_ms * 1e-3)
    torch.cuda.synchronize()
    it0 = sim.getNIteration()
    s0, _, ms0, _ = sim.getEfieldStats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(ext)
    sim.run((args.cp_warmup_ms + args.cp_ms) * 1e-3)
    e1.record(ext)
    e1.synchronize()
    wall = time.perf_counter() - w0
    ms = e0.elapsed_time(e1)
    windows = sim.getNIteration() - it0
    s1, iters, ms1, rr = sim.getEfieldStats()
    upd = mesh.ntets * 3 * windows
    out = {
        "metric": "tet-species updates/s; sim-ms per wall-s", "value": upd / (ms * 1e-3),
        "unit": "tet-species updates/s",
        "config": {"workload": f"coupled batched: {args.cp_nreal} realizations of {nx}x{ny}x{nz} Kuhn cubes "
                               f"({base.ntets} tets, {base.nverts} vertices each), Ca/CB/CaCB + membrane "
                               f"channels + {args.cp_method} EField",
                   "tets": mesh.ntets, "verts": mesh.nverts, "membrane_tris": int(len(mesh.getSurfTris())),
                   "timed_sim_ms": args.cp_ms, "warmup_sim_ms": args.cp_warmup_ms},
        "windows": windows, "efield_steps": s1 - s0, "ms": ms, "wall_s": wall, "setup_s": setup_s,
        "sim_ms_per_wall_s": args.cp_ms / wall,
        "efield_solve_ms_per_step": (ms1 - ms0) / max(s1 - s0, 1),
        "cg_iterations_per_step_overall": iters / max(s1, 1),
    }
    del sim
    return out


def run_coupled(args):
    print(json.dumps(coupled_extra(args)), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-windows", type=int, default=1,
                    help="reference arm: split windows per timed step (a bounded CPU sample of the 1 ms step)")
    ap.add_argument("--config", choices=["plain", "batched", "efield", "coupled", "windows"], default="plain")
    ap.add_argument("--windows", type=int, default=4, help="--config windows: windows after the warm-up")
    ap.add_argument("--split", type=int, default=1, help="--config windows: 1 split window kernels, 0 fused")
    ap.add_argument("--cp-dims", type=int, nargs=3, default=[50, 50, 80])
    ap.add_argument("--cp-nreal", type=int, default=16)
    ap.add_argument("--cp-ms", type=float, default=0.5, help="timed simulated ms (the configuration runs 20)")
    ap.add_argument("--cp-warmup-ms", type=float, default=0.02)
    ap.add_argument("--cpx-ms", type=float, default=0.03, help="coupled extra of the default line: timed simulated ms")
    ap.add_argument("--cp-method", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--ef-inner-tol", type=float, default=1e-4)
    ap.add_argument("--nreal", type=int, default=512)
    ap.add_argument("--bx-steps", type=int, default=3, help="batched: timed 1 ms steps")
    ap.add_argument("--bx-warmup", type=int, default=3, help="batched: warm-up 1 ms steps (the last autotunes)")
    ap.add_argument("--no-extra", action="store_true", help="default line without the batched / EField extras")
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--ef-dims", type=int, nargs=3, default=[20, 20, 200])
    ap.add_argument("--ef-steps", type=int, default=1000)
    ap.add_argument("--ef-reliable", type=int, default=1,
                    help="mixed method: 1 = one FP32 CG with reliable updates, 0 = restarted FP32 inner solves")
    ap.add_argument("--ef-ru-delta", type=float, default=0.1)
    ap.add_argument("--ef-tol", type=float, default=1e-10)
    ap.add_argument("--ef-persistent", type=int, default=1, help="1: each EField solve in one cooperative launch")
    args = ap.parse_args()
    if args.warmup < 3:
        print(f"bench.py: --warmup {args.warmup} raised to 3 (the timing rules need at least 3 warm-up steps)",
              file=sys.stderr)
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "efield":
        return run_efield(args)
    if args.config == "coupled":
        return run_coupled(args)
    if args.config == "windows":
        return run_windows(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
