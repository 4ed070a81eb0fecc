"""Benchmark: CloverLeaf3D hydro-cycle throughput (cell-updates/s) on B200.

Workload: the two-state shock of the reference decks (state 1 rho=0.2 e=1.0,
state 2 rho=1.0 e=2.5 in x<5, y<2, z<2) on [0,10]^3 at 512^3 cells,
initial/max timestep 0.04, timestep_rise 1.5, field summary every 10 steps.
A "step" is one full hydro step (hydro.f90:52-72, summaries included).

value      device-resident chunk (native API), inputs already in HBM, steps
           replayed from CUDA graphs; cells * steps / device time.
e2e        the configuration's whole run (200 steps at 512^3, --e2e-steps)
           through the drop-in C ABI with HOST arrays: the reference control
           flow calling clover_*_kernel, the first call of each array
           uploading it and a final copy back of every array, all inside the
           timed region.
roofline   dominant kernel group, algorithmic bytes / its event-timed duration
           (a profiled run of the same steps right after the timed one).
cpu_baseline  the oracle (C restatement of the reference, OpenMP) on the
           host cores over a bounded sample of the same problem.
bricks_decomposition  the same problem at 256^3 decomposed into 8 bricks
           (clover_decompose, device-side halo messages) against one chunk, both
           through the drop-in driver: the exchange's cost per step.
ensemble   batched decks (seeded draws of the same problem with drawn sizes,
           region, densities and energies): 64 decks of 24..128 cells per
           axis for 150 steps (FP64 and mixed) and 512 decks of 16..48 cells
           per axis for 100 steps (mixed, with its FP64 twin for the errors),
           each autotuned and graph-replayed, against the same decks run one
           after another as single chunks (graph-replayed too).

--impl reference times that CPU restatement alone (the Fortran reference
cannot be compiled on this image: no Fortran compiler).
Multi-GPU (--gpus N under torchrun): N independent replicas, one chunk per
GPU (the single-chunk path does not shard); weak scaling, max time over ranks.
The ensemble legs partition their decks over the ranks instead (each rank
its share, balanced by cells, no communication; strong scaling, max time over
ranks).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cloverleaf3d_ref_b200.replicas import deck_share, max_over_ranks  # noqa: E402

STATES = [
    dict(density=0.2, energy=1.0),
    dict(density=1.0, energy=2.5, geometry="cuboid", xmin=0.0, xmax=5.0, ymin=0.0, ymax=2.0,
         zmin=0.0, zmax=2.0),
]


def deck_values(n, steps):
    return dict(x_cells=n, y_cells=n, z_cells=n, xmin=0.0, ymin=0.0, zmin=0.0, xmax=10.0,
                ymax=10.0, zmax=10.0, initial_timestep=0.04, max_timestep=0.04,
                timestep_rise=1.5, end_step=steps, end_time=1.0e6, summary_frequency=10)


def workload_name(n, precision):
    """The workload both arms run: the benchmark problem at n^3 cells."""
    return "two-state shock %d^3, %s" % (n, precision)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return j.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for i, n in enumerate(names):
                if f[4 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(n_cells, seconds_target=12.0):
    """Oracle (OpenMP, all host threads) on a bounded sample of the problem."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    L = O.load(fast=True)
    L.oracle_run_timed.restype = ctypes.c_double
    cores = os.cpu_count() or 1
    # calibrate on 128^3, then size the sample to about seconds_target
    d = O.make_deck(dict(deck_values(128, 3), states=STATES))
    t = L.oracle_run_timed(ctypes.byref(d), 1, 2)
    rate = 128 ** 3 * 2 / t
    n = 256 if rate * seconds_target > 256 ** 3 * 2 else 128
    steps = max(2, min(20, int(rate * seconds_target / n ** 3)))
    d = O.make_deck(dict(deck_values(n, steps + 1), states=STATES))
    t = L.oracle_run_timed(ctypes.byref(d), 1, steps)
    return {"value": n ** 3 * steps / t, "unit": "cell-updates/s", "cores": cores,
            "kind": "port",
            "sample": "%d^3 cells x %d steps of the same two-state shock (oracle C restatement, "
                      "OpenMP %d threads, -O3 x86-64-v3)" % (n, steps, cores)}


def deck_dict(deck):
    """A library Deck as the oracle's deck mapping."""
    s = deck.s
    geo = {1: "cuboid", 2: "sphere", 3: "point"}
    states = []
    for i in range(s.number_of_states):
        states.append(dict(density=s.state_density[i], energy=s.state_energy[i],
                           xvel=s.state_xvel[i], yvel=s.state_yvel[i], zvel=s.state_zvel[i],
                           xmin=s.state_xmin[i], xmax=s.state_xmax[i], ymin=s.state_ymin[i],
                           ymax=s.state_ymax[i], zmin=s.state_zmin[i], zmax=s.state_zmax[i],
                           radius=s.state_radius[i], geometry=geo.get(s.state_geometry[i], "cuboid")))
    return dict(x_cells=s.x_cells, y_cells=s.y_cells, z_cells=s.z_cells, xmin=s.xmin, ymin=s.ymin,
                zmin=s.zmin, xmax=s.xmax, ymax=s.ymax, zmax=s.zmax,
                initial_timestep=s.initial_timestep, max_timestep=s.max_timestep,
                timestep_rise=s.timestep_rise, end_time=s.end_time, end_step=s.end_step,
                summary_frequency=s.summary_frequency, states=states)


def cpu_configs():
    """The oracle's timing build (OpenMP, all host threads) on the benchmark
    problem's configurations: 32^3 x 100 and 96^3 x 300 steps in full, 512^3
    for 3 steps after one, and the two ensembles on samples of their seeded
    decks run one after another (the rate over the sample's cells)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    import cloverleaf3d_ref_b200 as C
    L = O.load(fast=True)
    L.oracle_run_timed.restype = ctypes.c_double
    out = {"cores": os.cpu_count() or 1, "build": "oracle C restatement, -O3 x86-64-v3, OpenMP",
           "unit": "cell-updates/s"}

    def timed(d, warm, steps):
        od = O.make_deck(d)
        return L.oracle_run_timed(ctypes.byref(od), warm, steps)

    for key, n, steps, warm in (("config1_32", 32, 100, 0), ("config2_96", 96, 300, 0),
                                ("config3_512_sample", 512, 3, 1)):
        d = dict(deck_values(n, warm + steps + 1), states=STATES)
        t = timed(d, warm, steps)
        out[key] = {"value": n ** 3 * steps / t, "steps": steps, "seconds": t}
    for key, nd, cells, steps, seed, sample in (("config4_64_decks_sample", 64, (24, 128), 150, 2024, 8),
                                               ("config5_512_decks_sample", 512, (16, 48), 100, 4048, 64)):
        decks = C.draw_decks(nd, seed, cells=cells, end_step=steps, summary_frequency=10)[:sample]
        t = 0.0
        work = 0
        for dk in decks:
            d = deck_dict(dk)
            t += timed(d, 0, steps)
            work += dk.cells * steps
        out[key] = {"value": work / t, "decks_timed": sample, "steps": steps, "seconds": t}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    L = O.load(fast=True)
    L.oracle_run_timed.restype = ctypes.c_double
    cores = os.cpu_count() or 1
    # bounded sample: the configured size when the host holds it, else 256^3
    n = args.cells
    need = 31 * (n + 5) ** 3 * 8
    avail = 0
    try:
        with open("/proc/meminfo") as f:
            for l in f:
                if l.startswith("MemAvailable"):
                    avail = int(l.split()[1]) * 1024
    except OSError:
        pass
    if need * 1.5 > avail:
        n = 256
    # K timed steps after W warm-up ones, as the GPU arm; if the host would
    # need more than about four minutes for them (a calibration step first),
    # fewer steps, reported in "steps"
    d1 = O.make_deck(dict(deck_values(n, 3), states=STATES))
    per_step = L.oracle_run_timed(ctypes.byref(d1), 0, 1)
    budget = max(1, int(240.0 / max(per_step, 1e-9)))
    warm = min(args.warmup, max(0, budget - args.steps))
    steps = max(1, min(args.steps, budget - warm))
    d = O.make_deck(dict(deck_values(n, steps + warm + 1), states=STATES))
    t = L.oracle_run_timed(ctypes.byref(d), warm, steps)
    v = n ** 3 * steps / t
    line = {
        "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1000.0 * t / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: two-state shock deck generated on the host",
        "config": {"workload": workload_name(n, "fp64"),
                   "execution": "CPU restatement, OpenMP %d threads" % cores,
                   "size": "configured" if n == args.cells else
                           "reduced from %d^3: host memory" % args.cells},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                         "sample": "%d^3 cells x %d steps after %d warm-up (oracle C restatement of "
                                   "the reference; the Fortran reference needs a Fortran compiler, "
                                   "absent on this image)" % (n, steps, warm)},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def rel_err(a, b):
    """|a - b| / |b| per element; 0 where both are 0 (the kinetic energy at
    step 0 of a deck at rest)."""
    import numpy as np
    d = np.abs(a - b)
    s = np.abs(b)
    return np.where(s > 0, d / np.where(s > 0, s, 1.0), np.where(d > 0, np.inf, 0.0))


def accuracy_leg(C, n, steps):
    """The FP64 and the mixed-precision chunk run the same deck for `steps`
    steps (summary every 10); the relative error of every summary quantity at
    every summary step, the bar being 1e-5 after 200 steps."""
    deck = C.Deck.from_values(states=STATES, **deck_values(n, steps))
    out = {}
    for name, prec in (("fp64", C.PRECISION_FP64), ("mixed", C.PRECISION_MIXED)):
        ch = C.Chunk(deck, prec)
        assert ch.run() == steps
        out[name] = ch.summaries()
        ch.close()
    (a, st), (b, _) = out["fp64"], out["mixed"]
    rel = rel_err(b, a)
    names = ["vol", "mass", "ie", "ke", "press"]
    return {
        "steps": steps, "cells": "%d^3" % n, "summary_steps": [int(x) for x in st],
        "rel_err_per_summary": {q: [float(x) for x in rel[:, i]] for i, q in enumerate(names)},
        "max_rel_err": {q: float(rel[:, i].max()) for i, q in enumerate(names)},
        "within_1e-5": bool(rel.max() <= 1e-5),
    }


def mixed_leg(C, torch, deck, args, fp64_ms, fp64_sums, fp64_steps, barrier, world, dist):
    """The same workload with FP32 storage of the stencilled fields and the
    volume and mass fluxes (FP64 density, pre/post volumes, cell mass/energy
    update and node masses): timed the same way, and its field summaries
    compared with the FP64 run's at the same steps."""
    import numpy as np
    n = args.cells
    ch = C.Chunk(deck, C.PRECISION_MIXED)
    stream = torch.cuda.ExternalStream(ch.stream)
    ch.step(args.warmup)
    ch.sync()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ch.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    barrier()
    ms = max_over_ranks(ms, dist if world > 1 else None, "cuda")
    ch.profile(True)
    ch.step(args.steps)
    groups = ch.profile_report()
    ch.profile(False)
    sums, steps = ch.summaries()
    nbytes = ch.device_bytes
    ch.close()
    m = min(len(sums), len(fp64_sums))
    assert np.array_equal(steps[:m], fp64_steps[:m])
    rel = rel_err(sums[:m], fp64_sums[:m])
    step_bytes = sum(g["bytes"] for g in groups) / args.steps
    return {
        "value": world * n ** 3 * args.steps / (ms / 1000.0), "unit": "cell-updates/s",
        "ms_per_step": ms / args.steps, "speedup_vs_fp64": fp64_ms / ms,
        "dtype": "f32 storage and stencils (f64 density, volumes, cell update, node masses)",
        "device_gb": nbytes / 1e9,
        "step_algorithmic_bytes_per_cell": step_bytes / n ** 3,
        "step_achieved_gbs": step_bytes / (ms / args.steps / 1000.0) / 1e9,
        "summary_steps_compared": int(m),
        "max_rel_err_vs_fp64": dict(zip(["vol", "mass", "ie", "ke", "press"],
                                        [float(x) for x in rel.max(axis=0)])),
        "per_kernel": {g["name"]: {"ms_per_step": g["ms"] / args.steps,
                                   "gbs": g["bytes"] / max(g["ms"], 1e-9) / 1e6}
                       for g in groups},
    }


def timed_steps(torch, obj, steps):
    """Device time (ms) of obj.step(steps) with events on obj's stream."""
    stream = torch.cuda.ExternalStream(obj.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    obj.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def ensemble_leg(C, torch, n_decks, cells, steps, seed, precisions, seq_decks, warm=3,
                 world=1, rank=0, barrier=None, dist=None):
    """One ensemble configuration: per precision, the batched run (autotuned,
    then warm steps, then the rest of the steps timed); then the same decks
    one after another as single chunks (the first seq_decks of them, the
    rate scaled by their cells), and the per-deck summary error of the mixed
    run against the FP64 run at every summary step.

    With world > 1 every rank draws the same decks and runs its share of them
    (replicas.deck_share, balanced by cells) as its own ensemble, with no
    communication between ranks; the time is the slowest rank's (barrier
    before, max over ranks after) over the cells of all the decks, and the
    one-after-another baseline is left to the 1-GPU run."""
    import numpy as np
    all_decks = C.draw_decks(n_decks, seed, cells=cells, end_step=steps, summary_frequency=10)
    total = sum(d.cells for d in all_decks)
    mine = deck_share([d.cells for d in all_decks], rank, world)
    decks = [all_decks[i] for i in mine]
    timed = steps - warm
    out = {"decks": n_decks, "cells_per_axis": list(cells), "steps": steps, "seed": seed,
           "total_cells": total}
    if world > 1:
        out["partition"] = {"ranks": world, "scaling": "strong",
                            "rank0_decks": len(decks),
                            "rank0_cells": sum(d.cells for d in decks)}
    sums = {}
    for prec in precisions:
        key = "fp64" if prec == C.PRECISION_FP64 else "mixed"
        ens = C.Ensemble(decks, prec)
        t0 = time.perf_counter()
        ens.autotune(1)
        tune_s = time.perf_counter() - t0
        ens.step(warm)
        ens.sync()
        if barrier is not None:
            barrier()
        ms = timed_steps(torch, ens, timed)
        ms = max_over_ranks(ms, dist, "cuda")
        assert ens.run() == steps
        bad = [mine[d] for d in range(len(decks)) if ens.deck_status(d) != 0]
        sums[key] = [ens.deck_summaries(d)[0] for d in range(len(decks))]
        sched = ens.schedule()
        out[key] = {
            "value": total * timed / (ms / 1000.0), "unit": "cell-updates/s",
            "ms_per_step": ms / timed, "autotune_s": tune_s,
            "graph_nodes_per_step": ens.launches_per_step, "device_gb": ens.device_bytes / 1e9,
            "decks_with_status": bad,
            "schedule": {"launches": len(sched),
                         "order_counts": [sum(1 for x in sched if x["order"] == o)
                                          for o in range(3)],
                         "grid_div_counts": {str(v): sum(1 for x in sched if x["grid_div"] == v)
                                             for v in sorted({x["grid_div"] for x in sched})},
                         "segs": sorted({x["seg"] for x in sched if x["seg"] > 0})},
        }
        ens.close()
    if world > 1:
        if "fp64" in sums and "mixed" in sums:
            e = max(float(rel_err(a, b)[:, [0, 1, 2, 4]].max())
                    for a, b in zip(sums["mixed"], sums["fp64"]))
            out["mixed_rel_err_vs_fp64"] = {
                "all_summaries_max_over_decks_excluding_ke": max_over_ranks(e, dist, "cuda")}
        return out
    # the same decks one after another (single chunks, graph replay)
    prec = precisions[0]
    key = "fp64" if prec == C.PRECISION_FP64 else "mixed"
    sample = decks[:seq_decks]
    seq_ms = 0.0
    for d in sample:
        ch = C.Chunk(d, prec)
        ch.step(warm)
        ch.sync()
        seq_ms += timed_steps(torch, ch, timed)
        ch.close()
    seq_cells = sum(d.cells for d in sample)
    seq_value = seq_cells * timed / (seq_ms / 1000.0)
    out["sequential"] = {"precision": key, "value": seq_value, "unit": "cell-updates/s",
                         "decks_timed": len(sample),
                         "sample": "first %d of %d decks, rate over their cells" % (
                             len(sample), n_decks)}
    out["speedup_vs_sequential"] = out[key]["value"] / seq_value
    if "fp64" in sums and "mixed" in sums:
        e = np.stack([rel_err(a, b) for a, b in zip(sums["mixed"], sums["fp64"])])  # deck, summary, quantity
        last = e[:, -1, :]
        out["mixed_rel_err_vs_fp64"] = {
            "at_last_summary_max_over_decks": dict(zip(
                ["vol", "mass", "ie", "ke", "press"], [float(x) for x in last.max(axis=0)])),
            "all_summaries_max_over_decks_excluding_ke_at_step0": float(
                max(e[:, :, [0, 1, 2, 4]].max(), e[:, 1:, 3].max() if e.shape[1] > 1 else 0.0)),
        }
    return out


def e2e_dropin(C, args, n, steps):
    """The workload through the drop-in C ABI with host arrays, copies timed.

    Set-up (not timed): the reference's start() over host arrays, which
    allocates them (build_field), registers them as pinned memory on their
    first sight and initialises the chunk, and the warm-up steps; the state is
    then copied back and every mirror marked stale, so the timed run starts
    from the host arrays.
    Timed: the steps of the reference control flow through clover_*_kernel,
    whose first call on each array uploads it from the pinned host array (all
    of the state), the per-step scalar reads (dt, summaries), and the copy of
    every array back to the host at the end."""
    import numpy as np  # noqa: F401
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    warm = max(args.warmup if args is not None else 3, 1)
    deck = C.Deck.from_values(states=STATES, **deck_values(n, warm + steps + 1))
    L = C.lib()
    L.clover_gpu_release()
    L.clover_gpu_synchronize()
    ts = time.perf_counter()
    di = C.DropIn(deck)  # start(): first sight of every host array pins and uploads it
    di.run(warm)  # warm-up steps (the driver's step count is cumulative)
    L.clover_gpu_sync_to_host()
    L.clover_gpu_invalidate_all()
    t0 = time.perf_counter()
    taken = di.run(warm + steps) - warm
    L.clover_gpu_sync_to_host()  # every array back to the host
    t1 = time.perf_counter()
    arrays = ctypes.c_int(0)
    nbytes = ctypes.c_longlong(0)
    L.clover_gpu_mirror_stats(ctypes.byref(arrays), ctypes.byref(nbytes))
    host_bytes = 0
    nx = n
    cell = (nx + 4) ** 3 * 8
    vert = (nx + 5) ** 3 * 8
    face = (nx + 5) * (nx + 4) ** 2 * 8
    host_bytes = 8 * cell + 6 * vert + 9 * face + 7 * vert  # 3D arrays of build_field
    di.close()
    return {"value": n ** 3 * taken / (t1 - t0), "unit": "cell-updates/s",
            "h2d_bytes_per_step": host_bytes / taken,
            "d2h_bytes_per_step": (host_bytes + 8 * taken + 40 * (taken // 10 + 2)) / taken,
            "seconds": t1 - t0, "steps": taken, "cells": "%d^3" % n, "ranks": 1,
            "setup_seconds_untimed": t0 - ts,
            "timed": "the deck's whole run: upload of every host array (pinned) at its first "
                     "use, the steps, per-step dt and summary reads, every array copied back"}


def bricks_leg(C, n=256, n_bricks=8, steps=10):
    """The decomposed run of one deck (clover_decompose's bricks, halo
    messages exchanged between them on the device) against the same deck as
    one chunk, both through the drop-in driver on this GPU, FP64: what the
    exchange costs per step. The bricks share the GPU here; across GPUs each
    rank would hold one (ranks.RankBricks)."""
    deck = C.Deck.from_values(states=STATES, **deck_values(n, steps + 4))
    L = C.lib()
    out = {"cells": "%d^3" % n, "bricks": n_bricks, "steps_timed": steps, "precision": "fp64"}
    for key, make in (("one_chunk", lambda: C.DropIn(deck)),
                      ("bricks", lambda: C.Bricks(deck, n_bricks))):
        L.clover_gpu_release()
        w = make()
        w.run(2)
        L.clover_gpu_synchronize()
        t0 = time.perf_counter()
        w.run(2 + steps)
        L.clover_gpu_synchronize()
        dt = time.perf_counter() - t0
        out[key] = {"value": n ** 3 * steps / dt, "unit": "cell-updates/s",
                    "ms_per_step": 1e3 * dt / steps}
        if key == "bricks":
            out["grid"] = list(w.grid)
        w.close()
    out["bricks_over_one_chunk"] = out["bricks"]["ms_per_step"] / out["one_chunk"]["ms_per_step"]
    return out


def ensembles(C, torch, world=1, rank=0, barrier=None, dist=None):
    """The two ensemble configurations (64 decks FP64 + mixed; 512 small decks
    mixed with its FP64 twin), partitioned over the ranks when world > 1."""
    kw = dict(world=world, rank=rank, barrier=barrier, dist=dist)
    return {
        "decks64": ensemble_leg(C, torch, 64, (24, 128), 150, 2024,
                                [C.PRECISION_FP64, C.PRECISION_MIXED], 64, **kw),
        "decks512": ensemble_leg(C, torch, 512, (16, 48), 100, 4048,
                                 [C.PRECISION_MIXED, C.PRECISION_FP64], 64, **kw),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=512)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-bricks", action="store_true")
    ap.add_argument("--no-tma", action="store_true",
                    help="the register-marching forms of the stencils that stage their planes "
                         "by bulk-tensor copies")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the 200-step FP64 vs mixed comparison")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="only the ensemble legs (a separate JSON line)")
    ap.add_argument("--detail", default=None,
                    help="also write the line with the per-summary accuracy arrays to this file")
    ap.add_argument("--e2e-steps", type=int, default=200,
                    help="steps of the end-to-end run (the configuration's full deck: 200)")
    ap.add_argument("--cpu-configs", action="store_true",
                    help="only the CPU restatement on every configuration (a separate JSON line)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        return run_reference(args)
    if args.cpu_configs:
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"cpu_configs": cpu_configs()}))
        return 0

    import torch
    import torch.distributed as dist
    import cloverleaf3d_ref_b200 as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    if args.ensemble_only:
        ens = ensembles(C, torch, world, rank, barrier, dist)
        if rank == 0:
            print(json.dumps({"ensemble": ens, "n_gpus": world}))
        if world > 1:
            dist.destroy_process_group()
        return 0

    n = args.cells
    prec = C.PRECISION_MIXED if args.precision == "mixed" else C.PRECISION_FP64
    total = args.warmup + 2 * args.steps + 5
    deck = C.Deck.from_values(states=STATES, **deck_values(n, total))
    ch = C.Chunk(deck, prec)
    tma = ch.use_tma(not args.no_tma)
    stream = torch.cuda.ExternalStream(ch.stream)
    # the first step on its own (hydro.f90 reports it apart): wall time of
    # ch.step(1), which also captures and instantiates the step's CUDA graphs
    tf = time.perf_counter()
    ch.step(1)
    ch.sync()
    first_step_ms = 1e3 * (time.perf_counter() - tf)
    ch.step(args.warmup - 1)
    ch.sync()
    launches = ch.launches_per_step

    # timed region A: graph replay
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        ch.step(args.steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ms, dist if world > 1 else None, "cuda")
    clocks = clk.summary()

    # profiled region B: same steps with events around every kernel group
    ch.profile(True)
    ch.step(args.steps)
    groups = ch.profile_report()
    ch.profile(False)
    status = ch.status
    summaries, sum_steps = ch.summaries()
    ch.close()

    value = world * n ** 3 * args.steps / (ms / 1000.0)
    peak, peak_kind = load_peaks()
    top = max(groups, key=lambda g: g["ms"])
    # DRAM bytes per launch of the dominant group, from an ncu capture of its
    # kernels at 256^3 (dram__bytes_read.sum + dram__bytes_write.sum of one
    # direction's staged node pass and velocity pass, the mean over the five
    # of each in profiles/hydro_step_fused_fp64_256_launches.md: 2.356 GB),
    # scaled by the cells to 512^3
    traffic = None
    if top["name"] == "advec_mom_yz" and n == 512 and tma and prec == C.PRECISION_FP64:
        traffic = 2.356e9 * 8
    prof_total_ms = sum(g["ms"] for g in groups)
    achieved = top["bytes"] / (top["ms"] / 1000.0) / 1e9
    step_bytes = sum(g["bytes"] for g in groups) / args.steps
    roofline = {
        "kernel": top["name"], "bound": "hbm", "achieved": achieved, "peak": peak,
        "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
        "traffic": traffic,
        "traffic_source": "ncu capture at 256^3 scaled by cells" if traffic else None,
        "launches": top["launches"], "share": top["ms"] / prof_total_ms,
        "step_algorithmic_bytes_per_cell": step_bytes / n ** 3,
        "step_achieved_gbs": step_bytes / (ms / args.steps / 1000.0) / 1e9,
        "step_frac": step_bytes / (ms / args.steps / 1000.0) / 1e9 / peak,
        "reference_structured_frac": 2512.0 * n ** 3 / (ms / args.steps / 1000.0) / 1e9 / peak,
    }
    per_kernel = {g["name"]: {"ms_per_step": g["ms"] / args.steps,
                              "gbs": g["bytes"] / max(g["ms"], 1e-9) / 1e6,
                              "launches_per_step": g["launches"] / args.steps} for g in groups}

    mixed = None
    if prec == C.PRECISION_FP64 and not args.no_mixed:
        mixed = mixed_leg(C, torch, deck, args, ms, summaries, sum_steps, barrier, world, dist)
        if not args.no_accuracy and rank == 0:
            mixed["accuracy_200_steps"] = accuracy_leg(C, n, 200)

    # every rank takes part in the partitioned ensemble before rank 0 alone
    # runs the end-to-end and CPU legs
    ens = None
    if not args.no_ensemble:
        ens = ensembles(C, torch, world, rank, barrier, dist)
    # the end-to-end leg holds every reference array on the host (~33 GB at
    # 512^3), so it runs on rank 0 only, as the reference arm does
    e2e = None
    if not args.no_e2e and rank == 0:
        e2e = e2e_dropin(C, args, n, args.e2e_steps)
    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_baseline(n)
    bricks = None
    if not args.no_bricks and rank == 0 and world == 1:
        bricks = bricks_leg(C)

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "first_step": {"ms": first_step_ms, "includes": "CUDA graph capture and instantiation",
                           "clock": "host wall time"},
            "vs_baseline": None, "dtype": "f64" if prec == C.PRECISION_FP64 else "f32/f64 mixed",
            "data": "synthetic: two-state shock deck generated on the device",
            "config": {"workload": workload_name(n, args.precision),
                       "execution": "device-resident chunk, graph-replayed steps" +
                                    (", planes staged by bulk-tensor copies" if tma else ""),
                       "cells": n ** 3, "parallelism": "replicas only",
                       "l2": "inputs larger than L2 (each field %.2f GB)" % ((n + 5) ** 3 * 8 / 1e9)},
            "gpu_launches": launches * args.steps + 2 * (args.steps // 10 + 1),
            "clocks": clocks, "roofline": roofline, "per_kernel": per_kernel,
            "status": status,
            "last_summary": {"step": int(sum_steps[-1]), "vol_mass_ie_ke_press":
                             [float(x) for x in summaries[-1]]},
        }
        # bulky detail first, the headline figures last (a reader that keeps
        # only the end of the line keeps those)
        detail = {}
        if mixed and "accuracy_200_steps" in mixed:
            detail["mixed_fp32_accuracy_200_steps"] = mixed["accuracy_200_steps"]
            acc = mixed.pop("accuracy_200_steps")
            mixed["accuracy_200_steps"] = {k: acc[k] for k in ("steps", "cells", "max_rel_err",
                                                                "within_1e-5")}
        if ens:
            line["ensemble"] = ens
        if bricks:
            line["bricks_decomposition"] = bricks
        if mixed:
            line["mixed_fp32"] = mixed
        if cpu:
            line["cpu_baseline"] = cpu
        if e2e:
            line["e2e"] = e2e
        if mixed:
            line["mixed_fp32_summary"] = {
                k: mixed[k] for k in ("value", "ms_per_step", "speedup_vs_fp64")}
            if "accuracy_200_steps" in mixed:
                line["mixed_fp32_summary"]["max_rel_err_200_steps"] = \
                    mixed["accuracy_200_steps"]["max_rel_err"]
        line["roofline"] = line.pop("roofline")
        if args.detail:
            with open(args.detail, "w") as f:
                json.dump(dict(line, **detail), f, indent=1)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
