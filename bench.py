#!/usr/bin/env python
"""Throughput benchmark of the Biot/CPML stepper (one JSON line on stdout).

Workload: the 2D x-z layered model of 4000 x 2000 cells (+ a 20-cell CPML on
every face: 4040 x 2040 padded, 8.22 M updated cells per step), dx 5 m,
dt 0.4 ms, 25 Hz Ricker at (2000, 10) on txx/tzz and p, 2000 receivers at
depth 10, second-order stencil, seeded synthetic layers (seed 1).  A "step"
is one time step over the whole grid (velocity phase, stress phase, trace
recording and source injection).  The inputs (1.0 GB FP32 state + coefficients)
are larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       FP32 path (the headline `value`), COMP16 path and an FP64 run of
            the same steps for the seismogram relative L2 of both, device
            timed with CUDA events on the library's stream; `e2e` through the
            public API with pinned host buffers; `roofline` of the dominant
            kernel; `cpu_baseline` = the oracle (C++/OpenMP restatement of the
            reference arithmetic) on a bounded sample, on rank 0 at N = 1.
reference:  the reference's arithmetic on the host cores (the oracle, all
            threads), same workload and metric.  The reference itself is a
            CUDA program with no CPU implementation.
N > 1 runs independent replicas (one shot per GPU, no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mcell-updates/s"
WORKLOAD = "c1: 2D x-z layered 4000x2000 (+20-cell CPML), order 2, dt 0.4 ms, 25 Hz, 2000 receivers"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=4000)
    ap.add_argument("--nz", type=int, default=2000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=20)
    ap.add_argument("--min-timed-s", type=float, default=1.0,
                    help="c1: repeat the K-step timed region until the repetitions cover this many seconds")
    ap.add_argument("--no-batched", action="store_true", help="c1 line: skip the full-size c3 batched object")
    ap.add_argument("--workload", choices=["c0", "c1", "c2", "c3", "c4"], default="c1",
                    help="c1: one 2D shot (default, the headline); c0: the 3D 160^3 order-4 homogeneous shot; "
                         "c2: one 3D 512x512x384 shot; c3: 64 batched 2D shots; c4: serving stream")
    ap.add_argument("--crop-steps", type=int, default=1000, help="c2: steps of the 128^3 crop accuracy runs")
    ap.add_argument("--c0-steps", type=int, default=1000, help="c0: steps of each run (1000 in the configuration)")
    ap.add_argument("--scale", type=float, default=1.0, help="c3/c4: linear size scale of every shot")
    ap.add_argument("--requests", type=int, default=200, help="c4: number of requests")
    ap.add_argument("--precision", choices=["fp32", "comp16", "cbf16"], default="fp32", help="c3/c4 precision")
    ap.add_argument("--only", choices=["fp32", "comp16", "cbf16"], default=None,
                    help="time one precision only and skip the FP64, e2e and CPU legs (profiling runs)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def workload(precision, nt, nx, nz, host=False):
    """The c1 shot; host=True forms its medium without loading the CUDA library
    (the reference arm), with values bit-identical to the library's."""
    from mixedprecisionfaracoustic_b200.presets import config1
    return config1(precision=precision, seed=1, nx=nx, nz=nz, nt=nt, host=host)


def c1_config(args, ws):
    """The `config` object of the c1 line, the same in both arms."""
    return {"workload": WORKLOAD, "grid": [args.nx + 40, args.nz + 40], "order": 2,
            "global_batch": ws, "seq_len": None, "parallelism": f"replicas x{ws}",
            "l2_flush": "inputs larger than L2 (1.0 GB working set)"}


def ncu_traffic():
    """Per-launch DRAM bytes of the dominant kernels from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


C1_STEPS = 8000          # c1's configured run length


def run_ours(args, rank, ws):
    """The c1 line: FP32 (headline) and COMP16 on one shot per GPU.  The timed
    region is K steps bracketed by a barrier and events on the library's
    stream; it is repeated R times (the same R on every rank) so that the
    repetitions cover at least --min-timed-s seconds, and the median region
    gives the per-step time.  Then the FP64 run of the same steps (seismogram
    rel-L2), the per-phase profile, and e2e: the whole configured c1 job
    through the public API."""
    import torch
    from mixedprecisionfaracoustic_b200 import Simulation

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    K, W, P = args.steps, args.warmup, args.profile_steps
    peak, peak_kind = measured_peaks()
    res = {}
    sims = {}
    reps = None
    precs = (args.only,) if args.only else ("fp32", "comp16", "cbf16")
    for prec in precs:
        probe = 128                      # steps timed only to size R
        cfg, med = workload(prec, max(C1_STEPS, W + probe + 4 * K + P), args.nx, args.nz)
        cfg.device = dev
        s = Simulation(cfg, med)
        s.run_timed(W)
        per = max(s.run_timed(probe) / probe, 1e-4)     # after the warm-up: graphs built
        if reps is None:
            reps = max(1, int(np.ceil(args.min_timed_s * 1e3 / (K * per))))
            reps = max(1, min(reps, (cfg.nt - W - probe - P) // K))
            if ws > 1:
                t = torch.tensor([reps], device="cuda", dtype=torch.int64)
                torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
                reps = int(t.item())
        l0 = s.launch_count()
        regions = []
        with ClockSampler(dev) as clk:
            for _ in range(reps):
                if ws > 1:
                    torch.distributed.barrier()
                regions.append(s.run_timed(K))
        launches = (s.launch_count() - l0) // reps
        ms = float(np.median(regions))
        if ws > 1:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        (bv, bt), cells = s.algorithmic_bytes()
        family = s.kernel()
        if family == "fused":
            # one launch per step: the fused kernel is the dominant (only) kernel
            fms, fbpc = s.profile_fused(P)
            pv, pt, pp = fms, 0.0, 0.0
            dom, t_dom, b_dom = "fused_step", fms, fbpc * cells
            bv, bt = fbpc, 0.0
        else:
            pv, pt, pp = s.profile_phases(P)
            dom = "v_phase" if pv >= pt else "t_phase"
            t_dom = max(pv, pt)
            b_dom = (bv if pv >= pt else bt) * cells
        achieved = b_dom / (t_dom * 1e-3) / 1e9
        res[prec] = {
            "kernel_family": family,
            "value": cells * K * ws / (ms * 1e-3) / 1e6,
            "ms_per_step": ms / K,
            "timed_regions": {"count": reps, "steps_each": K, "ms_min": min(regions), "ms_median": ms,
                              "ms_max": max(regions)},
            "launches": launches,
            "clocks": clk.summary(),
            "phase_ms": ({"fused_step": pv} if family == "fused" else
                         {"v_phase": pv, "t_phase": pt, "record_inject": pp}),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "bytes_per_cell": ({"fused_step": bv} if family == "fused" else
                                            {"v_phase": bv, "t_phase": bt}),
                         "step_frac": (bv + bt) * cells / ((pv + pt) * 1e-3) / 1e9 / peak},
            "cells": cells,
            "medium": (f"indexed: {s.medium_tuples()} coefficient tuples, one index byte per cell"
                       if s.medium_tuples() else "per-cell coefficient arrays"),
        }
        sims[prec] = s
    if args.only:
        for s in sims.values():
            s.close()
        return res, None
    # the same FP32 shot reading its per-cell coefficient arrays (what the
    # indexed medium saves)
    cfg, med = workload("fp32", max(C1_STEPS, W + K + 64), args.nx, args.nz)
    cfg.device = dev
    cfg.medium = "dense"
    with Simulation(cfg, med) as sd:
        sd.run_timed(W)
        ms_d = sd.run_timed(K)
        (dv, dt_), _ = sd.algorithmic_bytes()
    res["fp32"]["dense_medium"] = {"value": res["fp32"]["cells"] * K / (ms_d * 1e-3) / 1e6, "unit": METRIC,
                                   "ms_per_step": ms_d / K, "bytes_per_cell": {"v_phase": dv, "t_phase": dt_},
                                   "timed_steps": K}
    # FP64 run of the same steps: seismogram relative L2 of both paths
    steps_run = W + 128 + reps * K + P
    cfg, med = workload("fp64", max(C1_STEPS, W + 128 + 4 * K + P), args.nx, args.nz)
    cfg.device = dev
    s64 = Simulation(cfg, med)
    s64.run(steps_run)
    s64.sync()
    for prec in ("fp32", "comp16", "cbf16"):
        res[prec]["rel_l2_vs_fp64"] = {c: sims[prec].trace_rel_l2(s64, c) for c in ("txx", "tzz", "vux", "vwx", "p")}
        res[prec]["rel_l2_steps"] = steps_run
    s64.close()
    for s in sims.values():
        s.close()
    # end to end through the public API: the whole configured c1 job (8000
    # steps), pinned host medium in, the five seismograms out into pinned buffers
    cfg, med = workload("fp32", C1_STEPS, args.nx, args.nz)
    cfg.device = dev
    pinned = {}
    for k, v in med.items():
        t = torch.empty(v.shape, dtype=torch.float32, pin_memory=True)
        t.numpy()[...] = v
        pinned[k] = t.numpy()
    from mixedprecisionfaracoustic_b200.biot import Medium
    pm = Medium(pinned)
    h2d = sum(a.nbytes for a in pinned.values())
    outs = [torch.empty((cfg.nrec, cfg.nt), dtype=torch.float32, pin_memory=True).numpy() for _ in range(5)]
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    s = Simulation(cfg, pm)
    s.run(cfg.nt)
    tr = [s.traces(c, out=o) for c, o in zip(("txx", "tzz", "vux", "vwx", "p"), outs)]
    s.close()
    e2e_s = time.perf_counter() - t0
    d2h = sum(a.nbytes for a in tr)
    if ws > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": res["fp32"]["cells"] * cfg.nt * ws / e2e_s / 1e6, "unit": METRIC,
           "h2d_bytes_per_step": h2d / cfg.nt, "d2h_bytes_per_step": d2h / cfg.nt, "steps": cfg.nt,
           "seconds": e2e_s,
           "path": f"bp_create(pinned host medium) + bp_run({cfg.nt}) + bp_get_traces x5 + bp_destroy: "
                   f"the whole c1 job"}
    return res, e2e


def run_batched(args):
    """c3 at full size in the default line: 64 2D shots (sizes from {1024^2,
    1536x1024, 2048^2, 3072x1536}, seed 3), one persistent launch per phase for
    all shots, FP32 and COMP16.  The autotuner runs first (its steps are real
    steps of the shots, outside the timed region); then max(K, 100) steps are
    timed with CUDA events on the batch's stream."""
    from mixedprecisionfaracoustic_b200 import Batch
    from mixedprecisionfaracoustic_b200.presets import config3_shots
    K = max(args.steps, 100)
    tune_budget = 800
    shots = config3_shots(seed=3, nshots=64, nt=4000, precision="fp32")
    cells = sum((c.padded[0] - 2) * (c.padded[2] - 2) for c, _ in shots)
    peak, peak_kind = measured_peaks()
    out = {"workload": "c3: 64 batched 2D shots at full size (seed 3), order 2, 4000-step shots",
           "cells_per_step": cells, "timed_steps": K}
    for prec in ("fp32", "comp16", "cbf16"):
        for c, _ in shots:
            c.precision = prec
        b = Batch([c for c, _ in shots], [m for _, m in shots])
        tune = b.autotune(tune_budget)
        # algorithmic bytes per updated cell of the step the chosen kernels run:
        # two phases (each array once per phase: the library's count, an
        # indexed medium's coefficients as one index byte per phase) or the
        # fused step (fields once each way, coefficients once)
        indexed = all(b.medium_tuples(i) > 0 for i in range(len(shots)))
        wb = 4.0 if prec == "fp32" else 3.0
        if tune["kernel"] == "fused":
            bpc = 2 * 8 * wb + (1.0 if indexed else 12 * wb)
        else:
            bpc = b.algorithmic_bytes() / cells
        b.run(max(args.warmup, 3))
        b.sync()
        with ClockSampler(0) as clk:
            ms = b.run_timed(K)
        b.sync()
        got = bpc * cells * K / (ms * 1e-3) / 1e9
        out[prec] = {"value": cells * K / (ms * 1e-3) / 1e6, "unit": METRIC, "ms_per_step": ms / K,
                     "tune": tune, "clocks": clk.summary(),
                     "medium": ("indexed: " + ", ".join(str(b.medium_tuples(i)) for i in range(3)) + ", ... tuples"
                                if indexed else "per-cell coefficient arrays"),
                     "roofline": {"bound": "hbm", "kernel": "step", "bytes_per_cell": bpc, "achieved": got,
                                  "peak": peak, "unit": "GB/s", "frac": got / peak, "peak_source": peak_kind}}
        b.close()
    out["speedup_comp16_vs_fp32"] = out["comp16"]["value"] / out["fp32"]["value"]
    out["speedup_cbf16_vs_fp32"] = out["cbf16"]["value"] / out["fp32"]["value"]
    return out


def cpu_baseline(args, budget_s=20.0):
    """The oracle (REF32, all host threads) on a bounded sample of the workload."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    cfg, med = workload("fp32", 8, args.nx, args.nz, host=True)
    probe = O.Oracle(cfg, med, O.REF32)
    probe.run(2)
    t0 = time.perf_counter()
    probe.run(3)
    per = (time.perf_counter() - t0) / 3
    probe.close()
    n = int(max(3, budget_s / max(per, 1e-6)))
    cfg, med = workload("fp32", n + 4, args.nx, args.nz, host=True)
    o = O.Oracle(cfg, med, O.REF32)
    o.run(2)
    t0 = time.perf_counter()
    o.run(n)
    el = time.perf_counter() - t0
    cells = (cfg.padded[0] - 2) * (cfg.padded[2] - 2)
    o.close()
    return {"value": cells * n / el / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"c1 full {cfg.padded[0]}x{cfg.padded[2]} grid, steps 2..{2 + n} ({el:.1f} s), REF32 arithmetic, "
                      f"{threads} OpenMP threads"}


def run_reference(args, rank, ws):
    """Reference arm: the reference's update equations (the oracle's REF32
    arithmetic) on all host cores, on the same c1 workload.  Nothing here loads
    the CUDA library: the medium is formed on the host."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    K, W = args.steps, args.warmup
    nz = args.nz
    cfg, med = workload("fp32", 4, args.nx, nz, host=True)
    probe = O.Oracle(cfg, med, O.REF32)
    probe.run(1)
    t0 = time.perf_counter()
    probe.run(1)
    per_full = time.perf_counter() - t0
    probe.close()
    budget = 150.0
    if (K + W) * per_full > budget:      # bounded sample: fewer rows, same nx and medium statistics
        nz = max(64, int(nz * budget / ((K + W) * per_full)))
    cfg, med = workload("fp32", K + W + 1, args.nx, nz, host=True)
    o = O.Oracle(cfg, med, O.REF32)
    o.run(W)
    t0 = time.perf_counter()
    o.run(K)
    el = time.perf_counter() - t0
    cells = (cfg.padded[0] - 2) * (cfg.padded[2] - 2)
    v = cells * K / el / 1e6
    sample = f"{cfg.padded[0]}x{cfg.padded[2]} grid ({nz} of {args.nz} physical rows), {K} steps, REF32"
    return {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus, "steps": K, "warmup": W,
            "ms_per_step": el / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": c1_config(args, ws),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def fp64_rel_l2(cfg, med, got, steps, min_signal=0.0):
    """Seismogram rel-L2 of traces `got` (component -> [nrec, >= steps]) against an FP64
    run of the same shot for `steps` steps; None if the FP64 traces never exceed
    `min_signal` (the wave has not reached the receivers yet)."""
    import copy
    from mixedprecisionfaracoustic_b200 import Simulation
    c = copy.copy(cfg)
    c.precision = "fp64"
    c.nt = steps
    with Simulation(c, med) as s:
        s.run(steps)
        out = {}
        for comp, a in got.items():
            ref = s.traces(comp).astype(np.float64)
            if np.abs(ref).max() <= min_signal:
                return None
            d = np.asarray(a, dtype=np.float64)[:, :steps]
            out[comp] = float(np.linalg.norm(d - ref) / max(np.linalg.norm(ref), 1e-300))
    return out


def run_batch(args, rank, ws):
    """c3: 64 2D shots (sizes from {1024^2, 1536x1024, 2048^2, 3072x1536}) in one
    persistent launch per phase and graph-replayed chunks; this rank's share of
    the shots (replicas.shard) when N > 1."""
    import torch
    from mixedprecisionfaracoustic_b200 import Batch
    from mixedprecisionfaracoustic_b200.presets import config3_shots
    from mixedprecisionfaracoustic_b200.replicas import max_over_ranks, my_shots, shot_cost
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    K, W = args.steps, args.warmup
    shots = config3_shots(seed=3, nshots=64, nt=W + K + 400, precision=args.precision, scale=args.scale)
    mine = my_shots([shot_cost(c) for c, _ in shots], rank, ws)
    cfgs = [shots[i][0] for i in mine]
    for c in cfgs:
        c.device = dev
    b = Batch(cfgs, [shots[i][1] for i in mine])
    b.run(W)                   # includes the autotuner's timed candidate steps
    b.sync()
    u0 = b.cell_updates()
    if ws > 1:
        torch.distributed.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with ClockSampler(dev) as clk:
        b.run(K)
        b.sync()
    el = max_over_ranks(time.perf_counter() - t0)
    upd = b.cell_updates() - u0
    # accuracy against FP64 runs of the same steps, for the first three of this
    # rank's shots whose receivers the wave has reached within those steps
    acc = {}
    for j in range(min(12, len(mine))):
        if len(acc) == 3:
            break
        i = mine[j]
        got = {c: b.traces(j, c) for c in ("txx", "p")}
        r = fp64_rel_l2(shots[i][0], shots[i][1], got, W + K, min_signal=1e-6)
        if r is not None:
            acc[f"shot{i}"] = r
    tot = upd
    if ws > 1:
        t = torch.tensor([float(upd)], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t)
        tot = int(t.item())
    tune = b.tune()
    b.close()
    return {"metric": METRIC, "value": tot / el / 1e6, "unit": METRIC, "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": el / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f16+i8 storage, f32 math", "data": "synthetic",
            "config": {"workload": f"c3: 64 batched 2D shots x{args.scale} size, {args.precision}",
                       "shots_on_rank0": len(mine), "tune": tune, "parallelism": f"shots sharded over {ws}"},
            "clocks": clk.summary(), "timing": "host wall clock around bp_batch_run + bp_batch_sync",
            "rel_l2_vs_fp64_sample": acc}


def run_c0(args):
    """c0: 3D homogeneous 160^3 (+20-cell CPML = 200^3), order 4, 1000 steps, FP32
    and COMP16: Mcell-updates/s, phase HBM GB/s vs the measured peak, and the
    seismogram rel-L2 of each against an FP64 run of the same 1000 steps."""
    import torch
    from mixedprecisionfaracoustic_b200 import Simulation
    from mixedprecisionfaracoustic_b200.presets import config0
    torch.cuda.set_device(0)
    nt = max(args.c0_steps, 30)
    peak, peak_kind = measured_peaks()
    runs = {}
    res = {}
    for prec in ("fp64", "fp32", "comp16"):
        cfg, med = config0(precision=prec, order=4, nt=nt)
        s = Simulation(cfg, med)
        s.run(5)
        s.sync()
        with ClockSampler(0) as clk:
            ms = s.run_timed(nt - 5 - 10)
        (bv, bt), cells = s.algorithmic_bytes()
        pv, pt, pp = s.profile_phases(10)
        s.sync()
        runs[prec] = s
        res[prec] = {"value": cells * (nt - 15) / (ms * 1e-3) / 1e6, "ms_per_step": ms / (nt - 15),
                     "phase_ms": {"v_phase": pv, "t_phase": pt, "record_inject": pp},
                     "frac": {"v_phase": bv * cells / (pv * 1e-3) / 1e9 / peak,
                              "t_phase": bt * cells / (pt * 1e-3) / 1e9 / peak,
                              "step": (bv + bt) * cells / ((pv + pt) * 1e-3) / 1e9 / peak},
                     "cells": cells, "clocks": clk.summary()}
    for prec in ("fp32", "comp16"):
        res[prec]["rel_l2_vs_fp64"] = {c: runs[prec].trace_rel_l2(runs["fp64"], c) for c in ("txx", "tzz", "vux", "p")}
    for s in runs.values():
        s.close()
    f32 = res["fp32"]
    return {"metric": METRIC, "value": f32["value"], "unit": METRIC, "n_gpus": 1, "steps": nt - 15, "warmup": 5,
            "ms_per_step": f32["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"c0: 3D homogeneous 160^3 (+20-cell CPML = 200^3), order 4, 128 receivers, "
                                   f"{nt} steps", "l2_flush": "inputs larger than L2 (1.9 GB working set)"},
            "roofline": {"bound": "hbm", "kernel": "step", "achieved": f32["frac"]["step"] * peak, "peak": peak,
                         "unit": "GB/s", "frac": f32["frac"]["step"], "peak_source": peak_kind},
            "fp32": f32, "comp16": res["comp16"], "fp64": {k: res["fp64"][k] for k in ("value", "ms_per_step")}}


def run_c2(args):
    """c2: the 3D 512x512x384 log-normal model (+20-cell CPML), COMP16 and FP32:
    Mcell-updates/s and the phase kernels' HBM GB/s against the measured peak;
    seismogram rel-L2 of COMP16 (and FP32) vs FP64 on a 128^3 crop of the same
    model around the source (the full model is too large for an FP64 run)."""
    import torch
    from mixedprecisionfaracoustic_b200 import Simulation
    from mixedprecisionfaracoustic_b200.presets import config2, config2_crop
    torch.cuda.set_device(0)
    K, W, P = min(args.steps, 300), max(args.warmup, 3), 5
    peak, peak_kind = measured_peaks()
    t0 = time.perf_counter()
    base, med = config2(precision="comp16", nt=W + K + P)
    gen_s = time.perf_counter() - t0
    res = {}
    for prec in ("comp16", "fp32"):
        base.precision = prec
        with Simulation(base, med) as s:
            s.run(W)
            s.sync()
            with ClockSampler(0) as clk:
                ms = s.run_timed(K)
            (bv, bt), cells = s.algorithmic_bytes()
            pv, pt, pp = s.profile_phases(P)
        res[prec] = {"value": cells * K / (ms * 1e-3) / 1e6, "ms_per_step": ms / K,
                     "phase_ms": {"v_phase": pv, "t_phase": pt, "record_inject": pp},
                     "hbm_GBps": {"v_phase": bv * cells / (pv * 1e-3) / 1e9, "t_phase": bt * cells / (pt * 1e-3) / 1e9,
                                  "step": (bv + bt) * cells / ((pv + pt) * 1e-3) / 1e9},
                     "bytes_per_cell": {"v_phase": bv, "t_phase": bt}, "cells": cells, "clocks": clk.summary()}
        for k in ("v_phase", "t_phase", "step"):
            res[prec].setdefault("frac", {})[k] = res[prec]["hbm_GBps"][k] / peak
    # accuracy on the crop
    acc = {}
    ref = None
    for prec in ("fp64", "comp16", "fp32"):
        c, m = config2_crop(base, med, size=128, precision=prec, nt=args.crop_steps)
        s = Simulation(c, m)
        s.run(c.nt)
        s.sync()
        if prec == "fp64":
            ref = s
            continue
        acc[prec] = {comp: s.trace_rel_l2(ref, comp) for comp in ("txx", "tzz", "vux", "p")}
        s.close()
    ref.close()
    c16 = res["comp16"]
    return {"metric": METRIC, "value": c16["value"], "unit": METRIC, "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": c16["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16+i8 storage, f32 math", "data": "synthetic",
            "config": {"workload": "c2: 3D log-normal 512x512x384 (+20-cell CPML = 552x552x424), order 2, "
                                   "65,536 surface receivers", "medium_generation_s": gen_s,
                       "l2_flush": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "kernel": "step", "achieved": c16["hbm_GBps"]["step"], "peak": peak,
                         "unit": "GB/s", "frac": c16["frac"]["step"], "peak_source": peak_kind},
            "comp16": c16, "fp32": res["fp32"], "speedup_comp16_vs_fp32": c16["value"] / res["fp32"]["value"],
            "rel_l2_vs_fp64_crop128": {"steps": args.crop_steps, **acc}}


def run_serve(args, rank):
    """c4: Poisson stream of shot requests into the server at ~80% of its measured
    capacity; p50/p99 latency and Mcell-updates/s (rank 0 only)."""
    import torch
    from mixedprecisionfaracoustic_b200 import Server
    from mixedprecisionfaracoustic_b200.presets import config4_requests
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    reqs = config4_requests(seed=4, n=args.requests, precision=args.precision, scale=args.scale, lazy=True)
    work = sum((c.padded[0] - 2) * max(c.padded[1] - 2, 1) * (c.padded[2] - 2) * c.nt for c, _ in reqs)
    srv = Server(hbm_budget_bytes=150 << 30, steps_per_sync=100, device=dev)
    # capacity probe: the first 6 2D and the first 2 3D requests, each class
    # back to back, and the stream's capacity as the work-weighted harmonic
    # mean of the two (a probe of the first 8 alone, mostly 2D, overstated the
    # capacity of a stream whose work is mostly 3D)
    def cells_of(c):
        return (c.padded[0] - 2) * max(c.padded[1] - 2, 1) * (c.padded[2] - 2) * c.nt
    cap_of = {}
    for dim, k in ((2, 6), (3, 2)):
        sample = [(c, m) for c, m in reqs if c.dim == dim][:k]
        if not sample:
            continue
        t0 = time.perf_counter()
        probe = [srv.submit(c, m()) for c, m in sample]
        for r in probe:
            srv.wait(r, 3600)
        cap_of[dim] = sum(cells_of(c) for c, _ in sample) / (time.perf_counter() - t0)
        for r in probe:
            srv.release(r)
    work_of = {d: sum(cells_of(c) for c, _ in reqs if c.dim == d) for d in cap_of}
    cap = sum(work_of.values()) / sum(work_of[d] / cap_of[d] for d in cap_of)
    rate = 0.8 * cap / (work / len(reqs))         # requests per second at 80% of capacity
    rng = np.random.default_rng(4)
    gaps = rng.exponential(1.0 / rate, len(reqs))
    ids = []
    with ClockSampler(dev) as clk:
        t0 = time.perf_counter()
        nxt = t0
        for (c, m), g in zip(reqs, gaps):
            nxt += g
            while time.perf_counter() < nxt:
                time.sleep(min(0.001, max(0.0, nxt - time.perf_counter())))
            ids.append(srv.submit(c, m()))
        for r in ids:
            srv.wait(r, 7200)
        el = time.perf_counter() - t0
    lat = sorted(srv.latency(r) for r in ids)
    # accuracy of a fixed sample of the requests (2D and 3D) against FP64 runs
    acc = {}
    sample = [i for i, (c, _) in enumerate(reqs) if c.dim == 2][:2] + [i for i, (c, _) in enumerate(reqs) if c.dim == 3][:1]
    for i in sample:
        c, m = reqs[i]
        got = {comp: srv.traces(ids[i], comp) for comp in ("txx", "p")}
        acc[f"req{i}_{c.dim}d"] = fp64_rel_l2(c, m(), got, c.nt)
    st = srv.stats()
    srv.close()
    return {"metric": METRIC, "value": work / el / 1e6, "unit": METRIC, "n_gpus": 1, "steps": None, "warmup": 8,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f16+i8 storage, f32 math", "data": "synthetic",
            "config": {"workload": f"c4: {len(reqs)} Poisson requests x{args.scale} size, {args.precision}",
                       "rate_per_s": rate, "capacity_cell_updates_per_s": cap,
                       "capacity_probe": {f"{d}d": v for d, v in cap_of.items()}, "hbm_budget_GB": 150},
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "server": {k: st[k] for k in ("completed", "max_resident", "busy_seconds", "cell_updates")},
            "clocks": clk.summary(), "elapsed_s": el, "requests_3d": sum(1 for c, _ in reqs if c.dim == 3),
            "timing": "host wall clock from first submit to last completion",
            "rel_l2_vs_fp64_sample": acc}


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.workload in ("c0", "c2") and args.impl == "ours":
        if rank == 0:
            print(json.dumps(run_c0(args) if args.workload == "c0" else run_c2(args)), flush=True)
        return 0
    if args.workload != "c1" and args.impl == "ours":
        if ws > 1:
            import torch
            import torch.distributed as dist
            from datetime import timedelta
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        out = run_batch(args, rank, ws) if args.workload == "c3" else (run_serve(args, rank) if rank == 0 else None)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return 0
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if args.impl == "reference":
            if rank != 0:
                return 0
        else:
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    if args.impl == "reference":
        print(json.dumps(run_reference(args, rank, ws)), flush=True)
        return 0
    res, e2e = run_ours(args, rank, ws)
    out = None
    if args.only and rank == 0:
        print(json.dumps({"metric": METRIC, "only": args.only, **res[args.only]}), flush=True)
    elif rank == 0:
        f32, c16 = res["fp32"], res["comp16"]
        batched = None if (args.no_batched or ws > 1) else run_batched(args)
        cpu = None if (args.no_cpu_baseline or ws > 1) else cpu_baseline(args)
        traffic = ncu_traffic()
        def tkey(prec, r):                 # ncu captures of the same medium representation
            return f"{prec}_{r['roofline']['kernel']}" + ("_indexed" if r["medium"].startswith("indexed") else "")
        roof = dict(f32["roofline"])
        roof["traffic"] = traffic.get(tkey("fp32", f32))
        c16roof = dict(c16["roofline"])
        c16roof["traffic"] = traffic.get(tkey("comp16", c16))
        b24 = res["cbf16"]
        b24roof = dict(b24["roofline"])
        b24roof["traffic"] = traffic.get(tkey("cbf16", b24))
        out = {
            "metric": METRIC, "value": f32["value"], "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": f32["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": c1_config(args, ws),
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": f32["launches"],
            "clocks": f32["clocks"],
            "rel_l2_vs_fp64": f32["rel_l2_vs_fp64"],
            "timed_regions": f32["timed_regions"],
            "phase_ms": f32["phase_ms"],
            "medium": f32["medium"],
            "dense_medium": f32["dense_medium"],
            "comp16": {"value": c16["value"], "ms_per_step": c16["ms_per_step"], "roofline": c16roof,
                       "medium": c16["medium"],
                       "rel_l2_vs_fp64": c16["rel_l2_vs_fp64"], "phase_ms": c16["phase_ms"],
                       "gpu_launches": c16["launches"], "clocks": c16["clocks"],
                       "timed_regions": c16["timed_regions"],
                       "speedup_vs_fp32": c16["value"] / f32["value"]},
            "cbf16": {"value": b24["value"], "ms_per_step": b24["ms_per_step"], "roofline": b24roof,
                      "medium": b24["medium"],
                      "storage": "bf16 hi + 8-bit residual (top 24 bits of fp32), fp32 math",
                      "rel_l2_vs_fp64": b24["rel_l2_vs_fp64"], "phase_ms": b24["phase_ms"],
                      "gpu_launches": b24["launches"], "clocks": b24["clocks"],
                      "timed_regions": b24["timed_regions"],
                      "speedup_vs_fp32": b24["value"] / f32["value"]},
            "batched": batched,
        }
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
