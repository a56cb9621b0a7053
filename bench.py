#!/usr/bin/env python
"""Throughput of the BSSN RK4 evolution step on B200 (zone-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                    [--workload amr|amr8|singleN|adjoint96] [--formulation bssn|z4c]
                    [--kernel split|fused] [--impl ours|reference] [--report mixed]

A step is one Berger-Oliger coarse step of the workload (every level
advanced to the next coarse time, with its AMR transfers).
`value` is interior zone-updates/s with the state resident in HBM, timed with
CUDA events on the engine's stream; `e2e` is the same metric through the
public engine API with the state copied in from pinned host memory and back out
every step.  Under torchrun each rank advances its own copy of the workload
(no data-path collective); the step time is the max over ranks.

--workload adjoint96 prints the adjoint step time over the forward step time
of the 96^3 gradient workload instead; --report mixed prints the mixed form's
field and constraint errors against FP64 after 20 coarse steps of the amr
hierarchy with m = 0.6, 0.4 and noise 1e-6.

--impl reference times the CPU restatement of the reference's Fortran path
(oracle/, the reference itself cannot be compiled in this image) on the host
cores, over a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nr-amssncku_b200"))

METRIC = "BSSN RK4 zone-updates/s on 1 B200: FP64 vs mixed, %HBM peak; adjoint/fwd ratio"
# algorithmic HBM bytes per zone-update: every field array read or written once per
# substep, 17 words per field per step.  Mixed: FP32 stages for all but the five
# wide fields (chi, alpha, beta^i), FP64 stages for those, FP64 U0/K/U_new:
# (nf - 5) * 112 + 5 * 136.
WIDE_FIELDS = 5


def bytes_per_zone(precision, nf):
    return 17 * nf * 8 if precision == "fp64" else (nf - WIDE_FIELDS) * 112 + WIDE_FIELDS * 136


def workload(name):
    """amr: coarse 96^3 on [-48, 48]^3 (dx = 1) plus 6
    box-in-box levels (48 cells per side per puncture, merged where their
    buffers meet) around Brill-Lindquist punctures m = 0.5 at (+-3, 0, 0), fine
    levels split into seeded uneven blocks; one step = one Berger-Oliger coarse
    step (level l takes 2^l RK4 steps).
    single64: one 64^3-interior block + 3 cells each side
    on [-8, 8]^3, Brill-Lindquist m = 1 at (0.1, 0.05, 0.02), noise 1e-8."""
    from amss_b200.hierarchy import box_in_box, single_block
    if name == "amr":
        # blocks of 24^3 to 80^3 points: 18 to 74 cells plus 3 ghost cells a side
        H = box_in_box(96, 48.0, [(-3.0, 0.0, 0.0), (3.0, 0.0, 0.0)], 7, box_cells=48, seed=1,
                       block_min=18, block_max=74)
        return dict(H=H, masses=[0.5, 0.5], pos=[[-3.0, 0.0, 0.0], [3.0, 0.0, 0.0]], noise=0.0, eps=0.1,
                    courant=0.25, desc="96^3 coarse on [-48,48]^3 + 6 box-in-box levels around "
                                       "BL m=0.5 at (+-3,0,0), uneven blocks of 24^3-80^3 points, dt0=0.25 dx0; "
                                       "step = one Berger-Oliger coarse step")
    if name == "amr8":
        H = box_in_box(96, 48.0, [(0.1, 0.05, 0.02)], 8, box_cells=64, seed=1, block_min=48, block_max=160)
        return dict(H=H, masses=[1.0], pos=[[0.1, 0.05, 0.02]], noise=1e-8, eps=0.1, courant=0.25,
                    desc="96^3 coarse on [-48,48]^3 + 7 box-in-box levels of 64^3 cells around BL m=1 at "
                         "(0.1,0.05,0.02), blocks 48-160 cells, dt0=0.25 dx0, noise 1e-8; step = one "
                         "Berger-Oliger coarse step")
    if name == "amr3":
        H = box_in_box(96, 48.0, [(-3.0, 0.0, 0.0), (3.0, 0.0, 0.0)], 7, box_cells=48, seed=1,
                       block_min=18, block_max=74)
        return dict(H=H, masses=[0.6, 0.4], pos=[[-3.0, 0.0, 0.0], [3.0, 0.0, 0.0]], noise=1e-6, eps=0.1,
                    courant=0.25, desc="the amr hierarchy with BL m=0.6, 0.4 at (+-3,0,0) and noise 1e-6")
    if name.startswith("single") and name[6:].isdigit():
        n = int(name[6:])
        H = single_block(n, -n / 8.0, n / 8.0, 3)
        return dict(H=H, masses=[1.0], pos=[[0.1, 0.05, 0.02]], noise=1e-8, eps=0.1, courant=0.25,
                    desc=f"{n}^3 interior + 3 ghosts ({n + 6}^3 points), one block on [-{n / 8:g},{n / 8:g}]^3, "
                         "BL m=1 at (0.1,0.05,0.02), dx=0.25, dt=0.25dx, eps=0.1, noise 1e-8")
    raise SystemExit(f"unknown workload {name}")


def make_initial(w, nf=24):
    """The workload's initial state per block: get_lousto_nbhs_ on the GPU plus
    the per-cell seeded noise (amss_b200.initial)."""
    from amss_b200 import initial
    return initial.initial_state(w["H"], w["masses"], w["pos"], noise=w["noise"], seed=1, nf=nf)


def make_initial_reference(w, nf=24):
    """The same initial state from the oracle's restatement (reference arm)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import amr as OA
    return OA.initial_state(w["H"], w["masses"], w["pos"], noise=w["noise"], seed=1, nf=nf)


def counts(H):
    """(interior zone-updates, array point-updates) of one coarse step."""
    zones = sum(H.interior_zones(l) * 2 ** l for l in range(len(H.levels)))
    pts = sum(H.points(l) * 2 ** l for l in range(len(H.levels)))
    return zones, pts


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def ncu_traffic(precision, formulation, workload):
    """DRAM bytes per interior zone-update of the substep kernels from the
    committed ncu summary (profiles/substep_traffic.json), with the workload
    and capture it was taken on; (None, why) when there is none for this
    precision and formulation."""
    p = os.path.join(ROOT, "profiles", "substep_traffic.json")
    if not os.path.exists(p):
        return None, "no ncu summary committed"
    d = json.load(open(p))
    key = precision if formulation == "bssn" else f"z4c_{precision}"
    for entry in d.get("captures", []):
        if entry.get("key") == key and entry.get("workload") == workload:
            return entry["bytes_per_zone_update"], entry["source"]
    for entry in d.get("captures", []):
        if entry.get("key") == key:
            return entry["bytes_per_zone_update"], entry["source"] + f" (a {entry['workload']} capture, not {workload})"
    return None, f"no ncu capture for {key}"


def max_over_ranks(value, world, device="cuda"):
    """The maximum of a per-rank value over all ranks; every rank gets it."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms_per_step):
    """Whole-job throughput: every rank advances its own replica of the
    workload, so the job does world x the units in the slowest rank's time."""
    return units_per_rank * world / (ms_per_step * 1e-3)


def time_engine(args, w, init, precision, rank, world, dev):
    """One engine form over the workload: warm-up, K coarse steps replayed as
    a CUDA graph (CUDA events on the engine's stream, bracketed by a barrier
    and a synchronize, max over ranks), then the end-to-end steps through the
    public API with pinned host buffers.  Returns the timings."""
    import torch
    import amss_b200

    H = w["H"]
    dt0 = w["courant"] * H.h0
    tiling = {}
    if args.tune and args.kernel == "split":
        # the stencil pass's tiling per level, measured on a scratch engine
        # before anything is timed (amss_b200.autotune)
        from amss_b200 import autotune
        tiling = autotune.tune(H, init, dt0, precision=precision, formulation=args.formulation, eps=w["eps"],
                               cache=args.tune_cache or None)
    eng = amss_b200.Engine.from_hierarchy(H, precision=precision, eps=w["eps"], kernel=args.kernel,
                                          formulation=args.formulation)
    for i, st in enumerate(init):
        eng.set_state(i, st)
    for lv, (tw, zs, oc, _) in tiling.items():
        eng.set_level_tiling(lv, tw, zs)
        eng.set_level_occupancy(lv, oc)
    if not tiling and args.occupancy is not None and args.kernel == "split":
        for lv in range(len(H.levels)):
            eng.set_level_occupancy(lv, args.occupancy)
    eng.set_punctures(w["pos"])   # Step tracks the punctures on the finest level (MAPBH 0)
    stream = torch.cuda.ExternalStream(eng.stream)

    for _ in range(args.warmup):
        eng.coarse_step(dt0)
    if eng.sync():
        raise SystemExit(f"{precision}: NaN during warm-up")
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = eng.launches
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        if args.graph:
            eng.run_coarse_graph(dt0, nsteps=1, replays=args.steps)
        else:
            for _ in range(args.steps):
                eng.coarse_step(dt0)
        ev1.record(stream)
        ev1.synchronize()
    nan = eng.sync()
    torch.cuda.synchronize()
    try:
        tracked = eng.punctures().tolist()
    except amss_b200.AmssError as exc:   # a puncture left the finest level
        tracked = str(exc)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    launches = eng.launches - launches0
    if world > 1:
        torch.distributed.barrier()

    # end to end through the public API: every block's state in from pinned host
    # memory, one coarse step, every block's state out
    host_in = [torch.empty(st.shape, dtype=torch.float64, pin_memory=True).numpy() for st in init]
    host_out = [torch.empty(st.shape, dtype=torch.float64, pin_memory=True).numpy() for st in init]
    for hi, st in zip(host_in, init):
        hi[...] = st
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for i, hi in enumerate(host_in):
            eng.set_state(i, hi)              # host -> device copy of the step's input
        eng.coarse_step(dt0)
        for i, ho in enumerate(host_out):
            eng.get_state(i, out=ho)          # device -> host copy of the step's result
    t1 = time.perf_counter()
    e2e_ms = max_over_ranks((t1 - t0) * 1e3 / e2e_steps, world)
    eng.close()
    return dict(ms_per_step=ms / args.steps, e2e_ms=e2e_ms, launches=launches, clocks=clk.summary(),
                nan=bool(nan), tracked=tracked,
                tiling={str(lv): [tw, zs, oc, round(t, 4)] for lv, (tw, zs, oc, t) in tiling.items()})


def roofline(precision, nf, zones, ms_per_step, npts, peak):
    """HBM roofline of a coarse step: algorithmic bytes per interior
    zone-update x interior zone-updates / step time.  Array-point bandwidth
    (ghost and buffer cells counted as work too) is reported beside it."""
    bpz = bytes_per_zone(precision, nf)
    achieved = bpz * zones / (ms_per_step * 1e-3) / 1e9
    return dict(achieved=achieved, frac=achieved / peak, algorithmic_bytes_per_zone_update=bpz,
                array_point_gbs=bpz * npts / (ms_per_step * 1e-3) / 1e9)


def run_ours(args, rank, world):
    import torch

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w = workload(args.workload)
    H = w["H"]
    nf = 25 if args.formulation == "z4c" else 24
    init = make_initial(w, nf)
    zones, npts = counts(H)
    hbm_peak, peak_kind = peaks()
    state_bytes = int(sum(st.nbytes for st in init))

    r = time_engine(args, w, init, args.precision, rank, world, dev)
    ms_per_step = r["ms_per_step"]
    value = job_rate(zones, world, ms_per_step)
    rf = roofline(args.precision, nf, zones, ms_per_step, npts, hbm_peak)
    traffic, traffic_src = ncu_traffic(args.precision, args.formulation, args.workload)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "zone-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-stencil/f64-state",
        "data": "synthetic (Brill-Lindquist punctures, generated in-process)",
        "config": {"workload": f"{args.workload}: {w['desc']}", "formulation": args.formulation,
                   "precision": args.precision, "kernel": args.kernel, "graph": bool(args.graph),
                   "zone_updates_per_step_per_gpu": zones, "point_updates_per_step": npts,
                   "levels": len(H.levels), "blocks": len(H.blocks),
                   "puncture_tracking": f"{len(w['pos'])} punctures on the finest level, every substep, "
                                        "inside the step",
                   "l2": "state + stages + K of the hierarchy (GBs) exceed the 126 MB L2; no flush",
                   "parallelism": f"replicas x{world} (no data-path collective)"},
        "roofline": {"bound": "hbm", "achieved": rf["achieved"], "peak": hbm_peak, "unit": "GB/s",
                     "frac": rf["frac"], "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_unit": "B/zone-update", "traffic_source": traffic_src,
                     "kernel": "whole coarse step: RK4 substeps (stencil pass + pointwise pass) and the AMR "
                               "transfers, timed together",
                     "algorithmic_bytes_per_zone_update": rf["algorithmic_bytes_per_zone_update"],
                     "achieved_per_array_point_gbs": rf["array_point_gbs"]},
        "e2e": {"value": job_rate(zones, world, r["e2e_ms"]), "unit": "zone-updates/s",
                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "path": "amss_b200.Engine set_state (pinned, every block) -> coarse_step -> get_state"},
        "gpu_launches": int(r["launches"]),
        "clocks": r["clocks"],
        "nan": r["nan"],
        "tiling": {"per_level": r["tiling"], "what": "stencil-pass tile width (0 = default), z-slabs per block, "
                                                    "occupancy form (0: 2 CTAs/SM, 1: 4 FP64 / 3 FP32) and the "
                                                    "tuner's ms per level step, chosen by amss_b200.autotune before "
                                                    "the timed region"},
        "punctures_after_warmup_and_timed_steps": r["tracked"],
    }
    if args.precision == "fp64" and args.formulation == "bssn" and not args.no_parts:
        # the metric's other two parts: the mixed form on the same workload, and
        # the adjoint/forward step ratio of the 96^3 gradient workload
        m = time_engine(args, w, init, "mixed", rank, world, dev)
        mrf = roofline("mixed", nf, zones, m["ms_per_step"], npts, hbm_peak)
        line["mixed"] = {"value": job_rate(zones, world, m["ms_per_step"]), "unit": "zone-updates/s",
                         "ms_per_step": m["ms_per_step"],
                         "e2e": job_rate(zones, world, m["e2e_ms"]), "roofline_frac": mrf["frac"],
                         "roofline_achieved": mrf["achieved"],
                         "algorithmic_bytes_per_zone_update": mrf["algorithmic_bytes_per_zone_update"],
                         "gpu_launches": int(m["launches"]), "clocks": m["clocks"], "nan": m["nan"],
                         "tiling": m["tiling"]}
        line["mixed_over_fp64"] = ms_per_step / m["ms_per_step"]
        if world == 1:
            a = run_adjoint(args, steps=1, warmup=1)
            line["adjoint"] = {k: a[k] for k in ("metric", "value", "unit", "forward_ms_per_step",
                                                 "adjoint_ms_per_step", "engine_forward_ms_per_step",
                                                 "adjoint_vs_engine_step", "gpu_launches", "clocks")}
            line["adjoint_over_forward"] = a["value"]
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, w, init)
    return line


def _oracle_sample(w, init, budget_s):
    """Time the oracle (C restatement of the reference's Fortran, OpenMP over
    k) on RK4 steps of the finest level until about budget_s have passed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import amr as OA
    H = w["H"]
    oh = OA.OracleHierarchy(H, eps=w["eps"], nf=init[0].shape[0])
    for i, st in enumerate(init):
        oh.set_state(i, st)
    lev = len(H.levels) - 1
    dt = w["courant"] * H.h(lev)
    oh.level_step(lev, dt)       # warm-up
    t0 = time.perf_counter()
    steps = 0
    while True:
        oh.level_step(lev, dt)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return H.interior_zones(lev) * steps / el, steps, lev


def cpu_baseline(args, w, init, budget_s=12.0):
    v, steps, lev = _oracle_sample(w, init, budget_s)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    return {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "port",
            "sample": f"{steps} RK4 step(s) of level {lev} of the workload ({w['H'].interior_zones(lev)} interior "
                      f"zones), FP64, OpenMP over {cores} threads"}


def run_adjoint(args, steps=None, warmup=None):
    """adjoint96: the gradient of L = sum_interior H^2 dV after 200 FP64 RK4
    steps (checkpoint every 20) on one 96^3-interior block on [-12, 12]^3,
    Brill-Lindquist m = 1 at (0.1, 0.05, 0.02) plus a Gaussian on gamma~_xx
    (amplitude 1e-4, width 2, centre uniform in the ball r < 4, seed 1).
    Reports the adjoint step (reverse sweep incl. the segment recompute, per
    step) over the forward step (with checkpointing), and over the engine's
    FP64 step of the same block."""
    import torch
    import amss_b200
    from amss_b200 import initial
    from amss_b200.adjoint import Adjoint
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, nsteps, ck = args.adj_n, args.adj_steps, args.adj_ck
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    X, st, bbox, h = initial.single_block_state(n, -n / 8.0, n / 8.0, 3, [1.0], [[0.1, 0.05, 0.02]])
    rng = np.random.default_rng(1)
    while True:
        c = rng.uniform(-4.0, 4.0, 3)
        if np.linalg.norm(c) < 4.0:
            break
    st[2] += initial.gaussian(X, X, X, 1e-4, 2.0, c)
    dt = 0.25 * h
    ex = (len(X),) * 3
    adj = Adjoint(ex, bbox)
    stream = torch.cuda.ExternalStream(adj.stream)
    for w_i in range(warmup):   # the last at full length: checkpoint and segment storage get allocated
        adj.set_state(st)
        if w_i == warmup - 1:
            adj.forward(dt, nsteps, ck)
        else:
            adj.forward(dt, min(nsteps, 2), 1)
        adj.backward()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), out

    fwd, bwd = [], []
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(steps):
            adj.set_state(st)
            l0 = adj.launches
            t, loss = timed(lambda: adj.forward(dt, nsteps, ck))
            fwd.append(t)
            lf = adj.launches - l0
            t, grad = timed(adj.backward)
            bwd.append(t)
            lb = adj.launches - l0 - lf
    adj.close()
    # the engine's FP64 step of the same block (split kernels, CUDA graph)
    eng = amss_b200.Engine(precision="fp64")
    b = eng.add_block(0, ex, bbox, bbox)
    eng.commit()
    eng.set_state(b, st)
    es = torch.cuda.ExternalStream(eng.stream)
    eng.run_graph(0, dt, 20, 1)
    eng.sync()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    eng.set_state(b, st)
    torch.cuda.synchronize()
    a.record(es)
    eng.run_graph(0, dt, nsteps, 1)
    e.record(es)
    torch.cuda.synchronize()
    eng_ms = a.elapsed_time(e) / nsteps
    eng.close()
    f_ms = max(fwd) / nsteps
    b_ms = max(bwd) / nsteps
    zones = n ** 3
    return {
        "metric": f"adjoint step time / forward step time (FP64, {n}^3, {nsteps} RK4 steps, checkpoint every {ck})",
        "value": round(b_ms / f_ms, 3), "unit": "ratio", "higher_is_better": False, "n_gpus": 1,
        "steps": steps, "warmup": warmup, "dtype": "f64", "data": "synthetic (Brill-Lindquist + "
        "Gaussian on gamma~_xx, generated in-process)",
        "forward_ms_per_step": round(f_ms, 4), "adjoint_ms_per_step": round(b_ms, 4),
        "engine_forward_ms_per_step": round(eng_ms, 4), "adjoint_vs_engine_step": round(b_ms / eng_ms, 3),
        "forward_zone_updates_per_s": zones / (f_ms * 1e-3), "loss": loss,
        "grad_norm": float(np.sqrt(np.sum(grad ** 2))),
        "gpu_launches": {"forward": int(lf), "backward": int(lb)}, "clocks": clk.summary(),
        "config": {"workload": "adjoint96: 96^3 interior + 3 ghosts on [-12,12]^3, BL m=1 at (0.1,0.05,0.02) + "
                               "Gaussian on gamma~_xx (1e-4, width 2), dt=0.25dx, 200 FP64 RK4 steps, checkpoint "
                               "every 20, loss sum_interior H^2 dV"},
    }


def level_constraints(eng, nlev):
    """Per level: the engine's constraint monitor (Parallel::L2Norm of the
    Hamiltonian, momentum and Gamma constraints); returns the Hamiltonian norm,
    the norm of the momentum-constraint magnitude and that of the Gamma
    constraint magnitude."""
    ham, mom, gam = [], [], []
    for lv in range(nlev):
        c = eng.constraint_norms(lv)
        ham.append(float(c[0]))
        mom.append(float(np.sqrt(c[1] ** 2 + c[2] ** 2 + c[3] ** 2)))
        gam.append(float(np.sqrt(c[4] ** 2 + c[5] ** 2 + c[6] ** 2)))
    return ham, mom, gam


def run_mixed_report(args):
    """amr3 (m = 0.6, 0.4, noise 1e-6): the mixed form against the FP64 form
    after `--report-steps` coarse steps from the same initial state: relative
    max-norm error of every field over all blocks, and per-level constraint L2
    norms of both."""
    import torch
    import amss_b200
    from amss_b200.dropin import STATE_NAMES
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    w = workload("amr3")
    H = w["H"]
    init = make_initial(w)
    dt0 = w["courant"] * H.h0
    out, cons = {}, {}
    for prec in ("fp64", "mixed"):
        eng = amss_b200.Engine.from_hierarchy(H, precision=prec, eps=w["eps"])
        for i, st in enumerate(init):
            eng.set_state(i, st)
        eng.run_coarse_graph(dt0, args.report_steps, 1)
        if eng.sync():
            raise SystemExit(f"{prec}: NaN in the state")
        out[prec] = [eng.get_state(i) for i in range(len(H.blocks))]
        cons[prec] = level_constraints(eng, len(H.levels))
        eng.close()
    err = {}
    for f, name in enumerate(STATE_NAMES):
        num = max(float(np.max(np.abs(m[f] - r[f]))) for m, r in zip(out["mixed"], out["fp64"]))
        den = max(float(np.max(np.abs(r[f]))) for r in out["fp64"])
        err[name] = num / den if den > 0 else num
    return {
        "metric": f"mixed vs FP64 after {args.report_steps} coarse steps: relative max-norm field error, "
                  "constraint L2 norms per level",
        "value": max(err.values()), "unit": "relative max-norm error (worst field)", "higher_is_better": False,
        "n_gpus": 1, "dtype": "f32 stencils / f64 state", "data": "synthetic (Brill-Lindquist + noise 1e-6)",
        "field_max_rel_err": err,
        "ham_l2": {p: cons[p][0] for p in cons}, "mom_l2": {p: cons[p][1] for p in cons},
        "gam_l2": {p: cons[p][2] for p in cons},
        "config": {"workload": f"amr3: {w['desc']}", "coarse_steps": args.report_steps},
    }


def run_reference(args, rank, world):
    """The reference arm: the oracle (the C restatement of the reference's
    Fortran) on all host cores, one finest-level RK4 step of the workload per
    bench step.  Only rank 0 works under torchrun."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import amr as OA
    w = workload(args.workload)
    H = w["H"]
    nf = 25 if args.formulation == "z4c" else 24
    init = make_initial_reference(w, nf)
    oh = OA.OracleHierarchy(H, eps=w["eps"], nf=nf)
    for i, st in enumerate(init):
        oh.set_state(i, st)
    lev = len(H.levels) - 1
    dt = w["courant"] * H.h(lev)
    for _ in range(args.warmup):
        oh.level_step(lev, dt)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oh.level_step(lev, dt)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    v = H.interior_zones(lev) / (ms * 1e-3)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {w['desc']}", "formulation": args.formulation,
                   "precision": "fp64",
                   "sample": f"one RK4 step of level {lev} per bench step"},
        "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "port",
                         "sample": f"one RK4 step of level {lev} of the workload per bench step: the C restatement "
                                   "of the reference's Fortran (oracle/), OpenMP over k; the Fortran itself cannot "
                                   "be compiled in this image"},
        "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--workload", default="amr",
                    help="amr | amr8 | singleN (one block of N^3 interior cells, e.g. single64, single320) | "
                         "adjoint96 (adjoint / forward step time)")
    ap.add_argument("--formulation", choices=["bssn", "z4c"], default="bssn")
    ap.add_argument("--kernel", choices=["split", "fused"], default="split")
    ap.add_argument("--graph", type=int, default=1, help="replay the timed steps as one CUDA graph")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune", type=int, default=1, help="pick each level's stencil-pass tiling with the autotuner")
    ap.add_argument("--tune-cache", default="", help="JSON cache of tuned tilings (default: none, tune every run)")
    ap.add_argument("--occupancy", type=int, choices=[0, 1], default=None,
                    help="with --tune 0: the stencil pass's occupancy form on every level (default: the engine's, 0)")
    ap.add_argument("--no-parts", action="store_true",
                    help="FP64 line only: skip the mixed-form and adjoint parts of the metric")
    ap.add_argument("--report", choices=["none", "mixed"], default="none",
                    help="mixed: the mixed form's field and constraint errors against FP64 (amr3 hierarchy)")
    ap.add_argument("--report-steps", type=int, default=20)
    ap.add_argument("--adj-n", type=int, default=96, help="adjoint96: interior cells per side (smaller for ncu)")
    ap.add_argument("--adj-steps", type=int, default=200, help="adjoint96: RK4 steps")
    ap.add_argument("--adj-ck", type=int, default=20, help="adjoint96: checkpoint interval")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.gpus != world:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}: launch N > 1 ranks with torchrun "
                         f"(python -m torch.distributed.run --nproc-per-node N bench.py --gpus N)")
    if args.report == "mixed":
        if rank == 0:
            print(json.dumps(run_mixed_report(args)))
        return
    if args.workload == "adjoint96":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint"}))
        elif rank == 0:
            print(json.dumps(run_adjoint(args)))
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line))
        return
    if world > 1:
        import torch
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=120))
    line = run_ours(args, rank, world)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
