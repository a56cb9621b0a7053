#!/usr/bin/env python
"""Throughput of the BSSN RK4 evolution step on B200 (zone-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                    [--workload single64] [--impl ours|reference]

A step is one full RK4 step (four fused substep launches) of the workload.
`value` is interior zone-updates/s with the state resident in HBM, timed with
CUDA events on the engine's stream; `e2e` is the same metric through the
public engine API with the state copied in from pinned host memory and back out
every step.  Under torchrun each rank advances its own copy of the workload
(no data-path collective); the step time is the max over ranks.

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
NF = 24
# algorithmic HBM bytes per zone-update: every field array read or written once per
# substep, 17 words per field per step.  Mixed: FP32 stages for 22 fields, FP64
# stages for chi and alpha, FP64 U0/K/U_new: 22 * 112 + 2 * 136.
BYTES_PER_ZONE = {"fp64": 17 * NF * 8, "mixed": 22 * 112 + 2 * 136}


def workload(name):
    """Config 1: one 64^3-interior block + 3 cells each side on [-8, 8]^3,
    Brill-Lindquist m = 1 at (0.1, 0.05, 0.02), noise 1e-8, dt = 0.25 dx."""
    if name == "single64":
        return dict(n_interior=64, lo=-8.0, hi=8.0, ghosts=3, masses=[1.0], pos=[[0.1, 0.05, 0.02]],
                    noise=1e-8, eps=0.1, courant=0.25)
    raise SystemExit(f"unknown workload {name}")


def make_initial(w):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # initial data only (Brill-Lindquist, get_lousto_nbhs)
    X, st, bbox, h = O.single_block_setup(w["n_interior"], w["lo"], w["hi"], w["ghosts"], w["masses"], w["pos"],
                                          noise=w["noise"], seed=1)
    return X, st, bbox, h


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


def ncu_traffic(precision):
    """Per-launch DRAM bytes of the substep kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "substep_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get(precision)
    return None


def run_ours(args, rank, world):
    import torch
    import amss_b200

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w = workload(args.workload)
    X, st0, bbox, h = make_initial(w)
    n = len(X)
    dt = w["courant"] * h
    zones = w["n_interior"] ** 3          # interior zones of the block
    npts = n ** 3                         # points the kernels update
    eng = amss_b200.Engine(precision=args.precision, eps=w["eps"])
    b = eng.add_block(0, (n, n, n), bbox, bbox)
    eng.commit()
    eng.set_state(b, st0)
    stream = torch.cuda.ExternalStream(eng.stream)

    # warm-up, then K timed steps bracketed by a barrier + synchronize
    for _ in range(args.warmup):
        eng.step(0, dt)
    if eng.sync():
        raise SystemExit("NaN during warm-up")
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = eng.launches
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            eng.step(0, dt)
        ev1.record(stream)
        ev1.synchronize()
    nan = eng.sync()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = eng.launches - launches0
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        torch.distributed.barrier()
    ms_per_step = ms / args.steps

    # end to end through the public API: pinned host state in, one step, state out
    host_in = torch.empty(st0.shape, dtype=torch.float64, pin_memory=True).numpy()
    host_out = torch.empty(st0.shape, dtype=torch.float64, pin_memory=True).numpy()
    host_in[...] = st0
    e2e_steps = max(2, min(args.steps, 10))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.set_state(b, host_in)          # host -> device copy of the step's input
        eng.step(0, dt)
        eng.get_state(b, out=host_out)     # device -> host copy of the step's result
    t1 = time.perf_counter()
    e2e_ms = (t1 - t0) * 1e3 / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    eng.close()

    value = zones * world / (ms_per_step * 1e-3)
    hbm_peak, peak_kind = peaks()
    alg_bytes_per_step = BYTES_PER_ZONE[args.precision] * npts
    achieved = alg_bytes_per_step / (ms_per_step * 1e-3) / 1e9
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
        "data": "synthetic (Brill-Lindquist puncture + seeded 1e-8 noise, generated in-process)",
        "config": {"workload": f"{args.workload}: 64^3 interior + 3 ghosts (70^3 points), one block, "
                               "BL m=1 at (0.1,0.05,0.02), dx=0.25, dt=0.25dx, eps=0.1",
                   "precision": args.precision, "zones_per_step_per_gpu": zones, "points_per_step": npts,
                   "l2": "working set 4 x 24 x 70^3 words (>= 264 MB FP64) exceeds the 126 MB L2; no flush",
                   "parallelism": f"replicas x{world} (no data-path collective)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                     "traffic": ncu_traffic(args.precision),
                     "kernel": "k_substep (fused RHS + RK4 substep)",
                     "algorithmic_bytes_per_point_step": BYTES_PER_ZONE[args.precision]},
        "e2e": {"value": zones * world / (e2e_ms * 1e-3), "unit": "zone-updates/s",
                "h2d_bytes_per_step": int(st0.nbytes), "d2h_bytes_per_step": int(st0.nbytes),
                "path": "amss_b200.Engine set_state (pinned) -> step -> get_state"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "nan": bool(nan),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, w)
    return line


def cpu_baseline(args, w, budget_s=12.0):
    """The oracle (C restatement of the reference's Fortran, OpenMP over k) on
    the host cores: RK4 steps of the full config-1 block until ~budget_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    X, st, bbox, h = make_initial(w)
    dt = w["courant"] * h
    O.bssn_step_single(X, X, X, bbox, st, dt, eps=w["eps"])   # warm-up
    t0 = time.perf_counter()
    steps = 0
    while True:
        O.bssn_step_single(X, X, X, bbox, st, dt, eps=w["eps"])
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt_s = time.perf_counter() - t0
    zones = w["n_interior"] ** 3
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    return {"value": zones * steps / dt_s, "unit": "zone-updates/s", "cores": cores, "kind": "port",
            "sample": f"{steps} RK4 step(s) of the full 70^3 config-1 block, FP64, OpenMP over {cores} threads"}


def run_reference(args, rank, world):
    """The reference arm: one RK4 step of the config-1 block per bench step,
    run by the oracle (the C restatement of the reference's Fortran) on all
    host cores.  Only rank 0 works under torchrun."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    w = workload(args.workload)
    X, st, bbox, h = make_initial(w)
    dt = w["courant"] * h
    for _ in range(args.warmup):
        O.bssn_step_single(X, X, X, bbox, st, dt, eps=w["eps"])
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.bssn_step_single(X, X, X, bbox, st, dt, eps=w["eps"])
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    zones = w["n_interior"] ** 3
    v = zones / (ms * 1e-3)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: 64^3 interior + 3 ghosts, one block (as the GPU arm)",
                   "precision": "fp64"},
        "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "port",
                         "sample": "one RK4 step of the full 70^3 config-1 block per bench step: the C "
                                   "restatement of the reference's Fortran (oracle/), OpenMP over k; the "
                                   "Fortran itself cannot be compiled in this image"},
        "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--workload", default="single64")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
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
