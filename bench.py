"""Throughput of the explicit structured-block update on B200.

Default workload: 256^3 ideal-air Euler block on the unit cube (Mach-3 inflow
at i-min, extrapolate outflow at i-max, slip walls elsewhere, density
perturbed by 8 seeded sines), HLLC flux, MUSCL/van Albada, predictor-corrector,
CFL 0.5.  A bench "step" is one full time step (both predictor-corrector
stages, ghost cells, decode and the dt control every 10 steps) over the block.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32_flux]
                  [--impl ours|reference] [--n 256] [--flux hllc|ausmdv]

Prints one JSON line (rank 0).  --impl reference times the CPU FP64
restatement of the reference algorithm (the D solver itself cannot be built:
no D compiler) on the host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s (256^3 Euler)"
UNIT = "cell-updates/s"
# Algorithmic bytes per cell-update (both stages): FP64 W (5) + U (5) per
# stage read/write as laid out in DESIGN.md: 45 doubles; FP32-flux form 280 B.
BYTES_PER_CELL_UPDATE = {"fp64": 360.0, "fp32_flux": 280.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_rate(n, steps, flux, threads=0, seed=None):
    """Cell-updates/s of the CPU FP64 oracle on an n^3 block of the workload."""
    from eilmer4_b200 import workloads as W
    from oracle import e4_oracle as O
    O.build()
    b = W.inflow_3d_block(n, n, n, seed if seed is not None else W.DEFAULT_SEED)
    cfg = O.default_config(dimensions=3, flux_calculator=O.FLUX_HLLC if flux == "hllc"
                           else O.FLUX_AUSMDV, n_threads=threads)
    sim = O.OracleSim(cfg)
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    sim.run(1)  # first touch / dt initialisation
    t0 = time.perf_counter()
    rc = sim.run(steps)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    return n ** 3 * steps / dt, cores, dt


def run_reference(args, rank, world):
    if rank != 0:
        return
    n = args.ref_sample
    rates = []
    for _ in range(args.warmup):
        cpu_oracle_rate(n, 1, args.flux)
    for _ in range(args.steps):
        r, cores, _ = cpu_oracle_rate(n, 1, args.flux)
        rates.append(r)
    value = statistics.median(rates)
    sample = f"{n}^3 sub-block of the {args.n}^3 workload, 1 time step per bench step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * args.n ** 3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"inflow_3d {args.n}^3 {args.flux} MUSCL/vanAlbada PC CFL0.5",
                   "sample": sample, "parallelism": "cpu-openmp"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch

    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    wl = W.inflow_3d(n=args.n, flux=args.flux)
    blk = wl.blocks[0]
    ncell = blk.ncell
    sim = Simulation.from_workload(wl, precision=args.precision, device=local_rank)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=local_rank)
    tile = sim.get_tile()
    if not args.no_autotune:
        # project autotuner: fastest fused tile shape; the state is restored
        tile, _ = sim.autotune(3)

    for _ in range(args.warmup):
        sim.run(1)
    sim.synchronize()

    # timed region: K full time steps, all on the device
    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    l0 = sim.kernel_launches()
    ev0.record(ext)
    sim.run(args.steps)
    ev1.record(ext)
    ev1.synchronize()
    launches = sim.kernel_launches() - l0
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_per_step = ms / args.steps
    value = world * ncell * args.steps / (ms * 1e-3)

    # dominant kernel: per-class device time over a few graph-free steps
    prof = sim.profile(args.profile_steps)
    cls = max(prof, key=lambda k: prof[k][0])
    cls_ms, cls_n = prof[cls]
    step_ms = sum(v[0] for v in prof.values()) / args.profile_steps
    hbm, peak_kind = peaks()
    bpc = BYTES_PER_CELL_UPDATE[args.precision]
    if cls == "stage":
        # stage 1 moves 20 doubles/cell, stage 2 25 doubles/cell (FP64 form)
        per_launch_bytes = bpc / 2.0 * ncell
    else:
        # unfused path: the step's algorithmic bytes over the whole step
        per_launch_bytes = bpc * ncell * (cls_ms / args.profile_steps) / step_ms / max(
            1, cls_n // args.profile_steps)
    achieved = per_launch_bytes / (cls_ms / cls_n * 1e-3) / 1e9
    step_achieved = bpc * ncell / (ms_per_step * 1e-3) / 1e9

    # end to end through the C ABI with host buffers: upload the state from
    # pinned memory, one step, download the state to pinned memory
    n = ncell
    host_in = torch.from_numpy(blk.prim).pin_memory()
    host_out = torch.empty((8, n), dtype=torch.float64).pin_memory()
    e2e_steps = max(2, min(args.steps, 5))
    sim.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.upload(0, host_in)
        sim.run(1)
        sim.download(0, prim=host_out, want_cons=False)
    e2e_s = time.perf_counter() - t0
    e2e_value = world * ncell * e2e_steps / e2e_s if world == 1 else None
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_value = world * ncell * e2e_steps / float(t.item())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, secs = cpu_oracle_rate(args.cpu_sample, args.cpu_steps, args.flux)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.cpu_sample}^3 block of the same workload, {args.cpu_steps} steps "
                         f"({secs:.1f} s), CPU FP64 restatement, OpenMP"}

    sim.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-flux/f64-accum",
            "data": "synthetic",
            "config": {"workload": f"inflow_3d {args.n}^3 ideal air, {args.flux}, MUSCL/vanAlbada, "
                                   f"PC, CFL 0.5, {args.precision}",
                       "cells": ncell, "l2": "inputs larger than L2 (each 5-double state array "
                       f"{5 * 8 * ncell / 1e6:.0f} MB > 126 MB)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single"},
            "tile": {"ti": tile[0], "tj": tile[1], "kc": tile[2],
                     "autotuned": not args.no_autotune},
            "roofline": {"bound": "hbm", "kernel": cls, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "traffic": None, "step_achieved": step_achieved,
                         "step_frac": step_achieved / hbm,
                         "bytes_per_cell_update": bpc},
            "profile_ms": {k: round(v[0] / args.profile_steps, 4) for k, v in prof.items()},
            "gpu_launches": launches,
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * 8 * ncell,
                    "d2h_bytes_per_step": 8 * 8 * ncell},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_flux"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--flux", default="hllc", choices=["hllc", "ausmdv"])
    ap.add_argument("--profile-steps", type=int, default=4)
    ap.add_argument("--cpu-sample", type=int, default=64)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--ref-sample", type=int, default=96)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
