"""Throughput of the explicit structured-block update on B200.

Default workload: 256^3 ideal-air Euler block on the unit cube (Mach-3 inflow
at i-min, extrapolate outflow at i-max, slip walls elsewhere, density
perturbed by 8 seeded sines), HLLC flux, MUSCL/van Albada, predictor-corrector,
CFL 0.5.  A bench "step" is one full time step (both predictor-corrector
stages, ghost cells, decode and the dt control every 10 steps) over the block.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32_flux]
                  [--impl ours|reference] [--n 256] [--flux hllc|ausmdv|hanel|adaptive_hanel_ausmdv]
                  [--headline-only]

Prints one JSON line (rank 0).  The headline (value, roofline, e2e, clocks,
gpu_launches) is the --precision form of the 256^3 block.  On one GPU the
same line also carries, each timed the same way on its own simulation:
  "fp32_flux" (or "plain_fp64"): the other precision form of the 256^3 block,
      its speed-up over FP64 and its max relative density difference from the
      FP64 run after the same steps;
  "ausmdv_fp64" (or "hllc_fp64"): the same block with the other of the two
      fluxes in the FP64 form (AUSMDV is the reference's own, its parity pinned);
  "adaptive_hanel_ausmdv_fp64": the same block with the reference's default
      flux (shock detector and per-face Hanel/AUSMDV choice) in the FP64 form;
  "batched": 64 uneven blocks (edges log-uniform in [16, 96]) in one
      persistent launch per stage inside a CUDA graph, autotuned tiles;
  "curvilinear": a 128^3 curvilinear block (the unit box with every vertex
      displaced by smooth sines) on the general path, with per-kernel-class
      times and the CPU oracle on a 96^3 block of the same grid;
  "reacting": the 512x256 5-species reacting ramp channel, 300 steps, with
      reacting cells/s, Newton iterations per reacting cell and the chemistry
      share of the step;
  "learned": the high-enthalpy variant of that channel (Mach 10 at 2000 K,
      20 kPa, where the air dissociates) with the learned chemistry seed:
      training on 1e7 pairs from the plain update, then the same run timed
      plain and seeded, Newton iterations, chemistry speed-up and the
      mass-fraction difference from the plain update.
--impl reference times the CPU FP64 restatement of the reference algorithm
(the D solver itself cannot be built: no D compiler) on the host cores, on the
bench's own 256^3 block (W warm-up steps, then K steps each timed alone; its
ms_per_step is the median measured step); its line also carries "gpu_chem",
the reference's own GPU chemistry (GPUChem and its alpha-QSS kernel, built
for sm_100a) on the high-enthalpy channel's cell states.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s (256^3 Euler)"
UNIT = "cell-updates/s"
# Algorithmic bytes per cell-update (both stages), ideal gas, FP64: stage 1
# reads W0 (5) and U0 (5), writes U1 (5) and W1 (5); stage 2 reads W1, U0 and
# U1, writes U2 and W2: 45 doubles = 360 B.  FP32-flux form (W in FP32): 280 B.
BYTES_PER_CELL_UPDATE = {"fp64": 360.0, "fp32_flux": 280.0}
# chemistry of one reacting cell: read rho, u, T, massf x5, dt_chem; write
# massf x5, T, p, u, a, dt_chem and rho*massf x5 (doubles)
BYTES_PER_REACTING_CELL = 8.0 * (9 + 15)
# DRAM bytes per launch of the fused stage kernel (dram__bytes_read.sum +
# dram__bytes_write.sum, mean of the stage-1 and stage-2 launches) from ncu
# captures, keyed by (precision, kernel class), for the autotuner's picks:
# FP64 (32x16 tile, 32-plane k-chunks) captured on the 128^3 block and scaled
# to 256^3 by the cell count (the kernel's traffic grows with the cells it
# processes); FP32-flux (the 32x8 tile of the edge-warp kernel, 32-plane
# k-chunks) captured on the 256^3 block itself.  Algorithmic bytes per launch
# at 256^3: 3020 MB (FP64), 2349 MB (FP32-flux).
TRAFFIC = {("fp64", "stage"): 2758515712, ("fp32_flux", "stage"): 2418098712}
# FP64 arithmetic per cell-update of the fused stage kernel (both stages),
# keyed by (precision, flux): DADD + DMUL + 2 x DFMA thread instructions per
# cycle times cycles, from the ncu capture of the 128^3 block with the 32x16
# tile (the count per cell does not depend on the block size for a tile
# shape).  Compiled without FMA contraction, the kernel's ceiling is half the
# FP64 peak (64 DFMA per SM per cycle, 2 FLOP each).
FP64_FLOP_PER_CELL_UPDATE = {("fp64", "hllc"): 2430.0}


def oracle_flux(O, flux):
    """The oracle's code of a flux calculator name."""
    return {"ausmdv": O.FLUX_AUSMDV, "hllc": O.FLUX_HLLC, "hanel": O.FLUX_HANEL,
            "adaptive_hanel_ausmdv": O.FLUX_ADAPTIVE_HANEL_AUSMDV}[flux]


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
    cfg = O.default_config(dimensions=3, flux_calculator=oracle_flux(O, flux), n_threads=threads)
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


def cpu_oracle_reacting(wl, steps):
    """Cell-updates/s of the CPU FP64 oracle (OpenMP, all cores) on the full
    reacting channel: `steps` time steps after the first (dt set-up)."""
    from oracle import e4_oracle as O
    O.build()
    cfg = O.default_config(dimensions=2, flux_calculator=O.FLUX_AUSMDV,
                           gas_model=O.GAS_THERM_PERF_5SP_AIR, reacting=1, n_threads=0)
    sim = O.OracleSim(cfg, wl.thermochem)
    b = wl.blocks[0]
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    sim.run(1)
    t0 = time.perf_counter()
    rc = sim.run(steps)
    secs = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return {"value": b.ncell * steps / secs, "unit": UNIT, "cores": os.cpu_count() or 1,
            "kind": "port", "sample": f"the full {b.ni}x{b.nj} channel, steps 2-{steps + 1} "
                                       f"({secs:.1f} s), CPU FP64 restatement, OpenMP"}


def reference_gpu_chem(ni, nj, steps):
    """The reference's own GPU chemistry path (GPUChem, cuda_gpu_chem.d:133-168,
    with its alpha-QSS kernel compiled for sm_100a from the reference's
    template) on the high-enthalpy channel after `steps` flow steps of the CPU
    oracle: the host preparation (concentrations, rate constants, step
    estimate; one cell after another as the D host does), the copies, the
    kernel (CUDA events) and the host's per-cell finish.  The sub-step loop of
    every cell is first bounded on the CPU by the kernel's NumPy restatement
    on the same inputs."""
    import torch

    from eilmer4_b200 import workloads as W
    from oracle import e4_oracle as O
    from oracle import ref_qss as RQ
    if not os.path.exists(RQ.LIB):
        return {"unavailable": "the reference kernel was not built (oracle/_ref)"}
    O.build()
    wl = W.reacting_channel_hot(ni=ni, nj=nj)
    tc = wl.thermochem
    cfg = O.default_config(dimensions=2, flux_calculator=O.FLUX_AUSMDV,
                           gas_model=O.GAS_THERM_PERF_5SP_AIR, reacting=1, n_threads=0)
    sim = O.OracleSim(cfg, tc)
    b = wl.blocks[0]
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    if sim.run(steps) != 0:
        return {"unavailable": "the oracle run that makes the cell states failed"}
    prim, _ = sim.get_flow(0)
    dt = sim.dt_global
    n = b.ncell
    rho, T, u, p, y = prim[0], prim[5], prim[6], prim[4], prim[8:13]
    t0 = time.perf_counter()
    conc, kf, kb, h = O.gpuchem_prepare(tc, rho, T, y, np.full(n, -1.0))
    prep_s = time.perf_counter() - t0
    _, _, passes = RQ.new_qss_numpy(tc, kf, kb, conc, h, dt, max_outer=20000)
    L = RQ.load()
    dev = torch.device("cuda:0")
    host = {"kf": kf, "kb": kb, "Y": conc, "h": h}
    pinned = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).pin_memory()
              for k, v in host.items()}
    names = ["kf", "kb", "MM", "Y", "Yp", "Yc", "h", "alpha", "q", "p", "qp", "pp", "q_bar",
             "p_bar", "alpha_bar", "Ypo"]
    rows = {"kf": tc.nreac, "kb": tc.nreac, "MM": tc.nreac, "h": 1}
    bufs = {k: torch.zeros(rows.get(k, tc.nsp) * n, dtype=torch.float64, device=dev)
            for k in names}
    dbg = torch.zeros(1, dtype=torch.float64, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    Yout = torch.empty(tc.nsp * n, dtype=torch.float64).pin_memory()
    hout = torch.empty(n, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    ev[0].record()
    for k in host:
        bufs[k].copy_(pinned[k], non_blocking=True)
    ev[1].record()
    L.kernel_launcher(*[bufs[k].data_ptr() for k in names], tc.nsp, tc.nreac, n, dt,
                      dbg.data_ptr(), 1, 1, n, 1)
    ev[2].record()
    Yout.copy_(bufs["Y"], non_blocking=True)
    hout.copy_(bufs["h"], non_blocking=True)
    ev[3].record()
    torch.cuda.synchronize()
    h2d_ms, kern_ms, d2h_ms = (ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]),
                               ev[2].elapsed_time(ev[3]))
    t0 = time.perf_counter()
    rc, _ = O.gpuchem_finish(tc, Yout.numpy().reshape(tc.nsp, n), hout.numpy(), rho, T, u, p)
    fin_s = time.perf_counter() - t0
    total_s = prep_s + fin_s + (h2d_ms + kern_ms + d2h_ms) * 1e-3
    return {
        "workload": f"reacting_channel_hot {ni}x{nj} after {steps} flow steps of the CPU oracle, "
                    f"one chemistry step of the flow dt ({dt:.3e} s), every cell",
        "kernel": "new_qss (alpha_qss_kernel_cuda_tmplt.cu), one cell per one-thread block, "
                  "nvcc defaults, sm_100a",
        "cells": n, "finish_rc": rc,
        "substeps_per_cell_mean": float(passes.mean()), "substeps_per_cell_max": int(passes.max()),
        "kernel_ms": kern_ms, "kernel_reacting_cells_per_s": n / (kern_ms * 1e-3),
        "h2d_ms": h2d_ms, "d2h_ms": d2h_ms, "host_prepare_ms": prep_s * 1e3,
        "host_finish_ms": fin_s * 1e3, "reacting_cells_per_s": n / total_s,
        "host_threads": 1,
    }


def run_reference(args, rank, world):
    """--impl reference: the CPU FP64 restatement of the reference's update
    (the D solver cannot be built here) on the bench's own block -- the same
    256^3 workload, flux and initial state -- with OpenMP on every host core.
    W untimed steps, then K steps each timed alone; ms_per_step is the median
    measured step.  Rank 0 alone runs it."""
    if rank != 0:
        return
    from eilmer4_b200 import workloads as W
    from oracle import e4_oracle as O
    O.build()
    n = args.ref_sample or args.n
    b = W.inflow_3d_block(n, n, n, W.DEFAULT_SEED)
    cfg = O.default_config(dimensions=3, flux_calculator=oracle_flux(O, args.flux), n_threads=0)
    sim = O.OracleSim(cfg)
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    del b
    for _ in range(args.warmup):
        if sim.run(1) != 0:
            raise RuntimeError("oracle failed in warm-up")
    secs = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rc = sim.run(1)
        secs.append(time.perf_counter() - t0)
        if rc != 0:
            raise RuntimeError(f"oracle failed: {rc}")
    del sim
    step_s = statistics.median(secs)
    value = n ** 3 / step_s
    cores = os.cpu_count() or 1
    workload = (f"inflow_3d {n}^3 ideal air, {args.flux}, MUSCL/vanAlbada, PC, CFL 0.5, "
                "fp64")
    sample = (f"the whole {n}^3 block, {args.steps} steps after {args.warmup} warm-up steps, "
              f"each timed alone (median {step_s:.2f} s, total {sum(secs):.1f} s)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * step_s, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload, "cells": n ** 3, "sample": sample,
                   "parallelism": "cpu-openmp", "same_config_as_ours": n == args.n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu_chem:
        line["gpu_chem"] = reference_gpu_chem(args.ref_chem_ni, args.ref_chem_nj,
                                              args.ref_chem_steps)
    print(json.dumps(line), flush=True)


def max_over_ranks(x, dist=None, device="cuda"):
    """Max of a host number over all ranks of the process group (x itself
    without one).  Every rank must call it at the same point."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, seconds):
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank in (the max over ranks of) `seconds`."""
    return world * units_per_rank / seconds


def _timed_steps(sim, ext, steps, dist=None, clocks=None):
    """Device time of `steps` time steps on the library stream (CUDA events),
    max over ranks; returns (ms, kernel launches)."""
    import torch
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    l0 = sim.kernel_launches()
    ev0.record(ext)
    sim.run(steps)
    ev1.record(ext)
    ev1.synchronize()
    launches = sim.kernel_launches() - l0
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist)
    if dist:
        dist.barrier()
    return ms, launches


def _roofline_stage(sim, ncell, bpc, profile_steps):
    """Achieved GB/s of the dominant kernel class from a graph-free profile."""
    prof = sim.profile(profile_steps)
    cls = max(prof, key=lambda k: prof[k][0])
    cls_ms, cls_n = prof[cls]
    step_ms = sum(v[0] for v in prof.values()) / profile_steps
    if cls == "stage":
        # one fused launch per stage: stage 1 moves 4/9, stage 2 5/9 of the
        # step's bytes; the average launch moves half
        per_launch_bytes = bpc / 2.0 * ncell
    else:
        per_launch_bytes = bpc * ncell * (cls_ms / profile_steps) / step_ms / max(
            1, cls_n // profile_steps)
    achieved = per_launch_bytes / (cls_ms / cls_n * 1e-3) / 1e9
    return cls, achieved, prof


def euler_case(args, precision, local_rank, dist, world, headline, flux=None):
    """256^3 (or --n) Mach-3 inflow block with the --flux calculator (or
    `flux`); returns a result dict and the downloaded density after warm-up +
    timed steps."""
    import torch

    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation

    flux = flux or args.flux
    wl = W.inflow_3d(n=args.n, flux=flux)
    blk = wl.blocks[0]
    ncell = blk.ncell
    sim = Simulation.from_workload(wl, precision=precision, device=local_rank)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=local_rank)
    tile = sim.get_tile()
    if args.tile:
        tile = tuple(int(x) for x in args.tile.split(","))
        sim.set_tile(*tile)
    elif not args.no_autotune:
        # project autotuner: fastest fused tile shape; the state is restored
        tile, _ = sim.autotune(3)
    for _ in range(args.warmup):
        sim.run(1)
    sim.synchronize()
    clocks = ClockSampler(local_rank) if headline else None
    ms, launches = _timed_steps(sim, ext, args.steps, dist, clocks)
    clk = clocks.stop() if clocks else None
    rho = sim.download(0, want_cons=False)[0][0].copy()
    ms_per_step = ms / args.steps
    value = replica_rate(ncell * args.steps, world, ms * 1e-3)
    bpc = BYTES_PER_CELL_UPDATE[precision]
    cls, achieved, prof = _roofline_stage(sim, ncell, bpc, args.profile_steps)
    hbm, peak_kind = peaks()
    step_achieved = bpc * ncell / (ms_per_step * 1e-3) / 1e9
    res = {
        "value": value, "unit": UNIT, "ms_per_step": ms_per_step, "steps": args.steps,
        "flux": flux, "dtype": "f64" if precision == "fp64" else "f32-flux/f64-accum",
        "tile": {"ti": tile[0], "tj": tile[1], "kc": tile[2],
                 "autotuned": not (args.no_autotune or args.tile)},
        "roofline": {"bound": "hbm", "kernel": cls, "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": TRAFFIC.get((precision, cls)),
                     "step_achieved": step_achieved, "step_frac": step_achieved / hbm,
                     "bytes_per_cell_update": bpc},
        "profile_ms": {k: round(v[0] / args.profile_steps, 4) for k, v in prof.items()},
        "gpu_launches": launches,
    }
    fpc = FP64_FLOP_PER_CELL_UPDATE.get((precision, flux))
    if fpc is not None and cls == "stage":
        # the second bound: FP64 FLOP/s of the same launches (same time base as
        # `roofline.achieved`) against the FP64 peak at the sampled SM clock
        mhz = (clk or {}).get("sm_mhz") or 1965.0
        nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
        peak_tf = nsm * 64 * 2 * mhz * 1e6 / 1e12
        ach_tf = achieved * fpc / bpc / 1e3
        res["fp64_roofline"] = {"bound": "fp64", "kernel": cls, "achieved": ach_tf,
                                "peak": peak_tf, "unit": "TFLOP/s", "frac": ach_tf / peak_tf,
                                "flop_per_cell_update": fpc, "no_fma_ceiling_frac": 0.5,
                                "peak_kind": "64 DFMA per SM per cycle at the sampled SM clock"}
    if clk is not None:
        res["clocks"] = clk
    if headline:
        # end to end through the C ABI with host buffers: every step uploads
        # the block's state from pinned memory, advances it one step and
        # downloads the new state to pinned memory.  The state crossing PCIe
        # is the conserved one (5 doubles per cell each way), decoded on the
        # device as a stage's end decodes it.
        _, cons0 = sim.download(0)
        host_in = torch.from_numpy(cons0).pin_memory()
        host_out = torch.empty((5, ncell), dtype=torch.float64).pin_memory()
        # enough steps that the pipeline's fill (the first upload) and drain
        # (the last download) do not dominate
        e2e_steps = max(2, min(args.steps, 30))
        sim.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            # the copies run on the library's two copy streams: a step's
            # upload overlaps the previous step's computation and download
            sim.upload_cons_async(0, host_in)
            sim.run_async(1)
            sim.download_async(0, cons=host_out)
        sim.wait_transfers()
        sim.run(0)   # raises if a step failed
        e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
        res["e2e"] = {"value": replica_rate(ncell * e2e_steps, world, e2e_s), "unit": UNIT,
                      "h2d_bytes_per_step": 5 * 8 * ncell, "d2h_bytes_per_step": 5 * 8 * ncell,
                      "state": "conserved (rho, rho*v, E) in and out"}
    sim.close()
    return res, rho


def batched_case(args, local_rank):
    """64 uneven blocks (edges log-uniform in [16, 96]) in one persistent launch."""
    import torch

    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation

    wl = W.batched_blocks()
    ncell = wl.ncell
    sim = Simulation.from_workload(wl, device=local_rank)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=local_rank)
    tile, _ = sim.autotune(3)
    for _ in range(args.warmup):
        sim.run(1)
    sim.synchronize()
    ms, launches = _timed_steps(sim, ext, args.batched_steps)
    bpc = BYTES_PER_CELL_UPDATE["fp64"]
    cls, achieved, prof = _roofline_stage(sim, ncell, bpc, args.profile_steps)
    hbm, _ = peaks()
    sim.close()
    return {
        "workload": f"{len(wl.blocks)} uneven 3-D blocks, edges log-uniform in [16,96], "
                    "ausmdv, CFL 0.5, fp64, one persistent launch per stage, CUDA graph",
        "cells": ncell, "steps": args.batched_steps,
        "value": ncell * args.batched_steps / (ms * 1e-3), "unit": UNIT,
        "ms_per_step": ms / args.batched_steps,
        "tile": {"ti": tile[0], "tj": tile[1], "kc": tile[2], "autotuned": True},
        "roofline": {"kernel": cls, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm},
        "gpu_launches": launches,
    }


def cpu_oracle_curvilinear(n, steps, flux):
    """Cell-updates/s of the CPU FP64 oracle (OpenMP, all cores) on an n^3
    curvilinear block (workloads.skewed_box_3d)."""
    from eilmer4_b200 import workloads as W
    from oracle import e4_oracle as O
    O.build()
    wl = W.skewed_box_3d(ni=n, nj=n, nk=n, flux=flux)
    b = wl.blocks[0]
    cfg = O.default_config(dimensions=3, flux_calculator=oracle_flux(O, flux), n_threads=0)
    sim = O.OracleSim(cfg)
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    sim.run(1)
    t0 = time.perf_counter()
    rc = sim.run(steps)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return n ** 3 * steps / dt, os.cpu_count() or 1, dt


def curvilinear_case(args, local_rank):
    """A curvilinear 3-D block (every vertex of the unit box displaced by
    smooth sines): the general path, whose face frames are no axis
    permutations, so the reference's in-place frame round trips are carried
    through every face."""
    import torch

    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation

    n = args.curv_n
    wl = W.skewed_box_3d(ni=n, nj=n, nk=n, flux=args.flux)
    ncell = wl.ncell
    sim = Simulation.from_workload(wl, device=local_rank)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=local_rank)
    for _ in range(args.warmup):
        sim.run(1)
    sim.synchronize()
    ms, launches = _timed_steps(sim, ext, args.curv_steps)
    prof = sim.profile(args.profile_steps)
    sim.close()
    res = {
        "workload": f"skewed_box_3d {n}^3 (curvilinear, amplitude 0.04), {args.flux}, "
                    "MUSCL/vanAlbada in the face frame, PC, CFL 0.5, fp64, general path",
        "cells": ncell, "steps": args.curv_steps,
        "value": ncell * args.curv_steps / (ms * 1e-3), "unit": UNIT,
        "ms_per_step": ms / args.curv_steps,
        "kernel_ms_per_step": {k: v[0] / args.profile_steps for k, v in prof.items() if v[1]},
        "gpu_launches": launches,
        "cpu_baseline": None,
    }
    if not args.no_cpu_baseline:
        rate, cores, secs = cpu_oracle_curvilinear(args.curv_cpu_n, args.curv_cpu_steps, args.flux)
        res["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": f"{args.curv_cpu_n}^3 block of the same grid, "
                                         f"{args.curv_cpu_steps} steps, {secs:.1f} s"}
    return res


def reacting_case(args, local_rank):
    """512x256 5-species reacting ramp channel: gas dynamics + point-implicit
    chemistry every step."""
    import torch

    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation

    wl = W.reacting_channel()
    ncell = wl.ncell
    sim = Simulation.from_workload(wl, reacting=True, device=local_rank)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=local_rank)
    for _ in range(args.warmup):
        sim.run(1)
    sim.synchronize()
    sim.chemistry_counters(reset=True)
    ms, launches = _timed_steps(sim, ext, args.reacting_steps)
    cells, newton, recovered, active = sim.chemistry_counters(reset=True)
    prof = sim.profile(args.profile_steps)
    pcells = sim.chemistry_counters(reset=True)[0]
    chem_ms = prof["chem"][0] + prof["chem_work"][0]
    step_ms = sum(v[0] for v in prof.values())
    prim = sim.download(0, want_cons=False)[0]
    sim.close()
    hbm, _ = peaks()
    chem_rate = pcells / (chem_ms * 1e-3) if chem_ms > 0 else None
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_oracle_reacting(wl, args.cpu_reacting_steps)
    out = {
        "workload": "reacting_channel 512x256, 5-species air, 5 reactions, M10 2 kPa 300 K, "
                    "15-deg ramp, ausmdv, PC, point-implicit chemistry every step",
        "cells": ncell, "steps": args.reacting_steps,
        "ms_per_step": ms / args.reacting_steps,
        "cell_updates_per_s": ncell * args.reacting_steps / (ms * 1e-3),
        "reacting_cells_per_s": cells / (ms * 1e-3),
        "reacting_cells_per_step": cells / args.reacting_steps,
        "newton_per_reacting_cell": newton / max(cells, 1),
        "newton_active_cells_per_step": active / args.reacting_steps,
        "recovered_cells": recovered,
        "chem_share": chem_ms / step_ms if step_ms > 0 else None,
        "chem_kernel": {"reacting_cells_per_s": chem_rate,
                        "achieved_GBps": (BYTES_PER_REACTING_CELL * pcells / (chem_ms * 1e-3)
                                          / 1e9) if chem_ms > 0 else None,
                        "peak_GBps": hbm, "bound": "fp64 latency"},
        "T_max": float(prim[5].max()),
        "gpu_launches": launches,
        "cpu_baseline": cpu,
    }
    return out, prim


def learned_case(args, local_rank):
    """High-enthalpy reacting channel (Mach 10 at 2000 K, 20 kPa): the plain
    point-implicit chemistry against the learned seed.  The network is trained
    here, on the device, on pairs that the plain update produces from the
    states of a plain run (sampled every 10 steps); then the same run is timed
    plain and seeded from the same initial state."""
    import torch

    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation

    nsteps = args.reacting_steps
    wl = W.reacting_channel_hot()
    ncell = wl.ncell
    t0 = time.perf_counter()
    sim = Simulation.from_workload(wl, reacting=True, device=local_rank)
    nsnap = max(1, nsteps // 10)
    per = max(1, args.seed_pairs // nsnap)
    for q in range(nsnap):
        sim.run(10)
        _, dt, _ = sim.state()
        sim.seed_collect([0], dt, per, seed=1000 + q)
    sim.synchronize()
    t_collect = time.perf_counter() - t0
    rep = sim.seed_train(epochs=args.seed_epochs, batch=args.seed_batch, lr=args.seed_lr, seed=1)
    params, norm = sim.seed_get()
    sim.close()

    runs = {}
    for seeded in (False, True):
        sim = Simulation.from_workload(wl, reacting=True, device=local_rank)
        if seeded:
            sim.seed_set(params, norm)
            sim.seed_enable(True)
        ext = torch.cuda.ExternalStream(sim.stream_handle(), device=local_rank)
        for _ in range(args.warmup):
            sim.run(1)
        sim.synchronize()
        sim.chemistry_counters(reset=True)
        ms, launches = _timed_steps(sim, ext, nsteps)
        cells, newton, recovered, active = sim.chemistry_counters(reset=True)
        prof = sim.profile(args.profile_steps)
        pcells = sim.chemistry_counters(reset=True)[0]
        prim = sim.download(0, want_cons=False)[0]
        chem_ms = prof["chem"][0] + prof["seed"][0] + prof["chem_work"][0]
        runs[seeded] = {
            "ms_per_step": ms / nsteps,
            "cell_updates_per_s": ncell * nsteps / (ms * 1e-3),
            "reacting_cells_per_s": cells / (ms * 1e-3),
            "newton_per_reacting_cell": newton / max(cells, 1),
            "newton_active_cells_per_step": active / nsteps,
            "newton_per_active_cell": newton / max(active, 1),
            "recovered_cells": recovered,
            "chem_ms_per_step": chem_ms / args.profile_steps,
            "seed_ms_per_step": prof["seed"][0] / args.profile_steps,
            # pass 1 (every cell: rate constants, the convergence test at the
            # start state; finished cells decoded) and pass 2 (the listed
            # cells' Newton work and decode)
            "pass1_ms_per_step": prof["chem"][0] / args.profile_steps,
            "pass2_ms_per_step": prof["chem_work"][0] / args.profile_steps,
            "chem_kernel_reacting_cells_per_s": pcells / (chem_ms * 1e-3) if chem_ms > 0 else None,
            "gpu_launches": launches,
            "_prim": prim,
        }
        sim.close()
    plain, seeded = runs[False], runs[True]
    # the chemistry update of one state (the plain run's last) with and
    # without the network: the surrogate's error against the plain update
    prim0 = plain["_prim"]
    sim = Simulation.from_workload(wl, reacting=True, device=local_rank)
    sim.seed_set(params, norm)
    out = {}
    for on in (False, True):
        sim.upload(0, prim0)
        sim.seed_enable(on)
        sim.chemistry_counters(reset=True)
        sim.chemistry_step([0], args.learned_check_dt)
        c = sim.chemistry_counters(reset=True)
        out[on] = (sim.download(0, want_cons=False)[0], c)
    sim.close()
    one_step_err = float(np.abs(out[True][0][8:] - out[False][0][8:]).max())
    run_err = float(np.abs(seeded["_prim"][8:] - plain["_prim"][8:]).max())
    for r in runs.values():
        r.pop("_prim")
    return {
        "workload": "reacting_channel_hot 512x256 (Mach 10 at 2000 K, 20 kPa), 5-species air, "
                    f"5 reactions, ausmdv, PC, {nsteps} steps",
        "cells": ncell, "steps": nsteps,
        "training": {"pairs": rep["n_train"] + rep["n_val"], "epochs": args.seed_epochs,
                     "batch": args.seed_batch, "train_loss": rep["train_loss"],
                     "val_loss": rep["val_loss"], "train_s": rep["seconds"],
                     "collect_s": t_collect, "optimizer_steps": rep["steps"]},
        "plain": plain, "seeded": seeded,
        "chem_speedup": plain["chem_ms_per_step"] / seeded["chem_ms_per_step"],
        # on the Newton-active work alone: plain pass 2 against pass 2 plus
        # the seed's inference
        "newton_work_speedup": plain["pass2_ms_per_step"] /
        max(seeded["pass2_ms_per_step"] + seeded["seed_ms_per_step"], 1e-12),
        "step_speedup": plain["ms_per_step"] / seeded["ms_per_step"],
        "massf_err_one_update": one_step_err,
        "newton_one_update": {"plain": out[False][1][1], "seeded": out[True][1][1],
                              "reacting_cells": out[False][1][0],
                              "active_cells": out[False][1][3]},
        "massf_diff_after_run": run_err,
    }


def run_ours(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.part != "all":
        # one part alone (profiling runs): its own JSON line
        fn = {"reacting": lambda: reacting_case(args, local_rank)[0],
              "learned": lambda: learned_case(args, local_rank),
              "batched": lambda: batched_case(args, local_rank),
              "curvilinear": lambda: curvilinear_case(args, local_rank)}[args.part]
        if rank == 0:
            print(json.dumps({"part": args.part, **fn()}), flush=True)
        return
    head, rho_head = euler_case(args, args.precision, local_rank, dist, world, headline=True)
    extra = {}
    if not args.headline_only and world == 1 and args.flux not in ("hllc", "ausmdv"):
        raise SystemExit("the full line (FP32-flux form included) runs with --flux hllc or "
                         "ausmdv; add --headline-only for the other fluxes")
    if not args.headline_only and world == 1:
        other = "fp32_flux" if args.precision == "fp64" else "fp64"
        res, rho_other = euler_case(args, other, local_rank, dist, world, headline=False)
        rho64, rho32 = (rho_head, rho_other) if args.precision == "fp64" else (rho_other, rho_head)
        res["rel_density_err_vs_fp64"] = float(np.max(np.abs(rho32 - rho64) / np.abs(rho64)))
        res["speedup_vs_fp64"] = (res["value"] / head["value"] if other == "fp32_flux"
                                  else head["value"] / res["value"])
        extra["fp32_flux" if other == "fp32_flux" else "plain_fp64"] = res
        # the reference's own flux calculator (AUSMDV, fluxcalc.d:376-529) on
        # the same block in the plain FP64 form
        other_flux = "ausmdv" if args.flux == "hllc" else "hllc"
        res, _ = euler_case(args, "fp64", local_rank, dist, world, headline=False,
                            flux=other_flux)
        extra[f"{other_flux}_fp64"] = res
        # the reference's default flux (adaptive Hanel/AUSMDV with the shock
        # detector, fluxcalc.d:824-838) on the fused path
        res, _ = euler_case(args, "fp64", local_rank, dist, world, headline=False,
                            flux="adaptive_hanel_ausmdv")
        extra["adaptive_hanel_ausmdv_fp64"] = res
        extra["batched"] = batched_case(args, local_rank)
        extra["curvilinear"] = curvilinear_case(args, local_rank)
        extra["reacting"], _ = reacting_case(args, local_rank)
        if not args.no_learned:
            extra["learned"] = learned_case(args, local_rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, secs = cpu_oracle_rate(args.cpu_sample, args.cpu_steps, args.flux)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.cpu_sample}^3 block of the same workload, {args.cpu_steps} steps "
                         f"({secs:.1f} s), CPU FP64 restatement, OpenMP"}
        # and one thread (the restatement's scalar rate)
        n1 = args.cpu_single_sample
        rate1, _, secs1 = cpu_oracle_rate(n1, args.cpu_single_steps, args.flux, threads=1)
        cpu["single_thread"] = {"value": rate1, "unit": UNIT, "cores": 1,
                                "sample": f"{n1}^3 block, {args.cpu_single_steps} steps "
                                          f"({secs1:.1f} s), one thread"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": head["dtype"], "data": "synthetic",
            "config": {"workload": f"inflow_3d {args.n}^3 ideal air, {args.flux}, MUSCL/vanAlbada, "
                                   f"PC, CFL 0.5, {args.precision}",
                       "cells": args.n ** 3, "l2": "inputs larger than L2 (each 5-double state "
                       f"array {5 * 8 * args.n ** 3 / 1e6:.0f} MB > 126 MB)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single"},
            "tile": head["tile"],
            "roofline": head["roofline"],
            "fp64_roofline": head.get("fp64_roofline"),
            "profile_ms": head["profile_ms"],
            "gpu_launches": head["gpu_launches"],
            "clocks": head.get("clocks"),
            "e2e": head["e2e"],
            "cpu_baseline": cpu,
        }
        line.update(extra)
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
    ap.add_argument("--flux", default="hllc", choices=["hllc", "ausmdv", "hanel", "adaptive_hanel_ausmdv"])
    ap.add_argument("--profile-steps", type=int, default=4)
    # CPU baseline samples: about 10 s of oracle work each on a 16-core host
    ap.add_argument("--cpu-sample", type=int, default=128)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--cpu-single-sample", type=int, default=64)
    ap.add_argument("--cpu-single-steps", type=int, default=10)
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="--impl reference: edge of the timed block (default: --n, the "
                         "bench's own block)")
    ap.add_argument("--cpu-reacting-steps", type=int, default=25)
    ap.add_argument("--no-ref-gpu-chem", action="store_true",
                    help="--impl reference: skip the reference's GPU chemistry kernel")
    ap.add_argument("--ref-chem-ni", type=int, default=256)
    ap.add_argument("--ref-chem-nj", type=int, default=128)
    ap.add_argument("--ref-chem-steps", type=int, default=60)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--tile", default="",
                    help="TI,TJ,KC: fixed fused tile shape for the 256^3 block (no autotuning)")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the --precision 256^3 line, no FP32/batched/reacting parts")
    ap.add_argument("--batched-steps", type=int, default=20)
    ap.add_argument("--curv-n", type=int, default=128,
                    help="edge of the curvilinear general-path block")
    ap.add_argument("--curv-steps", type=int, default=40)
    ap.add_argument("--curv-cpu-n", type=int, default=96)
    ap.add_argument("--curv-cpu-steps", type=int, default=5)
    ap.add_argument("--reacting-steps", type=int, default=300)
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--part", default="all",
                    choices=["all", "reacting", "learned", "batched", "curvilinear"],
                    help="run one sub-part alone (for profiling)")
    ap.add_argument("--seed-pairs", type=int, default=10_000_000)
    ap.add_argument("--seed-epochs", type=int, default=8)
    ap.add_argument("--seed-batch", type=int, default=4096)
    ap.add_argument("--seed-lr", type=float, default=2.0e-3)
    ap.add_argument("--learned-check-dt", type=float, default=1.0e-7)
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
