"""GPU parity on the benchmark configurations at their stated sizes.

C0  the 2-D Sod tube: 256x64 cells on the unit square, AUSMDV, 1000 steps
    (the whole configuration);
C1  the 256^3 Mach-3 inflow block on the unit cube, HLLC and AUSMDV, a few
    steps each, on the fused path with the tile shape the autotuner picks;
C2  the 64 uneven blocks of the batched configuration (edges log-uniform in
    [16, 96], 6.0 M cells), AUSMDV, one persistent launch per stage with the
    autotuned tile;
C3  the 512x256 reacting ramp channel (5-species air, point-implicit
    chemistry every step), and its high-enthalpy variant in which the air
    dissociates and the chemistry does Newton work.

Every primitive and conserved value, the step count, the simulation time and
dt_global are compared with == against the CPU oracle: the size-dependent
parts of the GPU path (work-item order over 148 persistent CTAs, k-chunk
remainders, 64-bit cell indices, the chemistry work list) are exercised at the
sizes the benchmark runs.  The oracle runs with OpenMP on every host core; the
256^3 block holds about 23 GB of host memory in the oracle's object layout.
"""
import warnings

import numpy as np
import pytest

from eilmer4_b200 import workloads as W
from parity import FLUX, assert_same, compare

pytestmark = pytest.mark.gpu

# host bytes per padded cell of the oracle's 3-D block (cell, three faces and
# a vertex in its object layout), with room for the comparison arrays
ORACLE_BYTES_PER_CELL = 1450


def largest_cube_that_fits(n):
    """Edge of the largest cube, at most n, whose oracle block fits in the
    host memory available now (the full size on a B200 host)."""
    import psutil
    avail = psutil.virtual_memory().available
    m = n
    while m > 64 and ORACLE_BYTES_PER_CELL * (m + 4) ** 3 > 0.8 * avail:
        m -= 32
    if m != n:
        warnings.warn(f"host memory ({avail / 2**30:.0f} GiB available) holds the oracle's "
                      f"{m}^3 block, not {n}^3")
    return m


def test_c0_sod_256x64_1000_steps(oracle, e4lib):
    wl = W.sod_2d(256, 64)
    info = compare(oracle, wl, 1000)
    assert info.steps_taken == 1000


def run_fused_pair(oracle, wl, nsteps):
    """The oracle and the GPU (autotuned tile, graphs) over nsteps."""
    from eilmer4_b200.simcore import Simulation
    cfg = oracle.default_config(dimensions=3, flux_calculator=FLUX[wl.flux_calculator],
                                n_threads=0)
    osim = oracle.OracleSim(cfg)
    for b in wl.blocks:
        h = osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
        osim.set_flow(h, b.prim)
    assert osim.run(nsteps) == 0
    with Simulation.from_workload(wl) as sim:
        tile, _ = sim.autotune(2)
        info = sim.run(nsteps)
        assert info.steps_taken == nsteps
        t, dt, st = sim.state()
        assert st == osim.step and t == osim.time and dt == osim.dt_global, \
            (st, osim.step, t, osim.time, dt, osim.dt_global)
        for h in range(len(wl.blocks)):
            gp, gc = sim.download(h)
            op, oc = osim.get_flow(h)
            assert_same(gc, oc, f"block {h} conserved (tile {tile})")
            assert_same(gp[:8], op[:8], f"block {h} primitive (tile {tile})")
            del gp, gc, op, oc
        prof = sim.profile(1)
    # the whole run took the fused path
    assert prof["flux"][1] == 0 and prof["stage"][1] == 2, prof
    return tile


@pytest.mark.parametrize("flux", ["hllc", "ausmdv"])
def test_c1_inflow_256cubed(oracle, e4lib, flux):
    n = largest_cube_that_fits(256)
    wl = W.inflow_3d(n=n, flux=flux)
    run_fused_pair(oracle, wl, 3)


def test_c2_batched_64_blocks(oracle, e4lib):
    wl = W.batched_blocks()
    assert len(wl.blocks) == 64 and wl.flux_calculator == "ausmdv"
    run_fused_pair(oracle, wl, 8)


@pytest.mark.parametrize("hot", [False, True])
def test_c3_reacting_channel_512x256(oracle, e4lib, hot):
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel_hot() if hot else W.reacting_channel()
    nsteps = 30
    cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV,
                                gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=1,
                                n_threads=0)
    osim = oracle.OracleSim(cfg, wl.thermochem)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(nsteps) == 0
    op, oc = osim.get_flow(0)
    with Simulation.from_workload(wl, reacting=True) as sim:
        sim.chemistry_counters(reset=True)
        sim.run(nsteps)
        gp, gc = sim.download(0)
        t, dt, st = sim.state()
        counters = sim.chemistry_counters()
    assert st == osim.step and t == osim.time and dt == osim.dt_global
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")
    if hot:
        # the chemistry did Newton work on dissociating cells
        assert counters[1] > 0 and counters[3] > 0, counters
        assert np.max(gp[12]) > 1.0e-4  # atomic oxygen behind the ramp shock


@pytest.mark.parametrize("hot", [False, True])
def test_c3_channel_against_the_libm_oracle(oracle, e4lib, hot):
    """How far the GPU's reacting path sits from the reference's arithmetic:
    the GPU (portable exp/log/pow, bit for bit the oracle's) against the
    oracle built on the C library's exp, log and pow, on the full 512x256
    channel after 30 steps.  The largest difference of each field, relative
    to the field's scale (the speed for a velocity component), is printed and
    bounded by 1e-8."""
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel_hot() if hot else W.reacting_channel()
    nsteps = 30
    cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV,
                                gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=1,
                                n_threads=0)
    osim = oracle.OracleSim(cfg, wl.thermochem, libm=True)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(nsteps) == 0
    op, _ = osim.get_flow(0)
    with Simulation.from_workload(wl, reacting=True) as sim:
        sim.run(nsteps)
        gp, _ = sim.download(0)
        assert sim.state()[2] == osim.step
    names = ["rho", "vx", "vy", "vz", "p", "T", "u", "a", "N2", "O2", "NO", "N", "O"]
    speed = np.abs(op[1:3]).max()
    diffs = {}
    for q, name in enumerate(names):
        scale = speed if q in (1, 2, 3) else np.abs(op[q]).max()
        if scale > 0.0:
            diffs[name] = float(np.abs(gp[q] - op[q]).max() / scale)
    print(f"\nGPU vs libm oracle, {'hot' if hot else 'cold'} channel 512x256, {nsteps} steps:",
          {k: f"{v:.2e}" for k, v in diffs.items()})
    assert max(diffs.values()) <= 1e-8, diffs
