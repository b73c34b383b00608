"""GPU parity on a curvilinear 3-D block (workloads.skewed_box_3d): every
vertex of the unit box displaced by smooth sines, so no face frame is an axis
permutation and every cell has its own volume and lengths.  This exercises the
hexahedral cell geometry (properties.d:568-648), the replay of the
reference's in-place frame round trips across all three face directions, the
slip-wall reflection in general frames and, with the thermally perfect
mixture, the 3-D reacting path -- bit for bit against the CPU oracle.  The
row-walking flux kernel of 3-D ideal-gas blocks is checked with forced run
lengths, on the curvilinear grid and on a stretched Cartesian one."""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W

pytestmark = pytest.mark.gpu


def assert_same(a, b, what):
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        q = tuple(bad[0])
        raise AssertionError(f"{what}: {len(bad)} values differ; first at {q}: "
                             f"gpu={a[q]!r} oracle={b[q]!r}")


@pytest.mark.parametrize("flux", ["ausmdv", "hllc", "adaptive_hanel_ausmdv"])
def test_skewed_box_ideal_gas_bitexact(oracle, e4lib, flux):
    from eilmer4_b200.simcore import Simulation
    wl = W.skewed_box_3d(flux=flux)
    fl = {"ausmdv": oracle.FLUX_AUSMDV, "hllc": oracle.FLUX_HLLC,
          "adaptive_hanel_ausmdv": oracle.FLUX_ADAPTIVE_HANEL_AUSMDV}[flux]
    cfg = oracle.default_config(dimensions=3, n_threads=0, flux_calculator=fl)
    osim = oracle.OracleSim(cfg)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(25) == 0
    op, oc = osim.get_flow(0)
    with Simulation.from_workload(wl) as sim:
        sim.run(25)
        gp, gc = sim.download(0)
        t, dt, st = sim.state()
    assert (t, dt, st) == (osim.time, osim.dt_global, osim.step)
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")


def test_skewed_box_reacting_bitexact(oracle, e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = W.skewed_box_3d(ni=10, nj=8, nk=6, reacting=True)
    cfg = oracle.default_config(dimensions=3, n_threads=0, flux_calculator=oracle.FLUX_AUSMDV,
                                gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=1)
    osim = oracle.OracleSim(cfg, wl.thermochem)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(20) == 0
    op, oc = osim.get_flow(0)
    assert op[12].max() > 1e-5   # atomic oxygen formed: the chemistry did work
    with Simulation.from_workload(wl, reacting=True) as sim:
        sim.run(20)
        gp, gc = sim.download(0)
        t, dt, st = sim.state()
    assert (t, dt, st) == (osim.time, osim.dt_global, osim.step)
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")


@pytest.fixture(scope="module")
def skewed_mid_oracle(oracle):
    """A 40x36x34 curvilinear block after 8 steps of the oracle, per flux."""
    out = {}
    for flux, fl in (("hllc", oracle.FLUX_HLLC),
                     ("adaptive_hanel_ausmdv", oracle.FLUX_ADAPTIVE_HANEL_AUSMDV)):
        wl = W.skewed_box_3d(ni=40, nj=36, nk=34, flux=flux)
        cfg = oracle.default_config(dimensions=3, n_threads=0, flux_calculator=fl)
        osim = oracle.OracleSim(cfg)
        b = wl.blocks[0]
        osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
        osim.set_flow(0, b.prim)
        assert osim.run(8) == 0
        out[flux] = (wl, osim.get_flow(0), (osim.time, osim.dt_global, osim.step))
    return out


@pytest.mark.parametrize("flux,runs", [("hllc", (8, 32)), ("hllc", (3, 5)), ("hllc", (1, 1)),
                                       ("hllc", (64, 64)),
                                       ("adaptive_hanel_ausmdv", (8, 32))])
def test_row_walk_any_run_length_bitexact(skewed_mid_oracle, e4lib, flux, runs):
    """The row-walking flux kernel carries the reference's in-place frame
    round trips along runs of faces (sfluidblock.d:2190-2344 loop order,
    onedinterp.d:445-454, 576-584).  Long runs, uneven runs (3 i-faces, 5 j/k
    faces per thread on rows of 41, 37 and 35 faces), one face per run, and
    runs longer than a row all give the oracle's bits."""
    from eilmer4_b200.simcore import Simulation
    wl, (op, oc), state = skewed_mid_oracle[flux]
    with Simulation.from_workload(wl) as sim:
        sim.set_flux_runs(*runs)
        sim.run(8)
        gp, gc = sim.download(0)
        assert tuple(sim.state()) == state
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")


def stretched_box(ni, nj, nk, flux):
    """A Cartesian block with cell sizes varying along each axis (vertex
    coordinate x -> x + 0.02 sin(2 pi x), likewise y and z): every face frame
    is an axis permutation, but the geometry is not uniform, so the block takes
    the general path."""
    import math
    b = W.inflow_3d_block(ni, nj, nk, 20261203)
    for c in range(3):
        b.vtx[:, c] = b.vtx[:, c] + 0.02 * np.sin(2.0 * math.pi * b.vtx[:, c])
    wl = W.Workload("stretched", 3, flux_calculator=flux)
    wl.blocks.append(b)
    return wl


@pytest.mark.parametrize("flux,runs", [("hllc", (0, 0)), ("hllc", (3, 5)),
                                       ("adaptive_hanel_ausmdv", (0, 0))])
def test_stretched_cartesian_row_walk_bitexact(oracle, e4lib, flux, runs):
    """Axis-permutation frames on a non-uniform grid: the row walk leaves the
    cells' velocities as they are (the reference copies rather than rotating
    in place for such frames) and gives the oracle's bits."""
    from eilmer4_b200.simcore import Simulation
    wl = stretched_box(40, 36, 34, flux)
    fl = {"hllc": oracle.FLUX_HLLC,
          "adaptive_hanel_ausmdv": oracle.FLUX_ADAPTIVE_HANEL_AUSMDV}[flux]
    cfg = oracle.default_config(dimensions=3, n_threads=0, flux_calculator=fl)
    osim = oracle.OracleSim(cfg)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(8) == 0
    op, oc = osim.get_flow(0)
    with Simulation.from_workload(wl) as sim:
        sim.set_flux_runs(*runs)
        sim.run(8)
        gp, gc = sim.download(0)
        assert tuple(sim.state()) == (osim.time, osim.dt_global, osim.step)
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")
