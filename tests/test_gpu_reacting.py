"""GPU parity on the reacting path: thermally perfect 5-species air on a
curvilinear 2-D grid (compression ramp) and the point-implicit chemistry,
checked bit for bit against the CPU oracle."""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W

pytestmark = pytest.mark.gpu


def assert_same(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        q = tuple(bad[0])
        rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
        raise AssertionError(f"{what}: {len(bad)} values differ; first at {q}: "
                             f"gpu={a[q]!r} oracle={b[q]!r}; max rel {rel:.3e}")


def run_pair(oracle, wl, nsteps, reacting):
    from eilmer4_b200.simcore import Simulation
    cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV,
                                gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=int(reacting),
                                n_threads=0)
    osim = oracle.OracleSim(cfg, wl.thermochem)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(nsteps) == 0
    op, oc = osim.get_flow(0)
    with Simulation.from_workload(wl, reacting=reacting) as sim:
        info = sim.run(nsteps)
        gp, gc = sim.download(0)
        t, dt, st = sim.state()
    assert st == osim.step and t == osim.time and dt == osim.dt_global
    return (gp, gc), (op, oc)


def test_therm_perf_ramp_channel_bitexact(oracle, e4lib):
    wl = W.reacting_channel(ni=48, nj=24)
    (gp, gc), (op, oc) = run_pair(oracle, wl, 30, reacting=False)
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")


def test_reacting_ramp_channel_bitexact(oracle, e4lib):
    wl = W.reacting_channel(ni=48, nj=24)
    (gp, gc), (op, oc) = run_pair(oracle, wl, 30, reacting=True)
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")


def test_chemistry_step_on_hot_air_bitexact(oracle, e4lib):
    """e4c_chemistry_step on hot air (2500-8000 K): every cell's mass
    fractions, T, u and p equal the oracle's thermochemical_increment."""
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel(ni=16, nj=8)
    tc = wl.thermochem
    b = wl.blocks[0]
    n = b.ncell
    rng = np.random.default_rng(5)
    mf0 = [0.767, 0.233, 0.0, 0.0, 0.0]
    for q in range(n):
        T = 2500.0 + 5500.0 * rng.random()
        p = 1.0e4 + 2.0e5 * rng.random()
        y = np.array(mf0) + np.array([0.0, -0.05, 0.02, 0.01, 0.02]) * rng.random()
        y = y / y.sum()
        rho, u, a = tc.state_pT(p, T, y)
        b.prim[:, q] = [rho, 0.0, 0.0, 0.0, p, T, u, a] + list(y)
    dt = 2.0e-7
    with Simulation.from_workload(wl, reacting=True) as sim:
        sim.chemistry_step([0], dt)
        gp, gc = sim.download(0)
    for q in range(n):
        rc, out = oracle.chem_cell(tc, 300.0, dt, b.prim[0, q], b.prim[5, q], b.prim[6, q],
                                   b.prim[4, q], b.prim[8:, q].copy(), 0.0)
        assert rc == 0
        assert_same(gp[8:, q], out["massf"], f"cell {q} mass fractions")
        assert gp[5, q] == out["T"] and gp[6, q] == out["u"] and gp[4, q] == out["p"], q
        assert_same(gc[5:, q], b.prim[0, q] * out["massf"], f"cell {q} species densities")
    # something happened: oxygen dissociated in the hottest cells
    assert gp[12].max() > 1.0e-4


def test_flow_file_round_trip_through_the_gpu(oracle, e4lib, tmp_path):
    """A flow file written from the GPU state (sfluidblock.d write_solution
    layout) and read into a fresh simulation gives back the same primitive
    state, mass fractions and per-cell chemistry step, bit for bit."""
    from eilmer4_b200 import _lib
    from eilmer4_b200 import flowfile as F
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel_hot(ni=32, nj=16)
    for fmt in ("gziptext", "rawbinary"):
        path = str(tmp_path / ("b.flow." + fmt))
        with Simulation.from_workload(wl, reacting=True) as sim:
            sim.run(15)
            sim.write_flow(0, path, fmt=fmt, label="ramp")
            p0, c0 = sim.download(0)
            d0 = np.zeros(wl.ncell)
            sim.L.e4c_block_get_dt_chem(0, _lib.dptr(d0))
            t0 = sim.state()[0]
        fl = F.read_flow(path, fmt)
        assert fl["sim_time"] == t0
        with Simulation.from_workload(wl, reacting=True) as sim2:
            assert sim2.read_flow(0, path, fmt=fmt) == t0
            p1, c1 = sim2.download(0)
            d1 = np.zeros(wl.ncell)
            sim2.L.e4c_block_get_dt_chem(0, _lib.dptr(d1))
        assert_same(p1, p0, "primitive")
        assert_same(d1, d0, "dt_chem")
        # the conserved state is re-encoded from the primitive one, as the
        # reference does on restart; the mixture's temperature iteration
        # leaves u at the energy of its last iterate (newton.d:40-99), so the
        # total energy comes back within that iteration's tolerance
        rel = np.abs(c1 - c0) / np.maximum(np.abs(c0), 1e-300)
        assert rel[:4].max() <= 1e-15 and rel[5:].max() <= 1e-15, rel.max()
        assert rel[4].max() <= 1e-9, rel[4].max()


def test_rkf_chemistry_step_on_hot_air_bitexact(oracle, e4lib):
    """The reference's own chemistry method (odeStep.method 'rkf':
    ChemistryUpdate.opCall's sub-cycling with RKFStep, chemistry_update.d:
    119-307, 362-461) on the device: every cell's mass fractions, T, u, p
    and dt_chem equal the oracle's, whose update of the hydrogen-iodide test
    problem gives the reference's golden value (test_oracle_kinetics_golden)."""
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel(ni=16, nj=8)
    tc = wl.thermochem
    b = wl.blocks[0]
    n = b.ncell
    rng = np.random.default_rng(8)
    mf0 = [0.767, 0.233, 0.0, 0.0, 0.0]
    for q in range(n):
        T = 2500.0 + 2500.0 * rng.random()
        p = 1.0e4 + 1.0e5 * rng.random()
        y = np.array(mf0) + np.array([0.0, -0.05, 0.02, 0.01, 0.02]) * rng.random()
        y = y / y.sum()
        rho, u, a = tc.state_pT(p, T, y)
        b.prim[:, q] = [rho, 0.0, 0.0, 0.0, p, T, u, a] + list(y)
    dt = 1.0e-7
    with Simulation.from_workload(wl, reacting=True, chem_method="rkf") as sim:
        sim.chemistry_step([0], dt)
        gp, gc = sim.download(0)
        dchem = np.zeros(n)
        from eilmer4_b200 import _lib
        sim.L.e4c_block_get_dt_chem(0, _lib.dptr(dchem))
    oracle.set_chem_method(1)
    try:
        for q in range(n):
            rc, out = oracle.chem_cell(tc, 300.0, dt, b.prim[0, q], b.prim[5, q], b.prim[6, q],
                                       b.prim[4, q], b.prim[8:, q].copy(), -1.0)
            assert rc == 0
            assert_same(gp[8:, q], out["massf"], f"cell {q} mass fractions")
            assert gp[5, q] == out["T"] and gp[6, q] == out["u"] and gp[4, q] == out["p"], q
            assert dchem[q] == out["dt_chem"], q
    finally:
        oracle.set_chem_method(0)
    assert gp[12].max() > 1.0e-5   # oxygen dissociated


def test_rkf_hot_ramp_channel_bitexact(oracle, e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel_hot(ni=48, nj=24)
    nsteps = 12
    cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV,
                                gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=1,
                                n_threads=0, chem_method=1)
    osim = oracle.OracleSim(cfg, wl.thermochem)
    b = wl.blocks[0]
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(nsteps) == 0
    op, oc = osim.get_flow(0)
    with Simulation.from_workload(wl, reacting=True, chem_method="rkf") as sim:
        sim.run(nsteps)
        gp, gc = sim.download(0)
        assert sim.state()[2] == osim.step and sim.state()[0] == osim.time
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")
