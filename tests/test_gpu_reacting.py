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
