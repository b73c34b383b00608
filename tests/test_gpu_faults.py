"""Faults made on the host side (nothing here faults, traps or hangs the GPU):
impossible time steps are refused at the C ABI with the state untouched, a
NaN in an uploaded state stops the run with the oracle's error class at the
oracle's step, and chemistry updates that defeat the whole-interval Newton
iteration take the reference's sub-cycling recovery, bit for bit as the
oracle does."""
import math

import numpy as np
import pytest

from eilmer4_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_impossible_dt_is_refused(e4lib):
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    with Simulation.from_workload(W.sod_2d(16, 8)) as sim:
        p0, c0 = sim.download(0)
        for dt in (0.0, -1.0e-6, math.nan, math.inf):
            with pytest.raises(_lib.E4CError) as ei:
                sim.gasdynamic_step([0], dt)
            assert ei.value.code == _lib.E4C_ERR_ARG, dt
        p1, c1 = sim.download(0)
        assert np.array_equal(c1, c0) and np.array_equal(p1, p0)
        # and the simulation still steps
        dt_allow, _ = sim.dt_allow([0], 1.0e-3, False)
        assert sim.gasdynamic_step([0], min(dt_allow, 1.0e-3)) == 0
    with Simulation.from_workload(W.reacting_channel(ni=16, nj=8), reacting=True) as sim:
        for dt in (0.0, math.nan):
            with pytest.raises(_lib.E4CError) as ei:
                sim.chemistry_step([0], dt)
            assert ei.value.code == _lib.E4C_ERR_ARG


def test_nan_in_the_uploaded_state_stops_like_the_oracle(oracle, e4lib):
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    wl = W.sod_2d(24, 8)
    b = wl.blocks[0]
    b.prim[0, 37] = math.nan
    cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV, n_threads=0)
    osim = oracle.OracleSim(cfg)
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    orc = osim.run(5)
    assert orc != 0
    with Simulation.from_workload(wl) as sim:
        with pytest.raises(_lib.E4CError) as ei:
            sim.run(5)
    # the oracle numbers its error classes on its own (e4_oracle_internal.h)
    oracle_class = {-2: _lib.E4C_ERR_BAD_MASS, -3: _lib.E4C_ERR_THERMO,
                    -4: _lib.E4C_ERR_BAD_CELLS, -5: _lib.E4C_ERR_CHEM}[orc]
    assert ei.value.code == oracle_class, (ei.value.code, orc)
    assert f"at step {osim.step}" in str(ei.value), (str(ei.value), osim.step)


def test_chemistry_recovery_path_bitexact(oracle, e4lib):
    """With no Newton iterations allowed for the whole-interval step
    (chem_newton_iterations = 0), every cell that needs Newton work is finished
    by opCall's sub-cycling (chemistry_update.d:119-307) with error-controlled
    point-implicit sub-steps; every cell's result equals the oracle's under the
    same setting, bit for bit."""
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel(ni=16, nj=8)
    tc = wl.thermochem
    b = wl.blocks[0]
    rng = np.random.default_rng(11)
    mf0 = np.array([0.767, 0.233, 0.0, 0.0, 0.0])
    for q in range(b.ncell):
        T = 3000.0 + 5000.0 * rng.random()
        p = 1.0e4 + 2.0e5 * rng.random()
        rho, u, a = tc.state_pT(p, T, mf0)
        b.prim[:, q] = [rho, 0.0, 0.0, 0.0, p, T, u, a] + list(mf0)
    dt = 2.0e-7
    with Simulation.from_workload(wl, reacting=True, chem_newton_iterations=0) as sim:
        sim.chemistry_counters(reset=True)
        sim.chemistry_step([0], dt)
        cells, newton, recovered, active = sim.chemistry_counters(reset=True)
        gp, _ = sim.download(0)
        dtc = np.zeros(b.ncell)
        from eilmer4_b200 import _lib
        sim.L.e4c_block_get_dt_chem(0, _lib.dptr(dtc))
    assert recovered > 50, (cells, newton, recovered, active)
    oracle.set_chem_newton_iterations(0)
    try:
        for q in range(b.ncell):
            rc, out = oracle.chem_cell(tc, 300.0, dt, b.prim[0, q], b.prim[5, q], b.prim[6, q],
                                       b.prim[4, q], b.prim[8:, q].copy(), -1.0)
            assert rc == 0
            assert np.array_equal(gp[8:, q], out["massf"]), q
            assert gp[5, q] == out["T"] and gp[6, q] == out["u"] and gp[4, q] == out["p"], q
            assert dtc[q] == out["dt_chem"], q
    finally:
        oracle.set_chem_newton_iterations(12)


def test_bad_flux_run_lengths_are_refused(e4lib):
    """e4c_set_flux_runs takes both lengths 0 (the per-block choice) or both
    in 1..4096; anything else is refused with E4C_ERR_ARG and changes
    nothing."""
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    with Simulation.from_workload(W.skewed_box_3d(ni=12, nj=10, nk=8)) as sim:
        for bad in ((0, 4), (4, 0), (-1, 8), (8, -1), (5000, 8), (8, 5000)):
            with pytest.raises(_lib.E4CError) as ei:
                sim.set_flux_runs(*bad)
            assert ei.value.code == _lib.E4C_ERR_ARG, bad
        sim.set_flux_runs(2, 3)
        sim.set_flux_runs(0, 0)
        assert sim.run(2).status == 0


def test_seed_inference_wait_runs_out_and_recovers(e4lib):
    """The seed inference kernel's bounded wait for the tensor cores, made to
    run out on a healthy device (first wait limited to 0 tries): the call
    reports E4C_ERR_TIMEOUT, the kernel's second, full wait lets the multiply
    it issued finish before it releases its tensor memory, and the next calls
    succeed and give the prediction of a call that never timed out."""
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    from oracle import e4_seed_oracle as SO
    rng = np.random.default_rng(9)
    params = SO.init_params(3)
    norm = np.zeros(SO.NNORM)
    norm[8:16] = 1.0
    norm[22:28] = 1.0
    norm[28] = 1.0e-9
    norm[29] = 1.0e-3
    n = 1000
    y = np.array([0.74, 0.2, 0.02, 0.01, 0.03]) + 0.01 * rng.random((n, 5))
    rows = np.column_stack([2500.0 + 5000.0 * rng.random(n), 1e4 + 1e5 * rng.random(n), y,
                            1e-7 * (1.0 + rng.random(n))])
    with Simulation.from_workload(W.sod_2d(16, 4)) as sim:
        sim.seed_set(params, norm)
        before = sim.seed_predict(rows)
        _lib.check(sim.L.e4c_seed_set_wait_limit(0))
        with pytest.raises(_lib.E4CError) as ei:
            sim.seed_predict(rows)
        assert ei.value.code == _lib.E4C_ERR_TIMEOUT
        _lib.check(sim.L.e4c_seed_set_wait_limit(-1))
        for _ in range(2):
            after = sim.seed_predict(rows)
            assert np.array_equal(after, before)
        # the simulation itself is untouched: it still steps
        info = sim.run(3)
        assert info.steps_taken == 3
