"""The CPU oracle against the reference's own golden values.

Pins the restatement (oracle/) before it is trusted as the checker:
  * src/gas/ideal_gas.d:220-239 (ideal air at p=1e5 Pa, T=300 K);
  * examples/eilmer/3D/sod-shock-tube/sg/sod-test.rb (75 +- 3 steps to
    t=0.6 ms; post-shock and expanded-driver probes within 1 %).
"""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W


def rel(a, b):
    return abs(a - b) / abs(b)


def test_ideal_air_golden(oracle):
    # ideal_gas.d:220-239, tolerance 1e-4 relative as in approxEqualNumbers there
    rho, u, a = oracle.ideal_gas_pT(0.02896, 1.4, 1.0e5, 300.0)
    assert rel(8.31451 / 0.02896, 287.086) < 1e-4
    assert rel(rho, 1.16109) < 1e-4
    assert rel(u, 215314.0) < 1e-4
    assert rel(a, 347.241) < 1e-4


def test_workload_state_matches_oracle_eos(oracle):
    gas = W.IdealGas()
    rho, u, a = gas.from_pT(1.0e5, 300.0)
    r2, u2, a2 = oracle.ideal_gas_pT(0.02896, 1.4, 1.0e5, 300.0)
    assert float(rho) == r2 and float(u) == u2 and float(a) == a2


def _run_sod3d(oracle, flux):
    wl = W.sod_3d_tube()
    cfg = oracle.default_config(dimensions=3, flux_calculator=flux)
    sim = oracle.OracleSim(cfg)
    b = wl.blocks[0]
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    rc = sim.run(600, 0.6e-3)
    assert rc == 0
    prim, _ = sim.get_flow(0)
    xc = W.cell_centres(b.vtx, b.ni, b.nj, b.nk, 3)[:, 0]
    return sim, prim, xc


def test_sod_tube_regression(oracle):
    sim, prim, xc = _run_sod3d(oracle, oracle.FLUX_AUSMDV)
    # sod-test.rb test_1_run: 75 +- 3 steps
    assert abs(sim.step - 75) < 3
    # test_2_post_shock_region at x=0.78 and test_3_expanded_driver_region at x=0.6
    for x, ref in ((0.78, {"rho": 0.2647, "p": 30.2e3, "T": 398.0, "velx": 293.0}),
                   (0.6, {"rho": 0.4271, "p": 30.2e3, "T": 247.0, "velx": 293.0})):
        q = int(np.argmin(np.abs(xc - x)))
        got = {"rho": prim[0, q], "velx": prim[1, q], "p": prim[4, q], "T": prim[5, q]}
        for k, v in ref.items():
            assert rel(got[k], v) < 1.0e-2, (x, k, got[k], v)


def test_hllc_sod_tube_close_to_ausmdv(oracle):
    # HLLC has no reference implementation; on the same deck it must land on
    # the same shock-tube solution within the regression test's 1 % band.
    sim, prim, xc = _run_sod3d(oracle, oracle.FLUX_HLLC)
    assert abs(sim.step - 75) < 4
    q = int(np.argmin(np.abs(xc - 0.78)))
    assert rel(prim[0, q], 0.2647) < 1.0e-2
    assert rel(prim[4, q], 30.2e3) < 1.0e-2


def test_uniform_geometry_is_exact(oracle):
    # Dyadic Cartesian grids give bit-identical geometry in every cell and face.
    wl = W.inflow_3d(n=8, nsteps=1)
    b = wl.blocks[0]
    sim = oracle.OracleSim(oracle.default_config(dimensions=3))
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    cells, faces = sim.geometry(0)
    assert np.all(cells[0] == cells[0, 0]) and cells[0, 0] == pytest.approx(1.0 / 512, rel=1e-15)
    assert np.all(cells[1] == 0.125)
    ni = nj = nk = 8
    nfi = (ni + 1) * nj * nk
    assert np.all(faces[:nfi, 0] == 1.0) and np.all(faces[:nfi, 9] == 1.0 / 64)


def test_oracle_conserves_mass_in_closed_box(oracle):
    wl = W.sod_2d(32, 8, nsteps=50)
    b = wl.blocks[0]
    sim = oracle.OracleSim(oracle.default_config(dimensions=2))
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    _, c0 = sim.get_flow(0)
    assert sim.run(50) == 0
    _, c1 = sim.get_flow(0)
    assert rel(c1[0].sum(), c0[0].sum()) < 1e-13
    assert rel(c1[4].sum(), c0[4].sum()) < 1e-13
