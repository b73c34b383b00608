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


@pytest.mark.parametrize("flux", ["hanel", "adaptive_hanel_ausmdv"])
def test_hanel_and_adaptive_sod_tube_regression(oracle, flux):
    # The reference's default flux calculator (adaptive_hanel_ausmdv,
    # globalconfig.d:533) and Hanel's: the Sod deck's regression values hold
    # within the test's 1 % band.
    f = oracle.FLUX_HANEL if flux == "hanel" else oracle.FLUX_ADAPTIVE_HANEL_AUSMDV
    sim, prim, xc = _run_sod3d(oracle, f)
    assert abs(sim.step - 75) < 4
    for x, ref in ((0.78, {"rho": 0.2647, "p": 30.2e3, "T": 398.0, "velx": 293.0}),
                   (0.6, {"rho": 0.4271, "T": 247.0})):
        q = int(np.argmin(np.abs(xc - x)))
        got = {"rho": prim[0, q], "velx": prim[1, q], "p": prim[4, q], "T": prim[5, q]}
        for k, v in ref.items():
            assert rel(got[k], v) < 1.0e-2, (flux, x, k, got[k], v)


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


# --- thermally perfect 5-species air and chemistry ---------------------------

def test_therm_perf_gas_golden(oracle):
    """src/gas/therm_perf_gas.d:457-480 on the 5-species air deck (1e-6 relative)."""
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    mf = [0.2] * 5
    s = oracle.tp_update(tc, 0, mf, p=1.0e6, T=2000.0)
    assert rel(s["u"], 11801825.6) < 1e-6 and rel(s["rho"], 1.2840117) < 1e-6
    s = oracle.tp_update(tc, 1, mf, rho=2.0, u=14.0e6, T=2000.0)
    assert rel(s["p"], 3373757.4) < 1e-6 and rel(s["T"], 4331.944) < 1e-6
    s = oracle.tp_update(tc, 2, mf, rho=1.5, T=10000.0)
    assert rel(s["p"], 5841068.3) < 1e-6 and rel(s["u"], 20340105.9) < 1e-6


def test_portable_math_accuracy(oracle):
    """The oracle's exp/log (also used on the GPU) stay within a few ulp of libm."""
    import ctypes
    L = oracle.lib()
    # exercised through the thermo curves: u(T) and the rhou Newton round trip
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    mf = [0.767, 0.233, 0.0, 0.0, 0.0]
    for T in (250.0, 600.0, 1000.0, 2500.0, 7000.0, 15000.0):
        s = oracle.tp_update(tc, 2, mf, rho=0.1, T=T)
        ref_u = sum(m * (tc.h(i, T) - tc.R[i] * T) for i, m in enumerate(mf))
        assert rel(s["u"], ref_u) < 1e-13, (T, s["u"], ref_u)
        back = oracle.tp_update(tc, 1, mf, rho=0.1, u=s["u"], T=T * 1.3)
        assert rel(back["T"], T) < 1e-9


def test_chemistry_relaxes_towards_dissociation(oracle):
    """Hot air at 6000 K dissociates O2 (and some N2); mass is conserved,
    energy is kept (constant rho, u) and T drops."""
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    mf = [0.767, 0.233, 0.0, 0.0, 0.0]
    s = oracle.tp_update(tc, 0, mf, p=1.0e5, T=6000.0)
    rc, out = oracle.chem_cell(tc, 300.0, 1.0e-6, s["rho"], 6000.0, s["u"], s["p"], mf)
    assert rc == 0
    y = out["massf"]
    assert abs(sum(y) - 1.0) < 1e-12
    assert y[4] > 1e-4 and y[1] < 0.233 and out["T"] < 6000.0
    # the whole-interval point-implicit step converged: the sub-cycling
    # recovery (the only user of the per-cell dt_chem) did not run
    assert out["dt_chem"] == -1.0
    # a frozen cell (T <= T_frozen) is left alone
    rc, out2 = oracle.chem_cell(tc, 300.0, 1.0e-6, 1.0, 300.0, 2.0e5, 1.0e5, mf)
    assert rc == 0 and list(out2["massf"]) == mf


def test_reacting_channel_oracle_runs(oracle):
    from eilmer4_b200 import workloads as W
    wl = W.reacting_channel(ni=24, nj=12)
    cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV,
                                gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=1)
    sim = oracle.OracleSim(cfg, wl.thermochem)
    b = wl.blocks[0]
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    assert sim.run(40) == 0
    prim, cons = sim.get_flow(0)
    assert np.all(np.isfinite(prim)) and prim[5].max() > 300.0
    assert np.allclose(prim[8:].sum(axis=0), 1.0, atol=1e-12)


def _thermo_only(species):
    """A ThermoChem with the given species' curves and no reactions."""
    from eilmer4_b200.thermochem import ThermoChem
    nsp, maxseg = len(species), 4
    T_break = np.zeros((nsp, maxseg + 1))
    T_blend = np.zeros((nsp, maxseg))
    coeffs = np.zeros((nsp, maxseg, 9))
    for i, s in enumerate(species):
        n = len(s["coeffs"])
        T_break[i, :n + 1] = s["T_break"]
        T_blend[i, :n - 1] = s["T_blend"]
        coeffs[i, :n] = s["coeffs"]
    return ThermoChem(
        species=[s["name"] for s in species], M=np.array([s["M"] for s in species]),
        nseg=np.array([len(s["coeffs"]) for s in species], dtype=np.int32),
        T_break=T_break, T_blend=T_blend, coeffs=coeffs,
        A_f=np.zeros(0), n_f=np.zeros(0), C_f=np.zeros(0), A_b=np.zeros(0), n_b=np.zeros(0),
        C_b=np.zeros(0), nu_r=np.zeros((0, nsp), dtype=np.int32),
        nu_p=np.zeros((0, nsp), dtype=np.int32), third_body=np.zeros(0, dtype=np.int32),
        eff=np.zeros((0, nsp)), T_lower=300.0, T_upper=50000.0)


def test_cea_curve_of_atomic_oxygen_golden(oracle):
    """cea_thermo_curves.d:173-189 (sample-data/O-thermo.lua, the same curves as
    the air data's O): Cp(500 K) = 1328.627 J/kg/K, h(3700 K) = 20030794.683 J/kg.
    The oracle's pure-O mixture gives h = u + R T and Cp from its frozen sound
    speed, a^2 = gamma R T."""
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    y = np.zeros(tc.nsp)
    y[tc.species.index("O")] = 1.0
    R = 8.31451 / 0.0159994
    s = oracle.tp_update(tc, 2, y, rho=0.1, T=3700.0)
    assert s["u"] + R * 3700.0 == pytest.approx(20030794.683, rel=1e-6)
    s = oracle.tp_update(tc, 2, y, rho=0.1, T=500.0)
    gamma = s["a"] ** 2 / (R * 500.0)
    assert gamma * R / (gamma - 1.0) == pytest.approx(1328.627, rel=1e-6)


def test_mixture_eos_golden(oracle):
    """therm_perf_gas_mix_eos.d:179-200 (sample-data/O2-N2-H2.lua, extracted to
    tests/golden/o2_n2_h2_thermo.json by tests/golden/make_o2_n2_h2.py): mass
    fractions 0.2, 0.7, 0.1 at 1000 K give u = 1031849.875 J/kg, and the
    temperature iteration started from 1500 K returns 1000 K."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "o2_n2_h2_thermo.json")
    with open(path) as f:
        tc = _thermo_only(json.load(f)["species"])
    y = [0.2, 0.7, 0.1]
    s = oracle.tp_update(tc, 2, y, rho=1.0, T=1000.0)
    assert s["u"] == pytest.approx(1031849.875, rel=1e-6)
    s2 = oracle.tp_update(tc, 1, y, rho=1.0, u=s["u"], T=1500.0)
    assert s2["T"] == pytest.approx(1000.0, rel=1e-6)
