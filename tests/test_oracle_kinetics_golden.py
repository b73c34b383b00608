"""The oracle's rate machinery against the reference's own kinetics tests on
the hydrogen-iodide system (src/kinetics/sample-input/H2-I2-HI.lua,
H2-I2-inp.lua):

* reaction.d:475-493 -- H2 + I2 -> 2 HI with k = 1.94e14 exp(-20620/T) both
  ways at 700 K and concentrations (4.54, 4.54, 0): HI produced at
  1287.8606, H2 and I2 lost at 643.9303 mol/m^3/s (relative 1e-6);
* chemistry_update.d:659-733 -- the same system with the mechanism's rate
  constants from 4.54 mol/m^3 each of H2 and I2 at 700 K: the analytic HI
  concentration after 60,000 s is 7.1420197868416215 mol/m^3.  The oracle's
  point-implicit update, repeated over shorter intervals, converges to it at
  first order (it is one backward-Euler step per interval)."""
import numpy as np
import pytest

M = np.array([0.00201588, 0.25380894, 0.12791241])   # H2, I2, HI (kg/mol)


def h2_i2(A_f, C_f, A_b, C_b):
    from eilmer4_b200.thermochem import ThermoChem
    nsp, maxseg = 3, 4
    T_break = np.zeros((nsp, maxseg + 1))
    T_break[:, 0], T_break[:, 1] = 200.0, 20000.0
    coeffs = np.zeros((nsp, maxseg, 9))
    coeffs[:, 0, 2] = 3.5          # Cp/R = 3.5 (not used by the rate tests)
    return ThermoChem(
        species=["H2", "I2", "HI"], M=M.copy(), nseg=np.ones(nsp, dtype=np.int32),
        T_break=T_break, T_blend=np.zeros((nsp, maxseg)), coeffs=coeffs,
        A_f=np.array([A_f]), n_f=np.array([0.0]), C_f=np.array([C_f]),
        A_b=np.array([A_b]), n_b=np.array([0.0]), C_b=np.array([C_b]),
        nu_r=np.array([[1, 1, 0]], dtype=np.int32), nu_p=np.array([[0, 0, 2]], dtype=np.int32),
        third_body=np.array([0], dtype=np.int32), eff=np.zeros((1, nsp)),
        T_lower=300.0, T_upper=50000.0)


def test_elementary_reaction_rates_golden(oracle):
    tc = h2_i2(1.94e14, 20620.0, 1.94e14, 20620.0)
    q, L = oracle.rates(tc, 700.0, [4.54, 4.54, 0.0])
    assert q[0] == 0.0 and q[1] == 0.0 and L[2] == 0.0
    assert q[2] == pytest.approx(1287.8606, rel=1e-6)
    assert L[0] == pytest.approx(643.9303, rel=1e-6)
    assert L[1] == pytest.approx(643.9303, rel=1e-6)


def test_hydrogen_iodide_update_converges_to_the_analytic_value(oracle):
    tc = h2_i2(1.93e8, 20620.0, 5.470705805110e-07, 0.0)
    T, c0, t_end = 700.0, 4.54, 60000.0
    analytic = 7.1420197868416215
    conc0 = np.array([c0, c0, 0.0])
    rho = float(conc0 @ M)
    errs = []
    for n in (200, 400, 800):
        y = conc0 * M / rho
        dtc = -1.0
        for _ in range(n):
            rc, y = oracle.chem_update(tc, t_end / n, rho, T, y, dtc)
            assert rc == 0
        c_hi = y[2] * rho / M[2]
        errs.append(c_hi - analytic)
    # first order: the error halves with the interval
    assert 1.8 < errs[0] / errs[1] < 2.2 and 1.8 < errs[1] / errs[2] < 2.2, errs
    assert abs(errs[2]) < 1e-3 * analytic, errs
    # Richardson extrapolation of the two finest runs lands on the analytic value
    assert abs((2.0 * (errs[2] + analytic) - (errs[1] + analytic)) - analytic) < 1e-5 * analytic


def test_newton_solver_golden(oracle):
    """nm/newton.d:109-135: the safeguarded Newton method (the one the
    mixture's temperature iteration uses) finds 1.732051 and 0.3604217."""
    rc, r = oracle.newton_test(0)
    assert rc == 0 and abs(r - 1.732051) < 1e-5
    rc, r = oracle.newton_test(1)
    assert rc == 0 and abs(r - 0.3604217) < 1e-5


def test_portable_math_against_libm_on_the_hot_channel(oracle):
    """The oracle with its portable exp/log/pow (which the GPU shares bit for
    bit) against its build on the C library's exp, log and pow, as the
    reference calls them: after 30 steps of the dissociating ramp channel
    every primitive field and mass fraction agrees to 1e-11 of its scale."""
    from eilmer4_b200 import workloads as W
    wl = W.reacting_channel_hot(48, 24)
    out = []
    for libm in (False, True):
        cfg = oracle.default_config(dimensions=2, flux_calculator=oracle.FLUX_AUSMDV,
                                    gas_model=oracle.GAS_THERM_PERF_5SP_AIR, reacting=1,
                                    n_threads=0)
        sim = oracle.OracleSim(cfg, wl.thermochem, libm=libm)
        b = wl.blocks[0]
        sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
        sim.set_flow(0, b.prim)
        assert sim.run(30) == 0
        out.append((sim.get_flow(0)[0], sim.step))
    (p0, s0), (p1, s1) = out
    assert s0 == s1
    speed = np.abs(p0[1:3]).max()
    for q in range(p0.shape[0]):
        scale = speed if q in (1, 2, 3) else np.abs(p0[q]).max()
        if scale == 0.0:
            continue
        assert np.abs(p1[q] - p0[q]).max() <= 1e-11 * scale, q


def test_rkf_step_order_golden(oracle):
    """chemistry_update.d:681-698: the RKF step on the hydrogen-iodide system,
    repeated with a fixed step to t = 60,000 s, with h = 287.175 and with
    h * 2^(-1/5): the errors against the analytic HI concentration fall by
    the ratio 1.96809 (to 1e-4), as a fifth-order method's do."""
    tc = h2_i2(1.93e8, 20620.0, 5.470705805110e-07, 0.0)
    T, c0, t_end = 700.0, 4.54, 60000.0
    analytic = 7.1420197868416215

    def estimate(dt):
        conc = np.array([c0, c0, 0.0])
        t = 0.0
        while (t_end - t) > 1.0e-9:
            dt = min(dt, t_end - t)
            _, conc, _ = oracle.rkf_step(tc, T, conc, dt)
            t += dt
        return conc[2]

    dt = 287.175
    err0 = analytic - estimate(dt)
    err1 = analytic - estimate(dt * 2.0 ** (-1.0 / 5.0))
    assert abs(err0 / err1 - 1.96809) <= 1e-4 * 1.96809, err0 / err1


def test_rkf_chemistry_update_golden(oracle):
    """chemistry_update.d:720-731: the complete chemistry update (opCall's
    sub-cycling with RKF steps, the reference's default method) over
    60,000 s from dt_chem = 200 s gives HI = 7.14201983840 mol/m^3 (to 1e-9)."""
    tc = h2_i2(1.93e8, 20620.0, 5.470705805110e-07, 0.0)
    T, c0 = 700.0, 4.54
    conc0 = np.array([c0, c0, 0.0])
    rho = float(conc0 @ M)
    oracle.set_chem_method(1)
    try:
        rc, y = oracle.chem_update(tc, 60000.0, rho, T, conc0 * M / rho, 200.0)
    finally:
        oracle.set_chem_method(0)
    assert rc == 0
    c_hi = y[2] * rho / M[2]
    assert abs(c_hi - 7.14201983840) <= 1e-9 * 7.14201983840, c_hi
