"""The point-implicit chemistry of the CPU oracle against an independent
integration of the same rate equations (SciPy's implicit Radau method at
tight tolerance), at constant temperature as ChemistryUpdate.opCall holds it
(src/kinetics/chemistry_update.d:119-307).

This pins what the reference has no test for here: the rate constants
(rate_constant.d:71-75 with the Gupta backward fits), the mass-action rates
with third bodies (reaction.d:275-400), the stoichiometry and the SI units of
the 5-species air mechanism.  The point-implicit step is one backward-Euler
step over dt, so it must (a) agree with the exact solution to first order in
dt and (b) land on the same equilibrium for long dt."""
import numpy as np
import pytest

scipy_integrate = pytest.importorskip("scipy.integrate")


def omega(tc, T, c):
    """dc/dt of the mechanism at temperature T (mol/m^3/s), NumPy restatement."""
    T = min(max(T, tc.T_lower), tc.T_upper)
    kf = tc.A_f * T ** tc.n_f * np.exp(-tc.C_f / T)
    kb = tc.A_b * T ** tc.n_b * np.exp(-tc.C_b / T)
    w = np.zeros(tc.nsp)
    for r in range(tc.nreac):
        M = float(tc.eff[r] @ c) if tc.third_body[r] else 1.0
        wf = kf[r] * M * np.prod(c ** tc.nu_r[r])
        wb = kb[r] * M * np.prod(c ** tc.nu_p[r])
        w += (tc.nu_p[r] - tc.nu_r[r]) * (wf - wb)
    return w


def exact_massf(tc, rho, T, y0, dt):
    c0 = np.asarray(y0) * rho / tc.M
    sol = scipy_integrate.solve_ivp(lambda t, c: omega(tc, T, c), (0.0, dt), c0, method="Radau",
                                    rtol=1e-11, atol=1e-14 * c0.sum())
    assert sol.success
    c = np.maximum(sol.y[:, -1], 0.0)
    y = c * tc.M / rho
    return y / y.sum()


def oracle_massf(oracle, tc, s, T, y0, dt):
    rc, y = oracle.chem_update(tc, dt, s["rho"], T, y0)
    assert rc == 0
    return y


@pytest.mark.parametrize("T", [4000.0, 6000.0])
def test_point_implicit_step_converges_to_exact_solution(oracle, T):
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    y0 = [0.767, 0.233, 0.0, 0.0, 0.0]
    s = oracle.tp_update(tc, 0, y0, p=1.0e5, T=T)
    errs = []
    for dt in (1.0e-8, 1.0e-9):
        ye = exact_massf(tc, s["rho"], T, y0, dt)
        yo = oracle_massf(oracle, tc, s, T, y0, dt)
        change = np.abs(ye - np.array(y0)).max()
        assert change > 1e-7, "the test state must react over dt"
        err = np.abs(yo - ye).max()
        errs.append(err / change)
        # same direction of every species' change
        sig = np.abs(ye - np.array(y0)) > 1e-3 * change
        assert np.all(np.sign(yo - y0)[sig] == np.sign(ye - y0)[sig])
    # first-order accurate: the relative error falls about tenfold with dt
    assert errs[1] < 0.05, errs
    assert errs[1] < 0.25 * errs[0], errs


def test_point_implicit_step_reaches_the_same_equilibrium(oracle):
    """Over a long dt at constant T the backward-Euler step lands on the
    equilibrium of the mechanism (its fixed point), as the exact solution
    does.  (Over such a dt the temperature update that follows the
    isothermal chemistry in thermochemical_increment would have no solution:
    the dissociation energy exceeds the cell's internal energy.)"""
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    T = 6000.0
    y0 = [0.767, 0.233, 0.0, 0.0, 0.0]
    s = oracle.tp_update(tc, 0, y0, p=1.0e5, T=T)
    dt = 1.0e-2        # many chemical times at 6000 K
    ye = exact_massf(tc, s["rho"], T, y0, dt)
    yo = oracle_massf(oracle, tc, s, T, y0, dt)
    assert ye[4] > 0.1    # oxygen dissociated
    assert np.abs(yo - ye).max() < 1e-5, (yo, ye)
