"""The premise of the bracket-sign shortcut in the GPU's mixture temperature
iteration: for the shipped 5-species air curves, each species' energy
e(T) = h(T) - R T, evaluated as the device evaluates it (blended segments,
linear beyond the curves), rises within any +-1000 K window by at least half
of Cv at the window's centre per kelvin (the library checks the same on the
host, on a finer grid, whenever curves are installed, and uses kappa = 1/4)."""
import numpy as np


def _coeffs(tc, s, T):
    tb, bl, c = tc.T_break[s], tc.T_blend[s], tc.coeffs[s]
    ns = int(tc.nseg[s])
    out = np.empty((T.size, 9))
    done = np.zeros(T.size, bool)
    m = T < tb[1] - 0.5 * bl[0]
    out[m] = c[0]
    done |= m
    m = (~done) & (T > tb[ns - 1] + 0.5 * bl[ns - 2])
    out[m] = c[ns - 1]
    done |= m
    for i in range(1, ns):
        lo, hi = tb[i] - 0.5 * bl[i - 1], tb[i] + 0.5 * bl[i - 1]
        m = (~done) & (T >= lo) & (T <= hi)
        wB = (T[m] - lo) / bl[i - 1]
        out[m] = (1.0 - wB)[:, None] * c[i - 1] + wB[:, None] * c[i]
        done |= m
        m = (~done) & (T > hi) & (T < tb[i + 1] - 0.5 * bl[i])
        out[m] = c[i]
        done |= m
    assert done.all()
    return out


def _h_in(tc, s, R, T):
    a = _coeffs(tc, s, T)
    hrt = (-a[:, 0] / (T * T) + a[:, 1] / T * np.log(T) + a[:, 2] + a[:, 3] * T / 2.0
           + a[:, 4] * T * T / 3.0 + a[:, 5] * T ** 3 / 4.0 + a[:, 6] * T ** 4 / 5.0 + a[:, 7] / T)
    return R * T * hrt


def _cp(tc, s, R, T):
    lo, hi = tc.T_break[s][0], tc.T_break[s][int(tc.nseg[s])]
    T = np.clip(T, lo, hi)
    a = _coeffs(tc, s, T)
    return R * (a[:, 0] / (T * T) + a[:, 1] / T + a[:, 2] + a[:, 3] * T + a[:, 4] * T * T
                + a[:, 5] * T ** 3 + a[:, 6] * T ** 4)


def _h(tc, s, R, T):
    lo, hi = tc.T_break[s][0], tc.T_break[s][int(tc.nseg[s])]
    out = _h_in(tc, s, R, np.clip(T, lo, hi))
    el, eh = np.array([lo]), np.array([hi])
    out = np.where(T < lo, _h_in(tc, s, R, el)[0] - _cp(tc, s, R, el)[0] * (lo - T), out)
    return np.where(T > hi, _h_in(tc, s, R, eh)[0] + _cp(tc, s, R, eh)[0] * (T - hi), out)


def test_air_energy_slope_bound():
    from numpy.lib.stride_tricks import sliding_window_view

    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    step = 1.0
    T = np.arange(20.0, 101501.0, step)
    W = int(1000 / step)
    for s in range(tc.nsp):
        R = 8.31451 / tc.M[s]
        cv = _cp(tc, s, R, T) - R
        assert cv.min() > 0.0, tc.species[s]
        slope = np.diff(_h(tc, s, R, T) - R * T) / step
        mins = sliding_window_view(slope, 2 * W).min(axis=1)
        ratio = mins / cv[W:W + mins.size]
        assert ratio.min() >= 0.5, (tc.species[s], ratio.min())
