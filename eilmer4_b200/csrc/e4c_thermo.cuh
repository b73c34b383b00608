// e4c_thermo.cuh -- thermally perfect mixture and finite-rate chemistry on the device.
//
// Reference code reproduced (paths in the reference project):
//   CEA thermo curves   src/gas/thermo/cea_thermo_curves.d:49-167
//   mixture EOS         src/gas/therm_perf_gas.d:182-191, 345-396,
//                       src/gas/thermo/therm_perf_gas_mix_eos.d:63-150,
//                       src/gas/thermo/perf_gas_mix_eos.d:43-62, gas_model.d:45-46, 196-230, 330-338
//   T Newton            src/nm/newton.d:40-99 (rtsafe with bisection); note that it leaves
//                       Q.u at the energy of the last evaluated iterate, as the reference does
//   rates               src/kinetics/rate_constant.d:71-75, reaction.d:79-114, 275-400,
//                       reaction_mechanism.d:47-82, 127-170
//   sub-cycling         src/kinetics/chemistry_update.d:119-307
//   cell increment      src/eilmer/fvcell.d:1510-1621
// The point-implicit step (backward Euler solved by Newton iteration with the
// analytic Jacobian) has no counterpart in the reference.
//
// exp and log are portable implementations written with + - * / only (Cody-
// Waite reduction + Taylor polynomial for exp; atanh series for log).  With
// -fmad=false they give the same bits as the CPU oracle's copies of the same
// methods (within a few ulp of libm).
#pragma once

#include <cfloat>
#include <math_constants.h>

#include "../../include/e4cuda.h"

namespace e4c {

// Inlining of the CEA curve evaluations and of exp/log.  The thermally perfect
// kernels are large enough for instruction fetch to matter: calling the CEA
// evaluations instead of inlining them measured 1.1x (cold channel) to 1.3x
// (reacting channel) faster.
#ifndef E4C_CEA_NOINLINE
#define E4C_CEA_NOINLINE 1
#endif
#if E4C_CEA_NOINLINE
#define E4C_CEA_FN __noinline__
#else
#define E4C_CEA_FN __forceinline__
#endif
// The segment/blend selection is inlined into each called evaluation, which
// keeps the nine coefficients in registers (1.27x on the reacting channel
// against calling it too).
#ifndef E4C_COEF_FN
#define E4C_COEF_FN __forceinline__
#endif
#ifndef E4C_PM_NOINLINE
#define E4C_PM_NOINLINE 0
#endif
#if E4C_PM_NOINLINE
#define E4C_PM_FN __noinline__
#else
#define E4C_PM_FN __forceinline__
#endif

// ---------------------------------------------------------------------------
// Portable exp / log / pow
// ---------------------------------------------------------------------------
static __device__ E4C_PM_FN double pm_log(double x) {
    if (!(x > 0.0)) return (x == 0.0) ? -HUGE_VAL : CUDART_NAN;
    if (isinf(x)) return x;
    int k;
    double m = frexp(x, &k);
    if (m < 0.70710678118654752440) { m = m * 2.0; k = k - 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    double p = 1.0 / 23.0;
    p = p * s2 + 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    p = p * s2 + 1.0;
    const double ln2_hi = 6.93147180369123816490e-01;
    const double ln2_lo = 1.90821492927058770002e-10;
    double kd = double(k);
    return kd * ln2_hi + (2.0 * s * p + kd * ln2_lo);
}

static __device__ E4C_PM_FN double pm_exp(double x) {
    if (x != x) return x;
    if (x > 709.78) return HUGE_VAL;
    if (x < -745.2) return 0.0;
    const double inv_ln2 = 1.44269504088896338700e+00;
    const double ln2_hi = 6.93147180369123816490e-01;
    const double ln2_lo = 1.90821492927058770002e-10;
    double kd = floor(x * inv_ln2 + 0.5);
    double r = (x - kd * ln2_hi) - kd * ln2_lo;
    double p = 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return ldexp(p, int(kd));
}

__device__ __forceinline__ double pm_pow(double x, double n) {
    if (n == 0.0) return 1.0;
    if (n == 1.0) return x;
    if (n == -1.0) return 1.0 / x;
    if (n == 2.0) return x * x;
    if (n == 0.5) return sqrt(x);
    if (n == -0.5) return 1.0 / sqrt(x);
    if (n == 1.5) return x * sqrt(x);
    if (n == -1.5) return 1.0 / (x * sqrt(x));
    return pm_exp(n * pm_log(x));
}

// pm_pow(x, n) given lx = pm_log(x): the same value, bit for bit
__device__ __forceinline__ double pm_pow_l(double x, double lx, double n) {
    if (n == 0.0) return 1.0;
    if (n == 1.0) return x;
    if (n == -1.0) return 1.0 / x;
    if (n == 2.0) return x * x;
    if (n == 0.5) return sqrt(x);
    if (n == -0.5) return 1.0 / sqrt(x);
    if (n == 1.5) return x * sqrt(x);
    if (n == -1.5) return 1.0 / (x * sqrt(x));
    return pm_exp(n * lx);
}

// ---------------------------------------------------------------------------
// CEA thermo curves
// ---------------------------------------------------------------------------
static __device__ E4C_COEF_FN void cea_coefficients(const e4c_thermochem& tc, int isp, double T,
                                                 double a[9]) {
    const int nseg = tc.nseg[isp];
    const double* tb = tc.T_break[isp];
    const double* bl = tc.T_blend[isp];
    if (T < (tb[1] - 0.5 * bl[0])) {
        for (int j = 0; j < 9; ++j) a[j] = tc.coeffs[isp][0][j];
        return;
    }
    if (T > (tb[nseg - 1] + 0.5 * bl[nseg - 2])) {
        for (int j = 0; j < 9; ++j) a[j] = tc.coeffs[isp][nseg - 1][j];
        return;
    }
    for (int i = 1; i < nseg; ++i) {
        double T_blend_low = tb[i] - 0.5 * bl[i - 1];
        double T_blend_high = tb[i] + 0.5 * bl[i - 1];
        if (T >= T_blend_low && T <= T_blend_high) {
            double wB = (1. / bl[i - 1]) * (T - T_blend_low);
            double wA = 1.0 - wB;
            for (int j = 0; j < 9; ++j) a[j] = wA * tc.coeffs[isp][i - 1][j] + wB * tc.coeffs[isp][i][j];
            return;
        }
        if (T > T_blend_high && T < (tb[i + 1] - 0.5 * bl[i])) {
            for (int j = 0; j < 9; ++j) a[j] = tc.coeffs[isp][i][j];
            return;
        }
    }
    for (int j = 0; j < 9; ++j) a[j] = CUDART_NAN;
}

// a / b rounded to nearest, from y = RN(1/b) computed once for the divisor.
// q = RN(a y) lies within 1.5 ulp of a/b; one correction with the FMA
// residual makes it faithful, and the second is RN(a/b) by Markstein's
// theorem (P. W. Markstein, IBM J. Res. Develop. 34(1), 1990: with y within
// half an ulp of 1/b and q within one ulp of a/b, r = a - q b is exact and
// RN(q + r y) = RN(a/b)).  For b positive, finite and normal with a/b normal
// (the CEA curve terms); a zero keeps the sign of the quotient.  The curve
// evaluations divide by T, T^2, 3 and 5 only, so each temperature pays for two
// true divisions instead of about thirty.
__device__ __forceinline__ double div_rn(double a, double b, double y) {
    double q = a * y;
    double r = fma(-q, b, a);
    q = fma(r, y, q);
    r = fma(-q, b, a);
    q = fma(r, y, q);
    return a == 0.0 ? a * y : q;
}

// A temperature with T^2 and the reciprocals of both, rounded to nearest.
struct TRecip {
    double T, T2, rT, rT2;
    __device__ explicit TRecip(double t) : T(t), T2(t * t), rT(1.0 / t), rT2(1.0 / (t * t)) {}
};

constexpr double kThird = 1.0 / 3.0, kFifth = 1.0 / 5.0;

// Cp/R and h/RT of one coefficient set at t (the operations of the
// reference's curves, cea_thermo_curves.d; each quotient as div_rn gives it)
__device__ __forceinline__ double cea_Cp_on_R(const double a[9], const TRecip& t) {
    const double T = t.T;
    double Cp_on_R = div_rn(a[0], t.T2, t.rT2) + div_rn(a[1], T, t.rT) + a[2] + a[3] * T;
    Cp_on_R += a[4] * T * T + a[5] * T * T * T + a[6] * T * T * T * T;
    return Cp_on_R;
}
__device__ __forceinline__ double cea_h_on_RT(const double a[9], const TRecip& t, double lT) {
    const double T = t.T;
    double h_on_RT = div_rn(-a[0], t.T2, t.rT2) + div_rn(a[1], T, t.rT) * lT + a[2] + a[3] * T / 2.0;
    h_on_RT += div_rn(a[4] * T * T, 3.0, kThird) + a[5] * T * T * T / 4.0 +
               div_rn(a[6] * T * T * T * T, 5.0, kFifth) + div_rn(a[7], T, t.rT);
    return h_on_RT;
}

static __device__ E4C_CEA_FN double cea_Cp(const e4c_thermochem& tc, int isp, double R, double T) {
    const int nseg = tc.nseg[isp];
    if (T < tc.T_break[isp][0]) T = tc.T_break[isp][0];
    if (T > tc.T_break[isp][nseg]) T = tc.T_break[isp][nseg];
    double a[9];
    cea_coefficients(tc, isp, T, a);
    return R * cea_Cp_on_R(a, TRecip(T));
}

// lT is pm_log(T), shared by the species of a mixture evaluated at one T
static __device__ E4C_CEA_FN double cea_h_in_range(const e4c_thermochem& tc, int isp, double R,
                                                 const TRecip& t, double lT) {
    double a[9];
    cea_coefficients(tc, isp, t.T, a);
    return R * t.T * cea_h_on_RT(a, t, lT);
}

static __device__ E4C_CEA_FN double cea_h(const e4c_thermochem& tc, int isp, double R,
                                        const TRecip& t, double lT) {
    const int nseg = tc.nseg[isp];
    const double T = t.T;
    if (T < tc.T_break[isp][0]) {
        double T_low = tc.T_break[isp][0];
        double h_low = cea_h_in_range(tc, isp, R, TRecip(T_low), pm_log(T_low));
        double Cp_low = cea_Cp(tc, isp, R, T_low);
        return h_low - Cp_low * (T_low - T);
    }
    if (T > tc.T_break[isp][nseg]) {
        double T_high = tc.T_break[isp][nseg];
        double h_high = cea_h_in_range(tc, isp, R, TRecip(T_high), pm_log(T_high));
        double Cp_high = cea_Cp(tc, isp, R, T_high);
        return h_high + Cp_high * (T - T_high);
    }
    return cea_h_in_range(tc, isp, R, t, lT);
}

// cea_h and cea_Cp of one species at one temperature with one coefficient
// selection (the same operations as the two functions)
static __device__ E4C_CEA_FN void cea_h_Cp(const e4c_thermochem& tc, int isp, double R,
                                          const TRecip& t, double lT, double& h, double& Cp) {
    const int nseg = tc.nseg[isp];
    const double T = t.T;
    if (T < tc.T_break[isp][0] || T > tc.T_break[isp][nseg]) {
        h = cea_h(tc, isp, R, t, lT);
        Cp = cea_Cp(tc, isp, R, T);
        return;
    }
    double a[9];
    cea_coefficients(tc, isp, T, a);
    Cp = R * cea_Cp_on_R(a, t);
    h = R * T * cea_h_on_RT(a, t, lT);
}

// ---------------------------------------------------------------------------
// Thermally perfect mixture
// ---------------------------------------------------------------------------
template <int NSP>
struct TPState {
    double rho, p, T, u, a;
    double massf[NSP];
};

// kappa of the bracket-sign shortcut of TPGas::solve_T, 0 when off: the
// installed curves raise each species' energy e(T) = h(T) - R T by at least
// 2 kappa Cv(x0) per kelvin anywhere within 1000 K of x0, for brackets up to
// 101,000 K (checked on the host when they are installed,
// set_thermochem_constants)
static __constant__ double c_bracket_kappa = 0.0;

// Per-species values passed by value (no address taken, so they stay in
// registers across the call).
template <int NSP>
struct SpVals {
    double v[NSP];
};
struct EnergySlope {
    double u, du;
};

// The mixture's energy e = sum Y_i (h_i - R_i T) and -sum Y_i (Cp_i - R_i)
// at T, every species in one call (one call boundary per temperature instead
// of one per species): the operations of TPGas::energy_dudT's loop over
// cea_h_Cp, in the same order.
template <int NSP>
static __device__ E4C_CEA_FN EnergySlope mix_energy_slope(const e4c_thermochem& tc, SpVals<NSP> R,
                                                          SpVals<NSP> massf, double T) {
    const double lT = pm_log(T);
    const TRecip t(T);
    double e[NSP], v[NSP];
#pragma unroll
    for (int i = 0; i < NSP; ++i) {
        double h, cp;
        const int nseg = tc.nseg[i];
        if (T < tc.T_break[i][0] || T > tc.T_break[i][nseg]) {
            h = cea_h(tc, i, R.v[i], t, lT);
            cp = cea_Cp(tc, i, R.v[i], T);
        } else {
            double a[9];
            cea_coefficients(tc, i, T, a);
            cp = R.v[i] * cea_Cp_on_R(a, t);
            h = R.v[i] * T * cea_h_on_RT(a, t, lT);
        }
        e[i] = h - R.v[i] * T;
        v[i] = cp - R.v[i];
    }
    double su = 0.0, sv = 0.0;
#pragma unroll
    for (int i = 0; i < NSP; ++i) su += massf.v[i] * e[i];
#pragma unroll
    for (int i = 0; i < NSP; ++i) sv += massf.v[i] * v[i];
    return EnergySlope{su, -1.0 * sv};
}

// The mixture's energy at T alone (TPGas::energy's loop over cea_h).
template <int NSP>
static __device__ E4C_CEA_FN double mix_energy(const e4c_thermochem& tc, SpVals<NSP> R,
                                               SpVals<NSP> massf, double T) {
    const double lT = pm_log(T);
    const TRecip t(T);
    double e[NSP];
#pragma unroll
    for (int i = 0; i < NSP; ++i) e[i] = cea_h(tc, i, R.v[i], t, lT) - R.v[i] * T;
    double su = 0.0;
#pragma unroll
    for (int i = 0; i < NSP; ++i) su += massf.v[i] * e[i];
    return su;
}

template <int NSP>
struct TPGas {
    const e4c_thermochem& tc;
    double R[NSP];
    __device__ explicit TPGas(const e4c_thermochem& t) : tc(t) {
#pragma unroll
        for (int i = 0; i < NSP; ++i) R[i] = 8.31451 / tc.M[i];
    }
    __device__ double mass_average(const double* massf, const double* phi) const {
        double result = 0.0;
#pragma unroll
        for (int i = 0; i < NSP; ++i) result += massf[i] * phi[i];
        return result;
    }
    __device__ double Rmix(const double* massf) const { return mass_average(massf, R); }
    __device__ SpVals<NSP> Rvals() const {
        SpVals<NSP> r;
#pragma unroll
        for (int i = 0; i < NSP; ++i) r.v[i] = R[i];
        return r;
    }
    __device__ static SpVals<NSP> vals(const double* x) {
        SpVals<NSP> r;
#pragma unroll
        for (int i = 0; i < NSP; ++i) r.v[i] = x[i];
        return r;
    }
    __device__ double energy(const double* massf, double T) const {
        return mix_energy<NSP>(tc, Rvals(), vals(massf), T);
    }
    // energy(massf, T) and dudT(massf, T) together
    __device__ void energy_dudT(const double* massf, double T, double& u, double& du) const {
        const EnergySlope r = mix_energy_slope<NSP>(tc, Rvals(), vals(massf), T);
        u = r.u;
        du = r.du;
    }
    __device__ double dudT(const double* massf, double T) const {
        double v[NSP];
#pragma unroll
        for (int i = 0; i < NSP; ++i) v[i] = cea_Cp(tc, i, R[i], T) - R[i];
        return -1.0 * mass_average(massf, v);
    }
    // nm/newton.d:40-99, f(T) = e_tgt - u(T); Q.T and Q.u follow every evaluation
    //
    // shortcut: the energies at the bracket ends serve only for their signs
    // (and zero tests).  With e = e_tgt - u(x0) and Cv = Cv(x0), the mixture's
    // u rises at no less than 2 kappa Cv per kelvin within the bracket, so
    // 0 <= e < kappa Cv (xMax - x0) gives e_tgt - u(xMin) > 0 > e_tgt - u(xMax)
    // (and likewise for e < 0), by margins of at least kappa Cv K that no
    // rounding reaches: those two evaluations are then skipped, with the same
    // outcome as when they are made.
    __device__ bool solve_T(TPState<NSP>& Q, double e_tgt, double x0, double xMin, double xMax,
                            double tol, double& root, bool shortcut = false) const {
        const int MAXIT = 30;
        double xL = xMin, xH = xMax;
        double fL = 0.0, fH = 0.0, u0 = 0.0, df0 = 0.0;
        bool have0 = false, signs = false;
        const double kappa = c_bracket_kappa;
        if (shortcut && kappa > 0.0 && x0 - xMin >= 1.0 && xMax - x0 >= 1.0 && xMax <= 101000.0) {
            energy_dudT(Q.massf, x0, u0, df0);
            have0 = true;
            const double e = e_tgt - u0, cv = -df0;
            if (cv > 0.0 && ((e >= 0.0 && e < kappa * cv * (xMax - x0)) ||
                             (e < 0.0 && -e < kappa * cv * (x0 - xMin)))) {
                fL = 1.0;
                fH = -1.0;
                signs = true;
            }
        }
        if (!signs) {
            Q.T = xL; Q.u = energy(Q.massf, Q.T);
            fL = e_tgt - Q.u;
            Q.T = xH; Q.u = energy(Q.massf, Q.T);
            fH = e_tgt - Q.u;
        }
        if ((fL > 0.0 && fH > 0.0) || (fL < 0.0 && fH < 0.0)) return false;
        if (fL == 0.0) { root = xMin; return true; }
        if (fH == 0.0) { root = xMax; return true; }
        if (fL < 0.0) { xL = xMin; xH = xMax; }
        else { xH = xMin; xL = xMax; }
        double rts = x0;
        double dxold = (xMax - xMin);
        double dx = dxold;
        if (!have0) energy_dudT(Q.massf, rts, u0, df0);
        Q.T = rts; Q.u = u0;
        double f0 = e_tgt - Q.u;
        for (int j = 0; j < MAXIT; ++j) {
            if ((((rts - xH) * df0 - f0) * ((rts - xL) * df0 - f0) > 0.0) ||
                (fabs(2.0 * f0) > fabs(dxold * df0))) {
                dxold = dx;
                dx = 0.5 * (xH - xL);
                rts = xL + dx;
                if (xL == rts) { root = rts; return true; }
            } else {
                dxold = dx;
                dx = f0 / df0;
                double tmp = rts;
                rts -= dx;
                if (tmp == rts) { root = rts; return true; }
            }
            if (fabs(dx) < tol) { root = rts; return true; }
            Q.T = rts; energy_dudT(Q.massf, Q.T, Q.u, df0);
            f0 = e_tgt - Q.u;
            if (f0 < 0.0) xL = rts;
            else xH = rts;
        }
        return false;
    }
    // ThermallyPerfectGasMixEOS.update_temperature (therm_perf_gas_mix_eos.d:70-150)
    __device__ bool update_temperature(TPState<NSP>& Q) const {
        double Tsave = Q.T;
        double e_tgt = Q.u;
        double T1 = fmax(Q.T - 0.5 * 1000.0, 20.0);
        double T2 = T1 + 1000.0;
        double root;
        if (solve_T(Q, e_tgt, Tsave, T1, T2, 1.0e-6, root, true)) { Q.T = root; return true; }
        if (solve_T(Q, e_tgt, Tsave, 20.0, 100000.0, 1.0e-6, root)) { Q.T = root; return true; }
        Q.T = Tsave;
        Q.u = energy(Q.massf, Q.T);
        return false;
    }
    __device__ bool rhou(TPState<NSP>& Q) const {
        if (!update_temperature(Q)) return false;
        Q.p = Q.rho * Rmix(Q.massf) * Q.T;
        return true;
    }
    __device__ void rhoT(TPState<NSP>& Q) const {
        Q.u = energy(Q.massf, Q.T);
        Q.p = Q.rho * Rmix(Q.massf) * Q.T;
    }
    __device__ double sound_speed(const double* massf, double T) const {
        double cp[NSP], cv[NSP];
#pragma unroll
        for (int i = 0; i < NSP; ++i) {
            double c = cea_Cp(tc, i, R[i], T);
            cp[i] = c;
            cv[i] = c - R[i];
        }
        double gamma = mass_average(massf, cp) / mass_average(massf, cv);
        double dpdrho = Rmix(massf) * T;
        return sqrt(gamma * dpdrho);
    }
};

// ---------------------------------------------------------------------------
// Reaction rates and the chemistry update
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ipow_d(double c, int n) {
    return (n == 1) ? c : ((n == 2) ? c * c : (n == 0 ? 1.0 : pm_pow(c, double(n))));
}

template <int NSP, int NR>
struct MechD {
    const e4c_thermochem& tc;
    double kf[NR], kb[NR];
    __device__ explicit MechD(const e4c_thermochem& t) : tc(t) {}
    __device__ void rate_constants(double T) {
        if (T < tc.T_lower) T = tc.T_lower;
        if (T > tc.T_upper) T = tc.T_upper;
        const double lT = pm_log(T);
        const double rT = 1.0 / T;
        for (int r = 0; r < NR; ++r) {
            kf[r] = tc.A_f[r] * pm_pow_l(T, lT, tc.n_f[r]) * pm_exp(div_rn(-tc.C_f[r], T, rT));
            kb[r] = tc.A_b[r] * pm_pow_l(T, lT, tc.n_b[r]) * pm_exp(div_rn(-tc.C_b[r], T, rT));
        }
    }
    __device__ void rates(int r, const double* c, double& wf, double& wb) const {
        if (tc.third_body[r]) {
            double M = 0.0;
            for (int i = 0; i < NSP; ++i) M += tc.eff[r][i] * c[i];
            wf = kf[r] * M;
            wb = kb[r] * M;
        } else {
            wf = kf[r];
            wb = kb[r];
        }
        for (int i = 0; i < NSP; ++i)
            if (tc.nu_r[r][i] > 0) wf *= ipow_d(c[i], tc.nu_r[r][i]);
        for (int i = 0; i < NSP; ++i)
            if (tc.nu_p[r][i] > 0) wb *= ipow_d(c[i], tc.nu_p[r][i]);
    }
    __device__ void split_rates(const double* c, double* q, double* L) const {
        for (int i = 0; i < NSP; ++i) { q[i] = 0.0; L[i] = 0.0; }
        for (int r = 0; r < NR; ++r) {
            double wf, wb;
            rates(r, c, wf, wb);
            for (int i = 0; i < NSP; ++i) {
                if (tc.nu_r[r][i] == 0 && tc.nu_p[r][i] == 0) continue;
                const double nu = double(tc.nu_p[r][i] - tc.nu_r[r][i]);
                double prod = 0.0, loss = 0.0;
                if (nu > 0.0) { prod = nu * wf; loss = nu * wb; }
                else if (nu < 0.0) { prod = -nu * wb; loss = -nu * wf; }
                q[i] += prod;
                L[i] += loss;
            }
        }
    }
    __device__ void jacobian(const double* c, double J[NSP][NSP]) const {
        for (int i = 0; i < NSP; ++i)
            for (int j = 0; j < NSP; ++j) J[i][j] = 0.0;
        for (int r = 0; r < NR; ++r) {
            double Pf = 1.0, Pb = 1.0;
            for (int i = 0; i < NSP; ++i) {
                if (tc.nu_r[r][i] > 0) Pf *= ipow_d(c[i], tc.nu_r[r][i]);
                if (tc.nu_p[r][i] > 0) Pb *= ipow_d(c[i], tc.nu_p[r][i]);
            }
            double M = 1.0;
            if (tc.third_body[r]) {
                M = 0.0;
                for (int i = 0; i < NSP; ++i) M += tc.eff[r][i] * c[i];
            }
            for (int j = 0; j < NSP; ++j) {
                double dPf = 0.0, dPb = 0.0;
                const int aj = tc.nu_r[r][j], bj = tc.nu_p[r][j];
                if (aj > 0) {
                    dPf = double(aj) * ipow_d(c[j], aj - 1);
                    for (int i = 0; i < NSP; ++i)
                        if (i != j && tc.nu_r[r][i] > 0) dPf *= ipow_d(c[i], tc.nu_r[r][i]);
                }
                if (bj > 0) {
                    dPb = double(bj) * ipow_d(c[j], bj - 1);
                    for (int i = 0; i < NSP; ++i)
                        if (i != j && tc.nu_p[r][i] > 0) dPb *= ipow_d(c[i], tc.nu_p[r][i]);
                }
                double ef = tc.third_body[r] ? tc.eff[r][j] : 0.0;
                double dwf = kf[r] * (M * dPf + ef * Pf);
                double dwb = kb[r] * (M * dPb + ef * Pb);
                for (int i = 0; i < NSP; ++i) {
                    const double nu = double(tc.nu_p[r][i] - tc.nu_r[r][i]);
                    if (nu != 0.0) J[i][j] += nu * (dwf - dwb);
                }
            }
        }
    }
    __device__ double estimate_step_size(const double* c) const {
        double q[NSP], L[NSP];
        split_rates(c, q, L);
        double min_dt = 1.0e6;
        for (int i = 0; i < NSP; ++i) {
            if (c[i] > 0.0 && (fabs(q[i] - L[i]) > 1.0e-30)) {
                double dt;
                if (q[i] > 10000.0 * L[i]) dt = c[i] / (L[i] + 1.0e-50);
                else dt = fabs(c[i] / (q[i] - L[i]));
                min_dt = fmin(min_dt, dt);
            }
        }
        double dt_chem = 1.0e-3 * min_dt;
        dt_chem = fmin(dt_chem, 1.0e-10);
        dt_chem = fmax(dt_chem, 1.0e-15);
        return dt_chem;
    }
};

template <int N>
__device__ bool solve_dense_d(double A[N][N], double* b) {
    for (int col = 0; col < N; ++col) {
        int piv = col;
        double best = fabs(A[col][col]);
        for (int r = col + 1; r < N; ++r)
            if (fabs(A[r][col]) > best) { best = fabs(A[r][col]); piv = r; }
        if (!(best > 0.0)) return false;
        if (piv != col) {
            for (int j = 0; j < N; ++j) { double t = A[col][j]; A[col][j] = A[piv][j]; A[piv][j] = t; }
            double t = b[col]; b[col] = b[piv]; b[piv] = t;
        }
        for (int r = col + 1; r < N; ++r) {
            double f = A[r][col] / A[col][col];
            for (int j = col; j < N; ++j) A[r][j] = A[r][j] - f * A[col][j];
            b[r] = b[r] - f * b[col];
        }
    }
    for (int r = N - 1; r >= 0; --r) {
        double s = b[r];
        for (int j = r + 1; j < N; ++j) s = s - A[r][j] * b[j];
        b[r] = s / A[r][r];
    }
    return true;
}

// Backward-Euler step solved by Newton iteration from the guess x0 (the start
// state c0 on the plain path).  Converged when max|F_i| / sum(c0) <= 1e-8.
template <int NSP, int NR>
__device__ bool point_implicit_step(const MechD<NSP, NR>& m, const double* c0, const double* x0,
                                    double h, double* cOut, double& h_suggest, int& iters) {
    double cscale = 0.0;
    for (int i = 0; i < NSP; ++i) cscale += c0[i];
    if (!(cscale > 0.0)) return false;
    double x[NSP];
    for (int i = 0; i < NSP; ++i) x[i] = x0[i];
    bool converged = false;
    iters = 0;
    for (int it = 0; it < 10; ++it) {
        double q[NSP], L[NSP], F[NSP];
        m.split_rates(x, q, L);
        double res = 0.0;
        for (int i = 0; i < NSP; ++i) {
            F[i] = x[i] - c0[i] - h * (q[i] - L[i]);
            res = fmax(res, fabs(F[i]));
        }
        if (res / cscale <= 1.0e-8) { converged = true; break; }
        double J[NSP][NSP], A[NSP][NSP];
        m.jacobian(x, J);
        for (int i = 0; i < NSP; ++i)
            for (int j = 0; j < NSP; ++j) A[i][j] = ((i == j) ? 1.0 : 0.0) - h * J[i][j];
        double dx[NSP];
        for (int i = 0; i < NSP; ++i) dx[i] = -F[i];
        if (!solve_dense_d<NSP>(A, dx)) return false;
        for (int i = 0; i < NSP; ++i) {
            x[i] = x[i] + dx[i];
            if (x[i] < 0.0) x[i] = 0.0;
        }
        ++iters;
    }
    if (!converged) return false;
    double q0[NSP], L0[NSP];
    m.split_rates(c0, q0, L0);
    // the distance from the explicit Euler prediction, measured as RKFStep
    // measures its error (chemistry_update.d:418-427): atol = rtol = errTol,
    // root mean square over the species
    double err = 0.0;
    for (int i = 0; i < NSP; ++i) {
        double xe = c0[i] + h * (q0[i] - L0[i]);
        double sk = 1.0e-3 + 1.0e-3 * fmax(fabs(c0[i]), fabs(x[i]));
        double e = (x[i] - xe) / sk;
        err += e * e;
    }
    err = sqrt(err / NSP);
    double fac = (err > 0.0) ? 0.9 / sqrt(err) : 5.0;
    fac = fmin(5.0, fmax(0.2, fac));
    h_suggest = h * fac;
    for (int i = 0; i < NSP; ++i) cOut[i] = x[i];
    return err <= 1.0;
}

// RKFStep.opCall (chemistry_update.d:362-461): Runge-Kutta-Fehlberg with the
// Cash-Karp coefficients on dc/dt = q - L, the fourth/fifth-order difference
// as the error (atol = rtol = 1e-3, RMS over the species) and the step-size
// suggestion (safety 0.9, exponent 0.2, scale limits [0.2, 10]); the same
// operations as the oracle's rkf_step.  Returns true on a successful step.
template <int NSP, int NR>
__device__ bool rkf_step_d(const MechD<NSP, NR>& m, const double* y0, double h, double* yOut,
                           double& hSuggest) {
    const double a21 = 1. / 5., a31 = 3. / 40., a32 = 9. / 40., a41 = 3. / 10., a42 = -9. / 10.,
                 a43 = 6. / 5., a51 = -11. / 54., a52 = 5. / 2., a53 = -70. / 27.,
                 a54 = 35. / 27., a61 = 1631. / 55296., a62 = 175. / 512., a63 = 575. / 13824.,
                 a64 = 44275. / 110592., a65 = 253. / 4096.;
    const double b51 = 37. / 378., b53 = 250. / 621., b54 = 125. / 594., b56 = 512. / 1771.,
                 b41 = 2825. / 27648., b43 = 18575. / 48384., b44 = 13525. / 55296.,
                 b45 = 277. / 14336., b46 = 1.0 / 4.0;
    const double tol = 1.0e-3;   // odeStep.errTol default, prep_chem.lua:51
    double k1[NSP], k2[NSP], k3[NSP], k4[NSP], k5[NSP], k6[NSP], yt[NSP], q[NSP], L[NSP];
    m.split_rates(y0, q, L);
    for (int i = 0; i < NSP; ++i) k1[i] = q[i] - L[i];
    for (int i = 0; i < NSP; ++i) yt[i] = y0[i] + h * (a21 * k1[i]);
    m.split_rates(yt, q, L);
    for (int i = 0; i < NSP; ++i) k2[i] = q[i] - L[i];
    for (int i = 0; i < NSP; ++i) yt[i] = y0[i] + h * (a31 * k1[i] + a32 * k2[i]);
    m.split_rates(yt, q, L);
    for (int i = 0; i < NSP; ++i) k3[i] = q[i] - L[i];
    for (int i = 0; i < NSP; ++i) yt[i] = y0[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
    m.split_rates(yt, q, L);
    for (int i = 0; i < NSP; ++i) k4[i] = q[i] - L[i];
    for (int i = 0; i < NSP; ++i)
        yt[i] = y0[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
    m.split_rates(yt, q, L);
    for (int i = 0; i < NSP; ++i) k5[i] = q[i] - L[i];
    for (int i = 0; i < NSP; ++i)
        yt[i] = y0[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
    m.split_rates(yt, q, L);
    for (int i = 0; i < NSP; ++i) k6[i] = q[i] - L[i];
    double err = 0.0;
    for (int i = 0; i < NSP; ++i) {
        yOut[i] = y0[i] + h * (b51 * k1[i] + b53 * k3[i] + b54 * k4[i] + b56 * k6[i]);
        const double yErr =
            yOut[i] - (y0[i] + h * (b41 * k1[i] + b43 * k3[i] + b44 * k4[i] + b45 * k5[i] +
                                    b46 * k6[i]));
        const double fa = fabs(y0[i]), fb = fabs(yOut[i]);
        const double sk = tol + tol * ((fa < fb) ? fb : fa);
        err += (yErr / sk) * (yErr / sk);
    }
    err = sqrt(err / NSP);
    const double maxscale = 10.0, minscale = 0.2, safe = 0.9, alpha = 0.2;
    double scale;
    if (err <= 1.0) {
        if (err == 0.0) {
            scale = maxscale;
        } else {
            scale = safe * pm_pow(err, -alpha);
            if (scale < minscale) scale = minscale;
            if (scale > maxscale) scale = maxscale;
        }
        hSuggest = scale * h;
        return true;
    }
    const double sc = safe * pm_pow(err, -alpha);
    scale = (sc < minscale) ? minscale : sc;
    hSuggest = scale * h;
    return false;
}

// Chemistry method (e4c_config.chem_method): 0 the point-implicit step over
// the whole interval with opCall's sub-cycled recovery; 1 the reference's
// odeStep.method 'rkf' (opCall's sub-cycling with RKF steps from the start).
static __constant__ int c_chem_method = 0;

// Outcomes of point_implicit_whole.
constexpr int PI_FAILED = 0;      // no convergence: the sub-cycled recovery takes over
constexpr int PI_CONVERGED = 1;
constexpr int PI_MORE = 2;        // probe: the start state is not converged
// thermochemical_increment_d in probe mode: the cell needs Newton work
constexpr int CHEM_NEEDS_WORK = 1;

// One backward-Euler step over the whole interval h by Newton iteration
// (at most 12 iterations, the convergence test of point_implicit_step, no
// error control): the point-implicit update proper.  In probe mode it
// returns PI_MORE, before anything else, unless the start state c0 already
// satisfies the convergence test.  The iteration starts
// from c0; with a guess (a prediction of the end concentrations; ignored
// unless every entry is finite and non-negative) it starts from whichever of
// c0 and the guess has the smaller residual.  Without a guess the operations are exactly the
// CPU oracle's.
// Newton iterations of the whole-interval step (e4c_config.chem_newton_iterations)
static __constant__ int c_chem_newton_iterations = 12;

template <int NSP, int NR>
__device__ int point_implicit_whole(const MechD<NSP, NR>& m, const double* c0,
                                    const double* guess, double h, double* cOut, int& iters,
                                    bool probe) {
    double cscale = 0.0;
    for (int i = 0; i < NSP; ++i) cscale += c0[i];
    iters = 0;
    if (!(cscale > 0.0)) return probe ? PI_MORE : PI_FAILED;
    double x[NSP];
    for (int i = 0; i < NSP; ++i) x[i] = c0[i];
    const int maxit = c_chem_newton_iterations;
    for (int it = 0; it <= maxit; ++it) {
        double q[NSP], L[NSP], F[NSP];
        m.split_rates(x, q, L);
        double res = 0.0;
        for (int i = 0; i < NSP; ++i) {
            F[i] = x[i] - c0[i] - h * (q[i] - L[i]);
            res = fmax(res, fabs(F[i]));
        }
        if (it == 0 && probe && !(res / cscale <= 1.0e-8)) return PI_MORE;
        bool use_guess = (it == 0 && guess != nullptr);
        if (use_guess)
            for (int i = 0; i < NSP; ++i)
                if (!(guess[i] >= 0.0) || isinf(guess[i])) use_guess = false;
        if (use_guess) {
            double xg[NSP], Fg[NSP];
            for (int i = 0; i < NSP; ++i) xg[i] = guess[i];
            m.split_rates(xg, q, L);
            double resg = 0.0;
            for (int i = 0; i < NSP; ++i) {
                Fg[i] = xg[i] - c0[i] - h * (q[i] - L[i]);
                resg = fmax(resg, fabs(Fg[i]));
            }
            if (resg < res) {
                res = resg;
                for (int i = 0; i < NSP; ++i) { x[i] = xg[i]; F[i] = Fg[i]; }
            }
        }
        if (res / cscale <= 1.0e-8) {
            for (int i = 0; i < NSP; ++i) cOut[i] = x[i];
            return PI_CONVERGED;
        }
        if (it == maxit) break;
        double J[NSP][NSP], A[NSP][NSP];
        m.jacobian(x, J);
        for (int i = 0; i < NSP; ++i)
            for (int j = 0; j < NSP; ++j) A[i][j] = ((i == j) ? 1.0 : 0.0) - h * J[i][j];
        double dx[NSP];
        for (int i = 0; i < NSP; ++i) dx[i] = -F[i];
        if (!solve_dense_d<NSP>(A, dx)) return PI_FAILED;
        for (int i = 0; i < NSP; ++i) {
            x[i] = x[i] + dx[i];
            if (x[i] < 0.0) x[i] = 0.0;
        }
        ++iters;
    }
    return PI_FAILED;
}

// Per-cell chemistry counters: Newton iterations of the whole-interval step
// and of the recovery sub-steps, and whether the recovery ran.
struct ChemCount {
    int newton = 0;
    int recovered = 0;
};

// The chemistry update of one cell over tInterval at the cell's temperature:
// the point-implicit step over the whole interval; when its Newton iteration
// does not converge, ChemistryUpdate.opCall's sub-cycling
// (chemistry_update.d:119-307) with error-controlled point-implicit sub-steps
// and the dt_chem warm start.  guess (optional): predicted end
// concentrations for the whole-interval step.  Returns 0, or E4C_ERR_CHEM
// with Q restored.
template <int NSP, int NR>
__device__ int chemistry_update_d(const e4c_thermochem& tc, TPState<NSP>& Q, double tInterval,
                                  double& dtChemSuggest, const double* guess, ChemCount* cnt,
                                  bool probe = false) {
    TPState<NSP> Qinit = Q;
    double conc0[NSP], concOut[NSP];
    if (isnan(Q.rho) || Q.rho <= 0.0) return E4C_ERR_CHEM;
    for (int i = 0; i < NSP; ++i) {
        conc0[i] = Q.massf[i] * Q.rho / tc.M[i];
        if (conc0[i] < 1.0e-30) conc0[i] = 0.0;
        concOut[i] = conc0[i];
    }
    const int method = c_chem_method;
    if (method == 1 && probe) return CHEM_NEEDS_WORK;   // every cell sub-cycles
    MechD<NSP, NR> m(tc);
    m.rate_constants(Q.T);
    if (method == 0) {
        int iters = 0;
        const int st =
            point_implicit_whole<NSP, NR>(m, conc0, guess, tInterval, concOut, iters, probe);
        if (st == PI_MORE) return CHEM_NEEDS_WORK;   // Q untouched
        if (cnt) cnt->newton += iters;
        if (st == PI_CONVERGED) {
            double total = 0.0;
            for (int i = 0; i < NSP; ++i) {
                Q.massf[i] = concOut[i] * tc.M[i] / Q.rho;
                if (Q.massf[i] < 1.0e-30) Q.massf[i] = 0.0;
                total += Q.massf[i];
            }
            if (fabs(total - 1.0) <= 1.0e-3) {
                for (int i = 0; i < NSP; ++i) Q.massf[i] /= total;
                return 0;
            }
            for (int i = 0; i < NSP; ++i) Q.massf[i] = Qinit.massf[i];
            for (int i = 0; i < NSP; ++i) concOut[i] = conc0[i];
        }
    }
    if (cnt) cnt->recovered = 1;
    double t = 0.0, h, dtSave = dtChemSuggest;
    if (dtChemSuggest > tInterval) h = tInterval;
    else if (dtChemSuggest <= 0.0) h = m.estimate_step_size(conc0);
    else h = dtChemSuggest;
    int cycle = 0;
    for (; cycle < 10000; ++cycle) {
        dtSave = dtChemSuggest;
        h = fmin(h, tInterval - t);
        int attempt = 0;
        for (; attempt < 4; ++attempt) {
            int iters = 0;
            const bool ok =
                (method == 1)
                    ? rkf_step_d<NSP, NR>(m, conc0, h, concOut, dtChemSuggest)
                    : point_implicit_step<NSP, NR>(m, conc0, conc0, h, concOut, dtChemSuggest,
                                                   iters);
            if (cnt) cnt->newton += iters;
            bool massf_ok = true;
            if (ok) {
                double total = 0.0;
                for (int i = 0; i < NSP; ++i) {
                    Q.massf[i] = concOut[i] * tc.M[i] / Q.rho;
                    if (Q.massf[i] < 1.0e-30) Q.massf[i] = 0.0;
                    total += Q.massf[i];
                }
                if (fabs(total - 1.0) > 1.0e-3) massf_ok = false;
            }
            if (ok && massf_ok) {
                t += h;
                for (int i = 0; i < NSP; ++i) conc0[i] = concOut[i];
                double hMax = h * (1.0 + 10.0 / 100.0);
                if (dtChemSuggest > h) h = fmin(dtChemSuggest, hMax);
                break;
            } else {
                h /= 10.0;
                if (h < 1.0e-15) { Q = Qinit; return E4C_ERR_CHEM; }
            }
        }
        if (attempt == 4) { Q = Qinit; return E4C_ERR_CHEM; }
        if (t >= tInterval) {
            if (cycle == 0) dtSave = dtChemSuggest;
            break;
        }
    }
    if (cycle == 10000) { Q = Qinit; return E4C_ERR_CHEM; }
    double total = 0.0;
    for (int i = 0; i < NSP; ++i) {
        Q.massf[i] = concOut[i] * tc.M[i] / Q.rho;
        if (Q.massf[i] < 1.0e-30) Q.massf[i] = 0.0;
        total += Q.massf[i];
    }
    for (int i = 0; i < NSP; ++i) Q.massf[i] /= total;
    dtChemSuggest = dtSave;
    return 0;
}

// FVCell.thermochemical_increment (fvcell.d:1510-1621): chemistry at constant
// rho and u, then T, p, a from the new composition.  probe: return
// CHEM_NEEDS_WORK, with Q untouched, for a cell whose start state does not
// already satisfy the point-implicit convergence test; every other cell is
// updated exactly as without probe.  guess (optional): six
// values, the predicted end concentrations and end temperature; the
// temperature only starts the rhou Newton iteration (when it lies within
// 500 K of the cell's temperature), so it changes T by no more than that
// iteration's tolerance.
template <int NSP, int NR>
__device__ int thermochemical_increment_d(const e4c_thermochem& tc, double T_frozen,
                                          TPState<NSP>& Q, double dt, double& dt_chem,
                                          const double* guess, ChemCount* cnt,
                                          bool probe = false) {
    if (Q.T <= T_frozen) return 0;
    const double T0 = Q.T;
    int rc = chemistry_update_d<NSP, NR>(tc, Q, dt, dt_chem, guess, cnt, probe);
    if (rc == CHEM_NEEDS_WORK) return rc;
    if (rc != 0) {
        dt_chem = -1.0;
        rc = chemistry_update_d<NSP, NR>(tc, Q, dt, dt_chem, nullptr, cnt);
        if (rc != 0) return rc;
    }
    TPGas<NSP> g(tc);
    if (guess != nullptr) {
        const double Tg = guess[NSP];
        if (Tg > 20.0 && Tg < 1.0e5 && fabs(Tg - T0) < 500.0) {
            const double u0 = Q.u;
            Q.T = Tg;
            if (g.rhou(Q)) {
                Q.a = g.sound_speed(Q.massf, Q.T);
                return 0;
            }
            Q.T = T0;
            Q.u = u0;
        }
    }
    if (!g.rhou(Q)) return E4C_ERR_THERMO;
    Q.a = g.sound_speed(Q.massf, Q.T);
    return 0;
}

}  // namespace e4c
