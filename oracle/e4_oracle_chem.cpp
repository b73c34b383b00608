/*
 * e4_oracle_chem.cpp -- thermally perfect gas and finite-rate chemistry of the
 * CPU FP64 oracle.  TEST INFRASTRUCTURE ONLY (see e4_oracle.cpp).
 *
 * Restates (paths inside the reference project):
 *   CEA thermo curves      src/gas/thermo/cea_thermo_curves.d:49-167
 *   mixture EOS            src/gas/therm_perf_gas.d:182-191, 345-396,
 *                          src/gas/thermo/therm_perf_gas_mix_eos.d:63-150,
 *                          src/gas/thermo/perf_gas_mix_eos.d:43-62,
 *                          src/gas/gas_model.d:45-46, 196-230, 330-338
 *   T Newton               src/nm/newton.d:40-99 (rtsafe with bisection)
 *   rates                  src/kinetics/rate_constant.d:71-75,
 *                          src/kinetics/reaction.d:79-114, 275-400,
 *                          src/kinetics/reaction_mechanism.d:47-82, 127-170
 *   sub-cycling            src/kinetics/chemistry_update.d:119-307
 *   cell increment         src/eilmer/fvcell.d:1510-1621
 *
 * The reference has no point-implicit ODE step; the step used here
 * (backward Euler solved by Newton iteration with the analytic 5x5
 * Jacobian) is this project's own and is the same in the CUDA library.
 *
 * exp and log are the project's portable versions (Cody-Waite argument
 * reduction with a Taylor polynomial for exp; an atanh series for log),
 * written with + - * / only and built without contraction, so the oracle
 * and the CUDA library produce identical bits.  They differ from the C
 * library's exp/log by at most a few ulp.
 */
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "e4_oracle_internal.h"

namespace e4o {

// ---------------------------------------------------------------------------
// Portable exp / log / pow
// ---------------------------------------------------------------------------
#ifdef E4O_LIBM
// The second build of the oracle (libe4oracle_libm.so): the C library's exp,
// log and pow in place of the portable restatements below, as the reference
// calls them (rate_constant.d:71-75, cea_thermo_curves.d:49-127).  It bounds
// how far the GPU's reacting path, which uses the portable forms, sits from
// the reference's arithmetic.
double pm_log(double x) { return std::log(x); }
double pm_exp(double x) { return std::exp(x); }
double pm_pow(double x, double n) { return std::pow(x, n); }
#else
double pm_log(double x) {
    // log(x) = k ln2 + 2 atanh(s), s = (m-1)/(m+1), x = m 2^k, m in [sqrt(1/2), sqrt(2))
    if (!(x > 0.0)) return (x == 0.0) ? -HUGE_VAL : NAN;
    if (std::isinf(x)) return x;
    int k;
    double m = std::frexp(x, &k);
    if (m < 0.70710678118654752440) { m = m * 2.0; k = k - 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    // 1 + s^2/3 + s^4/5 + ... + s^22/23
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
    const double ln2_hi = 6.93147180369123816490e-01;  // high bits of ln 2
    const double ln2_lo = 1.90821492927058770002e-10;  // ln 2 - ln2_hi
    double kd = double(k);
    return kd * ln2_hi + (2.0 * s * p + kd * ln2_lo);
}

double pm_exp(double x) {
    if (x != x) return x;
    if (x > 709.78) return HUGE_VAL;
    if (x < -745.2) return 0.0;
    const double inv_ln2 = 1.44269504088896338700e+00;
    const double ln2_hi = 6.93147180369123816490e-01;
    const double ln2_lo = 1.90821492927058770002e-10;
    double kd = std::floor(x * inv_ln2 + 0.5);
    double r = (x - kd * ln2_hi) - kd * ln2_lo;
    // Taylor polynomial of exp(r), |r| <= 0.35, degree 13
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
    return std::ldexp(p, int(kd));
}

double pm_pow(double x, double n) {
    // x^n for the exponents of the rate constants
    if (n == 0.0) return 1.0;
    if (n == 1.0) return x;
    if (n == -1.0) return 1.0 / x;
    if (n == 2.0) return x * x;
    if (n == 0.5) return std::sqrt(x);
    if (n == -0.5) return 1.0 / std::sqrt(x);
    if (n == 1.5) return x * std::sqrt(x);
    if (n == -1.5) return 1.0 / (x * std::sqrt(x));
    return pm_exp(n * pm_log(x));
}
#endif  // E4O_LIBM

// ---------------------------------------------------------------------------
// CEA thermo curves (cea_thermo_curves.d)
// ---------------------------------------------------------------------------
static void determine_coefficients(const e4o_thermochem& tc, int isp, double T, double a[9]) {
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
    for (int j = 0; j < 9; ++j) a[j] = NAN;
}

static double eval_Cp(const e4o_thermochem& tc, int isp, double R, double T) {
    const int nseg = tc.nseg[isp];
    if (T < tc.T_break[isp][0]) T = tc.T_break[isp][0];
    if (T > tc.T_break[isp][nseg]) T = tc.T_break[isp][nseg];
    double a[9];
    determine_coefficients(tc, isp, T, a);
    double Cp_on_R = a[0] / (T * T) + a[1] / T + a[2] + a[3] * T;
    Cp_on_R += a[4] * T * T + a[5] * T * T * T + a[6] * T * T * T * T;
    return R * Cp_on_R;
}

static double eval_h(const e4o_thermochem& tc, int isp, double R, double T) {
    const int nseg = tc.nseg[isp];
    if (T < tc.T_break[isp][0]) {
        double T_low = tc.T_break[isp][0];
        double h_low = eval_h(tc, isp, R, T_low);
        double Cp_low = eval_Cp(tc, isp, R, T_low);
        return h_low - Cp_low * (T_low - T);
    }
    if (T > tc.T_break[isp][nseg]) {
        double T_high = tc.T_break[isp][nseg];
        double h_high = eval_h(tc, isp, R, T_high);
        double Cp_high = eval_Cp(tc, isp, R, T_high);
        return h_high + Cp_high * (T - T_high);
    }
    double a[9];
    determine_coefficients(tc, isp, T, a);
    double h_on_RT = -a[0] / (T * T) + a[1] / T * pm_log(T) + a[2] + a[3] * T / 2.0;
    h_on_RT += a[4] * T * T / 3.0 + a[5] * T * T * T / 4.0 + a[6] * T * T * T * T / 5.0 + a[7] / T;
    return R * T * h_on_RT;
}

// ---------------------------------------------------------------------------
// Thermally perfect mixture (therm_perf_gas.d and the mixture EOS files)
// ---------------------------------------------------------------------------
// nm/newton.d:40-99 (rtsafe after Numerical Recipes): Newton's method
// safeguarded by bisection within a bracket; returns false where the reference
// throws (no bracket, no convergence in 30 iterations).
template <class F, class DF>
static bool rtsafe(F&& f, DF&& dfdx, double x0, double xMin, double xMax, double tol,
                   double& root) {
    const int MAXIT = 30;
    double xL = xMin, xH = xMax;
    double fL = f(xL);
    double fH = f(xH);
    if ((fL > 0.0 && fH > 0.0) || (fL < 0.0 && fH < 0.0)) return false;
    if (fL == 0.0) { root = xMin; return true; }
    if (fH == 0.0) { root = xMax; return true; }
    if (fL < 0.0) { xL = xMin; xH = xMax; }
    else { xH = xMin; xL = xMax; }
    double rts = x0;
    double dxold = (xMax - xMin);
    double dx = dxold;
    double f0 = f(rts);
    double df0 = dfdx(rts);
    for (int j = 0; j < MAXIT; ++j) {
        if ((((rts - xH) * df0 - f0) * ((rts - xL) * df0 - f0) > 0.0) ||
            (std::fabs(2.0 * f0) > std::fabs(dxold * df0))) {
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
        if (std::fabs(dx) < tol) { root = rts; return true; }
        f0 = f(rts);
        df0 = dfdx(rts);
        if (f0 < 0.0) xL = rts;
        else xH = rts;
    }
    return false;
}

struct TP {
    const e4o_thermochem& tc;
    double R[E4O_MAXSP];
    explicit TP(const e4o_thermochem& t) : tc(t) {
        for (int i = 0; i < tc.nsp; ++i) R[i] = R_universal / tc.M[i];
    }
    double mass_average(const GasState& Q, const double* phi) const {
        double result = 0.0;  // gas_model.d:330-338
        for (int i = 0; i < tc.nsp; ++i) result += Q.massf[i] * phi[i];
        return result;
    }
    double Rmix(const GasState& Q) const { return mass_average(Q, R); }
    void update_energy(GasState& Q) const {
        double e[E4O_MAXSP];
        for (int i = 0; i < tc.nsp; ++i) e[i] = eval_h(tc, i, R[i], Q.T) - R[i] * Q.T;
        Q.u = mass_average(Q, e);
    }
    double Cv(const GasState& Q) const {
        double v[E4O_MAXSP];
        for (int i = 0; i < tc.nsp; ++i) v[i] = eval_Cp(tc, i, R[i], Q.T) - R[i];
        return mass_average(Q, v);
    }
    double Cp(const GasState& Q) const {
        double v[E4O_MAXSP];
        for (int i = 0; i < tc.nsp; ++i) v[i] = eval_Cp(tc, i, R[i], Q.T);
        return mass_average(Q, v);
    }
    // nm/newton.d:40-99 with f = e_tgt - u(T) (Q.T, Q.u are set on each call)
    bool solve_T(GasState& Q, double e_tgt, double x0, double xMin, double xMax, double tol,
                 double& root) const {
        auto f = [&](double T) {
            Q.T = T;
            update_energy(Q);
            return e_tgt - Q.u;
        };
        auto dfdx = [&](double T) {
            double v[E4O_MAXSP];
            for (int i = 0; i < tc.nsp; ++i) v[i] = eval_Cp(tc, i, R[i], T) - R[i];
            return -1.0 * mass_average(Q, v);
        };
        return rtsafe(f, dfdx, x0, xMin, xMax, tol, root);
    }
    // ThermallyPerfectGasMixEOS.update_temperature (therm_perf_gas_mix_eos.d:70-150)
    bool update_temperature(GasState& Q) const {
        double Tsave = Q.T;
        const double TOL = 1.0e-6;
        double e_tgt = Q.u;
        double delT = 1000.0;
        double T1 = std::fmax(Q.T - 0.5 * delT, 20.0);
        double T2 = T1 + delT;
        double root;
        if (solve_T(Q, e_tgt, Tsave, T1, T2, TOL, root)) { Q.T = root; return true; }
        if (solve_T(Q, e_tgt, Tsave, 20.0, 100000.0, TOL, root)) { Q.T = root; return true; }
        Q.T = Tsave;
        update_energy(Q);
        return false;
    }
    bool update_thermo_from_pT(GasState& Q) const {
        double denom = Rmix(Q) * Q.T;  // perf_gas_mix_eos.d:55-62
        Q.rho = Q.p / denom;
        update_energy(Q);
        return true;
    }
    bool update_thermo_from_rhou(GasState& Q) const {
        if (!update_temperature(Q)) return false;
        Q.p = Q.rho * Rmix(Q) * Q.T;  // perf_gas_mix_eos.d:43-49
        return true;
    }
    bool update_thermo_from_rhoT(GasState& Q) const {
        update_energy(Q);
        Q.p = Q.rho * Rmix(Q) * Q.T;
        return true;
    }
    bool update_sound_speed(GasState& Q) const {
        // frozen sound speed, therm_perf_gas.d:345-355: sqrt(gamma * R T)
        double gamma = Cp(Q) / Cv(Q);
        double dpdrho = Rmix(Q) * Q.T;
        Q.a = std::sqrt(gamma * dpdrho);
        return true;
    }
};

void GasModel::init_therm_perf_air5() { kind = E4O_GAS_THERM_PERF_5SP_AIR; nsp = 5; }

bool GasModel::tp_update_thermo_from_pT(GasState& Q) const { return TP(tc).update_thermo_from_pT(Q); }
bool GasModel::tp_update_thermo_from_rhou(GasState& Q) const { return TP(tc).update_thermo_from_rhou(Q); }
bool GasModel::tp_update_thermo_from_rhoT(GasState& Q) const { return TP(tc).update_thermo_from_rhoT(Q); }
bool GasModel::tp_update_sound_speed(GasState& Q) const { return TP(tc).update_sound_speed(Q); }

// ---------------------------------------------------------------------------
// Reaction rates (rate_constant.d, reaction.d, reaction_mechanism.d)
// ---------------------------------------------------------------------------
static inline double ipow(double c, int n) {
    return (n == 1) ? c : ((n == 2) ? c * c : (n == 0 ? 1.0 : pm_pow(c, double(n))));
}

struct Mech {
    const e4o_thermochem& tc;
    double kf[E4O_MAXR], kb[E4O_MAXR];
    explicit Mech(const e4o_thermochem& t) : tc(t) {}
    void eval_rate_constants(double T) {
        // reaction_mechanism.d:47-57 limits, rate_constant.d:71-75 Arrhenius
        if (T < tc.T_lower) T = tc.T_lower;
        if (T > tc.T_upper) T = tc.T_upper;
        for (int r = 0; r < tc.nreac; ++r) {
            kf[r] = tc.A_f[r] * pm_pow(T, tc.n_f[r]) * pm_exp(-tc.C_f[r] / T);
            kb[r] = tc.A_b[r] * pm_pow(T, tc.n_b[r]) * pm_exp(-tc.C_b[r] / T);
        }
    }
    // forward and backward rates of reaction r (reaction.d:355-400)
    void rates(int r, const double* c, double& wf, double& wb, double& Mterm) const {
        Mterm = 1.0;
        if (tc.third_body[r]) {
            Mterm = 0.0;
            for (int i = 0; i < tc.nsp; ++i) Mterm += tc.eff[r][i] * c[i];
            wf = kf[r] * Mterm;
            wb = kb[r] * Mterm;
        } else {
            wf = kf[r];
            wb = kb[r];
        }
        for (int i = 0; i < tc.nsp; ++i)
            if (tc.nu_r[r][i] > 0) wf *= ipow(c[i], tc.nu_r[r][i]);
        for (int i = 0; i < tc.nsp; ++i)
            if (tc.nu_p[r][i] > 0) wb *= ipow(c[i], tc.nu_p[r][i]);
    }
    // eval_split_rates (reaction_mechanism.d:68-82)
    void split_rates(const double* c, double* q, double* L) const {
        for (int i = 0; i < tc.nsp; ++i) { q[i] = 0.0; L[i] = 0.0; }
        for (int r = 0; r < tc.nreac; ++r) {
            double wf, wb, M;
            rates(r, c, wf, wb, M);
            for (int i = 0; i < tc.nsp; ++i) {
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
    // d(q - L)_i / dc_j, the analytic Jacobian of the net production:
    // for w = k M prod_i c_i^a_i, dw/dc_j = k (M d(prod)/dc_j + eff_j prod)
    void jacobian(const double* c, double J[E4O_MAXSP][E4O_MAXSP]) const {
        const int n = tc.nsp;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) J[i][j] = 0.0;
        for (int r = 0; r < tc.nreac; ++r) {
            double Pf = 1.0, Pb = 1.0;
            for (int i = 0; i < n; ++i) {
                if (tc.nu_r[r][i] > 0) Pf *= ipow(c[i], tc.nu_r[r][i]);
                if (tc.nu_p[r][i] > 0) Pb *= ipow(c[i], tc.nu_p[r][i]);
            }
            double M = 1.0;
            if (tc.third_body[r]) {
                M = 0.0;
                for (int i = 0; i < n; ++i) M += tc.eff[r][i] * c[i];
            }
            for (int j = 0; j < n; ++j) {
                double dPf = 0.0, dPb = 0.0;
                const int aj = tc.nu_r[r][j], bj = tc.nu_p[r][j];
                if (aj > 0) {
                    dPf = double(aj) * ipow(c[j], aj - 1);
                    for (int i = 0; i < n; ++i)
                        if (i != j && tc.nu_r[r][i] > 0) dPf *= ipow(c[i], tc.nu_r[r][i]);
                }
                if (bj > 0) {
                    dPb = double(bj) * ipow(c[j], bj - 1);
                    for (int i = 0; i < n; ++i)
                        if (i != j && tc.nu_p[r][i] > 0) dPb *= ipow(c[i], tc.nu_p[r][i]);
                }
                double ef = tc.third_body[r] ? tc.eff[r][j] : 0.0;
                double dwf = kf[r] * (M * dPf + ef * Pf);
                double dwb = kb[r] * (M * dPb + ef * Pb);
                for (int i = 0; i < n; ++i) {
                    const double nu = double(tc.nu_p[r][i] - tc.nu_r[r][i]);
                    if (nu != 0.0) J[i][j] += nu * (dwf - dwb);
                }
            }
        }
    }
    // estimateStepSize (reaction_mechanism.d:127-170)
    double estimate_step_size(const double* c) const {
        const double MUCH_LARGER_FACTOR = 10000.0, ZERO_EPS = 1.0e-50, ZERO_TOL = 1.0e-30;
        const double EPS1 = 1.0e-3;
        double q[E4O_MAXSP], L[E4O_MAXSP];
        split_rates(c, q, L);
        double min_dt = 1.0e6;
        for (int i = 0; i < tc.nsp; ++i) {
            if (c[i] > 0.0 && (std::fabs(q[i] - L[i]) > ZERO_TOL)) {
                double dt;
                if (q[i] > MUCH_LARGER_FACTOR * L[i]) dt = c[i] / (L[i] + ZERO_EPS);
                else dt = std::fabs(c[i] / (q[i] - L[i]));
                min_dt = std::min(min_dt, dt);
            }
        }
        double dt_chem = EPS1 * min_dt;
        dt_chem = std::min(dt_chem, 1.0e-10);
        dt_chem = std::max(dt_chem, 1.0e-15);
        return dt_chem;
    }
};

// Solve A x = b (n x n) by Gaussian elimination with partial pivoting.
static bool solve_dense(int n, double A[E4O_MAXSP][E4O_MAXSP], double* b) {
    for (int col = 0; col < n; ++col) {
        int piv = col;
        double best = std::fabs(A[col][col]);
        for (int r = col + 1; r < n; ++r)
            if (std::fabs(A[r][col]) > best) { best = std::fabs(A[r][col]); piv = r; }
        if (!(best > 0.0)) return false;
        if (piv != col) {
            for (int j = 0; j < n; ++j) std::swap(A[col][j], A[piv][j]);
            std::swap(b[col], b[piv]);
        }
        for (int r = col + 1; r < n; ++r) {
            double f = A[r][col] / A[col][col];
            for (int j = col; j < n; ++j) A[r][j] = A[r][j] - f * A[col][j];
            b[r] = b[r] - f * b[col];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int j = r + 1; j < n; ++j) s = s - A[r][j] * b[j];
        b[r] = s / A[r][r];
    }
    return true;
}

// The point-implicit step: backward Euler, x = c0 + h w(x), solved by Newton
// iteration with the analytic Jacobian from the start guess x = c0.
// Returns true on convergence; cOut holds x and h_suggest the next step.
static const double PI_NEWTON_TOL = 1.0e-8;   // max |F_i| / sum(c0)
static const int PI_NEWTON_MAXIT = 10;
static const double PI_ERR_TOL = 1.0e-3;     // errTol default of prep_chem.lua:51

static bool point_implicit_step(const Mech& m, const double* c0, double h, double* cOut,
                                double& h_suggest, int& iters) {
    const int n = m.tc.nsp;
    double cscale = 0.0;
    for (int i = 0; i < n; ++i) cscale += c0[i];
    if (!(cscale > 0.0)) return false;
    double x[E4O_MAXSP];
    for (int i = 0; i < n; ++i) x[i] = c0[i];
    bool converged = false;
    iters = 0;
    for (int it = 0; it < PI_NEWTON_MAXIT; ++it) {
        double q[E4O_MAXSP], L[E4O_MAXSP], F[E4O_MAXSP];
        m.split_rates(x, q, L);
        double res = 0.0;
        for (int i = 0; i < n; ++i) {
            F[i] = x[i] - c0[i] - h * (q[i] - L[i]);
            res = std::fmax(res, std::fabs(F[i]));
        }
        if (res / cscale <= PI_NEWTON_TOL) { converged = true; break; }
        double J[E4O_MAXSP][E4O_MAXSP], A[E4O_MAXSP][E4O_MAXSP];
        m.jacobian(x, J);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) A[i][j] = ((i == j) ? 1.0 : 0.0) - h * J[i][j];
        double dx[E4O_MAXSP];
        for (int i = 0; i < n; ++i) dx[i] = -F[i];
        if (!solve_dense(n, A, dx)) return false;
        for (int i = 0; i < n; ++i) {
            x[i] = x[i] + dx[i];
            if (x[i] < 0.0) x[i] = 0.0;
        }
        ++iters;
    }
    if (!converged) return false;
    // error estimate: the distance from the explicit Euler prediction,
    // measured as RKFStep measures its error (chemistry_update.d:418-427):
    // atol = rtol = errTol, root mean square over the species
    double q0[E4O_MAXSP], L0[E4O_MAXSP];
    m.split_rates(c0, q0, L0);
    double err = 0.0;
    for (int i = 0; i < n; ++i) {
        double xe = c0[i] + h * (q0[i] - L0[i]);
        double sk = PI_ERR_TOL + PI_ERR_TOL * std::fmax(std::fabs(c0[i]), std::fabs(x[i]));
        double e = (x[i] - xe) / sk;
        err += e * e;
    }
    err = std::sqrt(err / n);
    double fac = (err > 0.0) ? 0.9 / std::sqrt(err) : 5.0;
    fac = std::fmin(5.0, std::fmax(0.2, fac));
    h_suggest = h * fac;
    for (int i = 0; i < n; ++i) cOut[i] = x[i];
    return err <= 1.0;
}

// RKFStep.opCall (chemistry_update.d:362-461): Runge-Kutta-Fehlberg with the
// Cash-Karp coefficients on dc/dt = q - L (eval_rates, reaction_mechanism.d:
// 59-66); the fifth-order solution, the difference from the fourth-order one
// as the error, measured with atol = rtol = tolerance as an RMS over the
// species, and the step-size suggestion with safety 0.9, exponent 0.2 and
// scale limits [0.2, 10].  Returns true on a successful step.
static const double RKF_TOL = 1.0e-3;   // odeStep.errTol default, prep_chem.lua:51

static bool rkf_step(const Mech& m, const double* y0, double h, double* yOut,
                     double& hSuggest) {
    const int n = m.tc.nsp;
    const double a21 = 1. / 5., a31 = 3. / 40., a32 = 9. / 40., a41 = 3. / 10., a42 = -9. / 10.,
                 a43 = 6. / 5., a51 = -11. / 54., a52 = 5. / 2., a53 = -70. / 27.,
                 a54 = 35. / 27., a61 = 1631. / 55296., a62 = 175. / 512., a63 = 575. / 13824.,
                 a64 = 44275. / 110592., a65 = 253. / 4096.;
    const double b51 = 37. / 378., b53 = 250. / 621., b54 = 125. / 594., b56 = 512. / 1771.,
                 b41 = 2825. / 27648., b43 = 18575. / 48384., b44 = 13525. / 55296.,
                 b45 = 277. / 14336., b46 = 1.0 / 4.0;
    double k1[E4O_MAXSP], k2[E4O_MAXSP], k3[E4O_MAXSP], k4[E4O_MAXSP], k5[E4O_MAXSP],
        k6[E4O_MAXSP], yt[E4O_MAXSP] = {}, q[E4O_MAXSP], L[E4O_MAXSP];
    auto eval = [&](const double* y, double* k) {
        m.split_rates(y, q, L);
        for (int i = 0; i < n; ++i) k[i] = q[i] - L[i];
    };
    eval(y0, k1);
    for (int i = 0; i < n; ++i) yt[i] = y0[i] + h * (a21 * k1[i]);
    eval(yt, k2);
    for (int i = 0; i < n; ++i) yt[i] = y0[i] + h * (a31 * k1[i] + a32 * k2[i]);
    eval(yt, k3);
    for (int i = 0; i < n; ++i) yt[i] = y0[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
    eval(yt, k4);
    for (int i = 0; i < n; ++i)
        yt[i] = y0[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
    eval(yt, k5);
    for (int i = 0; i < n; ++i)
        yt[i] = y0[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
    eval(yt, k6);
    double err = 0.0;
    for (int i = 0; i < n; ++i) {
        yOut[i] = y0[i] + h * (b51 * k1[i] + b53 * k3[i] + b54 * k4[i] + b56 * k6[i]);
        const double yErr =
            yOut[i] - (y0[i] + h * (b41 * k1[i] + b43 * k3[i] + b44 * k4[i] + b45 * k5[i] +
                                    b46 * k6[i]));
        const double sk = RKF_TOL + RKF_TOL * std::max(std::fabs(y0[i]), std::fabs(yOut[i]));
        err += (yErr / sk) * (yErr / sk);
    }
    err = std::sqrt(err / n);
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
    scale = std::max(safe * pm_pow(err, -alpha), minscale);
    hSuggest = scale * h;
    return false;
}

// One backward-Euler step over the whole interval h, x = c0 + h w(x), by
// Newton iteration from the start x = c0 (at most maxit iterations, 12 unless
// configured otherwise,
// same convergence test as point_implicit_step, no error control).  This is
// the point-implicit update proper; the sub-cycled recovery below runs only
// when it does not converge.
static bool point_implicit_whole(const Mech& m, const double* c0, double h, double* cOut,
                                 int& iters, int maxit) {
    const int n = m.tc.nsp;
    double cscale = 0.0;
    for (int i = 0; i < n; ++i) cscale += c0[i];
    iters = 0;
    if (!(cscale > 0.0)) return false;
    double x[E4O_MAXSP];
    for (int i = 0; i < n; ++i) x[i] = c0[i];
    for (int it = 0; it <= maxit; ++it) {
        double q[E4O_MAXSP], L[E4O_MAXSP], F[E4O_MAXSP];
        m.split_rates(x, q, L);
        double res = 0.0;
        for (int i = 0; i < n; ++i) {
            F[i] = x[i] - c0[i] - h * (q[i] - L[i]);
            res = std::fmax(res, std::fabs(F[i]));
        }
        if (res / cscale <= PI_NEWTON_TOL) {
            for (int i = 0; i < n; ++i) cOut[i] = x[i];
            return true;
        }
        if (it == maxit) break;
        double J[E4O_MAXSP][E4O_MAXSP], A[E4O_MAXSP][E4O_MAXSP];
        m.jacobian(x, J);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) A[i][j] = ((i == j) ? 1.0 : 0.0) - h * J[i][j];
        double dx[E4O_MAXSP];
        for (int i = 0; i < n; ++i) dx[i] = -F[i];
        if (!solve_dense(n, A, dx)) return false;
        for (int i = 0; i < n; ++i) {
            x[i] = x[i] + dx[i];
            if (x[i] < 0.0) x[i] = 0.0;
        }
        ++iters;
    }
    return false;
}

// The chemistry update of one cell over tInterval at the cell's temperature:
// first the point-implicit step over the whole interval; if its Newton
// iteration does not converge (or the mass fractions stop summing to one),
// ChemistryUpdate.opCall's sub-cycling (chemistry_update.d:119-307) takes
// over, with error-controlled point-implicit sub-steps and the per-cell
// dt_chem warm start.
// With method 1 (the reference's odeStep.method 'rkf') there is no
// whole-interval step: opCall's sub-cycling with RKF sub-steps from the start.
static int chemistry_update(const e4o_thermochem& tc, GasState& Q, double tInterval,
                            double& dtChemSuggest, int maxit, int method) {
    const int n = tc.nsp;
    GasState Qinit = Q;
    double conc0[E4O_MAXSP], concOut[E4O_MAXSP];
    if (std::isnan(Q.rho) || Q.rho <= 0.0) return E4O_ERR_CHEM;
    for (int i = 0; i < n; ++i) {  // massf2conc, gas_model.d:196-212
        conc0[i] = Q.massf[i] * Q.rho / tc.M[i];
        if (conc0[i] < 1.0e-30) conc0[i] = 0.0;
    }
    for (int i = 0; i < n; ++i) concOut[i] = conc0[i];
    Mech m(tc);
    m.eval_rate_constants(Q.T);
    if (method == 0) {
        int iters;
        if (point_implicit_whole(m, conc0, tInterval, concOut, iters, maxit)) {
            double total = 0.0;
            for (int i = 0; i < n; ++i) {
                Q.massf[i] = concOut[i] * tc.M[i] / Q.rho;
                if (Q.massf[i] < 1.0e-30) Q.massf[i] = 0.0;
                total += Q.massf[i];
            }
            if (std::fabs(total - 1.0) <= 1.0e-3) {
                for (int i = 0; i < n; ++i) Q.massf[i] /= total;
                return 0;
            }
            for (int i = 0; i < n; ++i) Q.massf[i] = Qinit.massf[i];
            for (int i = 0; i < n; ++i) concOut[i] = conc0[i];
        }
    }
    double t = 0.0, h, dtSave;
    if (dtChemSuggest > tInterval) h = tInterval;
    else if (dtChemSuggest <= 0.0) h = m.estimate_step_size(conc0);
    else h = dtChemSuggest;
    const int maxSubcycles = 10000, maxAttempts = 4;
    int cycle = 0;
    for (; cycle < maxSubcycles; ++cycle) {
        dtSave = dtChemSuggest;
        h = std::min(h, tInterval - t);
        int attempt = 0;
        for (; attempt < maxAttempts; ++attempt) {
            int iters = 0;
            bool ok = (method == 1) ? rkf_step(m, conc0, h, concOut, dtChemSuggest)
                                    : point_implicit_step(m, conc0, h, concOut, dtChemSuggest, iters);
            bool massf_ok = true;
            if (ok) {
                double total = 0.0;
                for (int i = 0; i < n; ++i) {  // conc2massf, gas_model.d:214-230
                    Q.massf[i] = concOut[i] * tc.M[i] / Q.rho;
                    if (Q.massf[i] < 1.0e-30) Q.massf[i] = 0.0;
                    total += Q.massf[i];
                }
                if (std::fabs(total - 1.0) > 1.0e-3) massf_ok = false;
            }
            if (ok && massf_ok) {
                t += h;
                for (int i = 0; i < n; ++i) conc0[i] = concOut[i];
                double hMax = h * (1.0 + 10.0 / 100.0);
                if (dtChemSuggest > h) h = std::min(dtChemSuggest, hMax);
                break;
            } else {
                h /= 10.0;
                if (h < 1.0e-15) { Q = Qinit; return E4O_ERR_CHEM; }
            }
        }
        if (attempt == maxAttempts) { Q = Qinit; return E4O_ERR_CHEM; }
        if (t >= tInterval) {
            if (cycle == 0) dtSave = dtChemSuggest;
            break;
        }
    }
    if (cycle == maxSubcycles) { Q = Qinit; return E4O_ERR_CHEM; }
    double total = 0.0;
    for (int i = 0; i < n; ++i) {
        Q.massf[i] = concOut[i] * tc.M[i] / Q.rho;
        if (Q.massf[i] < 1.0e-30) Q.massf[i] = 0.0;
        total += Q.massf[i];
    }
    for (int i = 0; i < n; ++i) Q.massf[i] /= total;
    dtChemSuggest = dtSave;
    return 0;
}

// FVCell.thermochemical_increment (fvcell.d:1510-1621)
static int thermochemical_increment(const e4o_thermochem& tc, double T_frozen, GasState& Q,
                                    double dt, double& dt_chem, int maxit, int method) {
    if (Q.T <= T_frozen) return 0;
    int rc = chemistry_update(tc, Q, dt, dt_chem, maxit, method);
    if (rc != 0) {
        dt_chem = -1.0;
        rc = chemistry_update(tc, Q, dt, dt_chem, maxit, method);
        if (rc != 0) return rc;
    }
    TP tp(tc);
    if (!tp.update_thermo_from_rhou(Q)) return E4O_ERR_THERMO;
    tp.update_sound_speed(Q);
    return 0;
}

int Sim::chemistry_step(double dt) {
    // simcore.d:1489-1505, every block and cell; then U.massf = rho*massf
    int err = 0;
    for (Block* b : blocks) {
#pragma omp parallel for collapse(2) schedule(dynamic, 4) reduction(min : err)
        for (int k = b->kmin; k <= b->kmax; ++k)
            for (int j = b->jmin; j <= b->jmax; ++j)
                for (int i = b->imin; i <= b->imax; ++i) {
                    Cell& c = b->cell(i, j, k);
                    // fvcell.d:1514: frozen cells return before U.massf is touched
                    if (c.fs.gas.T <= cfg.T_frozen) continue;
                    int rc = thermochemical_increment(gm.tc, cfg.T_frozen, c.fs.gas, dt, c.dt_chem,
                                                      cfg.chem_newton_iterations, cfg.chem_method);
                    if (rc != 0) { err = std::min(err, rc); continue; }
                    for (int s = 0; s < nsp_cons; ++s) c.U[0][5 + s] = c.fs.gas.rho * c.fs.gas.massf[s];
                }
    }
    return err;
}

}  // namespace e4o

using namespace e4o;

// Newton iterations of the whole-interval step for the single-cell entry
// points (a simulation uses its configuration's value).
static int g_chem_newton_iterations = 12;
static int g_chem_method = 0;

extern "C" {

int e4o_set_chem_method(int m) {
    if (m != 0 && m != 1) return E4O_ERR_ARG;
    g_chem_method = m;
    return 0;
}

int e4o_rkf_step(const e4o_thermochem* tc, double T, const double* conc0, double h,
                 double* concOut, double* h_suggest) {
    Mech m(*tc);
    m.eval_rate_constants(T);
    return rkf_step(m, conc0, h, concOut, *h_suggest) ? 0 : 1;
}

int e4o_set_chem_newton_iterations(int n) {
    g_chem_newton_iterations = n;
    return 0;
}

int e4o_set_thermochem(void* sim, const e4o_thermochem* tc) {
    Sim* s = static_cast<Sim*>(sim);
    s->gm.tc = *tc;
    return 0;
}

int e4o_tp_update(const e4o_thermochem* tc, int mode, const double* massf, double* rho,
                  double* p, double* T, double* u, double* a) {
    TP tp(*tc);
    GasState Q;
    for (int i = 0; i < tc->nsp; ++i) Q.massf[i] = massf[i];
    Q.rho = *rho; Q.p = *p; Q.T = *T; Q.u = *u;
    bool ok = true;
    if (mode == 0) ok = tp.update_thermo_from_pT(Q);
    else if (mode == 1) ok = tp.update_thermo_from_rhou(Q);
    else ok = tp.update_thermo_from_rhoT(Q);
    if (!ok) return E4O_ERR_THERMO;
    tp.update_sound_speed(Q);
    *rho = Q.rho; *p = Q.p; *T = Q.T; *u = Q.u; *a = Q.a;
    return 0;
}

int e4o_chem_update(const e4o_thermochem* tc, double dt, double rho, double T, double* massf,
                    double* dt_chem) {
    GasState Q;
    Q.rho = rho; Q.T = T; Q.u = 0.0; Q.p = 0.0;
    for (int i = 0; i < tc->nsp; ++i) Q.massf[i] = massf[i];
    int rc = chemistry_update(*tc, Q, dt, *dt_chem, g_chem_newton_iterations, g_chem_method);
    if (rc != 0) return rc;
    for (int i = 0; i < tc->nsp; ++i) massf[i] = Q.massf[i];
    return 0;
}

int e4o_chem_cell(const e4o_thermochem* tc, double T_frozen, double dt, double rho, double* T,
                  double* u, double* p, double* massf, double* dt_chem) {
    GasState Q;
    Q.rho = rho; Q.T = *T; Q.u = *u; Q.p = *p;
    for (int i = 0; i < tc->nsp; ++i) Q.massf[i] = massf[i];
    int rc = thermochemical_increment(*tc, T_frozen, Q, dt, *dt_chem, g_chem_newton_iterations,
                                      g_chem_method);
    if (rc != 0) return rc;
    *T = Q.T; *u = Q.u; *p = Q.p;
    for (int i = 0; i < tc->nsp; ++i) massf[i] = Q.massf[i];
    return 0;
}

// The two problems of the reference's Newton-solver unit test
// (nm/newton.d:109-135), solved by the same rtsafe the temperature iteration
// uses: x^3 + x^2 - 3x - 3 on [-5, 5] from 1, and 3x + sin(x) - exp(x) on
// [0, 1] from 0.2, with the solver's default tolerance 1e-9.
int e4o_newton_test(int which, double* root) {
    bool ok;
    if (which == 0) {
        ok = rtsafe([](double x) { return x * x * x + x * x - 3.0 * x - 3.0; },
                    [](double x) { return 3.0 * x * x + 2.0 * x - 3.0; }, 1.0, -5.0, 5.0, 1.0e-9,
                    *root);
    } else {
        const double a = 3.0;
        ok = rtsafe([&](double x) { return a * x + std::sin(x) - std::exp(x); },
                    [&](double x) { return a + std::cos(x) - std::exp(x); }, 0.2, 0.0, 1.0, 1.0e-9,
                    *root);
    }
    return ok ? 0 : E4O_ERR_THERMO;
}

// Production and loss rates of every species at temperature T and
// concentrations c (eval_rate_constants then eval_split_rates,
// reaction_mechanism.d:47-82): golden-vector tests of the rate machinery.
int e4o_rates(const e4o_thermochem* tc, double T, const double* c, double* q, double* L) {
    Mech m(*tc);
    m.eval_rate_constants(T);
    m.split_rates(c, q, L);
    return 0;
}

// GPUChem.prepareDataForGPU (src/eilmer/cuda_gpu_chem.d:183-205): per cell,
// one after another as the D host does, the concentrations (massf2conc,
// gas_model.d:196-212), the rate constants at the cell's temperature and the
// starting step h (the cell's dt_chem, else estimateStepSize).  Arrays are
// by cell, species or reaction outer: conc[s*n+i], kf[r*n+i].
int e4o_gpuchem_prepare(const e4o_thermochem* tc, int n, const double* rho, const double* T,
                        const double* massf, const double* dt_chem, double* conc, double* kf,
                        double* kb, double* h) {
    const int nsp = tc->nsp;
    Mech m(*tc);
    for (int i = 0; i < n; ++i) {
        if (std::isnan(rho[i]) || rho[i] <= 0.0) return E4O_ERR_CHEM;
        double c[E4O_MAXSP];
        for (int s = 0; s < nsp; ++s) {
            c[s] = massf[size_t(s) * n + i] * rho[i] / tc->M[s];
            if (c[s] < 1.0e-30) c[s] = 0.0;
            conc[size_t(s) * n + i] = c[s];
        }
        m.eval_rate_constants(T[i]);
        for (int r = 0; r < tc->nreac; ++r) {
            kf[size_t(r) * n + i] = m.kf[r];
            kb[size_t(r) * n + i] = m.kb[r];
        }
        h[i] = dt_chem[i] <= 0.0 ? m.estimate_step_size(c) : dt_chem[i];
    }
    return 0;
}

// The cell loop after the kernel (cuda_gpu_chem.d:156-167): conc2massf
// (gas_model.d:214-230), dt_chem = h, update_thermo_from_rhou (T holds the
// starting guess; u is left at the energy of the last iterate, p follows).
int e4o_gpuchem_finish(const e4o_thermochem* tc, int n, const double* conc, const double* h,
                       const double* rho, double* T, double* u, double* p, double* massf,
                       double* dt_chem) {
    const int nsp = tc->nsp;
    TP tp(*tc);
    int err = 0;
    for (int i = 0; i < n; ++i) {
        GasState Q;
        Q.rho = rho[i]; Q.T = T[i]; Q.u = u[i]; Q.p = p[i];
        for (int s = 0; s < nsp; ++s) {
            Q.massf[s] = conc[size_t(s) * n + i] * tc->M[s] / rho[i];
            if (Q.massf[s] < 1.0e-30) Q.massf[s] = 0.0;
        }
        dt_chem[i] = h[i];
        if (!tp.update_thermo_from_rhou(Q)) err = E4O_ERR_THERMO;
        T[i] = Q.T; u[i] = Q.u; p[i] = Q.p;
        for (int s = 0; s < nsp; ++s) massf[size_t(s) * n + i] = Q.massf[s];
    }
    return err;
}

}  // extern "C"
