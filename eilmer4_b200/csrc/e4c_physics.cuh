// e4c_physics.cuh -- device-side physics of the explicit structured-block update.
//
// Each function states the reference code it reproduces.  The FP64 kernels
// that include this header are compiled with -fmad=false and keep the
// reference's operation order, so their results are bit-identical to the
// reference algorithm run in IEEE double arithmetic.  The same templates
// instantiated with float serve the FP32 reconstruction/flux form.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "e4c_types.h"

namespace e4c {

template <typename R>
struct V3 {
    R x, y, z;
};

// Vector3.dot, src/geom/elements/vector3.d:409-414
template <typename R>
__device__ __forceinline__ R dot3(const V3<R>& a, const V3<R>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

// transform_to_local_frame, vector3.d:425-434
template <typename R>
__device__ __forceinline__ void to_local(V3<R>& v, const V3<R>& n, const V3<R>& t1,
                                         const V3<R>& t2) {
    R vx = dot3(v, n), vy = dot3(v, t1), vz = dot3(v, t2);
    v.x = vx; v.y = vy; v.z = vz;
}

// transform_to_global_frame, vector3.d:439-451
template <typename R>
__device__ __forceinline__ void to_global(V3<R>& v, const V3<R>& n, const V3<R>& t1,
                                          const V3<R>& t2) {
    R gx = v.x * n.x + v.y * t1.x + v.z * t2.x;
    R gy = v.x * n.y + v.y * t1.y + v.z * t2.y;
    R gz = v.x * n.z + v.y * t1.z + v.z * t2.z;
    v.x = gx; v.y = gy; v.z = gz;
}

template <typename R>
struct Frame {
    V3<R> n, t1, t2;
};

// Primitive state of a cell as the flux needs it (a FlowState subset,
// src/eilmer/flowstate.d:30).
template <typename R, int NSP>
struct Prim {
    R rho, p, u, a;
    R T;  // the starting guess of a thermally perfect rhou update
    V3<R> vel;
    R massf[NSP];
};

// RN(d / a) < tol for a shock detector's compression test, the quotient
// formed only where the outcome is not already certain: with a > 0 and
// P = RN(tol a) in the normal range, d < P - |P| 2^-49 puts d / a below tol by
// more than 2^-50 |tol| (so its rounded value is below tol as well), and
// d > P + |P| 2^-49 puts it above tol; in the band between, and for values
// outside the normal range, the division decides.  The outcome is the
// division's in every case.
__device__ __forceinline__ bool quotient_below(double d, double a, double tol) {
    const double P = tol * a;
    const double band = fabs(P) * 0x1p-49;
    if (a > 0.0 && tol != 0.0 && fabs(P) >= 0x1p-1000 && fabs(P) <= DBL_MAX && fabs(d) <= DBL_MAX) {
        if (d < P - band) return true;
        if (d > P + band) return false;
    }
    return (d / a) < tol;
}

// clip_to_limits, src/eilmer/limiters.d:31-38
template <typename R>
__device__ __forceinline__ R clip_to_limits(R q, R A, R B) {
    R lower = (A <= B) ? A : B;
    R upper = (A > B) ? A : B;
    R qc = (q > lower) ? q : lower;
    return (qc <= upper) ? qc : upper;
}

// l2r2_prepare, src/eilmer/onedinterp.d:118-133
template <typename R>
struct L2R2 {
    R aL0, aR0, lenL0, lenR0, tw_L0L1, tw_R0L0, tw_R1R0, two_L0_L1, two_R0_R1;
    __device__ __forceinline__ void prepare(R lenL1, R lenL0_, R lenR0_, R lenR1) {
        lenL0 = lenL0_;
        lenR0 = lenR0_;
        aL0 = R(0.5) * lenL0_ / (lenL1 + R(2.0) * lenL0_ + lenR0_);
        aR0 = R(0.5) * lenR0_ / (lenL0_ + R(2.0) * lenR0_ + lenR1);
        tw_L0L1 = R(2.0) / (lenL0_ + lenL1);
        tw_R0L0 = R(2.0) / (lenR0_ + lenL0_);
        tw_R1R0 = R(2.0) / (lenR1 + lenR0_);
        two_L0_L1 = (R(2.0) * lenL0_ + lenL1);
        two_R0_R1 = (R(2.0) * lenR0_ + lenR1);
    }
    // interp_l2r2_scalar, onedinterp.d:136-162 (van Albada, epsilon 1e-12 at :22)
    __device__ __forceinline__ void scalar(bool limiter, bool clip, R qL1, R qL0, R qR0, R qR1,
                                           R& qL, R& qR) const {
        const R eps = R(1.0e-12);
        R delLminus = (qL0 - qL1) * tw_L0L1;
        R del = (qR0 - qL0) * tw_R0L0;
        R delRplus = (qR1 - qR0) * tw_R1R0;
        R sL = R(1.0), sR = R(1.0);
        if (limiter) {
            sL = (delLminus * del + fabs(delLminus * del) + eps) /
                 (delLminus * delLminus + del * del + eps);
            sR = (del * delRplus + fabs(del * delRplus) + eps) /
                 (del * del + delRplus * delRplus + eps);
        }
        qL = qL0 + sL * aL0 * (del * two_L0_L1 + delLminus * lenR0);
        qR = qR0 - sR * aR0 * (delRplus * lenL0 + del * two_R0_R1);
        if (clip) {
            qL = clip_to_limits(qL, qL0, qR0);
            qR = clip_to_limits(qR, qL0, qR0);
        }
    }
    // With uniform cell lengths (tw_L0L1 == tw_R0L0 == tw_R1R0) the sL of a
    // face and the sR of the face before it are one van Albada value of their
    // shared cell, bit for bit: va() gives it from the cell and its two
    // neighbours, scalar_with() interpolates a face from the two values.
    __device__ __forceinline__ R va(R qm, R q0, R qp) const {
        const R eps = R(1.0e-12);
        R a = (q0 - qm) * tw_L0L1;
        R b = (qp - q0) * tw_R0L0;
        return (a * b + fabs(a * b) + eps) / (a * a + b * b + eps);
    }
    __device__ __forceinline__ void scalar_with(R sL, R sR, bool clip, R qL1, R qL0, R qR0, R qR1,
                                                R& qL, R& qR) const {
        R delLminus = (qL0 - qL1) * tw_L0L1;
        R del = (qR0 - qL0) * tw_R0L0;
        R delRplus = (qR1 - qR0) * tw_R1R0;
        qL = qL0 + sL * aL0 * (del * two_L0_L1 + delLminus * lenR0);
        qR = qR0 - sR * aR0 * (delRplus * lenL0 + del * two_R0_R1);
        if (clip) {
            qL = clip_to_limits(qL, qL0, qR0);
            qR = clip_to_limits(qR, qL0, qR0);
        }
    }
};

// IdealGas.update_thermo_from_rhou, src/gas/ideal_gas.d:98-106
template <typename R>
__device__ __forceinline__ bool ideal_rhou(const GasConsts& g, R rho, R u, R& p, R& T) {
    if (u <= R(0.0) || rho <= R(0.0)) return false;
    T = u * R(g.Cvinv);
    p = rho * R(g.Rgas) * T;
    return true;
}

// IdealGas.update_sound_speed, ideal_gas.d:137-144
template <typename R>
__device__ __forceinline__ R ideal_sound_speed(const GasConsts& g, R T) {
    return sqrt(R(g.gamma) * R(g.Rgas) * T);
}

// decode_conserved (fvcell.d:563-732) of one ideal-gas cell with the
// reference's defaults (adjust_invalid_cell_data = false,
// ignore_low_T_thermo_update_failure = true, suggested_low_T_value = 200 K):
// the primitive state from U, and U re-encoded where the low-temperature
// fallback applies.  The same operations as the stage kernels' decode.
// Returns false for a non-positive density (the state is then left zero).
__device__ __forceinline__ bool decode_ideal(const GasConsts& gas, double* Un, double& rho,
                                             double& vx, double& vy, double& vz, double& u,
                                             double& p, double& T, double& a) {
    rho = Un[0]; vx = 0.0; vy = 0.0; vz = 0.0; u = 0.0; p = 0.0; T = 0.0; a = 0.0;
    if (!(Un[0] > 0.0)) return false;
    const double dinv = 1.0 / rho;
    vx = Un[1] * dinv; vy = Un[2] * dinv; vz = Un[3] * dinv;
    u = Un[4] * dinv;
    const double ke = 0.5 * (vx * vx + vy * vy + vz * vz);
    u -= ke;
    if (!ideal_rhou<double>(gas, rho, u, p, T)) {
        T = 200.0;
        p = rho * gas.Rgas * T;
        u = gas.Cv * T;
        Un[0] = rho;
        Un[1] = rho * vx; Un[2] = rho * vy; Un[3] = rho * vz;
        const double ke2 = 0.5 * (vx * vx + vy * vy + vz * vz);
        Un[4] = rho * (u + ke2);
    }
    a = ideal_sound_speed<double>(gas, T);
    return true;
}

// gas_model.d:295-327 scale_mass_fractions (tolerance 0.0, assert tolerance 0.1)
template <typename R, int NSP>
__device__ __forceinline__ bool scale_mass_fractions(R* massf) {
    R sum = R(0.0);
#pragma unroll
    for (int i = 0; i < NSP; ++i) {
        massf[i] = massf[i] >= R(0.0) ? massf[i] : R(0.0);
        sum += massf[i];
    }
    if (fabs(sum - R(1.0)) > R(0.1)) return false;
    if (fabs(sum - R(1.0)) > R(0.0)) {
#pragma unroll
        for (int i = 0; i < NSP; ++i) massf[i] /= sum;
    }
    return true;
}

// AUSMDV flux in the face frame: src/eilmer/fluxcalc.d:376-529.
// Hanel's flux (fluxcalc.d:532-629; Hanel, Schwane & Seider 1987, in the
// form of Wada & Liou 1997), in the face frame.
template <typename R, int NSP, int NSPC>
__device__ __forceinline__ void hanel(const Prim<R, NSP>& Lf, const Prim<R, NSP>& Rt, R* F) {
    R rL = Lf.rho, pL = Lf.p;
    R pLrL = pL / rL;
    R uL = Lf.vel.x, vL = Lf.vel.y, wL = Lf.vel.z;
    R eL = Lf.u, aL = Lf.a;
    R keL = R(0.5) * (uL * uL + vL * vL + wL * wL);
    R HL = eL + pLrL + keL;
    R rR = Rt.rho, pR = Rt.p;
    R pRrR = pR / rR;
    R uR = Rt.vel.x, vR = Rt.vel.y, wR = Rt.vel.z;
    R eR = Rt.u, aR = Rt.a;
    R keR = R(0.5) * (uR * uR + vR * vR + wR * wR);
    R HR = eR + pRrR + keR;
    R pLplus, uLplus;
    if (fabs(uL) <= aL) {
        uLplus = R(1.0) / (R(4.0) * aL) * (uL + aL) * (uL + aL);
        pLplus = pL * uLplus * (R(1.0) / aL * (R(2.0) - uL / aL));
    } else {
        uLplus = R(0.5) * (uL + fabs(uL));
        pLplus = pL * uLplus * (R(1.0) / uL);
    }
    R pRminus, uRminus;
    if (fabs(uR) <= aR) {
        uRminus = -R(1.0) / (R(4.0) * aR) * (uR - aR) * (uR - aR);
        pRminus = pR * uRminus * (R(1.0) / aR * (-R(2.0) - uR / aR));
    } else {
        uRminus = R(0.5) * (uR - fabs(uR));
        pRminus = pR * uRminus * (R(1.0) / uR);
    }
    R p_half = pLplus + pRminus;
    F[0] = uLplus * rL + uRminus * rR;
    F[1] = uLplus * rL * uL + uRminus * rR * uR + p_half;
    F[2] = uLplus * rL * vL + uRminus * rR * vR;
    F[3] = uLplus * rL * wL + uRminus * rR * wR;
    F[4] = uLplus * rL * HL + uRminus * rR * HR;
#pragma unroll
    for (int i = 0; i < NSPC; ++i) F[5 + i] = uLplus * rL * Lf.massf[i] + uRminus * rR * Rt.massf[i];
}

// F: mass, xmom, ymom, zmom, energy, species (when NSPC > 0).
template <typename R, int NSP, int NSPC>
__device__ __forceinline__ void ausmdv(const Prim<R, NSP>& Lf, const Prim<R, NSP>& Rt, R* F) {
    R rL = Lf.rho, pL = Lf.p;
    R pLrL = pL / rL;
    R uL = Lf.vel.x, vL = Lf.vel.y, wL = Lf.vel.z;
    R eL = Lf.u, aL = Lf.a;
    R keL = R(0.5) * (uL * uL + vL * vL + wL * wL);
    R HL = eL + pLrL + keL;
    R rR = Rt.rho, pR = Rt.p;
    R pRrR = pR / rR;
    R uR = Rt.vel.x, vR = Rt.vel.y, wR = Rt.vel.z;
    R eR = Rt.u, aR = Rt.a;
    R keR = R(0.5) * (uR * uR + vR * vR + wR * wR);
    R HR = eR + pRrR + keR;
    R alphaL = R(2.0) * pLrL / (pLrL + pRrR);
    R alphaR = R(2.0) * pRrR / (pLrL + pRrR);
    R am = fmax(aL, aR);
    R ML = uL / am;
    R MR = uR / am;
    R pLplus, uLplus;
    R duL = R(0.5) * (uL + fabs(uL));
    if (fabs(ML) <= R(1.0)) {
        pLplus = pL * (ML + R(1.0)) * (ML + R(1.0)) * (R(2.0) - ML) * R(0.25);
        uLplus = alphaL * ((uL + am) * (uL + am) / (R(4.0) * am) - duL) + duL;
    } else {
        pLplus = pL * duL / uL;
        uLplus = duL;
    }
    R pRminus, uRminus;
    R duR = R(0.5) * (uR - fabs(uR));
    if (fabs(MR) <= R(1.0)) {
        pRminus = pR * (MR - R(1.0)) * (MR - R(1.0)) * (R(2.0) + MR) * R(0.25);
        uRminus = alphaR * (-(uR - am) * (uR - am) / (R(4.0) * am) - duR) + duR;
    } else {
        pRminus = pR * duR / uR;
        uRminus = duR;
    }
    R ru_half = uLplus * rL + uRminus * rR;
    R p_half = pLplus + pRminus;
    R dp = pL - pR;
    dp = R(10.0) * fabs(dp) / fmin(pL, pR);
    R s = R(0.5) * fmin(R(1.0), dp);
    R ru2_AUSMV = uLplus * rL * uL + uRminus * rR * uR;
    R ru2_AUSMD = R(0.5) * (ru_half * (uL + uR) - fabs(ru_half) * (uR - uL));
    R ru2_half = (R(0.5) + s) * ru2_AUSMV + (R(0.5) - s) * ru2_AUSMD;
    F[0] = ru_half;
    F[1] = ru2_half + p_half;
    if (ru_half >= R(0.0)) {
        F[2] = ru_half * vL; F[3] = ru_half * wL; F[4] = ru_half * HL;
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] = ru_half * Lf.massf[i];
    } else {
        F[2] = ru_half * vR; F[3] = ru_half * wR; F[4] = ru_half * HR;
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] = ru_half * Rt.massf[i];
    }
    // entropy fix, Wada & Liou sec. 3.5 (fluxcalc.d:499-528), C_EFIX = 0.125
    bool caseA = ((uL - aL) < R(0.0)) && ((uR - aR) > R(0.0));
    bool caseB = ((uL + aL) < R(0.0)) && ((uR + aR) > R(0.0));
    R d_ua = R(0.0);
    if (caseA && !caseB) d_ua = R(0.125) * ((uR - aR) - (uL - aL));
    if (caseB && !caseA) d_ua = R(0.125) * ((uR + aR) - (uL + aL));
    if (d_ua != R(0.0)) {
        F[0] -= d_ua * (rR - rL);
        F[1] -= d_ua * (rR * uR - rL * uL);
        F[2] -= d_ua * (rR * vR - rL * vL);
        F[3] -= d_ua * (rR * wR - rL * wL);
        F[4] -= d_ua * (rR * HR - rL * HL);
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] -= d_ua * (rR * Rt.massf[i] - rL * Lf.massf[i]);
    }
}

// HLLC flux in the face frame.  The reference has no HLLC; this is Toro's
// HLLC (Riemann Solvers and Numerical Methods for Fluid Dynamics, 3rd ed.,
// sec. 10.4-10.6) with Davis wave-speed bounds and the flux form
// F*K = FK + SK (U*K - UK).  Species ride on the star-state mass flux.
template <typename R, int NSP, int NSPC>
__device__ __forceinline__ void hllc(const Prim<R, NSP>& Lf, const Prim<R, NSP>& Rt, R* F) {
    R rL = Lf.rho, pL = Lf.p, uL = Lf.vel.x, vL = Lf.vel.y, wL = Lf.vel.z, aL = Lf.a;
    R eL = Lf.u + R(0.5) * (uL * uL + vL * vL + wL * wL);  // total energy per mass
    R EL = rL * eL;
    R rR = Rt.rho, pR = Rt.p, uR = Rt.vel.x, vR = Rt.vel.y, wR = Rt.vel.z, aR = Rt.a;
    R eR = Rt.u + R(0.5) * (uR * uR + vR * vR + wR * wR);
    R ER = rR * eR;
    R SL = fmin(uL - aL, uR - aR);
    R SR = fmax(uL + aL, uR + aR);
    if (SL >= R(0.0)) {
        R m = rL * uL;
        F[0] = m; F[1] = m * uL + pL; F[2] = m * vL; F[3] = m * wL; F[4] = uL * (EL + pL);
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] = m * Lf.massf[i];
        return;
    }
    if (SR <= R(0.0)) {
        R m = rR * uR;
        F[0] = m; F[1] = m * uR + pR; F[2] = m * vR; F[3] = m * wR; F[4] = uR * (ER + pR);
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] = m * Rt.massf[i];
        return;
    }
    // subsonic: the contact speed (computed only here; the supersonic faces
    // above do not use it)
    R mL = rL * (SL - uL);
    R mR = rR * (SR - uR);
    R Sstar = (pR - pL + mL * uL - mR * uR) / (mL - mR);
    if (Sstar >= R(0.0)) {
        R m = rL * uL;
        R coef = mL / (SL - Sstar);
        R Estar = coef * (eL + (Sstar - uL) * (Sstar + pL / mL));
        F[0] = m + SL * (coef - rL);
        F[1] = (m * uL + pL) + SL * (coef * Sstar - m);
        F[2] = m * vL + SL * (coef * vL - rL * vL);
        F[3] = m * wL + SL * (coef * wL - rL * wL);
        F[4] = uL * (EL + pL) + SL * (Estar - EL);
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] = F[0] * Lf.massf[i];
    } else {
        R m = rR * uR;
        R coef = mR / (SR - Sstar);
        R Estar = coef * (eR + (Sstar - uR) * (Sstar + pR / mR));
        F[0] = m + SR * (coef - rR);
        F[1] = (m * uR + pR) + SR * (coef * Sstar - m);
        F[2] = m * vR + SR * (coef * vR - rR * vR);
        F[3] = m * wR + SR * (coef * wR - rR * wR);
        F[4] = uR * (ER + pR) + SR * (Estar - ER);
#pragma unroll
        for (int i = 0; i < NSPC; ++i) F[5 + i] = F[0] * Rt.massf[i];
    }
}

// Order-preserving encoding of non-negative doubles for atomicMin/atomicMax.
__device__ __forceinline__ unsigned long long dbits(double x) {
    return static_cast<unsigned long long>(__double_as_longlong(x));
}

}  // namespace e4c
