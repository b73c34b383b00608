// e4c_tp.cu -- kernels of the general-geometry path for the thermally
// perfect 5-species mixture: face fluxes and cell updates with the mixture's
// EOS, the point-implicit chemistry (two passes: every cell, then the cells
// that need Newton work) and the training-pair kernels of the chemistry seed.
//
// Compiled with -fmad=false, as e4c_general.cu: the results match the CPU
// FP64 oracle bit for bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "e4c_cells.cuh"

namespace e4c {

// Host check for the bracket-sign shortcut of TPGas::solve_T: the least
// slope of each species' energy e(T) = h(T) - R T, as the device evaluates h
// (blended segments, linear continuation beyond the curves), over any window
// of +-1000 K around x0, divided by Cv(x0) (Cp clamped to the curves, minus R);
// on a 0.25 K grid from 20 K to 101,500 K, slopes taken as the minimum over
// 100 K blocks that meet the window (a lower bound of the window minimum).
// Returns the smallest ratio over the species, or 0 if a Cv is not positive.
namespace {
void host_coeffs(const e4c_thermochem& tc, int s, double T, double a[9]) {
    const int ns = tc.nseg[s];
    const double* tb = tc.T_break[s];
    const double* bl = tc.T_blend[s];
    if (T < tb[1] - 0.5 * bl[0]) { for (int j = 0; j < 9; ++j) a[j] = tc.coeffs[s][0][j]; return; }
    if (T > tb[ns - 1] + 0.5 * bl[ns - 2]) {
        for (int j = 0; j < 9; ++j) a[j] = tc.coeffs[s][ns - 1][j];
        return;
    }
    for (int i = 1; i < ns; ++i) {
        const double lo = tb[i] - 0.5 * bl[i - 1], hi = tb[i] + 0.5 * bl[i - 1];
        if (T >= lo && T <= hi) {
            const double wB = (T - lo) / bl[i - 1];
            for (int j = 0; j < 9; ++j) a[j] = (1.0 - wB) * tc.coeffs[s][i - 1][j] + wB * tc.coeffs[s][i][j];
            return;
        }
        if (T > hi && T < tb[i + 1] - 0.5 * bl[i]) {
            for (int j = 0; j < 9; ++j) a[j] = tc.coeffs[s][i][j];
            return;
        }
    }
    for (int j = 0; j < 9; ++j) a[j] = 0.0;
}
double host_cp(const e4c_thermochem& tc, int s, double R, double T) {
    T = std::min(std::max(T, tc.T_break[s][0]), tc.T_break[s][tc.nseg[s]]);
    double a[9];
    host_coeffs(tc, s, T, a);
    return R * (a[0] / (T * T) + a[1] / T + a[2] + a[3] * T + a[4] * T * T + a[5] * T * T * T +
                a[6] * T * T * T * T);
}
double host_h_in(const e4c_thermochem& tc, int s, double R, double T) {
    double a[9];
    host_coeffs(tc, s, T, a);
    const double hrt = -a[0] / (T * T) + a[1] / T * std::log(T) + a[2] + a[3] * T / 2.0 +
                       a[4] * T * T / 3.0 + a[5] * T * T * T / 4.0 +
                       a[6] * T * T * T * T / 5.0 + a[7] / T;
    return R * T * hrt;
}
double host_h(const e4c_thermochem& tc, int s, double R, double T) {
    const double lo = tc.T_break[s][0], hi = tc.T_break[s][tc.nseg[s]];
    if (T < lo) return host_h_in(tc, s, R, lo) - host_cp(tc, s, R, lo) * (lo - T);
    if (T > hi) return host_h_in(tc, s, R, hi) + host_cp(tc, s, R, hi) * (T - hi);
    return host_h_in(tc, s, R, T);
}
double bracket_slope_ratio(const e4c_thermochem& tc) {
    const double T0 = 20.0, step = 0.25, Tend = 101500.0;
    const int n = int((Tend - T0) / step) + 1;
    const int per_block = 400, nblk = (n - 1 + per_block - 1) / per_block;
    const int W = int(1000.0 / step);
    double worst = 1.0e300;
    std::vector<double> e(n), cv(n), bmin(nblk);
    for (int s = 0; s < tc.nsp; ++s) {
        const double R = 8.31451 / tc.M[s];
        for (int k = 0; k < n; ++k) {
            const double T = T0 + step * k;
            e[k] = host_h(tc, s, R, T) - R * T;
            cv[k] = host_cp(tc, s, R, T) - R;
            if (!(cv[k] > 0.0)) return 0.0;
        }
        for (int b = 0; b < nblk; ++b) bmin[b] = 1.0e300;
        for (int k = 0; k + 1 < n; ++k)
            bmin[k / per_block] = std::min(bmin[k / per_block], (e[k + 1] - e[k]) / step);
        for (int k = 0; k < n; ++k) {
            const int b0 = std::max(0, k - W) / per_block;
            const int b1 = std::min(n - 2, k + W) / per_block;
            double m = 1.0e300;
            for (int b = b0; b <= b1; ++b) m = std::min(m, bmin[b]);
            worst = std::min(worst, m / cv[k]);
        }
    }
    return worst;
}
}  // namespace

int set_chem_newton_iterations(int n) {
    return cudaMemcpyToSymbol(c_chem_newton_iterations, &n, sizeof(n)) == cudaSuccess ? 0 : -1;
}

int set_chem_method(int m) {
    return cudaMemcpyToSymbol(c_chem_method, &m, sizeof(m)) == cudaSuccess ? 0 : -1;
}

int set_thermochem_constants(const e4c_thermochem& tc) {
    if (cudaMemcpyToSymbol(c_tc, &tc, sizeof(tc)) != cudaSuccess) return -1;
    // the shortcut with kappa = 1/4 needs a slope ratio of at least 1/2
    const double kappa = bracket_slope_ratio(tc) >= 0.5 ? 0.25 : 0.0;
    return cudaMemcpyToSymbol(c_bracket_kappa, &kappa, sizeof(kappa)) == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------------------
// Training pairs of the learned chemistry seed
// ---------------------------------------------------------------------------
// Cells hotter than T_frozen whose start state does not satisfy the
// point-implicit convergence test over dt: the cells the seed is used for.
__global__ void k_seed_active_list(BlockView b, double T_frozen, double dt, int* list,
                                   int* count) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const size_t c = interior_cell(b, t);
        TPState<5> Q;
        load_tp(b, c, Q);
        if (Q.T <= T_frozen) continue;
        double dtc = -1.0;
        if (thermochemical_increment_d<5, 5>(c_tc, T_frozen, Q, dt, dtc, nullptr, nullptr, true) ==
            CHEM_NEEDS_WORK)
            list[atomicAdd(count, 1)] = int(c);
    }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    // splitmix64 finaliser (Steele, Lea & Flood 2014)
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Sample r: a cell drawn uniformly from the active list and a step dt * f with
// log f uniform in [log 1/4, log 4]; the plain chemistry update (no guess)
// gives the target.  feat = (log T, log p, Y[5], log dt), targ = (dY[5], dT);
// a failed update leaves a NaN first feature.
__global__ void k_seed_collect(BlockView b, const int* hot, int nhot, long long n,
                               unsigned long long seed, double dt, double T_frozen, double* feat,
                               double* targ) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
         r += (long long)gridDim.x * blockDim.x) {
        const unsigned long long h1 = mix64(seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(2 * r + 1));
        const unsigned long long h2 = mix64(seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(2 * r + 2));
        const size_t c = size_t(hot[h1 % (unsigned long long)nhot]);
        const double u = double(h2 >> 11) * (1.0 / 9007199254740992.0);
        const double dts = dt * exp(log(0.25) + u * log(16.0));
        TPState<5> Q;
        Q.rho = b.W[W_RHO * b.npad + c];
        Q.p = b.W[W_P * b.npad + c];
        Q.T = b.W[W_T * b.npad + c];
        Q.u = b.W[W_U * b.npad + c];
        Q.a = b.W[W_A * b.npad + c];
#pragma unroll
        for (int s = 0; s < 5; ++s) Q.massf[s] = b.W[(W_NBASE + s) * b.npad + c];
        double* f = feat + r * 8;
        double* g = targ + r * 6;
        f[0] = log(Q.T);
        f[1] = log(Q.p);
#pragma unroll
        for (int s = 0; s < 5; ++s) f[2 + s] = Q.massf[s];
        f[7] = log(dts);
        TPState<5> Q1 = Q;
        double dtc = -1.0;
        const int rc = thermochemical_increment_d<5, 5>(c_tc, T_frozen, Q1, dts, dtc, nullptr,
                                                        nullptr);
#pragma unroll
        for (int s = 0; s < 5; ++s) g[s] = Q1.massf[s] - Q.massf[s];
        g[5] = Q1.T - Q.T;
        if (rc != 0) f[0] = CUDART_NAN;
    }
}

static int grid_for(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 64) g = 148LL * 64;
    if (g < 1) g = 1;
    return int(g);
}

void launch_flux_tp(const BlockView& b, const SimDev* sim, const FluxOpts& o, int dir, int g,
                    int T, cudaStream_t s) {
    if (o.flux == 1) k_flux<5, 1, 1><<<g, T, 0, s>>>(b, sim, o, dir);
    else if (o.flux == 2) k_flux<5, 2, 1><<<g, T, 0, s>>>(b, sim, o, dir);
    else if (o.flux == 3) k_flux<5, 3, 1><<<g, T, 0, s>>>(b, sim, o, dir);
    else k_flux<5, 0, 1><<<g, T, 0, s>>>(b, sim, o, dir);
}

static int boundary_cells(const BlockView& b) {
    const int m1 = b.ni * b.nk, m2 = b.nj * b.nk, m3 = b.ni * b.nj;
    return m1 > m2 ? (m1 > m3 ? m1 : m3) : (m2 > m3 ? m2 : m3);
}

void launch_bc_linear_tp(const BlockView& b, SimDev* sim, const GasConsts& gas, cudaStream_t s) {
    dim3 grid((boundary_cells(b) + 127) / 128, b.dim == 3 ? 6 : 4);
    k_bc_linear<5, 1><<<grid, 128, 0, s>>>(b, sim, gas);
}

void launch_ghost_defaults_tp(const BlockView& b, const GasConsts& gas, cudaStream_t s) {
    dim3 grid((boundary_cells(b) + 127) / 128, b.dim == 3 ? 6 : 4);
    k_ghost_defaults<5, 1><<<grid, 128, 0, s>>>(b, gas);
}

void launch_update_tp(const BlockView& b, SimDev* sim, const GasConsts& gas, int stage,
                      int final_stage, int g, int T, cudaStream_t s) {
    k_update<5, 1><<<g, T, 0, s>>>(b, sim, gas, stage, final_stage);
}

void launch_seed_active_list(const BlockView& b, double T_frozen, double dt, int* list, int* count,
                             cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_seed_active_list<<<grid_for(n, 128), 128, 0, s>>>(b, T_frozen, dt, list, count);
}

void launch_seed_collect(const BlockView& b, const int* hot, int nhot, long long n,
                         unsigned long long seed, double dt, double T_frozen, double* feat,
                         double* targ, cudaStream_t s) {
    k_seed_collect<<<grid_for(n, 64), 64, 0, s>>>(b, hot, nhot, n, seed, dt, T_frozen, feat, targ);
}

int launch_chem(const BlockView& b, SimDev* sim, double T_frozen, const double* dt, int nreac,
                int* work, int* nwork, unsigned long long* stats, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    if (b.nsp != 5 || nreac != 5) return -1;
    k_chem<5, 5><<<grid_for(n, 128), 128, 0, s>>>(b, sim, T_frozen, dt, work, nwork, stats);
    return 0;
}

int launch_chem_work(const BlockView& b, SimDev* sim, double T_frozen, const double* dt,
                     int nreac, const int* work, const int* nwork, const double* guess,
                     unsigned long long* stats, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    if (b.nsp != 5 || nreac != 5) return -1;
    // the list length is known only on the device: a grid of up to two
    // 64-thread CTAs per SM strides over it
    long long g = (n + 63) / 64;
    if (g > 148 * 16) g = 148 * 16;
    k_chem_work<5, 5><<<int(g), 64, 0, s>>>(b, sim, T_frozen, dt, work, nwork, guess, stats);
    return 0;
}

}  // namespace e4c
