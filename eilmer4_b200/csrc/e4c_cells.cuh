// e4c_cells.cuh -- device code shared by the general-path translation units:
// cell indexing, the face-flux and cell-update kernels (templates over the
// species count, flux calculator and gas model) and the chemistry kernels.
// e4c_general.cu instantiates the ideal-gas forms, e4c_tp.cu the thermally
// perfect and reacting ones.  Each unit has its own copy of the constant
// c_tc; only e4c_tp.cu's is used (and set).
#pragma once

#include <cfloat>

#include "e4c_kernels.h"
#include "e4c_physics.cuh"
#include "e4c_thermo.cuh"

namespace e4c {

// Thermally perfect mixture and mechanism of the context (e4c_set_thermochem).
static __constant__ e4c_thermochem c_tc;

__device__ __forceinline__ size_t pidx(const BlockView& b, int i, int j, int k) {
    return (size_t(k) * b.njdim + j) * b.nidim + i;
}

__device__ __forceinline__ void set_status(SimDev* sim, int code) {
    if (atomicCAS(&sim->status, 0, code) == 0) sim->status_step = sim->step;
}

// ---------------------------------------------------------------------------
// Face flux: reconstruction + flux for one face
// (sfluidblock.d:2190-2344, onedinterp.d:435-585, fluxcalc.d:26-128)
// ---------------------------------------------------------------------------
template <int NSP>
__device__ __forceinline__ void load_prim(const BlockView& b, size_t c, Prim<double, NSP>& s) {
    s.rho = b.W[W_RHO * b.npad + c];
    s.vel = {b.W[W_VX * b.npad + c], b.W[W_VY * b.npad + c], b.W[W_VZ * b.npad + c]};
    s.p = b.W[W_P * b.npad + c];
    s.u = b.W[W_U * b.npad + c];
    s.a = b.W[W_A * b.npad + c];
    s.T = b.W[W_T * b.npad + c];
    if (NSP > 1) {
#pragma unroll
        for (int q = 0; q < NSP; ++q) s.massf[q] = b.W[(W_NBASE + q) * b.npad + c];
    } else {
        s.massf[0] = 1.0;
    }
}

// interp_l2r2 rotates the velocities of its four stencil cells into the face
// frame and back again in place (onedinterp.d:445-454, 576-584), so a cell
// enters each face with the round-off of every earlier face, in the loop order
// of sfluidblock.d:2190-2344, that it took part in.  For frames made of signed
// unit axes a round trip is exact (up to the sign of a zero) and is skipped.
__device__ __forceinline__ bool frame_is_axis(const double* fg, size_t npad, size_t f) {
    for (int v = 0; v < 3; ++v) {
        int ones = 0;
        for (int c = 0; c < 3; ++c) {
            const double x = fg[(3 * v + c) * npad + f];
            if (x == 1.0 || x == -1.0) ++ones;
            else if (x != 0.0) return false;
        }
        if (ones != 1) return false;
    }
    return true;
}

__device__ __forceinline__ void roundtrip(V3<double>& v, const double* fg, size_t npad, size_t f) {
    if (frame_is_axis(fg, npad, f)) return;
    const V3<double> n{fg[0 * npad + f], fg[1 * npad + f], fg[2 * npad + f]};
    const V3<double> t1{fg[3 * npad + f], fg[4 * npad + f], fg[5 * npad + f]};
    const V3<double> t2{fg[6 * npad + f], fg[7 * npad + f], fg[8 * npad + f]};
    to_local(v, n, t1, t2);
    to_global(v, n, t1, t2);
}

// Velocity of stencil cell (ci,cj,ck) as the reference holds it when it
// reaches the face of direction dir at index fpos along dir.  The round trips
// of the earlier directions' faces (their loops cover interior rows only, so
// only cells interior along dir took part) come precomputed per cell in
// b.Vrt (k_replay_base); this applies the earlier faces of direction dir in
// the same row, in loop order.
__device__ __forceinline__ void replay_roundtrips(const BlockView& b, int dir, int fpos, int ci,
                                                  int cj, int ck, size_t c, V3<double>& v) {
    const int cd = dir == 0 ? ci : (dir == 1 ? cj : ck);
    const int lo = dir == 0 ? b.imin : (dir == 1 ? b.jmin : b.kmin);
    const int hi = dir == 0 ? b.imax : (dir == 1 ? b.jmax : b.kmax);
    if (dir > 0 && cd >= lo && cd <= hi) {
        const double* V = b.Vrt + size_t(3 * (dir - 1)) * b.npad;
        v = {V[c], V[b.npad + c], V[2 * b.npad + c]};
    }
    const double* fg = dir == 0 ? b.fgi : (dir == 1 ? b.fgj : b.fgk);
    for (int g = cd - 1; g <= cd + 2 && g < fpos; ++g) {
        if (g < lo || g > hi + 1) continue;
        int p[3] = {ci, cj, ck};
        p[dir] = g;
        roundtrip(v, fg, b.npad, pidx(b, p[0], p[1], p[2]));
    }
}

// Velocity of an interior cell as the reference holds it after all of a
// stage's convective-flux loops: the round trips of every face it took part
// in, i faces, then j, then k, each in loop order.
static __device__ void replay_all_roundtrips(const BlockView& b, int ci, int cj, int ck,
                                             V3<double>& v) {
    const int c[3] = {ci, cj, ck};
    const int lo[3] = {b.imin, b.jmin, b.kmin}, hi[3] = {b.imax, b.jmax, b.kmax};
    const double* fgs[3] = {b.fgi, b.fgj, b.fgk};
    for (int d = 0; d < b.dim; ++d)
        for (int g = c[d] - 1; g <= c[d] + 2; ++g) {
            if (g < lo[d] || g > hi[d] + 1) continue;
            int p[3] = {c[0], c[1], c[2]};
            p[d] = g;
            roundtrip(v, fgs[d], b.npad, pidx(b, p[0], p[1], p[2]));
        }
}

__device__ __forceinline__ void load_frame(const double* fg, size_t npad, size_t f, Frame<double>& fr) {
    fr.n = {fg[0 * npad + f], fg[1 * npad + f], fg[2 * npad + f]};
    fr.t1 = {fg[3 * npad + f], fg[4 * npad + f], fg[5 * npad + f]};
    fr.t2 = {fg[6 * npad + f], fg[7 * npad + f], fg[8 * npad + f]};
}

// update_thermo_from_rhou of a reconstructed state: ideal gas, or the
// thermally perfect mixture started from the cell-centre temperature (the
// state was copied from the cell, onedinterp.d / sfluidblock.d:2199-2208)
template <int NSP, int GAS>
__device__ __forceinline__ bool rhou_update(const FluxOpts& o, Prim<double, NSP>& s) {
    if (GAS == 0) {
        double T;
        return ideal_rhou<double>(o.gas, s.rho, s.u, s.p, T);
    }
    TPState<NSP> Q;
    Q.rho = s.rho; Q.u = s.u; Q.T = s.T; Q.p = s.p; Q.a = s.a;
#pragma unroll
    for (int i = 0; i < NSP; ++i) Q.massf[i] = s.massf[i];
    TPGas<NSP> g(c_tc);
    if (!g.rhou(Q)) return false;
    s.p = Q.p; s.T = Q.T; s.u = Q.u;
    return true;
}

// Faces of direction dir, or of every direction of the block in one launch
// (dir < 0: i faces, then j, then k, one index space).
template <int NSP, int FLUX, int GAS>
__global__ void k_flux(BlockView b, const SimDev* sim, FluxOpts o, int dir_arg) {
    if (sim->status != 0 || sim->finished) return;
    long long nd[3];
    for (int d = 0; d < 3; ++d)
        nd[d] = (long long)(b.ni + (d == 0)) * (b.nj + (d == 1)) * (b.nk + (d == 2));
    if (b.dim == 2) nd[2] = 0;
    const long long n = dir_arg >= 0 ? nd[dir_arg] : nd[0] + nd[1] + nd[2];
    constexpr int NSPC = NSP > 1 ? NSP : 0;
    for (long long tt = blockIdx.x * (long long)blockDim.x + threadIdx.x; tt < n;
         tt += (long long)gridDim.x * blockDim.x) {
        int dir = dir_arg;
        long long t = tt;
        if (dir < 0) {
            dir = 0;
            if (t >= nd[0]) { t -= nd[0]; dir = 1; }
            if (dir == 1 && t >= nd[1]) { t -= nd[1]; dir = 2; }
        }
        const int ni = b.ni + (dir == 0), nj = b.nj + (dir == 1);
        const size_t stride = dir == 0 ? 1 : (dir == 1 ? size_t(b.nidim) : size_t(b.nidim) * b.njdim);
        const double* fg = dir == 0 ? b.fgi : (dir == 1 ? b.fgj : b.fgk);
        double* Fo = dir == 0 ? b.Fi : (dir == 1 ? b.Fj : b.Fk);
        int i = b.imin + int(t % ni);
        int j = b.jmin + int((t / ni) % nj);
        int k = b.kmin + int(t / ((long long)ni * nj));
        const size_t f = pidx(b, i, j, k);
        const size_t cR0 = f, cL0 = f - stride, cL1 = f - 2 * stride, cR1 = f + stride;
        const int fpos = dir == 0 ? i : (dir == 1 ? j : k);
        const int di = dir == 0, dj = dir == 1, dk = dir == 2;
        const bool replay = o.local_frame && !b.axis_frames;
        Frame<double> fr;
        load_frame(fg, b.npad, f, fr);
        // a stencil cell's state as the reconstruction holds it: velocity after
        // the earlier faces' round trips and in this face's frame
        auto cell_state = [&](size_t c, int ci, int cj, int ck, Prim<double, NSP>& s) {
            load_prim<NSP>(b, c, s);
            if (o.order2) {
                if (replay) replay_roundtrips(b, dir, fpos, ci, cj, ck, c, s.vel);
                if (o.local_frame) to_local(s.vel, fr.n, fr.t1, fr.t2);
            }
        };
        Prim<double, NSP> Lf, Rt;
        cell_state(cL0, i - di, j - dj, k - dk, Lf);
        cell_state(cR0, i, j, k, Rt);
        if (o.order2) {
            {
                // the outer cells live only for the reconstruction; the inner
                // ones are reloaded where the reference falls back on them
                Prim<double, NSP> sL1, sL0 = Lf, sR0 = Rt, sR1;
                cell_state(cL1, i - 2 * di, j - 2 * dj, k - 2 * dk, sL1);
                cell_state(cR1, i + di, j + dj, k + dk, sR1);
                const double* len = b.cgeom + size_t(1 + dir) * b.npad;
                L2R2<double> r;
                r.prepare(len[cL1], len[cL0], len[cR0], len[cR1]);
                r.scalar(o.limiter, o.clip, sL1.vel.x, sL0.vel.x, sR0.vel.x, sR1.vel.x, Lf.vel.x, Rt.vel.x);
                r.scalar(o.limiter, o.clip, sL1.vel.y, sL0.vel.y, sR0.vel.y, sR1.vel.y, Lf.vel.y, Rt.vel.y);
                r.scalar(o.limiter, o.clip, sL1.vel.z, sL0.vel.z, sR0.vel.z, sR1.vel.z, Lf.vel.z, Rt.vel.z);
                if (NSP > 1) {
#pragma unroll
                    for (int q = 0; q < NSP; ++q)
                        r.scalar(o.limiter, o.clip, sL1.massf[q], sL0.massf[q], sR0.massf[q],
                                 sR1.massf[q], Lf.massf[q], Rt.massf[q]);
                    if (!scale_mass_fractions<double, NSP>(Lf.massf))
                        for (int q = 0; q < NSP; ++q) Lf.massf[q] = sL0.massf[q];
                    if (!scale_mass_fractions<double, NSP>(Rt.massf))
                        for (int q = 0; q < NSP; ++q) Rt.massf[q] = sR0.massf[q];
                } else {
                    Lf.massf[0] = 1.0;
                    Rt.massf[0] = 1.0;
                }
                r.scalar(o.limiter, o.clip, sL1.rho, sL0.rho, sR0.rho, sR1.rho, Lf.rho, Rt.rho);
                r.scalar(o.limiter, o.clip, sL1.u, sL0.u, sR0.u, sR1.u, Lf.u, Rt.u);
            }
            // codeForThermoUpdateBoth("rhou"), onedinterp.d:1039-1068: on failure
            // the cell-centre state (its velocity as above) is taken
            if (!rhou_update<NSP, GAS>(o, Lf)) {
                load_frame(fg, b.npad, f, fr);
                cell_state(cL0, i - di, j - dj, k - dk, Lf);
            }
            if (!rhou_update<NSP, GAS>(o, Rt)) {
                load_frame(fg, b.npad, f, fr);
                cell_state(cR0, i, j, k, Rt);
            }
            load_frame(fg, b.npad, f, fr);
            if (o.local_frame) {
                to_global(Lf.vel, fr.n, fr.t1, fr.t2);
                to_global(Rt.vel, fr.n, fr.t1, fr.t2);
            }
        }
        // compute_interface_flux, fluxcalc.d:26-128 (fixed grid)
        to_local(Lf.vel, fr.n, fr.t1, fr.t2);
        to_local(Rt.vel, fr.n, fr.t1, fr.t2);
        double F[5 + NSPC];
        if (FLUX == 1) {
            hllc<double, NSP, NSPC>(Lf, Rt, F);
        } else if (FLUX == 2) {
            hanel<double, NSP, NSPC>(Lf, Rt, F);
        } else if (FLUX == 3) {
            // adaptive_hanel_ausmdv (fluxcalc.d:824-838); the states carry the
            // shock flags of the cells they were reconstructed from
            // (the shear matters only at shock points)
            bool use_hanel = false;
            if (b.S[cL0] == 1 || b.S[cR0] == 1) {
                const double sound_speed = 0.5 * (Lf.a + Rt.a);
                const double shear_y = fabs(Lf.vel.y - Rt.vel.y) / sound_speed;
                const double shear_z = fabs(Lf.vel.z - Rt.vel.z) / sound_speed;
                use_hanel = fmax(shear_y, shear_z) <= o.shear_tol;
            }
            if (use_hanel)
                hanel<double, NSP, NSPC>(Lf, Rt, F);
            else
                ausmdv<double, NSP, NSPC>(Lf, Rt, F);
        } else {
            ausmdv<double, NSP, NSPC>(Lf, Rt, F);
        }
        V3<double> m{F[1], F[2], F[3]};
        to_global(m, fr.n, fr.t1, fr.t2);
        F[1] = m.x; F[2] = m.y; F[3] = m.z;
#pragma unroll
        for (int q = 0; q < 5 + NSPC; ++q) Fo[q * b.npad + f] = F[q];
    }
}

// ---------------------------------------------------------------------------
// OutFlowBC_SimpleExtrapolate{xOrder=1}: ExtrapolateCopy with x_order 1
// (src/eilmer/bc/ghost_cell_effect/extrapolate_copy.d:206-258 for the east
// face, the same steps for every face).  Each ghost layer is extrapolated
// linearly from the two cells before it (the second layer from the first
// ghost and the boundary cell): rho, u and the mass fractions (scaled), then
// T and p by update_thermo_from_rhou (from the ghost's own T for a mixture),
// then the velocity.  The sound speed and the shock flag stay as they were:
// the ghost cell's initial FlowState (k_ghost_defaults).  A failed thermo
// update or mass-fraction scaling (the reference throws) stops the run with
// E4C_ERR_THERMO.
// ---------------------------------------------------------------------------
template <int NSP, int GAS>
__global__ void k_bc_linear(BlockView b, SimDev* sim, GasConsts gas) {
    if (sim->status != 0 || sim->finished) return;
    const int which = blockIdx.y;
    if (b.dim == 2 && which >= 4) return;
    if (b.bc[which] != E4C_BC_OUTFLOW_EXTRAPOLATE_LINEAR) return;
    int n1, n2;
    if (which == NORTH || which == SOUTH) { n1 = b.ni; n2 = b.nk; }
    else if (which == EAST || which == WEST) { n1 = b.nj; n2 = b.nk; }
    else { n1 = b.ni; n2 = b.nj; }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n1 * n2) return;
    const int a1 = t % n1, a2 = t / n1;
    int i, j, k, di = 0, dj = 0, dk = 0;
    switch (which) {
        case NORTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmax; dj = 1; break;
        case SOUTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmin; dj = -1; break;
        case EAST: j = b.jmin + a1; k = b.kmin + a2; i = b.imax; di = 1; break;
        case WEST: j = b.jmin + a1; k = b.kmin + a2; i = b.imin; di = -1; break;
        case TOP: i = b.imin + a1; j = b.jmin + a2; k = b.kmax; dk = 1; break;
        default: i = b.imin + a1; j = b.jmin + a2; k = b.kmin; dk = -1; break;
    }
    size_t c1 = pidx(b, i, j, k), c2 = pidx(b, i - di, j - dj, k - dk);
    const size_t dst[2] = {pidx(b, i + di, j + dj, k + dk), pidx(b, i + 2 * di, j + 2 * dj, k + 2 * dk)};
    double* W = b.W;
    const size_t np = b.npad;
    for (int g = 0; g < 2; ++g) {
        const size_t d = dst[g];
        const double rho = 2.0 * W[W_RHO * np + c1] - W[W_RHO * np + c2];
        const double u = 2.0 * W[W_U * np + c1] - W[W_U * np + c2];
        bool ok = true;
        double p, T;
        if (GAS == 0) {
            ok = ideal_rhou<double>(gas, rho, u, p, T);
            W[W_U * np + d] = u;
        } else {
            TPState<NSP> Q;
            Q.rho = rho; Q.u = u; Q.T = W[W_T * np + d]; Q.p = W[W_P * np + d]; Q.a = W[W_A * np + d];
#pragma unroll
            for (int q = 0; q < NSP; ++q)
                Q.massf[q] = 2.0 * W[(W_NBASE + q) * np + c1] - W[(W_NBASE + q) * np + c2];
            if (NSP > 1) ok = scale_mass_fractions<double, NSP>(Q.massf);
            if (ok) {
                TPGas<NSP> gm(c_tc);
                ok = gm.rhou(Q);
            }
            p = Q.p; T = Q.T;
            W[W_U * np + d] = Q.u;
#pragma unroll
            for (int q = 0; q < NSP; ++q) W[(W_NBASE + q) * np + d] = Q.massf[q];
        }
        if (!ok) {
            set_status(sim, E4C_ERR_THERMO);
            return;
        }
        W[W_RHO * np + d] = rho;
        W[W_P * np + d] = p;
        W[W_T * np + d] = T;
        W[W_VX * np + d] = 2.0 * W[W_VX * np + c1] - W[W_VX * np + c2];
        W[W_VY * np + d] = 2.0 * W[W_VY * np + c1] - W[W_VY * np + c2];
        W[W_VZ * np + d] = 2.0 * W[W_VZ * np + c1] - W[W_VZ * np + c2];
        c2 = c1;
        c1 = d;
    }
}

// Both ghost layers of the block's x_order 1 boundaries as a cell's initial
// FlowState (fvcell.d:168-170 with flowstate.d:46-60 and gas_state.d:64-88):
// 100 kPa, 300 K, at rest, mass fractions (1, 0, ...), rho and u from
// update_thermo_from_pT, a from update_sound_speed, shock flag clear.
template <int NSP, int GAS>
__global__ void k_ghost_defaults(BlockView b, GasConsts gas) {
    const int which = blockIdx.y;
    if (b.dim == 2 && which >= 4) return;
    if (b.bc[which] != E4C_BC_OUTFLOW_EXTRAPOLATE_LINEAR) return;
    int n1, n2;
    if (which == NORTH || which == SOUTH) { n1 = b.ni; n2 = b.nk; }
    else if (which == EAST || which == WEST) { n1 = b.nj; n2 = b.nk; }
    else { n1 = b.ni; n2 = b.nj; }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n1 * n2) return;
    const int a1 = t % n1, a2 = t / n1;
    int i, j, k, di = 0, dj = 0, dk = 0;
    switch (which) {
        case NORTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmax; dj = 1; break;
        case SOUTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmin; dj = -1; break;
        case EAST: j = b.jmin + a1; k = b.kmin + a2; i = b.imax; di = 1; break;
        case WEST: j = b.jmin + a1; k = b.kmin + a2; i = b.imin; di = -1; break;
        case TOP: i = b.imin + a1; j = b.jmin + a2; k = b.kmax; dk = 1; break;
        default: i = b.imin + a1; j = b.jmin + a2; k = b.kmin; dk = -1; break;
    }
    const double p = 100.0e3, T = 300.0;
    double rho, u, a, massf[NSP > 1 ? NSP : 1];
    massf[0] = 1.0;
    for (int q = 1; q < NSP; ++q) massf[q] = 0.0;
    if (GAS == 0) {
        rho = p / (T * gas.Rgas);   // ideal_gas.d:89-97
        u = gas.Cv * T;
        a = ideal_sound_speed<double>(gas, T);
    } else {
        TPGas<NSP> gm(c_tc);
        rho = p / (gm.Rmix(massf) * T);   // perf_gas_mix_eos.d:55-62
        u = gm.energy(massf, T);
        a = gm.sound_speed(massf, T);
    }
    for (int g = 1; g <= 2; ++g) {
        const size_t d = pidx(b, i + g * di, j + g * dj, k + g * dk);
        b.W[W_RHO * b.npad + d] = rho;
        b.W[W_VX * b.npad + d] = 0.0;
        b.W[W_VY * b.npad + d] = 0.0;
        b.W[W_VZ * b.npad + d] = 0.0;
        b.W[W_P * b.npad + d] = p;
        b.W[W_T * b.npad + d] = T;
        b.W[W_U * b.npad + d] = u;
        b.W[W_A * b.npad + d] = a;
        if (NSP > 1)
            for (int q = 0; q < NSP; ++q) b.W[(W_NBASE + q) * b.npad + d] = massf[q];
        b.S[d] = 0;
    }
}

// 8-byte asynchronous global -> shared copies of one thread (cp.async; the
// thread waits for its own copies only).
__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Values a run fetches ahead for its next face: the entering cell's rho,
// velocity (its replayed base where it has one), p, u, a, T and length along
// the row, and the face frame n, t1, t2.
constexpr int kRowPrefetch = 18;
constexpr int kRowThreads = 128;

// Faces of a 3-D ideal-gas block (second order, reconstruction in the face
// frame), a run of consecutive faces of one row per thread.  The
// reference's in-place round trips (onedinterp.d:445-454, 576-584) are taken
// literally: the thread holds its four stencil cells with their velocities as
// the reference holds them, turns them into the face frame for the
// reconstruction and back afterwards, and moves on to the next face of the
// row, as the loops of sfluidblock.d:2190-2344 do.  The first face of a run
// starts from the replayed velocities (replay_roundtrips).  Runs of the
// i faces are interleaved across threads (neighbouring threads take
// neighbouring runs of a row); j and k faces are taken with i fastest.
// runs[d]: runs per row of direction d.
// The next face's loads are issued into shared memory (two slots, by face
// parity) before the current face is computed, so their latency hides behind
// its arithmetic.  Launched with kRowThreads threads per block.
// MUTATE: the block's frames are general (b.Vrt holds the replayed bases).
template <int NSP, int FLUX, int GAS, bool MUTATE>
__global__ void __launch_bounds__(kRowThreads) k_flux_rows(BlockView b, const SimDev* sim,
                                                          FluxOpts o, int3 runs) {
    static_assert(NSP == 1, "the row walk serves ideal-gas blocks");
    __shared__ double s_pf[2][kRowPrefetch][kRowThreads];
    const int tid = threadIdx.x;
    if (sim->status != 0 || sim->finished) return;
    // blocks whose frames are all signed unit axes: the round trips are exact
    // (up to the sign of a zero) and the reference copies instead of
    // mutating (its in-place form only serves general frames), so the cells
    // keep their velocities
    constexpr bool mutate = MUTATE;
    const int nrun[3] = {runs.x, runs.y, runs.z};
    long long nd[3];
    for (int d = 0; d < 3; ++d) {
        const long long rows = d == 0 ? (long long)b.nj * b.nk
                                      : (d == 1 ? (long long)b.ni * b.nk : (long long)b.ni * b.nj);
        nd[d] = (d < b.dim) ? rows * nrun[d] : 0;
    }
    const long long n = nd[0] + nd[1] + nd[2];
    constexpr int NSPC = NSP > 1 ? NSP : 0;
    for (long long tt = blockIdx.x * (long long)blockDim.x + threadIdx.x; tt < n;
         tt += (long long)gridDim.x * blockDim.x) {
        int dir = 0;
        long long t = tt;
        if (t >= nd[0]) { t -= nd[0]; dir = 1; }
        if (dir == 1 && t >= nd[1]) { t -= nd[1]; dir = 2; }
        int run, a1, a2;  // run index; the row's coordinates (i, j, k without dir)
        if (dir == 0) {
            run = int(t % nrun[0]);
            a1 = b.jmin + int((t / nrun[0]) % b.nj);
            a2 = b.kmin + int(t / ((long long)nrun[0] * b.nj));
        } else if (dir == 1) {
            a1 = b.imin + int(t % b.ni);
            run = int((t / b.ni) % nrun[1]);
            a2 = b.kmin + int(t / ((long long)b.ni * nrun[1]));
        } else {
            a1 = b.imin + int(t % b.ni);
            a2 = b.jmin + int((t / b.ni) % b.nj);
            run = int(t / ((long long)b.ni * b.nj));
        }
        const int lo = dir == 0 ? b.imin : (dir == 1 ? b.jmin : b.kmin);
        // faces lo .. lo + nf - 1 of the row, in nr runs
        const int nf = (dir == 0 ? b.ni : (dir == 1 ? b.nj : b.nk)) + 1;
        const int nr = dir == 0 ? runs.x : (dir == 1 ? runs.y : runs.z);
        const int g0 = lo + int((long long)run * nf / nr);
        const int g1 = lo + int((long long)(run + 1) * nf / nr);
        const size_t stride = dir == 0 ? 1 : (dir == 1 ? size_t(b.nidim) : size_t(b.nidim) * b.njdim);
        const double* fg = dir == 0 ? b.fgi : (dir == 1 ? b.fgj : b.fgk);
        double* Fo = dir == 0 ? b.Fi : (dir == 1 ? b.Fj : b.Fk);
        const double* len = b.cgeom + size_t(1 + dir) * b.npad;
        auto coords = [&](int x, int& ci, int& cj, int& ck) {
            if (dir == 0) { ci = x; cj = a1; ck = a2; }
            else if (dir == 1) { ci = a1; cj = x; ck = a2; }
            else { ci = a1; cj = a2; ck = x; }
        };
        // stencil window: cells g-2, g-1, g, g+1 of face g, velocities as held
        Prim<double, NSP> w[4];
        double wl[4];
        {
            int ci, cj, ck;
            coords(g0, ci, cj, ck);
            const size_t f0 = pidx(b, ci, cj, ck);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int x = g0 - 2 + q;
                coords(x, ci, cj, ck);
                const size_t c = f0 + (q - 2) * (long long)stride;
                load_prim<NSP>(b, c, w[q]);
                if (mutate) replay_roundtrips(b, dir, g0, ci, cj, ck, c, w[q].vel);
                wl[q] = len[c];
            }
        }
        const int hi = dir == 0 ? b.imax : (dir == 1 ? b.jmax : b.kmax);
        size_t f;
        {
            int ci, cj, ck;
            coords(g0, ci, cj, ck);
            f = pidx(b, ci, cj, ck);
        }
        for (int g = g0; g < g1; ++g, f += stride) {
            Frame<double> fr;
            if (g > g0) {
                // the entering cell g+1 (it has met no face of this row yet:
                // its velocity is its base) and the frame of face g
                cp_async_wait_all();
                const int sl = g & 1;
#pragma unroll
                for (int q = 0; q < 3; ++q) { w[q] = w[q + 1]; wl[q] = wl[q + 1]; }
                w[3].rho = s_pf[sl][0][tid];
                w[3].vel = {s_pf[sl][1][tid], s_pf[sl][2][tid], s_pf[sl][3][tid]};
                w[3].p = s_pf[sl][4][tid];
                w[3].u = s_pf[sl][5][tid];
                w[3].a = s_pf[sl][6][tid];
                w[3].T = s_pf[sl][7][tid];
                w[3].massf[0] = 1.0;
                wl[3] = s_pf[sl][8][tid];
                fr.n = {s_pf[sl][9][tid], s_pf[sl][10][tid], s_pf[sl][11][tid]};
                fr.t1 = {s_pf[sl][12][tid], s_pf[sl][13][tid], s_pf[sl][14][tid]};
                fr.t2 = {s_pf[sl][15][tid], s_pf[sl][16][tid], s_pf[sl][17][tid]};
            } else {
                load_frame(fg, b.npad, f, fr);
            }
            if (g + 1 < g1) {
                // face g+1: its entering cell g+2 (within the two ghost layers)
                // and its frame
                const int sl = (g + 1) & 1;
                const size_t fn = f + stride, c = fn + stride;
                const int x = g + 2;
                const double* V = (mutate && dir > 0 && x >= lo && x <= hi)
                                      ? b.Vrt + size_t(3 * (dir - 1)) * b.npad
                                      : b.W + size_t(W_VX) * b.npad;
                cp_async8(&s_pf[sl][0][tid], b.W + size_t(W_RHO) * b.npad + c);
                cp_async8(&s_pf[sl][1][tid], V + c);
                cp_async8(&s_pf[sl][2][tid], V + b.npad + c);
                cp_async8(&s_pf[sl][3][tid], V + 2 * b.npad + c);
                cp_async8(&s_pf[sl][4][tid], b.W + size_t(W_P) * b.npad + c);
                cp_async8(&s_pf[sl][5][tid], b.W + size_t(W_U) * b.npad + c);
                cp_async8(&s_pf[sl][6][tid], b.W + size_t(W_A) * b.npad + c);
                cp_async8(&s_pf[sl][7][tid], b.W + size_t(W_T) * b.npad + c);
                cp_async8(&s_pf[sl][8][tid], len + c);
#pragma unroll
                for (int q = 0; q < 9; ++q) cp_async8(&s_pf[sl][9 + q][tid], fg + q * b.npad + fn);
                cp_async_commit();
            }
            Prim<double, NSP> sL1 = w[0], sL0 = w[1], sR0 = w[2], sR1 = w[3];
            to_local(sL1.vel, fr.n, fr.t1, fr.t2);
            to_local(sL0.vel, fr.n, fr.t1, fr.t2);
            to_local(sR0.vel, fr.n, fr.t1, fr.t2);
            to_local(sR1.vel, fr.n, fr.t1, fr.t2);
            Prim<double, NSP> Lf = sL0, Rt = sR0;
            {
                L2R2<double> r;
                r.prepare(wl[0], wl[1], wl[2], wl[3]);
                r.scalar(o.limiter, o.clip, sL1.vel.x, sL0.vel.x, sR0.vel.x, sR1.vel.x, Lf.vel.x, Rt.vel.x);
                r.scalar(o.limiter, o.clip, sL1.vel.y, sL0.vel.y, sR0.vel.y, sR1.vel.y, Lf.vel.y, Rt.vel.y);
                r.scalar(o.limiter, o.clip, sL1.vel.z, sL0.vel.z, sR0.vel.z, sR1.vel.z, Lf.vel.z, Rt.vel.z);
                if (NSP > 1) {
#pragma unroll
                    for (int q = 0; q < NSP; ++q)
                        r.scalar(o.limiter, o.clip, sL1.massf[q], sL0.massf[q], sR0.massf[q],
                                 sR1.massf[q], Lf.massf[q], Rt.massf[q]);
                    if (!scale_mass_fractions<double, NSP>(Lf.massf))
                        for (int q = 0; q < NSP; ++q) Lf.massf[q] = sL0.massf[q];
                    if (!scale_mass_fractions<double, NSP>(Rt.massf))
                        for (int q = 0; q < NSP; ++q) Rt.massf[q] = sR0.massf[q];
                } else {
                    Lf.massf[0] = 1.0;
                    Rt.massf[0] = 1.0;
                }
                r.scalar(o.limiter, o.clip, sL1.rho, sL0.rho, sR0.rho, sR1.rho, Lf.rho, Rt.rho);
                r.scalar(o.limiter, o.clip, sL1.u, sL0.u, sR0.u, sR1.u, Lf.u, Rt.u);
            }
            // codeForThermoUpdateBoth("rhou"), onedinterp.d:1039-1068: on failure
            // the cell-centre state (its velocity in the face frame) is taken
            if (!rhou_update<NSP, GAS>(o, Lf)) Lf = sL0;
            if (!rhou_update<NSP, GAS>(o, Rt)) Rt = sR0;
            to_global(Lf.vel, fr.n, fr.t1, fr.t2);
            to_global(Rt.vel, fr.n, fr.t1, fr.t2);
            // the stencil cells back to the global frame in place; cell g-2
            // leaves the window and is not needed again
            if (mutate) {
                to_global(sL0.vel, fr.n, fr.t1, fr.t2);
                to_global(sR0.vel, fr.n, fr.t1, fr.t2);
                to_global(sR1.vel, fr.n, fr.t1, fr.t2);
                w[1].vel = sL0.vel; w[2].vel = sR0.vel; w[3].vel = sR1.vel;
            }
            // compute_interface_flux, fluxcalc.d:26-128 (fixed grid)
            to_local(Lf.vel, fr.n, fr.t1, fr.t2);
            to_local(Rt.vel, fr.n, fr.t1, fr.t2);
            double F[5 + NSPC];
            if (FLUX == 1) {
                hllc<double, NSP, NSPC>(Lf, Rt, F);
            } else if (FLUX == 2) {
                hanel<double, NSP, NSPC>(Lf, Rt, F);
            } else if (FLUX == 3) {
                // (the shear matters only at shock points)
                bool use_hanel = false;
                if (b.S[f - stride] == 1 || b.S[f] == 1) {
                    const double sound_speed = 0.5 * (Lf.a + Rt.a);
                    const double shear_y = fabs(Lf.vel.y - Rt.vel.y) / sound_speed;
                    const double shear_z = fabs(Lf.vel.z - Rt.vel.z) / sound_speed;
                    use_hanel = fmax(shear_y, shear_z) <= o.shear_tol;
                }
                if (use_hanel)
                    hanel<double, NSP, NSPC>(Lf, Rt, F);
                else
                    ausmdv<double, NSP, NSPC>(Lf, Rt, F);
            } else {
                ausmdv<double, NSP, NSPC>(Lf, Rt, F);
            }
            V3<double> m{F[1], F[2], F[3]};
            to_global(m, fr.n, fr.t1, fr.t2);
            F[1] = m.x; F[2] = m.y; F[3] = m.z;
#pragma unroll
            for (int q = 0; q < 5 + NSPC; ++q) Fo[q * b.npad + f] = F[q];
        }
    }
}

// ---------------------------------------------------------------------------
// Cell update: time_derivatives + stage update + decode + validity check
// (fvcell.d:735-875, 1153-1311, 563-732; fluidblock.d:433-499)
// ---------------------------------------------------------------------------
template <int NSP, int GAS>
__global__ void k_update(BlockView b, SimDev* sim, GasConsts gas, int stage, int final_stage) {
    if (sim->status != 0 || sim->finished) return;
    constexpr int NSPC = NSP > 1 ? NSP : 0;
    constexpr int NV = 5 + NSPC;
    const long long n = (long long)b.ni * b.nj * b.nk;
    const double dt = sim->dt_global;
    int bad = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        const size_t c = pidx(b, i, j, k);
        // faces north, east, south, west, top, bottom (sfluidblock.d:506-517)
        const size_t sj = b.nidim, sk = size_t(b.nidim) * b.njdim;
        const double* Fq[6] = {b.Fj, b.Fi, b.Fj, b.Fi, b.Fk, b.Fk};
        const double* Gq[6] = {b.fgj, b.fgi, b.fgj, b.fgi, b.fgk, b.fgk};
        const size_t fq[6] = {c + sj, c + 1, c, c, c + sk, c};
        const double outsign[6] = {1.0, 1.0, -1.0, -1.0, 1.0, -1.0};
        const int nf = (b.dim == 3) ? 6 : 4;
        double integral[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) integral[v] = 0.0;
        for (int q = 0; q < nf; ++q) {
            double area = outsign[q] * Gq[q][9 * b.npad + fq[q]];
            const double* F = Fq[q];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                if (v == 3 && b.dim != 3) continue;
                integral[v] -= F[v * b.npad + fq[q]] * area;
            }
        }
        double vol_inv = 1.0 / b.cgeom[c];
        double Un[NV];
        if (stage == 1) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double d0 = vol_inv * integral[v];
                if (!final_stage) b.dUdt0[v * b.npad + c] = d0;
                Un[v] = b.U0[v * b.npad + c] + dt * 1.0 * d0;
            }
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                double d1 = vol_inv * integral[v];
                Un[v] = b.U0[v * b.npad + c] + dt * (0.5 * b.dUdt0[v * b.npad + c] + 0.5 * d1);
            }
        }
        // decode_conserved (ideal gas; adjust_invalid_cell_data = false,
        // ignore_low_T_thermo_update_failure = true, suggested_low_T_value = 200 K)
        bool data_bad = false;
        double rho = Un[0], vx = 0, vy = 0, vz = 0, u = 0, p = 0, T = 0, a = 0;
        double massf[NSP];
        massf[0] = 1.0;
        if (!(Un[0] > 0.0)) {
            set_status(sim, -5);
            data_bad = true;
        } else {
            double dinv = 1.0 / rho;
            vx = Un[1] * dinv; vy = Un[2] * dinv; vz = Un[3] * dinv;
            u = Un[4] * dinv;
            double ke = 0.5 * (vx * vx + vy * vy + vz * vz);
            u -= ke;
            if (NSPC > 0) {
#pragma unroll
                for (int s = 0; s < NSPC; ++s) massf[s] = Un[5 + s] * dinv;
                if (!scale_mass_fractions<double, NSP>(massf)) { set_status(sim, -6); data_bad = true; }
            }
            bool ok_thermo;
            if (GAS == 0) {
                ok_thermo = ideal_rhou<double>(gas, rho, u, p, T);
            } else {
                // thermally perfect: the Newton starts from the cell's previous T
                TPState<NSP> Q;
                Q.rho = rho; Q.u = u; Q.T = b.W[W_T * b.npad + c];
#pragma unroll
                for (int s = 0; s < NSP; ++s) Q.massf[s] = massf[s];
                TPGas<NSP> g(c_tc);
                ok_thermo = g.rhou(Q);
                p = Q.p; T = Q.T; u = Q.u;
            }
            if (!ok_thermo) {
                T = 200.0;
                if (GAS == 0) {
                    p = rho * gas.Rgas * T;
                    u = gas.Cv * T;
                } else {
                    TPState<NSP> Q;
                    Q.rho = rho; Q.T = T;
#pragma unroll
                    for (int s = 0; s < NSP; ++s) Q.massf[s] = massf[s];
                    TPGas<NSP> g(c_tc);
                    g.rhoT(Q);
                    p = Q.p; u = Q.u;
                }
                // encode_conserved(gtl, ftl)
                Un[0] = rho;
                Un[1] = rho * vx; Un[2] = rho * vy; Un[3] = rho * vz;
                double ke2 = 0.5 * (vx * vx + vy * vy + vz * vz);
                Un[4] = rho * (u + ke2);
#pragma unroll
                for (int s = 0; s < NSPC; ++s) Un[5 + s] = rho * massf[s];
            }
            if (GAS == 0) {
                a = ideal_sound_speed<double>(gas, T);
            } else {
                TPGas<NSP> g(c_tc);
                a = g.sound_speed(massf, T);
            }
        }
        // write the new state
        double* W = b.W;
        W[W_RHO * b.npad + c] = rho;
        W[W_VX * b.npad + c] = vx; W[W_VY * b.npad + c] = vy; W[W_VZ * b.npad + c] = vz;
        W[W_P * b.npad + c] = p; W[W_T * b.npad + c] = T;
        W[W_U * b.npad + c] = u; W[W_A * b.npad + c] = a;
#pragma unroll
        for (int s = 0; s < NSPC; ++s) W[(W_NBASE + s) * b.npad + c] = massf[s];
        if (final_stage) {
#pragma unroll
            for (int v = 0; v < NV; ++v) b.U0[v * b.npad + c] = Un[v];
        }
        // count_invalid_cells / FlowState.check_data (flowstate.d:345-388,
        // gas_state.d:199-241, limits fvcore.d:20-27)
        bool ok = !data_bad;
        if (!isfinite(rho) || rho < 1.01 * 0.0) ok = false;
        if (!isfinite(T) || T < 1.01 * 1.0) ok = false;
        if (!isfinite(p)) ok = false;
        if (!isfinite(a)) ok = false;
        double fsum = 0.0;
        for (int s = 0; s < NSP; ++s) fsum += massf[s];
        if (fsum < 0.99 || fsum > 1.01 || !isfinite(fsum)) ok = false;
        if (fabs(vx) > 30000.0 || fabs(vy) > 30000.0 || fabs(vz) > 30000.0) ok = false;
        if (T < 0.0 || T > 50000.0) ok = false;
        if (!ok) ++bad;
    }
    if (bad) atomicAdd(&sim->bad_cells, bad);
}

// ---------------------------------------------------------------------------
// Chemistry: FVCell.thermochemical_increment for every interior cell
// (simcore.d:1489-1505, fvcell.d:1510-1621), one cell per thread
// ---------------------------------------------------------------------------
template <int NSP>
__device__ __forceinline__ void load_tp(const BlockView& b, size_t c, TPState<NSP>& Q) {
    Q.rho = b.W[W_RHO * b.npad + c];
    Q.p = b.W[W_P * b.npad + c];
    Q.T = b.W[W_T * b.npad + c];
    Q.u = b.W[W_U * b.npad + c];
    Q.a = b.W[W_A * b.npad + c];
#pragma unroll
    for (int s = 0; s < NSP; ++s) Q.massf[s] = b.W[(W_NBASE + s) * b.npad + c];
}

template <int NSP>
__device__ __forceinline__ void store_tp(const BlockView& b, size_t c, const TPState<NSP>& Q,
                                         double dt_chem) {
    b.dt_chem[c] = dt_chem;
    b.W[W_P * b.npad + c] = Q.p;
    b.W[W_T * b.npad + c] = Q.T;
    b.W[W_U * b.npad + c] = Q.u;
    b.W[W_A * b.npad + c] = Q.a;
#pragma unroll
    for (int s = 0; s < NSP; ++s) {
        b.W[(W_NBASE + s) * b.npad + c] = Q.massf[s];
        b.U0[(5 + s) * b.npad + c] = Q.rho * Q.massf[s];
    }
}

__device__ __forceinline__ size_t interior_cell(const BlockView& b, long long t) {
    const int i = b.imin + int(t % b.ni);
    const int j = b.jmin + int((t / b.ni) % b.nj);
    const int k = b.kmin + int(t / ((long long)b.ni * b.nj));
    return pidx(b, i, j, k);
}

__device__ __forceinline__ void add_stats(unsigned long long* stats, int slot, unsigned int v) {
    v = __reduce_add_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && v > 0) atomicAdd(stats + slot, (unsigned long long)v);
}

// Pass 1 over every interior cell: cells whose start state already satisfies
// the point-implicit convergence test are updated here (exactly as the full
// update would); the others are listed in work[] (interior index, i fastest)
// for pass 2, so that the Newton work runs in full warps.
template <int NSP, int NR>
__global__ void k_chem(BlockView b, SimDev* sim, double T_frozen, const double* dt_p, int* work,
                       int* nwork, unsigned long long* stats) {
    if (sim->status != 0 || sim->finished) return;
    const long long n = (long long)b.ni * b.nj * b.nk;
    const double dt = *dt_p;
    unsigned int my_cells = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const size_t c = interior_cell(b, t);
        TPState<NSP> Q;
        load_tp(b, c, Q);
        if (Q.T <= T_frozen) continue;
        my_cells += 1;
        double dt_chem = b.dt_chem[c];
        int rc = thermochemical_increment_d<NSP, NR>(c_tc, T_frozen, Q, dt, dt_chem, nullptr,
                                                     nullptr, true);
        if (rc == CHEM_NEEDS_WORK) {
            work[atomicAdd(nwork, 1)] = int(t);
            continue;
        }
        if (rc != 0) {
            set_status(sim, rc);
            continue;
        }
        store_tp(b, c, Q, dt_chem);
    }
    if (stats) add_stats(stats, 0, my_cells);
}

// Pass 2 over the listed cells: the full point-implicit update, started from
// guess[s * n + w] (w = position in the list; NSP concentrations and T) when
// a guess is given.
template <int NSP, int NR>
__global__ void k_chem_work(BlockView b, SimDev* sim, double T_frozen, const double* dt_p,
                            const int* work, const int* nwork, const double* guess,
                            unsigned long long* stats) {
    if (sim->status != 0 || sim->finished) return;
    const long long n = (long long)b.ni * b.nj * b.nk;
    const int nw = *nwork;
    const double dt = *dt_p;
    unsigned int my_active = 0, my_newton = 0, my_recovered = 0;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
        const size_t c = interior_cell(b, work[w]);
        TPState<NSP> Q;
        load_tp(b, c, Q);
        double g[NSP + 1];
        if (guess) {
#pragma unroll
            for (int s = 0; s <= NSP; ++s) g[s] = guess[s * n + w];
        }
        double dt_chem = b.dt_chem[c];
        ChemCount cnt;
        int rc = thermochemical_increment_d<NSP, NR>(c_tc, T_frozen, Q, dt, dt_chem,
                                                     guess ? g : nullptr, &cnt);
        my_active += 1;
        my_newton += cnt.newton;
        my_recovered += cnt.recovered;
        if (rc != 0) {
            set_status(sim, rc);
            continue;
        }
        store_tp(b, c, Q, dt_chem);
    }
    if (stats) {
        add_stats(stats, 1, my_newton);
        add_stats(stats, 2, my_recovered);
        add_stats(stats, 3, my_active);
    }
}

}  // namespace e4c
