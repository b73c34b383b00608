// e4c_fused.cuh -- fused stage kernel for blocks with uniform, axis-aligned
// geometry (every cell and every face of a direction has identical bits).
//
// One launch performs a whole predictor-corrector stage for every such block:
// ghost cells (computed in the tile loader from the boundary condition),
// MUSCL/van Albada reconstruction, the face flux, the flux divergence in the
// reference's face order, the stage update and the conserved->primitive
// decode.  CTAs are persistent over work items (block, i-j tile, k chunk);
// within an item the CTA marches in k, keeping a ring of four halo planes of
// the primitive state in shared memory, so each plane is read from HBM once
// and each face flux is computed once.
//
// R = double: the plain FP64 form (compiled with -fmad=false; bit-identical
//             to the general path and to the reference algorithm).
// R = float:  the FP32 reconstruction/flux form; fluxes are accumulated,
//             the state updated and decoded in FP64.
#pragma once

#include <cfloat>

#include "e4c_kernels.h"
#include "e4c_physics.cuh"

namespace e4c {

// Fields kept per cell in shared memory: rho, vx, vy, vz, u, a.
constexpr int NF = 6;

template <typename R, int TI, int TJ>
struct FusedSmem {
    static constexpr int PI = TI + 4, PJ = TJ + 4;
    static constexpr int PLANE = NF * PI * PJ;
    // per-cell van Albada values of a plane for its i-faces ([5][TJ][TI+2],
    // cells -1..TI of each row) and j-faces ([5][TJ+2][TI])
    static constexpr int NVI = TJ * (TI + 2), NVJ = (TJ + 2) * TI;
    static constexpr size_t base() {
        return sizeof(R) * (size_t(4) * PLANE + 5 * TJ * (TI + 1) + 5 * (TJ + 1) * TI);
    }
    static constexpr size_t va_bytes() { return sizeof(R) * 5 * size_t(NVI + NVJ); }
};

template <typename R>
__device__ __forceinline__ void reflect_normal(R& vx, R& vy, R& vz, const double* n,
                                               const double* t1, const double* t2) {
    // reflect_normal_velocity, ghost_cell.d:34-44
    V3<R> v{vx, vy, vz};
    Frame<R> fr{{R(n[0]), R(n[1]), R(n[2])}, {R(t1[0]), R(t1[1]), R(t1[2])},
                {R(t2[0]), R(t2[1]), R(t2[2])}};
    to_local(v, fr.n, fr.t1, fr.t2);
    v.x = -(v.x);
    to_global(v, fr.n, fr.t1, fr.t2);
    vx = v.x; vy = v.y; vz = v.z;
}

// Load halo plane kk of a tile into shared-memory slot s.  Ghost cells are
// built from the boundary condition of the face they lie beyond; corner
// ghosts and cells beyond the second ghost layer are never read and skipped.
template <typename R, int TI, int TJ>
__device__ __forceinline__ void load_plane(const FusedDesc* __restrict__ descs, int stage,
                                           const FusedDesc& d, const R* __restrict__ W, int use_a0,
                                           const GasConsts& gas, R* plane, int i0, int j0,
                                           int kk) {
    constexpr int PI = TI + 4, PJ = TJ + 4;
    const size_t nc = size_t(d.ni) * d.nj * d.nk;
    for (int e = threadIdx.x; e < PI * PJ; e += blockDim.x) {
        const int li = e % PI, lj = e / PI;
        int gi = i0 - 2 + li, gj = j0 - 2 + lj, gk = kk;
        const bool oi = gi < 0 || gi >= d.ni;
        const bool oj = gj < 0 || gj >= d.nj;
        const bool ok = gk < 0 || gk >= d.nk;
        if (int(oi) + int(oj) + int(ok) > 1) continue;
        int which = -1, layer = 0;  // boundary and ghost layer (0: first, 1: second)
        if (oi) {
            if (gi < 0) { which = WEST; layer = -gi - 1; }
            else { which = EAST; layer = gi - d.ni; }
        } else if (oj) {
            if (gj < 0) { which = SOUTH; layer = -gj - 1; }
            else { which = NORTH; layer = gj - d.nj; }
        } else if (ok) {
            if (gk < 0) { which = BOTTOM; layer = -gk - 1; }
            else { which = TOP; layer = gk - d.nk; }
        }
        if (layer > 1) continue;
        R rho, vx, vy, vz, u, a;
        int type = which >= 0 ? d.bc[which] : -1;
        if (type == 3) {
            // full-face copy (full_face_copy.d, opposite faces, orientation 0):
            // the partner block's first two cells beyond the joint face
            const FusedDesc& o = descs[d.ex[which]];
            int si = gi, sj = gj, sk = gk;
            switch (which) {
                case WEST: si = o.ni - 1 - layer; break;
                case EAST: si = layer; break;
                case SOUTH: sj = o.nj - 1 - layer; break;
                case NORTH: sj = layer; break;
                case BOTTOM: sk = o.nk - 1 - layer; break;
                default: sk = layer; break;
            }
            const size_t onc = size_t(o.ni) * o.nj * o.nk;
            const size_t c = (size_t(sk) * o.nj + sj) * o.ni + si;
            const R* OW = static_cast<const R*>(stage == 1 ? o.WA : o.WB);
            rho = OW[0 * onc + c]; vx = OW[1 * onc + c]; vy = OW[2 * onc + c];
            vz = OW[3 * onc + c]; u = OW[4 * onc + c];
            if (stage == 1 && *o.use_a0) {
                a = R(o.A0[c]);
            } else {
                R T = u * R(gas.Cvinv);
                a = sqrt(R(gas.gamma) * R(gas.Rgas) * T);
            }
        } else if (type == 1) {  // supersonic inflow: both ghost layers hold the inflow state
            rho = R(d.inflow[0]); vx = R(d.inflow[1]); vy = R(d.inflow[2]); vz = R(d.inflow[3]);
            u = R(d.inflow[4]); a = R(d.inflow[5]);
        } else {
            // source cell: the mirror cell for a slip wall, the first interior
            // cell for the zero-order extrapolation outflow
            if (which >= 0) {
                const int src = (type == 2) ? 0 : layer;
                switch (which) {
                    case WEST: gi = src; break;
                    case EAST: gi = d.ni - 1 - src; break;
                    case SOUTH: gj = src; break;
                    case NORTH: gj = d.nj - 1 - src; break;
                    case BOTTOM: gk = src; break;
                    default: gk = d.nk - 1 - src; break;
                }
            }
            const size_t c = (size_t(gk) * d.nj + gj) * d.ni + gi;
            rho = W[0 * nc + c]; vx = W[1 * nc + c]; vy = W[2 * nc + c]; vz = W[3 * nc + c];
            u = W[4 * nc + c];
            if (use_a0) {
                a = R(d.A0[c]);
            } else {
                // a of the decoded state: update_thermo_from_rhou then update_sound_speed
                R T = u * R(gas.Cvinv);
                a = sqrt(R(gas.gamma) * R(gas.Rgas) * T);
            }
            if (type == 0) {
                // reflect_normal_velocity (ghost_cell.d:34-44) with an axis frame:
                // the normal component changes sign
                if (which == WEST || which == EAST) vx = -vx;
                else if (which == SOUTH || which == NORTH) vy = -vy;
                else vz = -vz;
            }
        }
        R* p = plane + lj * PI + li;
        constexpr int FS = PI * PJ;
        p[0 * FS] = rho; p[1 * FS] = vx; p[2 * FS] = vy; p[3 * FS] = vz; p[4 * FS] = u; p[5 * FS] = a;
    }
}

// Face frames of a Cartesian block are exact cyclic unit permutations:
// i-faces (x, y, z), j-faces (y, z, x), k-faces (z, x, y) as (n, t1, t2).
// transform_to_local_frame / transform_to_global_frame with such a frame
// reduce to a permutation: v.x*1 + v.y*0 + v.z*0 equals v.x up to the sign of
// a zero, which no later operation turns into a different non-zero value.
template <int DIR, typename R>
__device__ __forceinline__ void axis_to_local(V3<R>& v) {
    if (DIR == 1) { R t = v.x; v.x = v.y; v.y = v.z; v.z = t; }
    if (DIR == 2) { R t = v.x; v.x = v.z; v.z = v.y; v.y = t; }
}
template <int DIR, typename R>
__device__ __forceinline__ void axis_to_global(V3<R>& v) {
    if (DIR == 1) { R t = v.z; v.z = v.y; v.y = v.x; v.x = t; }
    if (DIR == 2) { R t = v.x; v.x = v.y; v.y = v.z; v.z = t; }
}

template <typename R>
__device__ __forceinline__ void get_cell(const R* plane, int off, int FS, const GasConsts& gas,
                                         Prim<R, 1>& s) {
    s.rho = plane[off];
    s.vel = {plane[FS + off], plane[2 * FS + off], plane[3 * FS + off]};
    s.u = plane[4 * FS + off];
    s.a = plane[5 * FS + off];
    s.p = R(0.0);  // filled in only when needed (cell_pressure)
    s.massf[0] = R(1.0);
    (void)gas;
}

// Cell-centre pressure of a decoded cell (update_thermo_from_rhou); read only
// when a reconstructed state fails its thermo update and the reference falls
// back to a copy of the cell-centre FlowState.
template <typename R>
__device__ __forceinline__ void cell_pressure(Prim<R, 1>& s, const GasConsts& gas) {
    R T = s.u * R(gas.Cvinv);
    s.p = s.rho * R(gas.Rgas) * T;
}

// Reconstruction + flux of one face from four cells (general-path semantics,
// sfluidblock.d:2190-2344 with onedinterp.d:435-585 and fluxcalc.d:26-128),
// with the face frame of direction DIR applied as a permutation.
//
// vaL, vaR (optional, with the limiter on): the van Albada values of the
// cells L0 and R0 for this direction, at stride vs, in the order rho, vx, vy,
// vz, u of the global frame (L2R2::va).
template <typename R, int FLUX, int DIR>
__device__ __forceinline__ void face_flux(Prim<R, 1> sL1, Prim<R, 1> sL0, Prim<R, 1> sR0,
                                          Prim<R, 1> sR1, const L2R2<R>& w, const FluxOpts& o,
                                          R* F, const R* vaL = nullptr, const R* vaR = nullptr,
                                          int vs = 0, int shock = 0) {
    Prim<R, 1> Lf = sL0, Rt = sR0;
    if (o.order2) {
        if (o.local_frame) {
            axis_to_local<DIR>(sL1.vel);
            axis_to_local<DIR>(sL0.vel);
            axis_to_local<DIR>(sR0.vel);
            axis_to_local<DIR>(sR1.vel);
        }
        const bool lim = o.limiter, clip = o.clip;
        if (vaL) {
            // local x, y, z are the global components DIR, DIR+1, DIR+2 (mod 3)
            const int cx = o.local_frame ? DIR : 0;
            const int c0 = 1 + cx, c1 = 1 + (cx + 1) % 3, c2 = 1 + (cx + 2) % 3;
            w.scalar_with(vaL[c0 * vs], vaR[c0 * vs], clip, sL1.vel.x, sL0.vel.x, sR0.vel.x,
                          sR1.vel.x, Lf.vel.x, Rt.vel.x);
            w.scalar_with(vaL[c1 * vs], vaR[c1 * vs], clip, sL1.vel.y, sL0.vel.y, sR0.vel.y,
                          sR1.vel.y, Lf.vel.y, Rt.vel.y);
            w.scalar_with(vaL[c2 * vs], vaR[c2 * vs], clip, sL1.vel.z, sL0.vel.z, sR0.vel.z,
                          sR1.vel.z, Lf.vel.z, Rt.vel.z);
        } else {
            w.scalar(lim, clip, sL1.vel.x, sL0.vel.x, sR0.vel.x, sR1.vel.x, Lf.vel.x, Rt.vel.x);
            w.scalar(lim, clip, sL1.vel.y, sL0.vel.y, sR0.vel.y, sR1.vel.y, Lf.vel.y, Rt.vel.y);
            w.scalar(lim, clip, sL1.vel.z, sL0.vel.z, sR0.vel.z, sR1.vel.z, Lf.vel.z, Rt.vel.z);
        }
        Lf.massf[0] = R(1.0);
        Rt.massf[0] = R(1.0);
        if (vaL) {
            w.scalar_with(vaL[0], vaR[0], clip, sL1.rho, sL0.rho, sR0.rho, sR1.rho, Lf.rho, Rt.rho);
            w.scalar_with(vaL[4 * vs], vaR[4 * vs], clip, sL1.u, sL0.u, sR0.u, sR1.u, Lf.u, Rt.u);
        } else {
            w.scalar(lim, clip, sL1.rho, sL0.rho, sR0.rho, sR1.rho, Lf.rho, Rt.rho);
            w.scalar(lim, clip, sL1.u, sL0.u, sR0.u, sR1.u, Lf.u, Rt.u);
        }
        R T;
        if (!ideal_rhou<R>(o.gas, Lf.rho, Lf.u, Lf.p, T)) { Lf = sL0; cell_pressure(Lf, o.gas); }
        if (!ideal_rhou<R>(o.gas, Rt.rho, Rt.u, Rt.p, T)) { Rt = sR0; cell_pressure(Rt, o.gas); }
        // transform back to the global frame (onedinterp.d:576-584) and into the
        // face frame again (fluxcalc.d:50-52): together an identity here
        if (!o.local_frame) {
            axis_to_local<DIR>(Lf.vel);
            axis_to_local<DIR>(Rt.vel);
        }
    } else {
        cell_pressure(Lf, o.gas);
        cell_pressure(Rt, o.gas);
        axis_to_local<DIR>(Lf.vel);
        axis_to_local<DIR>(Rt.vel);
    }
    if (FLUX == 1) {
        hllc<R, 1, 0>(Lf, Rt, F);
    } else if (FLUX == 2) {
        hanel<R, 1, 0>(Lf, Rt, F);
    } else if (FLUX == 3) {
        // adaptive_hanel_ausmdv (fluxcalc.d:824-838): Hanel where either
        // cell is a shock point and the shear is small, AUSMDV elsewhere
        // (the shear matters only at shock points)
        bool use_hanel = false;
        if (shock) {
            const R sound_speed = R(0.5) * (Lf.a + Rt.a);
            const R shear_y = fabs(Lf.vel.y - Rt.vel.y) / sound_speed;
            const R shear_z = fabs(Lf.vel.z - Rt.vel.z) / sound_speed;
            use_hanel = fmax(shear_y, shear_z) <= R(o.shear_tol);
        }
        if (use_hanel) hanel<R, 1, 0>(Lf, Rt, F);
        else ausmdv<R, 1, 0>(Lf, Rt, F);
    } else {
        ausmdv<R, 1, 0>(Lf, Rt, F);
    }
    V3<R> m{F[1], F[2], F[3]};
    axis_to_global<DIR>(m);
    F[1] = m.x; F[2] = m.y; F[3] = m.z;
}

// detect_shock_points (fluidblock.d:415-431) with PJ_ShockDetector
// (shockdetectors.d:20-59) for the cell at offset off of plane p0 (pm and pp
// the planes below and above): a face flags compression when
// (uR - uL) / min(aL, aR) < tol, u the velocity along the face normal (an
// axis here, so the component itself: v.n = v.x*1 + v.y*0 + v.z*0 differs
// from it at most in the sign of a zero, which the test cannot see); the
// cell is a shock point if any of its six faces does.
template <typename R, int PI>
__device__ __forceinline__ int cell_shock(const R* pm, const R* p0, const R* pp, int off, int FS,
                                          double tol) {
    auto face = [tol](double uL, double uR, double aL, double aR) {
        const double a_min = (aL < aR) ? aL : aR;
        return quotient_below(uR - uL, a_min, tol) ? 1 : 0;
    };
    const R a = p0[5 * FS + off];
    int S = 0;
    S |= face(p0[FS + off - 1], p0[FS + off], p0[5 * FS + off - 1], a);
    S |= face(p0[FS + off], p0[FS + off + 1], a, p0[5 * FS + off + 1]);
    S |= face(p0[2 * FS + off - PI], p0[2 * FS + off], p0[5 * FS + off - PI], a);
    S |= face(p0[2 * FS + off], p0[2 * FS + off + PI], a, p0[5 * FS + off + PI]);
    S |= face(pm[3 * FS + off], p0[3 * FS + off], pm[5 * FS + off], a);
    S |= face(p0[3 * FS + off], pp[3 * FS + off], a, pp[5 * FS + off]);
    return S;
}

// The flag of the first ghost cell beyond one face of block d at (gi, gj,
// gk) (exactly one index outside): what the boundary condition copied at the
// start of the stage, i.e. the previous stage's flag of the cell the ghost
// copies (the mirror or first interior cell for walls and outflow, the
// partner's cell across a joint), 0 for an inflow.
__device__ __forceinline__ int ghost_shock(const FusedDesc* __restrict__ descs, const FusedDesc& d,
                                           int stage, int gi, int gj, int gk) {
    const int prev = (stage == 1) ? 1 : 0;
    int which;
    if (gi < 0) which = WEST;
    else if (gi >= d.ni) which = EAST;
    else if (gj < 0) which = SOUTH;
    else if (gj >= d.nj) which = NORTH;
    else if (gk < 0) which = BOTTOM;
    else which = TOP;
    const int type = d.bc[which];
    if (type == 1) return 0;
    if (type == 3) {
        const FusedDesc& o = descs[d.ex[which]];
        if (!o.S[prev]) return 0;
        int si = gi, sj = gj, sk = gk;
        switch (which) {
            case WEST: si = o.ni - 1; break;
            case EAST: si = 0; break;
            case SOUTH: sj = o.nj - 1; break;
            case NORTH: sj = 0; break;
            case BOTTOM: sk = o.nk - 1; break;
            default: sk = 0; break;
        }
        return o.S[prev][(size_t(sk) * o.nj + sj) * o.ni + si];
    }
    switch (which) {
        case WEST: gi = 0; break;
        case EAST: gi = d.ni - 1; break;
        case SOUTH: gj = 0; break;
        case NORTH: gj = d.nj - 1; break;
        case BOTTOM: gk = 0; break;
        default: gk = d.nk - 1; break;
    }
    return d.S[prev][(size_t(gk) * d.nj + gj) * d.ni + gi];
}

template <typename R>
__device__ __forceinline__ Frame<R> frame_of(const FusedDesc& d, int dir) {
    Frame<R> f;
    f.n = {R(d.fn[dir][0]), R(d.fn[dir][1]), R(d.fn[dir][2])};
    f.t1 = {R(d.ft1[dir][0]), R(d.ft1[dir][1]), R(d.ft1[dir][2])};
    f.t2 = {R(d.ft2[dir][0]), R(d.ft2[dir][1]), R(d.ft2[dir][2])};
    return f;
}

__device__ __forceinline__ int find_block(const FusedDesc* descs, int nblocks, long long item) {
    int lo = 0, hi = nblocks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (descs[mid].item0 <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Threads of a fused CTA: one per cell of the tile.
template <int TI, int TJ>
struct FusedThreads {
    static constexpr int cells = TI * TJ;
    static constexpr int total = TI * TJ;
};

// The i- and j-faces of a plane, (TI+1)*TJ + TI*(TJ+1) of them, are one list.
// Full passes use every thread; the TI+TJ faces left over for the last pass go
// to the first threads, one each, so only the first warps take that pass and
// the others go on to their k-face (dense: 1.7 % faster on the 256^3 block
// with the 32x16 tile than three faces in each of the 16 warps).
template <int TI, int TJ>
struct FaceList {
    static constexpr int NT = TI * TJ;
    static constexpr int N = (TI + 1) * TJ + TI * (TJ + 1);
    static constexpr int FULL = N / NT;                 // passes with every thread
    static constexpr int REM = N - FULL * NT;           // faces left for the last pass
    __device__ static int face(int pass, int tid) {
        if (pass < FULL) return pass * NT + tid;
        const int f = FULL * NT + tid;
        return f < N ? f : -1;
    }
    static constexpr int passes = FULL + (REM > 0 ? 1 : 0);
};

// Blocks per SM the launch bounds ask for: a resident-warp target per SM
// (FP64: 16 warps, i.e. 128 registers; FP32: 32 warps, 64 registers without
// spills, measured 2 % ahead of 24 warps and 20 % ahead of 16) divided by the
// warps of one CTA of the tile shape.
#ifndef E4C_FUSED_WARPS64
#define E4C_FUSED_WARPS64 16
#endif
#ifndef E4C_FUSED_WARPS32
#define E4C_FUSED_WARPS32 32
#endif
template <typename R, int TI, int TJ>
struct FusedMinBlocks {
    static constexpr int warps = (sizeof(R) == 8 ? E4C_FUSED_WARPS64 : E4C_FUSED_WARPS32);
    static constexpr int per_cta = (TI * TJ) / 32;
    static constexpr int value = warps / per_cta > 0 ? warps / per_cta : 1;
};

// The per-cell limiter values take shared memory of their own and a barrier
// per plane; they halve the FP64 divisions of the limiter (measured 3 % on the
// 256^3 block with the 32x16 tile), while in FP32 (approximate division) the
// barrier costs more than they save.  A tile shape keeps them where they fit
// beside the CTAs per SM its launch bounds ask for (228 KB per SM, 1 KB
// reserved per CTA, 227 KB per CTA).
template <typename R, int TI, int TJ>
struct FusedShareVA {
    using S = FusedSmem<R, TI, TJ>;
    static constexpr size_t with = S::base() + S::va_bytes();
    static constexpr bool value = sizeof(R) == 8 && with <= 227 * 1024 &&
                                  FusedMinBlocks<R, TI, TJ>::value * (with + 1024) <= 228 * 1024;
    static constexpr size_t bytes() { return value ? with : S::base(); }
};

// The fused stage.  stage 1: W=WA -> WB, writes dUdt0; stage 2: W=WB -> WA,
// writes U0 (the end-of-step state).
template <typename R, int FLUX, int TI, int TJ>
__global__ void __launch_bounds__(FusedThreads<TI, TJ>::total, FusedMinBlocks<R, TI, TJ>::value)
k_fused_stage(const FusedDesc* __restrict__ descs, int nblocks, long long nitems, int kc,
              SimDev* sim, GasConsts gas, FluxOpts o, int stage, const int* __restrict__ order) {
    // one decision per CTA (another CTA may set the status while this one
    // starts): every thread leaves, or none
    __shared__ int s_stop;
    if (threadIdx.x == 0) s_stop = (sim->status != 0 || sim->finished) ? 1 : 0;
    __syncthreads();
    if (s_stop) return;
    // CTAs take work items from a counter, costliest first; the other stage's
    // counter is reset for its next launch (it is not in use now)
    if (blockIdx.x == 0 && threadIdx.x == 0) sim->item_next[stage == 1 ? 1 : 0] = 0u;
    __shared__ unsigned int s_item;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using S = FusedSmem<R, TI, TJ>;
    constexpr int PI = S::PI, PJ = S::PJ, FS = PI * PJ;
    R* planes = reinterpret_cast<R*>(smem_raw);
    R* Fi = planes + 4 * S::PLANE;              // [5][TJ][TI+1]
    R* Fj = Fi + 5 * TJ * (TI + 1);             // [5][TJ+1][TI]
    R* VAi = Fj + 5 * (TJ + 1) * TI;            // [5][TJ][TI+2] (FusedShareVA)
    R* VAj = VAi + 5 * S::NVI;                  // [5][TJ+2][TI]
    const bool share_va = FusedShareVA<R, TI, TJ>::value && o.order2 && o.limiter;
    const bool cell_thread = threadIdx.x < FusedThreads<TI, TJ>::cells;
    const int ti = threadIdx.x % TI, tj = threadIdx.x / TI;
    const double dt = sim->dt_global;
    int bad = 0;
    // adaptive flux: shock flags of two planes (the tile and its one-cell
    // ring, pitch TI + 2), this thread's cell's in registers
    constexpr bool ADAPT = (FLUX == 3);
    constexpr int SP = TI + 2;
    constexpr int RING = 2 * (TI + TJ);
    static_assert(RING <= TI * TJ, "the ring's flags take one thread each");
    __shared__ unsigned char s_S[2][ADAPT ? SP * (TJ + 2) : 1];

    for (;;) {
        __syncthreads();  // s_item of the previous item has been read by all
        if (threadIdx.x == 0) s_item = atomicAdd(&sim->item_next[stage == 1 ? 0 : 1], 1u);
        __syncthreads();
        if (s_item >= (unsigned long long)nitems) break;
        const long long item = order[s_item];
        const int b = find_block(descs, nblocks, item);
        const FusedDesc& d = descs[b];
        long long local = item - d.item0;
        const int kch = int(local % d.kchunks);
        local /= d.kchunks;
        const int tile_i = int(local % d.tiles_i), tile_j = int(local / d.tiles_i);
        const int i0 = tile_i * TI, j0 = tile_j * TJ;
        const int k0 = kch * kc, k1 = min(k0 + kc, d.nk);
        const int i = i0 + ti, j = j0 + tj;
        const bool active = cell_thread && i < d.ni && j < d.nj;
        const size_t nc = size_t(d.ni) * d.nj * d.nk;
        const R* __restrict__ Win = static_cast<const R*>(stage == 1 ? d.WA : d.WB);
        R* __restrict__ Wout = static_cast<R*>(stage == 1 ? d.WB : d.WA);
        const int use_a0 = (stage == 1) ? *d.use_a0 : 0;

        // l2r2_prepare with the (uniform) cell lengths of each direction
        L2R2<R> w[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) w[q].prepare(R(d.len[q]), R(d.len[q]), R(d.len[q]), R(d.len[q]));

        // prologue: planes k0-2 .. k0+1
        __syncthreads();
        for (int kk = k0 - 2; kk <= k0 + 1; ++kk)
            load_plane<R, TI, TJ>(descs, stage, d, Win, use_a0, gas, planes + ((kk + 8) & 3) * S::PLANE, i0, j0, kk);
        __syncthreads();
        // the shock flag of tile position (li, lj) (-1..TI, -1..TJ) in plane
        // kk, from planes kk-1..kk+1; the first ghost cell beyond a face
        // takes its boundary's copy
        auto flag_at = [&](int li, int lj, int kk) -> int {
            const int gi = i0 + li, gj = j0 + lj;
            const int out = int(gi < 0 || gi >= d.ni) + int(gj < 0 || gj >= d.nj) +
                            int(kk < 0 || kk >= d.nk);
            if (out == 1) return ghost_shock(descs, d, stage, gi, gj, kk);
            if (out > 1) return 0;
            return cell_shock<R, PI>(planes + ((kk - 1 + 8) & 3) * S::PLANE,
                                     planes + ((kk + 8) & 3) * S::PLANE,
                                     planes + ((kk + 1 + 8) & 3) * S::PLANE,
                                     (lj + 2) * PI + (li + 2), FS, o.compression_tol);
        };
        // flags of plane kk into slot kk & 1: each thread its own position,
        // the first threads the ring; returns this thread's own flag
        auto flag_plane = [&](int kk) -> int {
            int own = 0;
            if (cell_thread) {
                own = flag_at(ti, tj, kk);
                s_S[kk & 1][(tj + 1) * SP + ti + 1] = (unsigned char)own;
            }
            if (threadIdx.x < RING) {
                int li, lj;
                const int r = threadIdx.x;
                if (r < 2 * TJ) { li = (r & 1) ? TI : -1; lj = r >> 1; }
                else { li = (r - 2 * TJ) >> 1; lj = ((r - 2 * TJ) & 1) ? TJ : -1; }
                s_S[kk & 1][(lj + 1) * SP + li + 1] = (unsigned char)flag_at(li, lj, kk);
            }
            return own;
        };
        int s_cur = 0, s_below = 0;
        if (ADAPT) {
            if (active) s_below = flag_at(ti, tj, k0 - 1);
            s_cur = flag_plane(k0);
        }
        R Fbot[5];
        const int coff = (tj + 2) * PI + (ti + 2);
        if (active) {
            Prim<R, 1> c0, c1, c2, c3;
            get_cell(planes + ((k0 - 2 + 8) & 3) * S::PLANE, coff, FS, gas, c0);
            get_cell(planes + ((k0 - 1 + 8) & 3) * S::PLANE, coff, FS, gas, c1);
            get_cell(planes + ((k0 + 8) & 3) * S::PLANE, coff, FS, gas, c2);
            get_cell(planes + ((k0 + 1 + 8) & 3) * S::PLANE, coff, FS, gas, c3);
            face_flux<R, FLUX, 2>(c0, c1, c2, c3, w[2], o, Fbot, nullptr, nullptr, 0,
                                  s_below | s_cur);
        }
        __syncthreads();  // plane k0-2 is overwritten by the first load below
        for (int k = k0; k < k1; ++k) {
            // plane k+2 replaces plane k-2 (not read since the previous iteration)
            load_plane<R, TI, TJ>(descs, stage, d, Win, use_a0, gas, planes + ((k + 2 + 8) & 3) * S::PLANE, i0, j0,
                                  k + 2);
            const R* pk = planes + ((k + 8) & 3) * S::PLANE;
            if (share_va) {
                // van Albada values of the cells of this plane that the i- and
                // j-faces below use (cells -1..n of each direction)
                for (int e = threadIdx.x; e < S::NVI + S::NVJ; e += blockDim.x) {
                    int off, step, dir;
                    R* dst;
                    int vs;
                    if (e < S::NVI) {
                        const int ci = e % (TI + 2), cj = e / (TI + 2);
                        if (i0 + ci - 1 > d.ni || j0 + cj >= d.nj) continue;
                        off = (cj + 2) * PI + (ci + 1);
                        step = 1; dir = 0; dst = VAi + e; vs = S::NVI;
                    } else {
                        const int g = e - S::NVI;
                        const int ci = g % TI, cj = g / TI;
                        if (i0 + ci >= d.ni || j0 + cj - 1 > d.nj) continue;
                        off = (cj + 1) * PI + (ci + 2);
                        step = PI; dir = 1; dst = VAj + g; vs = S::NVJ;
                    }
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const R* q = pk + f * FS + off;
                        dst[f * vs] = w[dir].va(q[-step], q[0], q[step]);
                    }
                }
            }
            // plane k+2 and the limiter values of plane k are in place (plane k
            // was loaded two iterations ago: the values need no barrier of
            // their own, and the loads overlap their divisions)
            __syncthreads();
            // shock flags of plane k+1 (slot (k+1) & 1, last read by the
            // previous plane's faces); the ring's are read after the next
            // plane's barrier, this thread's own at once
            int s_next = 0;
            if (ADAPT) s_next = flag_plane(k + 1);
            const unsigned char* sk_ = s_S[k & 1];
            // i-faces, (TI+1) x TJ (face fi is the west face of cell i0+fi), then
            // j-faces, TI x (TJ+1) (face fj is the south face of cell j0+fj), as
            // one list over all the CTA's threads
            constexpr int NFI = (TI + 1) * TJ;
            for (int pass = 0; pass < FaceList<TI, TJ>::passes; ++pass) {
                const int f = FaceList<TI, TJ>::face(pass, threadIdx.x);
                if (f < 0) continue;
                if (f < NFI) {
                    const int fi = f % (TI + 1), fj = f / (TI + 1);
                    if (i0 + fi > d.ni || j0 + fj >= d.nj) continue;
                    const int off = (fj + 2) * PI + fi;
                    Prim<R, 1> a0, a1, a2, a3;
                    get_cell(pk, off, FS, gas, a0);
                    get_cell(pk, off + 1, FS, gas, a1);
                    get_cell(pk, off + 2, FS, gas, a2);
                    get_cell(pk, off + 3, FS, gas, a3);
                    R F[5];
                    const int sh = ADAPT ? (sk_[(fj + 1) * SP + fi] | sk_[(fj + 1) * SP + fi + 1]) : 0;
                    if (share_va) {
                        const R* v = VAi + fj * (TI + 2) + fi;
                        face_flux<R, FLUX, 0>(a0, a1, a2, a3, w[0], o, F, v, v + 1, S::NVI, sh);
                    } else {
                        face_flux<R, FLUX, 0>(a0, a1, a2, a3, w[0], o, F, nullptr, nullptr, 0, sh);
                    }
#pragma unroll
                    for (int v = 0; v < 5; ++v) Fi[(v * TJ + fj) * (TI + 1) + fi] = F[v];
                } else {
                    const int g = f - NFI;
                    const int fi = g % TI, fj = g / TI;
                    if (i0 + fi >= d.ni || j0 + fj > d.nj) continue;
                    const int off = fj * PI + (fi + 2);
                    Prim<R, 1> a0, a1, a2, a3;
                    get_cell(pk, off, FS, gas, a0);
                    get_cell(pk, off + PI, FS, gas, a1);
                    get_cell(pk, off + 2 * PI, FS, gas, a2);
                    get_cell(pk, off + 3 * PI, FS, gas, a3);
                    R F[5];
                    const int sh = ADAPT ? (sk_[fj * SP + fi + 1] | sk_[(fj + 1) * SP + fi + 1]) : 0;
                    if (share_va) {
                        const R* v = VAj + fj * TI + fi;
                        face_flux<R, FLUX, 1>(a0, a1, a2, a3, w[1], o, F, v, v + TI, S::NVJ, sh);
                    } else {
                        face_flux<R, FLUX, 1>(a0, a1, a2, a3, w[1], o, F, nullptr, nullptr, 0, sh);
                    }
#pragma unroll
                    for (int v = 0; v < 5; ++v) Fj[(v * (TJ + 1) + fj) * TI + fi] = F[v];
                }
            }
            // k-face on top of cell k, from planes k-1 .. k+2 of this column
            R Ftop[5];
            if (active) {
                Prim<R, 1> c0, c1, c2, c3;
                get_cell(planes + ((k - 1 + 8) & 3) * S::PLANE, coff, FS, gas, c0);
                get_cell(pk, coff, FS, gas, c1);
                get_cell(planes + ((k + 1 + 8) & 3) * S::PLANE, coff, FS, gas, c2);
                get_cell(planes + ((k + 2 + 8) & 3) * S::PLANE, coff, FS, gas, c3);
                face_flux<R, FLUX, 2>(c0, c1, c2, c3, w[2], o, Ftop, nullptr, nullptr, 0,
                                      s_cur | s_next);
            }
            __syncthreads();
            if (active) {
                // time_derivatives: faces north, east, south, west, top, bottom
                const double aN = d.area[1], aE = d.area[0], aT = d.area[2];
                double integral[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    double s = 0.0;
                    s -= double(Fj[(v * (TJ + 1) + tj + 1) * TI + ti]) * (1.0 * aN);
                    s -= double(Fi[(v * TJ + tj) * (TI + 1) + ti + 1]) * (1.0 * aE);
                    s -= double(Fj[(v * (TJ + 1) + tj) * TI + ti]) * (-1.0 * aN);
                    s -= double(Fi[(v * TJ + tj) * (TI + 1) + ti]) * (-1.0 * aE);
                    s -= double(Ftop[v]) * (1.0 * aT);
                    s -= double(Fbot[v]) * (-1.0 * aT);
                    integral[v] = s;
                }
                const double vol_inv = 1.0 / d.vol;
                const size_t c = (size_t(k) * d.nj + j) * d.ni + i;
                double Un[5];
                if (stage == 1) {
#pragma unroll
                    for (int v = 0; v < 5; ++v) {
                        const double d0 = vol_inv * integral[v];
                        d.dUdt0[v * nc + c] = d0;
                        Un[v] = d.U0[v * nc + c] + dt * 1.0 * d0;
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < 5; ++v) {
                        const double d1 = vol_inv * integral[v];
                        Un[v] = d.U0[v * nc + c] + dt * (0.5 * d.dUdt0[v * nc + c] + 0.5 * d1);
                    }
                }
                // decode_conserved (fvcell.d:563-732), ideal gas
                bool ok = true;
                double rho = Un[0], vx = 0.0, vy = 0.0, vz = 0.0, u = 0.0, p = 0.0, T = 0.0, a = 0.0;
                if (!(Un[0] > 0.0)) {
                    if (atomicCAS(&sim->status, 0, -5) == 0) sim->status_step = sim->step;
                    ok = false;
                } else {
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
                }
                Wout[0 * nc + c] = R(rho);
                Wout[1 * nc + c] = R(vx); Wout[2 * nc + c] = R(vy); Wout[3 * nc + c] = R(vz);
                Wout[4 * nc + c] = R(u);
                if (stage == 2) {
#pragma unroll
                    for (int v = 0; v < 5; ++v) d.U0[v * nc + c] = Un[v];
                }
                // FlowState.check_data (flowstate.d:345-388)
                if (!isfinite(rho) || rho < 0.0) ok = false;
                if (!isfinite(T) || T < 1.01) ok = false;
                if (!isfinite(p) || !isfinite(a)) ok = false;
                if (fabs(vx) > 30000.0 || fabs(vy) > 30000.0 || fabs(vz) > 30000.0) ok = false;
                if (T > 50000.0) ok = false;
                if (!ok) ++bad;
#pragma unroll
                for (int v = 0; v < 5; ++v) Fbot[v] = Ftop[v];
                if (ADAPT) d.S[stage == 1 ? 0 : 1][c] = (unsigned char)s_cur;
            }
            s_cur = s_next;
            // no barrier here: the update reads only Fi/Fj (rewritten after the
            // next plane's load barrier) and its own registers; the next load
            // overwrites plane k-1, last read by this plane's k-faces
        }
    }
    if (stage == 2 && blockIdx.x == 0 && threadIdx.x == 0) {
        // from now on the sound speed comes from the decoded state
        for (int b = 0; b < nblocks; ++b) *descs[b].use_a0 = 0;
    }
    if (bad) atomicAdd(&sim->bad_cells, bad);
}

// signal_frequency + block min/max of one fused block (fvcell.d:1624-1705,
// fluidblock.d:776-862): the cells this thread strides over, a warp
// reduction, one atomic per warp into acc[0] (min dt) and acc[1] (max CFL);
// the last cell's signal goes to acc[2].
template <typename R>
__device__ __forceinline__ void fused_dt_cells(const FusedDesc& d, const GasConsts& gas,
                                               double cfl_value, double dt_current,
                                               unsigned long long* acc) {
    const long long nc = (long long)d.ni * d.nj * d.nk;
    const R* W = static_cast<const R*>(d.WA);
    const V3<double> nN{d.fn[1][0], d.fn[1][1], d.fn[1][2]};
    const V3<double> nE{d.fn[0][0], d.fn[0][1], d.fn[0][2]};
    const V3<double> nT{d.fn[2][0], d.fn[2][1], d.fn[2][2]};
    const int use_a0 = *d.use_a0;
    double dmin = DBL_MAX, cmax = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
         c += (long long)gridDim.x * blockDim.x) {
        V3<double> v{double(W[1 * nc + c]), double(W[2 * nc + c]), double(W[3 * nc + c])};
        double a;
        if (use_a0) {
            a = d.A0[c];
        } else {
            double T = double(W[4 * nc + c]) * gas.Cvinv;
            a = sqrt(gas.gamma * gas.Rgas * T);
        }
        const double un_N = fabs(dot3(v, nN));
        const double un_E = fabs(dot3(v, nE));
        const double un_T = fabs(dot3(v, nT));
        double signal = 0.0;
        signal = fmax(signal, (un_N + a) / d.len[1]);
        signal = fmax(signal, (un_E + a) / d.len[0]);
        signal = fmax(signal, (un_T + a) / d.len[2]);
        dmin = fmin(dmin, cfl_value / signal);
        cmax = fmax(cmax, dt_current * signal);
        if (c == nc - 1) acc[2] = dbits(signal);
    }
    for (int off = 16; off > 0; off >>= 1) {
        dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, off));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&acc[0], dbits(dmin));
        atomicMax(&acc[1], dbits(cmax));
    }
}

// The dt reduction for the fused layout.  With a descriptor table, one launch
// covers all fused blocks (blockIdx.y picks the block, accumulators from the
// descriptor).  Without one (descs == nullptr), the launch covers the single
// block `one` passed by value, into the accumulators `one_acc`: the
// allocation-free dt control uses this form, so both give the same bits.
template <typename R>
__global__ void k_fused_dt(const FusedDesc* __restrict__ descs, FusedDesc one,
                           unsigned long long* one_acc, SimDev* sim, GasConsts gas,
                           double cfl_value, const double* dt_current_p) {
    if (sim && (sim->status != 0 || sim->finished)) return;
    const double dt_current = *dt_current_p;
    if (descs) {
        const FusedDesc& d = descs[blockIdx.y];
        fused_dt_cells<R>(d, gas, cfl_value, dt_current, d.acc);
    } else {
        fused_dt_cells<R>(one, gas, cfl_value, dt_current, one_acc);
    }
}

}  // namespace e4c
