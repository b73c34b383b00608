// e4c_fused_ws.cuh -- the fused stage of the FP32-flux form for tiles 32 cells
// wide (i) and TJ rows (j), marching in k over a chunk of planes.
//
// The CTA has two kinds of warps:
//   cell warps (TJ of them): warp w owns tile row j = w, lane l the cell
//     i = l.  Per plane each thread reconstructs its own cell once per
//     direction (the MUSCL values at the cell's low and high faces, with the
//     cell's van Albada value), computes the west, south and top faces of
//     its cell, and updates and decodes the cell;
//   edge warps (two): load the halo plane three planes ahead into a ring of
//     four shared-memory slots with cp.async (ghost cells from the boundary
//     conditions), reconstruct the halo cells around the tile, and compute
//     the faces on the tile's east and north edges.
// So every cell thread does exactly three faces per plane; a face reads the
// reconstructed values of its two cells rather than reconstructing from four,
// and each warp reads one 32-cell row of shared memory at a time (no bank
// conflicts).  Two barriers per plane: after the reconstruction (and the
// halo), and after the faces.
//
// On uniform grids the left state of a face is a function of its left cell
// and that cell's two neighbours alone (the MUSCL weights and the van Albada
// value are those of the cell: onedinterp.d:136-162 with equal lengths), so
// reconstructing per cell gives what the per-face form gives; the FP32 form
// is checked against the FP64 oracle with a tolerance.
#pragma once

#include "e4c_fused.cuh"

namespace e4c {
namespace ws {

constexpr int TI = 32;
constexpr int PI = TI + 4;     // ring row pitch: cells i0-2 .. i0+33
constexpr int NEW = 2;         // edge warps per CTA
constexpr int NE = 32 * NEW;   // edge threads

#ifndef E4C_WS_WARPS
// resident warps per SM the launch bounds aim at: 20 (two 10-warp CTAs of the
// 32x8 tile, up to 96 registers a thread, no spills) measured 4.6 % ahead of
// 30 warps at 64 registers with spills on the 256^3 block
#define E4C_WS_WARPS 20
#endif

template <int TJ>
struct Lay {
    // two bits per plane position an edge thread handles (queue_plane)
    static_assert(PI * (TJ + 4) <= 16 * NE, "tile too tall for the edge threads' fixups");
    static constexpr int PJ = TJ + 4;             // ring rows: j0-2 .. j0+TJ+1
    static constexpr int PLANE = PI * PJ;         // one field of one plane
    static constexpr int QI = TJ * (TI + 2);      // [row 0..TJ-1][i -1..32]
    static constexpr int QJ = (TJ + 2) * TI;      // [row -1..TJ][i 0..31]
    static constexpr int AN = (TJ + 2) * (TI + 2);  // [row -1..TJ][i -1..32]
    static constexpr int FI = TJ * (TI + 1);      // i-faces [row][face 0..32]
    static constexpr int FJ = (TJ + 1) * TI;      // j-faces [face row 0..TJ][i]
    static constexpr int o_qip = 20 * PLANE;      // ring: 4 slots x 5 fields
    static constexpr int o_qim = o_qip + 5 * QI;
    static constexpr int o_qjp = o_qim + 5 * QI;
    static constexpr int o_qjm = o_qjp + 5 * QJ;
    static constexpr int o_a = o_qjm + 5 * QJ;
    static constexpr int o_fi = o_a + AN;
    static constexpr int o_fj = o_fi + 5 * FI;
    static constexpr int words = o_fj + 5 * FJ;
    static constexpr size_t bytes = sizeof(float) * size_t(words);
    static constexpr int threads = 32 * (TJ + NEW);
    static constexpr int min_blocks =
        (E4C_WS_WARPS / (TJ + NEW)) > 0 ? E4C_WS_WARPS / (TJ + NEW) : 1;
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// MUSCL values of one scalar at a cell's high (hi) and low (lo) faces from
// the cell and its two neighbours along one direction (interp_l2r2_scalar,
// onedinterp.d:136-162, for a uniform grid: the left state of a face is its
// left cell's hi, the right state its right cell's lo).  With equal cell
// lengths len the weights reduce to hi = q0 + s (3 b + a) / 8 and
// lo = q0 - s (b + 3 a) / 8 on the raw differences a = q0 - qm, b = qp - q0,
// and the van Albada value s to (ab + |ab| + e)/(a^2 + b^2 + e) with
// e = 1e-12 len^2 (the reference's epsilon on the length-scaled differences).
__device__ __forceinline__ void muscl_cell(float eps_l2, bool lim, float qm, float q0, float qp,
                                           float& hi, float& lo) {
    const float a = q0 - qm;
    const float b = qp - q0;
    float s = 0.125f;
    if (lim) {
        const float ab = a * b;
        s = 0.125f * (ab + fabsf(ab) + eps_l2) / (a * a + b * b + eps_l2);
    }
    hi = q0 + s * (3.0f * b + a);
    lo = q0 - s * (b + 3.0f * a);
}

__device__ __forceinline__ float clip2(float q, float A, float B, bool clip) {
    return clip ? clip_to_limits(q, A, B) : q;
}

// A face from its two cells' reconstructed values: hL (left cell's hi), cL
// (left cell's state), aL; lR (right cell's lo), cR, aR; the 5 values in the
// order rho, vx, vy, vz, u of the global frame.  Extrema clipping, the
// thermo update of each side (falling back to the cell state as
// interp_l2r2 does), the face frame of direction DIR as a permutation, the
// flux, and the momentum flux back in the global frame.
template <int FLUX, int DIR>
__device__ __forceinline__ void face_cells(const float* hL, const float* cL, float aL,
                                           const float* lR, const float* cR, float aR,
                                           const FluxOpts& o, float* F) {
    Prim<float, 1> Lf, Rt;
    const bool clip = o.clip;
    Lf.rho = clip2(hL[0], cL[0], cR[0], clip);
    Lf.vel = {clip2(hL[1], cL[1], cR[1], clip), clip2(hL[2], cL[2], cR[2], clip),
              clip2(hL[3], cL[3], cR[3], clip)};
    Lf.u = clip2(hL[4], cL[4], cR[4], clip);
    Rt.rho = clip2(lR[0], cL[0], cR[0], clip);
    Rt.vel = {clip2(lR[1], cL[1], cR[1], clip), clip2(lR[2], cL[2], cR[2], clip),
              clip2(lR[3], cL[3], cR[3], clip)};
    Rt.u = clip2(lR[4], cL[4], cR[4], clip);
    Lf.a = aL;
    Rt.a = aR;
    Lf.massf[0] = 1.0f;
    Rt.massf[0] = 1.0f;
    const float Rg = float(o.gas.Rgas), Cvi = float(o.gas.Cvinv);
    if (!(Lf.u > 0.0f && Lf.rho > 0.0f)) {
        Lf.rho = cL[0]; Lf.vel = {cL[1], cL[2], cL[3]}; Lf.u = cL[4];
    }
    Lf.p = Lf.rho * Rg * (Lf.u * Cvi);
    if (!(Rt.u > 0.0f && Rt.rho > 0.0f)) {
        Rt.rho = cR[0]; Rt.vel = {cR[1], cR[2], cR[3]}; Rt.u = cR[4];
    }
    Rt.p = Rt.rho * Rg * (Rt.u * Cvi);
    axis_to_local<DIR>(Lf.vel);
    axis_to_local<DIR>(Rt.vel);
    if (FLUX == 1) hllc<float, 1, 0>(Lf, Rt, F);
    else ausmdv<float, 1, 0>(Lf, Rt, F);
    V3<float> m{F[1], F[2], F[3]};
    axis_to_global<DIR>(m);
    F[1] = m.x; F[2] = m.y; F[3] = m.z;
}

__device__ __forceinline__ float sound_speed(float u, const GasConsts& g) {
    return sqrtf(float(g.gamma) * float(g.Rgas) * (u * float(g.Cvinv)));
}

// Edge threads: queue the copies of halo plane kk of a tile into ring slot
// `slot` (5 fields), the ghost cells made from the boundary conditions as
// load_plane makes them.  Inflow ghosts are stored at once; every other cell
// is copied from its source with cp.async.  Returns, two bits per position
// this thread handles, the velocity component a slip wall negates once the
// copies have landed (fixup_plane).
template <int TJ>
__device__ __forceinline__ unsigned queue_plane(const FusedDesc* __restrict__ descs, int stage,
                                                const FusedDesc& d, const float* __restrict__ W,
                                                float* slot, int i0, int j0, int kk, int et) {
    constexpr int NPOS = Lay<TJ>::PLANE;
    const size_t nc = size_t(d.ni) * d.nj * d.nk;
    unsigned fix = 0u;
    int m = 0;
    for (int e = et; e < NPOS; e += NE, ++m) {
        const int x = e % PI, r = e / PI;
        int gi = i0 - 2 + x, gj = j0 - 2 + r, gk = kk;
        const bool oi = gi < 0 || gi >= d.ni;
        const bool oj = gj < 0 || gj >= d.nj;
        const bool ok = gk < 0 || gk >= d.nk;
        if (int(oi) + int(oj) + int(ok) > 1) continue;
        int which = -1, layer = 0;
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
        const int type = which >= 0 ? d.bc[which] : -1;
        if (type == 1) {  // supersonic inflow: both ghost layers hold the inflow state
#pragma unroll
            for (int f = 0; f < 5; ++f) slot[f * NPOS + e] = float(d.inflow[f]);
            continue;
        }
        const float* src;
        size_t c, snc;
        if (type == 3) {  // full-face copy from the partner block (opposite faces)
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
            snc = size_t(o.ni) * o.nj * o.nk;
            c = (size_t(sk) * o.nj + sj) * o.ni + si;
            src = static_cast<const float*>(stage == 1 ? o.WA : o.WB);
        } else {
            if (which >= 0) {
                // the mirror cell for a slip wall, the first interior cell for
                // the zero-order extrapolation outflow
                const int s = (type == 2) ? 0 : layer;
                switch (which) {
                    case WEST: gi = s; break;
                    case EAST: gi = d.ni - 1 - s; break;
                    case SOUTH: gj = s; break;
                    case NORTH: gj = d.nj - 1 - s; break;
                    case BOTTOM: gk = s; break;
                    default: gk = d.nk - 1 - s; break;
                }
                if (type == 0) {
                    // reflect_normal_velocity with an axis frame
                    const unsigned comp = (which == WEST || which == EAST) ? 1u
                                          : (which == SOUTH || which == NORTH) ? 2u : 3u;
                    fix |= comp << (2 * m);
                }
            }
            snc = nc;
            c = (size_t(gk) * d.nj + gj) * d.ni + gi;
            src = W;
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) cp_async4(slot + f * NPOS + e, src + f * snc + c);
    }
    return fix;
}

// After cp_async_wait_all: negate the normal velocity of this thread's
// slip-wall ghost cells.
template <int TJ>
__device__ __forceinline__ void fixup_plane(float* slot, unsigned fix, int et) {
    constexpr int NPOS = Lay<TJ>::PLANE;
    int m = 0;
    for (int e = et; e < NPOS && fix; e += NE, ++m) {
        const unsigned comp = (fix >> (2 * m)) & 3u;
        if (comp) {
            float* p = slot + comp * NPOS + e;
            *p = -*p;
            fix &= ~(3u << (2 * m));
        }
    }
}

template <int FLUX, int TJ>
__global__ void __launch_bounds__(Lay<TJ>::threads, Lay<TJ>::min_blocks)
k_fused_stage_ws(const FusedDesc* __restrict__ descs, int nblocks, long long nitems, int kc,
                 SimDev* sim, GasConsts gas, FluxOpts o, int stage,
                 const int* __restrict__ order) {
    using L = Lay<TJ>;
    constexpr int NPOS = L::PLANE;
    // one decision per CTA (another CTA may set the status while this one
    // starts): every thread leaves, or none
    __shared__ int s_stop;
    if (threadIdx.x == 0) s_stop = (sim->status != 0 || sim->finished) ? 1 : 0;
    __syncthreads();
    if (s_stop) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) sim->item_next[stage == 1 ? 1 : 0] = 0u;
    __shared__ unsigned int s_item;
    __shared__ double s_volinv, s_area[3];   // of the current work item's block
    extern __shared__ __align__(16) float sm[];
    float* ring = sm;
    float* Qip = sm + L::o_qip;   // hi of the i-direction, cells i -1..31 (and lo of 32)
    float* Qim = sm + L::o_qim;
    float* Qjp = sm + L::o_qjp;
    float* Qjm = sm + L::o_qjm;
    float* As = sm + L::o_a;
    float* Fi = sm + L::o_fi;
    float* Fj = sm + L::o_fj;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool edge = warp >= TJ;
    const int et = threadIdx.x - 32 * TJ;   // edge thread index (edge warps)
    const int ti = lane, tj = warp;          // cell warps
    const double dt = sim->dt_global;
    const bool lim = o.limiter != 0;
    int bad = 0;
    // ring slot of plane kk
    auto slot_of = [&](int kk) { return ring + ((kk + 8) & 3) * (5 * NPOS); };

    for (;;) {
        __syncthreads();
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
        const size_t nc = size_t(d.ni) * d.nj * d.nk;
        if (threadIdx.x == 0) {
            // read after the prologue's barriers
            s_volinv = 1.0 / d.vol;
            s_area[0] = d.area[0]; s_area[1] = d.area[1]; s_area[2] = d.area[2];
        }
        const float* __restrict__ Win = static_cast<const float*>(stage == 1 ? d.WA : d.WB);
        float* __restrict__ Wout = static_cast<float*>(stage == 1 ? d.WB : d.WA);
        // the van Albada epsilon of each direction on raw differences
        float w[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) w[q] = float(1.0e-12 * d.len[q] * d.len[q]);

        // prologue: planes k0-2 .. k0+1
        if (edge) {
            unsigned fx[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                fx[q] = queue_plane<TJ>(descs, stage, d, Win, slot_of(k0 - 2 + q), i0, j0,
                                        k0 - 2 + q, et);
            cp_async_wait_all();
#pragma unroll
            for (int q = 0; q < 4; ++q) fixup_plane<TJ>(slot_of(k0 - 2 + q), fx[q], et);
        }
        __syncthreads();
        const int cx = ti + 2, cr = tj + 2;     // own cell in the ring
        const int coff = cr * PI + cx;
        float hK[5];       // hi (k-direction) of the own cell at the current plane
        float aK = 0.0f;   // sound speed of the own cell at the current plane
        float Fbot[5];
        if (!edge) {
            float c0[5], c1[5], c2[5], c3[5];
            const float* s0 = slot_of(k0 - 2);
            const float* s1 = slot_of(k0 - 1);
            const float* s2 = slot_of(k0);
            const float* s3 = slot_of(k0 + 1);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                c0[f] = s0[f * NPOS + coff]; c1[f] = s1[f * NPOS + coff];
                c2[f] = s2[f * NPOS + coff]; c3[f] = s3[f * NPOS + coff];
            }
            float hB[5], lo0[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                float lo_unused;
                muscl_cell(w[2], lim, c0[f], c1[f], c2[f], hB[f], lo_unused);
                muscl_cell(w[2], lim, c1[f], c2[f], c3[f], hK[f], lo0[f]);
            }
            const float aB = sound_speed(c1[4], gas);
            aK = sound_speed(c2[4], gas);
            face_cells<FLUX, 2>(hB, c1, aB, lo0, c2, aK, o, Fbot);
        }
        __syncthreads();   // plane k0-2's slot takes plane k0+2 next
        if (edge) {
            float* s = slot_of(k0 + 2);
            const unsigned fx = queue_plane<TJ>(descs, stage, d, Win, s, i0, j0, k0 + 2, et);
            cp_async_wait_all();
            fixup_plane<TJ>(s, fx, et);
        }
        __syncthreads();

        const bool active = !edge && (i0 + ti) < d.ni && (j0 + tj) < d.nj;
        for (int k = k0; k < k1; ++k) {
            const float* sk = slot_of(k);
            unsigned fx_next = 0u;
            const bool load_next = k + 3 <= k1 + 1;
            float q0[5], Ftop[5];
            // ---- phase A: reconstruction ------------------------------------------
            if (edge) {
                if (load_next)
                    fx_next = queue_plane<TJ>(descs, stage, d, Win, slot_of(k + 3), i0, j0, k + 3,
                                              et);
                // halo cells: rows -1 and TJ (j-direction), columns -1 and 32
                // (i-direction), with their sound speed
                for (int t = et; t < 64 + 2 * TJ; t += NE) {
                    int hi_, hj_, dir;
                    if (t < 64) { hi_ = t & 31; hj_ = (t < 32) ? -1 : TJ; dir = 1; }
                    else { const int u = t - 64; hj_ = u % TJ; hi_ = (u < TJ) ? -1 : TI; dir = 0; }
                    const int off = (hj_ + 2) * PI + (hi_ + 2);
                    const int st = dir == 0 ? 1 : PI;
                    const bool want_hi = (dir == 0) ? (hi_ < 0) : (hj_ < 0);
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const float* q = sk + f * NPOS + off;
                        float h, l;
                        muscl_cell(w[dir], lim, q[-st], q[0], q[st], h, l);
                        if (dir == 0) {
                            if (want_hi) Qip[f * L::QI + hj_ * (TI + 2) + 0] = h;
                            else Qim[f * L::QI + hj_ * (TI + 2) + (TI + 1)] = l;
                        } else {
                            if (want_hi) Qjp[f * L::QJ + 0 * TI + hi_] = h;
                            else Qjm[f * L::QJ + (TJ + 1) * TI + hi_] = l;
                        }
                    }
                    As[(hj_ + 1) * (TI + 2) + (hi_ + 1)] = sound_speed(sk[4 * NPOS + off], gas);
                }
            } else {
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    const float* q = sk + f * NPOS + coff;
                    q0[f] = q[0];
                    float h, l;
                    muscl_cell(w[0], lim, q[-1], q0[f], q[1], h, l);
                    Qip[f * L::QI + tj * (TI + 2) + ti + 1] = h;
                    Qim[f * L::QI + tj * (TI + 2) + ti + 1] = l;
                    muscl_cell(w[1], lim, q[-PI], q0[f], q[PI], h, l);
                    Qjp[f * L::QJ + (tj + 1) * TI + ti] = h;
                    Qjm[f * L::QJ + (tj + 1) * TI + ti] = l;
                }
                As[(tj + 1) * (TI + 2) + ti + 1] = aK;
                // k-direction: the cell above (plane k+1) and the top face
                const float* s1 = slot_of(k + 1);
                const float* s2 = slot_of(k + 2);
                float c1[5], hN[5], lN[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    c1[f] = s1[f * NPOS + coff];
                    muscl_cell(w[2], lim, q0[f], c1[f], s2[f * NPOS + coff], hN[f], lN[f]);
                }
                const float aN = sound_speed(c1[4], gas);
                face_cells<FLUX, 2>(hK, q0, aK, lN, c1, aN, o, Ftop);
#pragma unroll
                for (int f = 0; f < 5; ++f) hK[f] = hN[f];
                aK = aN;
            }
            __syncthreads();
            // ---- phase B: faces ---------------------------------------------------
            if (edge) {
                // the faces on the tile's east edge (i-face 32 of each row) and
                // north edge (j-face TJ of each column)
                for (int t = et; t < TJ + TI; t += NE) {
                    float hL[5], cL[5], lR[5], cR[5], F[5];
                    if (t < TJ) {
                        const int off = (t + 2) * PI + (TI + 1);
#pragma unroll
                        for (int f = 0; f < 5; ++f) {
                            hL[f] = Qip[f * L::QI + t * (TI + 2) + TI];
                            lR[f] = Qim[f * L::QI + t * (TI + 2) + TI + 1];
                            cL[f] = sk[f * NPOS + off];
                            cR[f] = sk[f * NPOS + off + 1];
                        }
                        face_cells<FLUX, 0>(hL, cL, As[(t + 1) * (TI + 2) + TI], lR, cR,
                                            As[(t + 1) * (TI + 2) + TI + 1], o, F);
#pragma unroll
                        for (int f = 0; f < 5; ++f) Fi[f * L::FI + t * (TI + 1) + TI] = F[f];
                    } else {
                        const int i = t - TJ;
                        const int off = (TJ + 1) * PI + (i + 2);
#pragma unroll
                        for (int f = 0; f < 5; ++f) {
                            hL[f] = Qjp[f * L::QJ + TJ * TI + i];
                            lR[f] = Qjm[f * L::QJ + (TJ + 1) * TI + i];
                            cL[f] = sk[f * NPOS + off];
                            cR[f] = sk[f * NPOS + off + PI];
                        }
                        face_cells<FLUX, 1>(hL, cL, As[TJ * (TI + 2) + i + 1], lR, cR,
                                            As[(TJ + 1) * (TI + 2) + i + 1], o, F);
#pragma unroll
                        for (int f = 0; f < 5; ++f) Fj[f * L::FJ + TJ * TI + i] = F[f];
                    }
                }
                // the plane queued in phase A must be in place before the next
                // plane's phase A reads it
                if (load_next) {
                    cp_async_wait_all();
                    fixup_plane<TJ>(slot_of(k + 3), fx_next, et);
                }
            } else {
                float Fw[5], Fs[5];
                {   // west face: cells i-1 and i
                    float hL[5], cL[5], lR[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        hL[f] = Qip[f * L::QI + tj * (TI + 2) + ti];
                        cL[f] = sk[f * NPOS + coff - 1];
                        lR[f] = Qim[f * L::QI + tj * (TI + 2) + ti + 1];
                    }
                    face_cells<FLUX, 0>(hL, cL, As[(tj + 1) * (TI + 2) + ti], lR, q0,
                                        As[(tj + 1) * (TI + 2) + ti + 1], o, Fw);
                }
                {   // south face: cells j-1 and j
                    float hL[5], cL[5], lR[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        hL[f] = Qjp[f * L::QJ + tj * TI + ti];
                        cL[f] = sk[f * NPOS + coff - PI];
                        lR[f] = Qjm[f * L::QJ + (tj + 1) * TI + ti];
                    }
                    face_cells<FLUX, 1>(hL, cL, As[tj * (TI + 2) + ti + 1], lR, q0,
                                        As[(tj + 1) * (TI + 2) + ti + 1], o, Fs);
                }
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    Fi[f * L::FI + tj * (TI + 1) + ti] = Fw[f];
                    Fj[f * L::FJ + tj * TI + ti] = Fs[f];
                }
            }
            __syncthreads();
            // ---- phase C: update and decode (cell warps) --------------------------
            if (active) {
                const int i = i0 + ti, j = j0 + tj;
                // time_derivatives (faces north, east, south, west, top,
                // bottom, fvcell.d:735-875) on the uniform grid: each
                // direction's two face fluxes enter as one difference, formed
                // in FP32 (the fluxes' own precision); the accumulation over
                // directions, the stage update and the decode are FP64
                double integral[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    const float dj = Fj[v * L::FJ + (tj + 1) * TI + ti] - Fj[v * L::FJ + tj * TI + ti];
                    const float di = Fi[v * L::FI + tj * (TI + 1) + ti + 1] -
                                     Fi[v * L::FI + tj * (TI + 1) + ti];
                    const float dk = Ftop[v] - Fbot[v];
                    integral[v] = -(double(dj) * s_area[1] + double(di) * s_area[0] +
                                    double(dk) * s_area[2]);
                }
                const double vol_inv = s_volinv;
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
                double rho = Un[0], vx = 0.0, vy = 0.0, vz = 0.0, u = 0.0, p = 0.0, T = 0.0,
                       a = 0.0;
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
                Wout[0 * nc + c] = float(rho);
                Wout[1 * nc + c] = float(vx); Wout[2 * nc + c] = float(vy);
                Wout[3 * nc + c] = float(vz);
                Wout[4 * nc + c] = float(u);
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
            }
            if (!edge) {
#pragma unroll
                for (int f = 0; f < 5; ++f) Fbot[f] = Ftop[f];
            }
            // no barrier here: phase C reads only the face arrays, which the next
            // plane writes after its phase-A barrier
        }
    }
    if (stage == 2 && blockIdx.x == 0 && threadIdx.x == 0) {
        for (int b = 0; b < nblocks; ++b) *descs[b].use_a0 = 0;
    }
    if (bad) atomicAdd(&sim->bad_cells, bad);
}

}  // namespace ws
}  // namespace e4c
