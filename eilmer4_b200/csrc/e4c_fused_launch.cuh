// e4c_fused_launch.cuh -- instantiations and launchers of the fused kernels
// for one arithmetic type (included by e4c_fused.cu with double and by
// e4c_fused32.cu with float; each file is its own translation unit with its
// own floating-point contract).
#pragma once

#include "e4c_fused.cuh"
#if E4C_FUSED_WS
#include "e4c_fused_ws.cuh"
#endif

#ifndef E4C_FUSED_R
#error "define E4C_FUSED_R (double or float) before including this file"
#endif

namespace e4c {
namespace E4C_FUSED_NS {

using RT = E4C_FUSED_R;

template <int FLUX, int TI, int TJ>
static int launch_one(const FusedLaunch& L, SimDev* sim, const GasConsts& gas, const FluxOpts& o,
                      int stage, cudaStream_t s) {
    constexpr size_t smem = FusedShareVA<RT, TI, TJ>::bytes();
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_fused_stage<RT, FLUX, TI, TJ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        attr_set = true;
    }
    k_fused_stage<RT, FLUX, TI, TJ><<<L.grid, FusedThreads<TI, TJ>::total, smem, s>>>(
        static_cast<const FusedDesc*>(L.descs), L.nblocks, L.nitems, L.kc, sim, gas, o, stage,
        L.order);
    return 0;
}

template <int FLUX, int TI, int TJ>
static int occupancy_one() {
    constexpr size_t smem = FusedShareVA<RT, TI, TJ>::bytes();
    cudaFuncSetAttribute(k_fused_stage<RT, FLUX, TI, TJ>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_stage<RT, FLUX, TI, TJ>,
                                                      FusedThreads<TI, TJ>::total, smem) != cudaSuccess)
        return 0;
    return n;
}

#if E4C_FUSED_WS
// 32-wide tiles of the FP32-flux form: the kernel with edge warps and per-cell
// reconstruction (second-order reconstruction only)
template <int FLUX, int TJ>
static int launch_ws(const FusedLaunch& L, SimDev* sim, const GasConsts& gas, const FluxOpts& o,
                     int stage, cudaStream_t s) {
    constexpr size_t smem = ws::Lay<TJ>::bytes;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(ws::k_fused_stage_ws<FLUX, TJ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        attr_set = true;
    }
    ws::k_fused_stage_ws<FLUX, TJ><<<L.grid, ws::Lay<TJ>::threads, smem, s>>>(
        static_cast<const FusedDesc*>(L.descs), L.nblocks, L.nitems, L.kc, sim, gas, o, stage,
        L.order);
    return 0;
}

template <int FLUX, int TJ>
static int occupancy_ws() {
    constexpr size_t smem = ws::Lay<TJ>::bytes;
    cudaFuncSetAttribute(ws::k_fused_stage_ws<FLUX, TJ>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ws::k_fused_stage_ws<FLUX, TJ>,
                                                      ws::Lay<TJ>::threads, smem) != cudaSuccess)
        return 0;
    return n;
}

#define E4C_WS_TILES(X) X(4) X(8) X(16)
#endif

// Tile shapes available to the autotuner: (TI, TJ).
#define E4C_TILES(X) X(32, 8) X(32, 4) X(16, 8) X(64, 4) X(16, 16) X(32, 16)

int fused_stage(const FusedLaunch& L, SimDev* sim, const GasConsts& gas, const FluxOpts& o,
                int stage, cudaStream_t s) {
#if E4C_FUSED_WS
    if (L.ti == 32 && o.order2) {
#define E4C_WS_CASE(TJ_)                                                            \
        if (L.tj == TJ_) {                                                          \
            if (o.flux == 1) return launch_ws<1, TJ_>(L, sim, gas, o, stage, s);    \
            return launch_ws<0, TJ_>(L, sim, gas, o, stage, s);                     \
        }
        E4C_WS_TILES(E4C_WS_CASE)
#undef E4C_WS_CASE
    }
#endif
// Hanel and the adaptive Hanel/AUSMDV flux: the FP64 form only
#define E4C_CASE(TI_, TJ_)                                                        \
    if (L.ti == TI_ && L.tj == TJ_) {                                            \
        if (o.flux == 1) return launch_one<1, TI_, TJ_>(L, sim, gas, o, stage, s); \
        if constexpr (sizeof(RT) == 8) {                                         \
            if (o.flux == 2) return launch_one<2, TI_, TJ_>(L, sim, gas, o, stage, s); \
            if (o.flux == 3) return launch_one<3, TI_, TJ_>(L, sim, gas, o, stage, s); \
        }                                                                        \
        return launch_one<0, TI_, TJ_>(L, sim, gas, o, stage, s);                  \
    }
    E4C_TILES(E4C_CASE)
#undef E4C_CASE
    return -1;
}

int fused_occupancy(int flux, int ti, int tj) {
#if E4C_FUSED_WS
    if (ti == 32) {
#define E4C_WS_CASE(TJ_)                                                            \
        if (tj == TJ_) return flux == 1 ? occupancy_ws<1, TJ_>() : occupancy_ws<0, TJ_>();
        E4C_WS_TILES(E4C_WS_CASE)
#undef E4C_WS_CASE
    }
#endif
#define E4C_CASE(TI_, TJ_)                                          \
    if (ti == TI_ && tj == TJ_) {                                  \
        if constexpr (sizeof(RT) == 8) {                           \
            if (flux == 2) return occupancy_one<2, TI_, TJ_>();    \
            if (flux == 3) return occupancy_one<3, TI_, TJ_>();    \
        }                                                          \
        return flux == 1 ? occupancy_one<1, TI_, TJ_>() : occupancy_one<0, TI_, TJ_>(); \
    }
    E4C_TILES(E4C_CASE)
#undef E4C_CASE
    return 0;
}

void fused_dt(const void* descs, int nfused, int gx, SimDev* sim, const GasConsts& gas,
              double cfl_value, const double* dt_current, cudaStream_t s) {
    k_fused_dt<RT><<<dim3(gx, nfused), 256, 0, s>>>(static_cast<const FusedDesc*>(descs),
                                                   FusedDesc{}, nullptr, sim, gas, cfl_value,
                                                   dt_current);
}

void fused_dt_one(const FusedDesc& d, unsigned long long* acc, int gx, const GasConsts& gas,
                  double cfl_value, const double* dt_current, cudaStream_t s) {
    k_fused_dt<RT><<<dim3(gx, 1), 256, 0, s>>>(nullptr, d, acc, nullptr, gas, cfl_value,
                                              dt_current);
}

// prim (rho, vx, vy, vz, p, T, u, a) -> W (R), A0 and the encoded U0
// (encode_conserved, fvcell.d:494-560)
__global__ void k_fused_upload(const double* prim, size_t nc, RT* W, double* A0, double* U0) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < nc;
         c += size_t(gridDim.x) * blockDim.x) {
        const double rho = prim[0 * nc + c], vx = prim[1 * nc + c], vy = prim[2 * nc + c];
        const double vz = prim[3 * nc + c], u = prim[6 * nc + c], a = prim[7 * nc + c];
        W[0 * nc + c] = RT(rho); W[1 * nc + c] = RT(vx); W[2 * nc + c] = RT(vy);
        W[3 * nc + c] = RT(vz); W[4 * nc + c] = RT(u);
        A0[c] = a;
        U0[0 * nc + c] = rho;
        U0[1 * nc + c] = rho * vx;
        U0[2 * nc + c] = rho * vy;
        U0[3 * nc + c] = rho * vz;
        const double ke = 0.5 * (vx * vx + vy * vy + vz * vz);
        U0[4 * nc + c] = rho * (u + ke);
    }
}

// U (dense) -> U0 and the decoded W (R) of a fused block (decode_ideal, the
// operations of the stage's decode); the sound speed then comes from W
__global__ void k_fused_upload_cons(const double* cons, size_t nc, RT* W, double* U0, SimDev* sim,
                                    GasConsts gas) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < nc;
         c += size_t(gridDim.x) * blockDim.x) {
        double Un[5];
        for (int v = 0; v < 5; ++v) Un[v] = cons[v * nc + c];
        double rho, vx, vy, vz, u, p, T, a;
        if (!decode_ideal(gas, Un, rho, vx, vy, vz, u, p, T, a)) {
            if (atomicCAS(&sim->status, 0, -5) == 0) sim->status_step = sim->step;
        }
        W[0 * nc + c] = RT(rho); W[1 * nc + c] = RT(vx); W[2 * nc + c] = RT(vy);
        W[3 * nc + c] = RT(vz); W[4 * nc + c] = RT(u);
        for (int v = 0; v < 5; ++v) U0[v * nc + c] = Un[v];
    }
}

// W (R) -> prim with p, T, a from update_thermo_from_rhou + update_sound_speed
__global__ void k_fused_download(const RT* W, const double* A0, const int* use_a0,
                                 const double* U0, size_t nc, GasConsts gas, double* prim,
                                 double* cons) {
    const int a0 = *use_a0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < nc;
         c += size_t(gridDim.x) * blockDim.x) {
        if (prim) {
            const double rho = double(W[0 * nc + c]), u = double(W[4 * nc + c]);
            const double T = u * gas.Cvinv;
            prim[0 * nc + c] = rho;
            prim[1 * nc + c] = double(W[1 * nc + c]);
            prim[2 * nc + c] = double(W[2 * nc + c]);
            prim[3 * nc + c] = double(W[3 * nc + c]);
            prim[4 * nc + c] = rho * gas.Rgas * T;
            prim[5 * nc + c] = T;
            prim[6 * nc + c] = u;
            prim[7 * nc + c] = a0 ? A0[c] : sqrt(gas.gamma * gas.Rgas * T);
        }
        if (cons)
            for (int v = 0; v < 5; ++v) cons[v * nc + c] = U0[v * nc + c];
    }
}

void fused_upload(const double* prim, size_t nc, void* W, double* A0, double* U0, cudaStream_t s) {
    int g = int((nc + 255) / 256);
    if (g > 148 * 32) g = 148 * 32;
    k_fused_upload<<<g, 256, 0, s>>>(prim, nc, static_cast<RT*>(W), A0, U0);
}

void fused_upload_cons(const double* cons, size_t nc, void* W, double* U0, SimDev* sim,
                       const GasConsts& gas, cudaStream_t s) {
    int g = int((nc + 255) / 256);
    if (g > 148 * 32) g = 148 * 32;
    k_fused_upload_cons<<<g, 256, 0, s>>>(cons, nc, static_cast<RT*>(W), U0, sim, gas);
}

void fused_download(const void* W, const double* A0, const int* use_a0, const double* U0,
                    size_t nc, const GasConsts& gas, double* prim, double* cons, cudaStream_t s) {
    int g = int((nc + 255) / 256);
    if (g > 148 * 32) g = 148 * 32;
    k_fused_download<<<g, 256, 0, s>>>(static_cast<const RT*>(W), A0, use_a0, U0, nc, gas, prim,
                                        cons);
}

}  // namespace E4C_FUSED_NS
}  // namespace e4c
