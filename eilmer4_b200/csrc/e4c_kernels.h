// e4c_kernels.h -- launchers of the libe4cuda kernels (internal to the library).
#pragma once

#include <cuda_runtime.h>

#include "../../include/e4cuda.h"
#include "e4c_types.h"

namespace e4c {

struct FluxOpts {
    int flux;          // 0 ausmdv, 1 hllc, 2 hanel, 3 adaptive_hanel_ausmdv
    int order2;        // interpolation_order > 1
    int limiter;       // apply_limiter
    int clip;          // extrema_clipping
    int local_frame;   // interpolate_in_local_frame
    GasConsts gas;
    double shear_tol;        // adaptive flux: shear_tolerance
    double compression_tol;  // shock detector: compression_tolerance
    int row_run_i, row_run_jk;  // faces per run of k_flux_rows (0: chosen per block)
};

// general-geometry FP64 path (e4c_general.cu)
void launch_geometry(const BlockView& b, const double* vtx, cudaStream_t s);
void launch_upload(const BlockView& b, const double* prim, cudaStream_t s);
void launch_download(const BlockView& b, double* prim, double* cons, cudaStream_t s);
// conserved state of the interior cells (ideal gas) -> U0 and the decoded W
void launch_upload_cons(const BlockView& b, const double* cons, SimDev* sim, const GasConsts& gas,
                        cudaStream_t s);
void launch_bc(const BlockView& b, const SimDev* sim, cudaStream_t s);
// x_order 1 extrapolation boundaries of a general block, after launch_bc
void launch_bc_linear(const BlockView& b, SimDev* sim, const GasConsts& gas, cudaStream_t s);
void launch_bc_linear_tp(const BlockView& b, SimDev* sim, const GasConsts& gas, cudaStream_t s);
// the ghost cells of its x_order 1 boundaries as a cell's initial FlowState
void launch_ghost_defaults(const BlockView& b, const GasConsts& gas, cudaStream_t s);
void launch_ghost_defaults_tp(const BlockView& b, const GasConsts& gas, cudaStream_t s);
// shock points (detect_shock_points with the PJ detector)
void launch_shock(const BlockView& b, const SimDev* sim, double tol, cudaStream_t s);
// velocities of the interior cells after their i (and j) face round trips
// (blocks with general face frames, before the flux launch)
void launch_replay_base(const BlockView& b, const SimDev* sim, cudaStream_t s);
// face fluxes of direction dir, or of every direction when dir < 0
void launch_flux(const BlockView& b, const SimDev* sim, const FluxOpts& o, int dir, cudaStream_t s);
// boundary-face fluxes of OutFlowBC_SimpleFlux boundaries (after launch_flux)
void launch_bc_flux(const BlockView& b, const SimDev* sim, const FluxOpts& o, cudaStream_t s);
void launch_update(const BlockView& b, SimDev* sim, const GasConsts& gas, int stage,
                   int final_stage, cudaStream_t s);
void launch_dt_reset(unsigned long long* acc, int nb, cudaStream_t s);
// dt accumulators are indexed by block handle; hlist lists the handles to reduce over
void launch_dt(const BlockView& b, const SimDev* sim, double cfl_value, const double* dt_current,
               unsigned long long* acc, cudaStream_t s);
void launch_dt_finalize(SimDev* sim, const unsigned long long* acc, const int* hlist, int nb,
                        double cfl_allow, double dt_init, double dt_max, int check_cfl, int step0,
                        double* out_dt_allow, double* out_cfl_max, cudaStream_t s);
void launch_reset_bad(SimDev* sim, cudaStream_t s);
void launch_stage_check(SimDev* sim, int max_invalid, cudaStream_t s);
void launch_end_step(SimDev* sim, cudaStream_t s);
void launch_begin_run(SimDev* sim, double max_time, cudaStream_t s);
// compare every cell's and face's geometry with the first one; flag[0] != 0 if any
// differs, flag[1] != 0 if some face frame is not made of signed unit axes
void launch_check_uniform(const BlockView& b, int* flag, cudaStream_t s);
// thermally perfect mixture / mechanism into constant memory; chemistry of one block
int set_thermochem_constants(const e4c_thermochem& tc);
int set_chem_newton_iterations(int n);
int set_chem_method(int m);
// ghost-cell geometry of an exchange boundary from the partner block
void launch_exchange_geometry(const BlockView& b, int which, cudaStream_t s);
// per-cell chemistry step suggestions to (to_dense = 1) or from a dense array
void launch_dt_chem_copy(const BlockView& b, double* dense, int to_dense, cudaStream_t s);
// thermally perfect face fluxes / cell updates (e4c_tp.cu)
void launch_flux_tp(const BlockView& b, const SimDev* sim, const FluxOpts& o, int dir, int g,
                    int T, cudaStream_t s);
void launch_update_tp(const BlockView& b, SimDev* sim, const GasConsts& gas, int stage,
                      int final_stage, int g, int T, cudaStream_t s);
// training pairs of the chemistry seed: list of the cells needing Newton work
// over dt, then sampled plain chemistry updates (features [n][8], targets [n][6])
void launch_seed_active_list(const BlockView& b, double T_frozen, double dt, int* list,
                             int* count, cudaStream_t s);
void launch_seed_collect(const BlockView& b, const int* hot, int nhot, long long n,
                         unsigned long long seed, double dt, double T_frozen, double* feat,
                         double* targ, cudaStream_t s);
// chemistry: pass 1 (every cell; lists cells needing Newton work) and
// pass 2 (the listed cells, optionally from a guess)
int launch_chem(const BlockView& b, SimDev* sim, double T_frozen, const double* dt, int nreac,
                int* work, int* nwork, unsigned long long* stats, cudaStream_t s);
int launch_chem_work(const BlockView& b, SimDev* sim, double T_frozen, const double* dt,
                     int nreac, const int* work, const int* nwork, const double* guess,
                     unsigned long long* stats, cudaStream_t s);

// fused uniform path (e4c_fused.cu: FP64, e4c_fused32.cu: FP32 flux)
struct FusedLaunch {
    const void* descs;      // device array of FusedDesc
    int nblocks;
    long long nitems;       // (block, tile, k-chunk) work items
    int kc;                 // k-chunk length
    int ti, tj;             // tile shape
    int grid;               // persistent CTAs
    const int* order;       // work items, costliest first (device array of nitems)
};

#define E4C_DECLARE_FUSED(NS)                                                                \
    namespace NS {                                                                           \
    int fused_stage(const FusedLaunch& L, SimDev* sim, const GasConsts& gas, const FluxOpts& o, \
                    int stage, cudaStream_t s);                                              \
    int fused_occupancy(int flux, int ti, int tj);                                           \
    void fused_dt(const void* descs, int nfused, int gx, SimDev* sim, const GasConsts& gas,  \
                  double cfl_value, const double* dt_current, cudaStream_t s);              \
    void fused_dt_one(const FusedDesc& d, unsigned long long* acc, int gx,                   \
                      const GasConsts& gas, double cfl_value, const double* dt_current,      \
                      cudaStream_t s);                                                       \
    void fused_upload(const double* prim, size_t nc, void* W, double* A0, double* U0,        \
                      cudaStream_t s);                                                       \
    void fused_upload_cons(const double* cons, size_t nc, void* W, double* U0, SimDev* sim,  \
                           const GasConsts& gas, cudaStream_t s);                            \
    void fused_download(const void* W, const double* A0, const int* use_a0, const double* U0, \
                        size_t nc, const GasConsts& gas, double* prim, double* cons,        \
                        cudaStream_t s);                                                     \
    }
E4C_DECLARE_FUSED(f64)
E4C_DECLARE_FUSED(f32)
#undef E4C_DECLARE_FUSED

}  // namespace e4c
