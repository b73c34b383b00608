// e4c_kernels.h -- launchers of the libe4cuda kernels (internal to the library).
#pragma once

#include <cuda_runtime.h>

#include "e4c_types.h"

namespace e4c {

struct FluxOpts {
    int flux;          // 0 ausmdv, 1 hllc
    int order2;        // interpolation_order > 1
    int limiter;       // apply_limiter
    int clip;          // extrema_clipping
    int local_frame;   // interpolate_in_local_frame
    GasConsts gas;
};

// general-geometry FP64 path (e4c_general.cu)
void launch_geometry(const BlockView& b, const double* vtx, cudaStream_t s);
void launch_upload(const BlockView& b, const double* prim, cudaStream_t s);
void launch_download(const BlockView& b, double* prim, double* cons, cudaStream_t s);
void launch_bc(const BlockView& b, const SimDev* sim, cudaStream_t s);
void launch_flux(const BlockView& b, const SimDev* sim, const FluxOpts& o, int dir, cudaStream_t s);
void launch_update(const BlockView& b, SimDev* sim, const GasConsts& gas, int stage,
                   int final_stage, cudaStream_t s);
void launch_dt_reset(unsigned long long* acc, int nb, cudaStream_t s);
void launch_dt(const BlockView& b, const SimDev* sim, double cfl_value, const double* dt_current,
               unsigned long long* acc, cudaStream_t s);
void launch_dt_finalize(SimDev* sim, const unsigned long long* acc, int nb, double cfl_allow,
                        double dt_init, double dt_max, int check_cfl, int step0,
                        double* out_dt_allow, double* out_cfl_max, cudaStream_t s);
void launch_reset_bad(SimDev* sim, cudaStream_t s);
void launch_stage_check(SimDev* sim, int max_invalid, cudaStream_t s);
void launch_end_step(SimDev* sim, cudaStream_t s);
void launch_begin_run(SimDev* sim, double max_time, cudaStream_t s);

}  // namespace e4c
