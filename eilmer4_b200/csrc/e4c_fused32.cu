// e4c_fused32.cu -- the FP32 reconstruction/flux form of the fused stage
// kernel: primitive state, reconstruction and face fluxes in FP32; flux
// accumulation, the stage update and the decode stay in FP64.  Compiled with
// contraction allowed (fused multiply-adds) since this form is checked
// against the FP64 oracle with a tolerance.
#define E4C_FUSED_R float
#define E4C_FUSED_NS f32
// 32-wide tiles take the kernel with edge warps and per-cell reconstruction
#define E4C_FUSED_WS 1
#include "e4c_fused_launch.cuh"
