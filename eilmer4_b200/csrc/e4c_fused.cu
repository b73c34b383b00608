// e4c_fused.cu -- the plain FP64 form of the fused stage kernel.
// Compiled with -fmad=false so that its arithmetic is bit-identical to the
// general path and to the reference algorithm.
#define E4C_FUSED_R double
#define E4C_FUSED_NS f64
#include "e4c_fused_launch.cuh"
