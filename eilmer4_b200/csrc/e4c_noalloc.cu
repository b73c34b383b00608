// e4c_noalloc.cu -- e4c_dt_allow_noalloc: the time-step control reduction
// without any device allocation.
//
// Who needs it: a host that has handed all of the GPU's memory to its own
// pool (or runs under a fixed memory budget) cannot let a library call
// cudaMalloc in the middle of its time loop -- the call may fail or fragment
// the pool.  e4c_dt_allow may allocate its per-block accumulators on first
// use; this variant never does.  Its scratch (per-block accumulators, the
// block list, dt_current and the two results) is one file-scope device array
// of fixed size, so at most E4C_NOALLOC_MAX_BLOCKS blocks can be reduced in
// one call.  The kernels are the ones e4c_dt_allow launches (the fused
// blocks' dt kernel in its single-descriptor form, the general path's dt
// kernel and the finalising kernel), so the results are the same bits.
//
// The array is shared by every call and keeps the last call's contents; each
// call resets the accumulators it uses before the reduction.  Calls that
// overlap on the GPU (from several host threads, or queued on several
// streams) would race on the array; the library runs everything on its own
// single stream and is documented as single-threaded.
//
// In host code the name e4c_noalloc_scratch is only a host-side stand-in, not
// a device address.  e4c_init resolves the device address with
// cudaGetSymbolAddress, with the library's device current, and keeps it in
// the library context (cleared by e4c_finalize, resolved again by the next
// e4c_init).  Resolving it also loads this file's device code, so the array
// is reserved at e4c_init rather than on the first call inside a time loop.
#include <cfloat>
#include <cstring>

#include "e4c_internal.h"
#include "e4c_physics.cuh"

namespace e4c {

// Scratch layout, in 8-byte words: [accumulators 3*MAX][block list MAX/2 words]
// [dt_current][dt_allow][cfl_max][pad]
constexpr int kNoallocMaxBlocks = E4C_NOALLOC_MAX_BLOCKS;
constexpr int kAccWords = 3 * kNoallocMaxBlocks;
constexpr int kListWords = kNoallocMaxBlocks / 2;  // int block list
constexpr int kScalarWords = 4;
constexpr int kScratchWords = kAccWords + kListWords + kScalarWords;

static __device__ __align__(256) unsigned long long e4c_noalloc_scratch[kScratchWords];

// Device address of the scratch array on the current device (called by
// e4c_init with the library's device current).
int noalloc_setup(void** out) {
    *out = nullptr;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, e4c_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(e4c_noalloc_scratch)");
    *out = p;
    return E4C_OK;
}

}  // namespace e4c

using namespace e4c;

extern "C" int e4c_dt_allow_noalloc(const int* h, int nb, double dt_current, int check_cfl,
                                    double* dt_allow, double* cfl_max) {
    Ctx& c = g_ctx;
    if (!c.initialised || !c.noalloc_scratch) return fail(E4C_ERR_STATE, "not initialised");
    if (!h || nb <= 0 || !dt_allow || !cfl_max) return fail(E4C_ERR_ARG, "bad arguments");
    if (nb > kNoallocMaxBlocks)
        return fail(E4C_ERR_ARG, "e4c_dt_allow_noalloc reduces over at most "
                                 "E4C_NOALLOC_MAX_BLOCKS (1024) blocks per call");
    for (int q = 0; q < nb; ++q)
        if (h[q] < 0 || h[q] >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    // the scratch address and the library stream belong to the device that
    // e4c_init selected
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev != c.cfg.device)
        return fail(E4C_ERR_STATE, "e4c_dt_allow_noalloc called with another device current "
                                   "than the one e4c_init selected");
    unsigned long long* scratch = static_cast<unsigned long long*>(c.noalloc_scratch);
    unsigned long long* acc = scratch;
    int* list = reinterpret_cast<int*>(scratch + kAccWords);
    double* scal = reinterpret_cast<double*>(scratch + kAccWords + kListWords);
    // inputs into the scratch: dt_current and the identity block list (the
    // accumulators are indexed by position in the call's block list)
    int ident[kNoallocMaxBlocks];
    for (int q = 0; q < nb; ++q) ident[q] = q;
    e = cudaMemcpyAsync(list, ident, size_t(nb) * sizeof(int), cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scal, &dt_current, sizeof(double), cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "e4c_dt_allow_noalloc inputs");
    launch_dt_reset(acc, nb, c.stream);
    for (int q = 0; q < nb; ++q) {
        const BlockHost& b = c.blocks[h[q]];
        unsigned long long* a = acc + 3 * q;
        if (b.fused) {
            const long long ncell = (long long)b.ncell;
            int g = int((ncell + 255) / 256);
            if (g > 148 * 8) g = 148 * 8;
            if (g < 1) g = 1;
            if (c.cfg.precision == E4C_PREC_FP32_FLUX)
                f32::fused_dt_one(b.f, a, g, c.gas, c.cfg.cfl_value, scal, c.stream);
            else
                f64::fused_dt_one(b.f, a, g, c.gas, c.cfg.cfl_value, scal, c.stream);
        } else {
            launch_dt(b.v, nullptr, c.cfg.cfl_value, scal, a, c.stream);
        }
    }
    const double cfl_allow = (c.cfg.gasdynamic_update_scheme == E4C_UPDATE_PC) ? 1.2 : 0.9;
    launch_dt_finalize(nullptr, acc, list, nb, cfl_allow, c.cfg.dt_init, c.cfg.dt_max,
                       check_cfl ? 1 : 0, 0, scal + 1, scal + 2, c.stream);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "e4c_dt_allow_noalloc kernels");
    double out[2] = {0.0, 0.0};
    e = cudaMemcpyAsync(out, scal + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "e4c_dt_allow_noalloc result");
    *dt_allow = out[0];
    *cfl_max = out[1];
    return E4C_OK;
}
