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
// one call.
//
// The array is shared by every call and keeps the last call's contents; each
// call resets the accumulators it uses before the reduction.  Calls that
// overlap on the GPU (from several host threads, or queued on several
// streams) would race on the array; the library runs everything on its own
// single stream and is documented as single-threaded.
//
// In host code the name e4c_noalloc_scratch is only a host-side stand-in, not
// a device address.  The device address is obtained once per device with
// cudaGetSymbolAddress (with that device current) the first time the entry
// point runs on it; make that first call before any stream capture.
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

// Per-device address of the scratch array (set up once per device).
static unsigned long long* g_scratch_addr[64] = {nullptr};

static int scratch_for_current_device(unsigned long long** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(E4C_ERR_ARG, "device ordinal out of range");
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, e4c_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(e4c_noalloc_scratch)");
        g_scratch_addr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_scratch_addr[dev];
    return E4C_OK;
}

// signal_frequency + min/max for one fused (uniform) block, accumulating into
// an explicit accumulator triple: the fused dt kernel with its accumulators
// taken from the caller instead of the block descriptor.
template <typename R>
__global__ void k_fused_dt_explicit(FusedDesc d, GasConsts gas, double cfl_value,
                                    const double* dt_current_p, unsigned long long* acc) {
    const double dt_current = *dt_current_p;
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

}  // namespace e4c

using namespace e4c;

extern "C" int e4c_dt_allow_noalloc(const int* h, int nb, double dt_current, int check_cfl,
                                    double* dt_allow, double* cfl_max) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!h || nb <= 0 || !dt_allow || !cfl_max) return fail(E4C_ERR_ARG, "bad arguments");
    if (nb > kNoallocMaxBlocks)
        return fail(E4C_ERR_ARG, "e4c_dt_allow_noalloc reduces over at most "
                                 "E4C_NOALLOC_MAX_BLOCKS (1024) blocks per call");
    for (int q = 0; q < nb; ++q)
        if (h[q] < 0 || h[q] >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    unsigned long long* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != E4C_OK) return rc;
    unsigned long long* acc = scratch;
    int* list = reinterpret_cast<int*>(scratch + kAccWords);
    double* scal = reinterpret_cast<double*>(scratch + kAccWords + kListWords);
    // inputs into the scratch: dt_current and the identity block list (the
    // accumulators are indexed by position in the call's block list)
    int ident[kNoallocMaxBlocks];
    for (int q = 0; q < nb; ++q) ident[q] = q;
    cudaError_t e = cudaMemcpyAsync(list, ident, size_t(nb) * sizeof(int), cudaMemcpyHostToDevice,
                                    c.stream);
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
                k_fused_dt_explicit<float><<<g, 256, 0, c.stream>>>(b.f, c.gas, c.cfg.cfl_value, scal, a);
            else
                k_fused_dt_explicit<double><<<g, 256, 0, c.stream>>>(b.f, c.gas, c.cfg.cfl_value, scal, a);
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
