// e4c_seed.cu -- the learned chemistry seed: a small multilayer perceptron
// that predicts the end state of a cell's chemistry update, used as the
// Newton starting point of the point-implicit step.  No counterpart in the
// reference.
//
// Network: input (log T, log p, Y[5], log dt) normalised by the training-set
// mean and spread; three hidden layers of 64 units with the tanh-form GELU
// (Hendrycks & Gimpel 2016); output 6 values, the normalised transforms
// asinh(dY_s / sY) (5 species) and asinh(dT / sT).  Weights are kept in FP32
// (master copy for Adam) and run as BF16 on the tensor cores with FP32
// accumulation.  Inference (the chemistry step and e4c_seed_predict) and
// training both run on the 5th-generation tensor cores: tcgen05.mma issued
// by one thread, accumulators in tensor memory, operands in shared memory in
// the canonical K-major layout, 128 rows per CTA.  Training does forward and
// backward in one kernel per mini-batch (k_seed_train_tc): the pre-activations
// stay in tensor memory for the backward pass, the data gradients are
// products with the transposed weight copies, and the weight gradients
// products of transposed copies of the output gradients and activations that
// the threads write.
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "e4c_internal.h"

namespace e4c {

#define E4C_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// ---------------------------------------------------------------------------
// Parameter layout (FP32 master vector) and the packed BF16 image
// ---------------------------------------------------------------------------
constexpr int P_W1 = 0;               // [64][8]
constexpr int P_B1 = P_W1 + 64 * 8;   // [64]
constexpr int P_W2 = P_B1 + 64;       // [64][64]
constexpr int P_B2 = P_W2 + 64 * 64;
constexpr int P_W3 = P_B2 + 64;       // [64][64]
constexpr int P_B3 = P_W3 + 64 * 64;
constexpr int P_W4 = P_B3 + 64;       // [6][64]
constexpr int P_B4 = P_W4 + 6 * 64;   // [6]
constexpr int P_N = P_B4 + 6;
static_assert(P_N == E4C_SEED_NPARAM, "parameter count");

// Packed image (bf16 elements), copied as is into shared memory.  Row strides
// of 24 and 72 elements keep the fragment loads free of bank conflicts.
constexpr int S16 = 24, S64 = 72;
constexpr int OFF_W1 = 0;                      // W1  [64][24], cols 8.. zero
constexpr int OFF_W2 = OFF_W1 + 64 * S16;      // W2  [64][72]
constexpr int OFF_W3 = OFF_W2 + 64 * S64;      // W3  [64][72]
constexpr int OFF_W4 = OFF_W3 + 64 * S64;      // W4  [8][72], rows 6, 7 zero
constexpr int OFF_W2T = OFF_W4 + 8 * S64;      // W2^T [64][72]
constexpr int OFF_W3T = OFF_W2T + 64 * S64;    // W3^T [64][72]
constexpr int OFF_W4T = OFF_W3T + 64 * S64;    // W4^T [64][24], cols 6.. zero
constexpr int PACKED_N = OFF_W4T + 64 * S16;   // 22080
constexpr int PACKED_FWD = OFF_W2T;            // the forward part
static_assert((PACKED_N * 2) % 16 == 0 && (PACKED_FWD * 2) % 16 == 0, "uint4 copies");
constexpr int NBIAS = 200;                     // b1, b2, b3 (64 each), b4 (6) + 2 zeros

// Norm vector: mu_in[8], sd_in[8], mu_out[6], sd_out[6], sY, sT.
constexpr int N_MU_IN = 0, N_SD_IN = 8, N_MU_OUT = 16, N_SD_OUT = 22, N_SY = 28, N_ST = 29;
static_assert(E4C_SEED_NNORM == 30, "norm layout");

// ---------------------------------------------------------------------------
// BF16 and GELU helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_to_f(uint16_t r) {
    return __uint_as_float(uint32_t(r) << 16);
}

__device__ __forceinline__ float gelu_f(float x) {
    const float c = 0.7978845608028654f;  // sqrt(2/pi)
    const float u = c * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad_f(float x) {
    const float c = 0.7978845608028654f;
    const float x2 = x * x;
    const float th = tanhf(c * (x + 0.044715f * x2 * x));
    return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * c * (1.0f + 3.0f * 0.044715f * x2);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
// FP32 master parameters -> packed BF16 image (forward and transposed copies).
__global__ void k_seed_pack(const float* __restrict__ w, uint16_t* __restrict__ packed) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < PACKED_N; e += gridDim.x * blockDim.x) {
        float v = 0.0f;
        if (e < OFF_W2) {
            const int r = (e - OFF_W1) / S16, c = (e - OFF_W1) % S16;
            if (c < 8) v = w[P_W1 + r * 8 + c];
        } else if (e < OFF_W3) {
            const int r = (e - OFF_W2) / S64, c = (e - OFF_W2) % S64;
            if (c < 64) v = w[P_W2 + r * 64 + c];
        } else if (e < OFF_W4) {
            const int r = (e - OFF_W3) / S64, c = (e - OFF_W3) % S64;
            if (c < 64) v = w[P_W3 + r * 64 + c];
        } else if (e < OFF_W2T) {
            const int r = (e - OFF_W4) / S64, c = (e - OFF_W4) % S64;
            if (r < 6 && c < 64) v = w[P_W4 + r * 64 + c];
        } else if (e < OFF_W3T) {
            const int r = (e - OFF_W2T) / S64, c = (e - OFF_W2T) % S64;
            if (c < 64) v = w[P_W2 + c * 64 + r];
        } else if (e < OFF_W4T) {
            const int r = (e - OFF_W3T) / S64, c = (e - OFF_W3T) % S64;
            if (c < 64) v = w[P_W3 + c * 64 + r];
        } else {
            const int r = (e - OFF_W4T) / S16, c = (e - OFF_W4T) % S16;
            if (c < 6) v = w[P_W4 + c * 64 + r];
        }
        __nv_bfloat16 b = __float2bfloat16_rn(v);
        packed[e] = *reinterpret_cast<uint16_t*>(&b);
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; clears the gradient.
__global__ void k_seed_adam(float* __restrict__ w, float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float beta1, float beta2,
                            float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = grad[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        grad[i] = 0.0f;
    }
}

// Cell source for inference: a structured block's primitive state.
struct BlockCells {
    const double* W;
    size_t npad;
    int ni, nj, imin, jmin, kmin, nidim, njdim;
    __device__ size_t cell(long long q) const {
        const int i = imin + int(q % ni);
        const int j = jmin + int((q / ni) % nj);
        const int k = kmin + int(q / ((long long)ni * nj));
        return (size_t(k) * njdim + j) * nidim + i;
    }
};

__device__ __forceinline__ void seed_features(double T, double p, const double* Y, double dt,
                                              const double* norm, float* x) {
    double f[8] = {log(T), log(p), Y[0], Y[1], Y[2], Y[3], Y[4], log(dt)};
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = float((f[q] - norm[N_MU_IN + q]) / norm[N_SD_IN + q]);
}

// Rows of the chemistry step: the cells of the pass-1 work list of a block.
// Output: guess[s * n + q] (s < 5) = predicted end concentration of species
// s of the q-th listed cell, guess[5 * n + q] = its predicted end temperature.
struct WorkRows {
    BlockCells b;
    long long n;           // interior cells of the block (stride of guess)
    const int* work;
    const int* nwork;
    const double* dt_p;
    SeedMolar mol;
    double* guess;
    double rho, T, Y[5];
    __device__ long long count() const { return *nwork; }
    __device__ void load(long long q, const double* norm, float* x) {
        const size_t c = b.cell(work[q]);
        rho = b.W[W_RHO * b.npad + c];
        T = b.W[W_T * b.npad + c];
        const double p = b.W[W_P * b.npad + c];
#pragma unroll
        for (int s = 0; s < 5; ++s) Y[s] = b.W[(W_NBASE + s) * b.npad + c];
        seed_features(T, p, Y, *dt_p, norm, x);
    }
    __device__ void store(long long q, const float* z, const double* norm) const {
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const double zz = double(z[s]) * norm[N_SD_OUT + s] + norm[N_MU_OUT + s];
            const double y = Y[s] + norm[N_SY] * sinh(zz);
            guess[s * n + q] = fmax(y, 0.0) * rho / mol.M[s];
        }
        const double zT = double(z[5]) * norm[N_SD_OUT + 5] + norm[N_MU_OUT + 5];
        guess[5 * n + q] = T + norm[N_ST] * sinh(zT);
    }
};

// Rows given by the host: (T, p, Y[5], dt) -> out[q][6] = predicted dY[5], dT.
struct HostRows {
    const double* rows;
    long long n;
    double* out;
    __device__ long long count() const { return n; }
    __device__ void load(long long q, const double* norm, float* x) {
        const double* r = rows + q * 8;
        seed_features(r[0], r[1], r + 2, r[7], norm, x);
    }
    __device__ void store(long long q, const float* z, const double* norm) const {
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const double zz = double(z[s]) * norm[N_SD_OUT + s] + norm[N_MU_OUT + s];
            out[q * 6 + s] = norm[s < 5 ? N_SY : N_ST] * sinh(zz);
        }
    }
};

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05): 128 rows per CTA
// tile, M = 128 x N = 64 (N = 16 for the output layer) x K = 16 BF16
// instructions issued by one thread, FP32 accumulators in tensor memory
// (64 columns), operands in shared memory in the canonical K-major layout
// without swizzle: 8-row x 16-byte core matrices, consecutive along the rows
// (stride 128 B), the K chunks of 8 elements LBO bytes apart.  Each warp
// reads its 32 rows of the accumulator back with tcgen05.ld, adds the bias,
// applies GELU and writes the next layer's BF16 operand.
// ---------------------------------------------------------------------------
constexpr int TC_W1 = 0;          // W1: 64 rows x 16 (2 chunks), LBO 1024
constexpr int TC_W2 = 2048;       // W2: 64 x 64 (8 chunks), LBO 1024
constexpr int TC_W3 = 10240;      // W3
constexpr int TC_W4 = 18432;      // W4: 16 rows (6 used) x 64, LBO 256
constexpr int TC_X0 = 20480;      // input rows: 128 x 16, LBO 2048
constexpr int TC_H = 24576;       // hidden rows: 128 x 64, LBO 2048
constexpr int TC_BIAS = 40960;    // NBIAS floats
constexpr int TC_MBAR = 41984;    // mbarrier (8 B)
constexpr int TC_TSLOT = 41992;   // tensor-memory address written by tcgen05.alloc
constexpr int TC_FLAG = 41996;    // MMA completion seen by thread 0
constexpr int TC_SMEM = 42000 + 1024;   // + slack to align the base to 1 KB
constexpr uint32_t TC_COLS = 64;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, leading (K chunk) and stride
// (8-row group) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for an mbarrier phase (each try_wait itself suspends for a
// while): false after `tries` tries (~1e6 by default).
constexpr int kMbarTries = 1 << 20;
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int tries = kMbarTries) {
    for (int it = 0; it < tries; ++it)
        if (mbar_try(mbar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void proxy_fence() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 lanes x 64 columns of FP32 from TMEM (this warp's lane quarter).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&r)[64]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// 32 lanes x 16 columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Row r of a K-major canonical operand: chunk c (8 BF16) at
// (c * groups + r / 8) * 128 + (r % 8) * 16.
__device__ __forceinline__ uint32_t tc_row_chunk(int r, int c, int groups) {
    return uint32_t((c * groups + (r >> 3)) * 128 + (r & 7) * 16);
}

template <class Src>
__global__ void __launch_bounds__(128) k_seed_infer_tc(Src src, const float* __restrict__ params,
                                                       const uint16_t* __restrict__ packed,
                                                       const double* __restrict__ norm,
                                                       SimDev* sim, int first_wait_tries) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const long long nrows = src.count();
    if ((long long)blockIdx.x * 128 >= nrows) return;   // before any tensor-memory use
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
    unsigned char* sm = smem_raw + pad;
    const uint32_t sb = raw + pad;
    const int tid = threadIdx.x, warp = tid >> 5;

    // weights into the canonical layouts, biases
    const uint4* pk = reinterpret_cast<const uint4*>(packed);
    const uint4 zero4 = make_uint4(0u, 0u, 0u, 0u);
    for (int e = tid; e < 128; e += 128) {   // W1: 64 rows x 2 chunks
        const int r = e >> 1, c = e & 1;
        *reinterpret_cast<uint4*>(sm + TC_W1 + tc_row_chunk(r, c, 8)) = pk[(OFF_W1 + r * S16 + 8 * c) / 8];
    }
    for (int e = tid; e < 512; e += 128) {   // W2, W3: 64 rows x 8 chunks
        const int r = e >> 3, c = e & 7;
        *reinterpret_cast<uint4*>(sm + TC_W2 + tc_row_chunk(r, c, 8)) = pk[(OFF_W2 + r * S64 + 8 * c) / 8];
        *reinterpret_cast<uint4*>(sm + TC_W3 + tc_row_chunk(r, c, 8)) = pk[(OFF_W3 + r * S64 + 8 * c) / 8];
    }
    for (int e = tid; e < 128; e += 128) {   // W4: 16 rows (8.. zero) x 8 chunks
        const int r = e >> 3, c = e & 7;
        *reinterpret_cast<uint4*>(sm + TC_W4 + tc_row_chunk(r, c, 2)) =
            r < 8 ? pk[(OFF_W4 + r * S64 + 8 * c) / 8] : zero4;
    }
    float* bias = reinterpret_cast<float*>(sm + TC_BIAS);
    for (int q = tid; q < NBIAS; q += 128) {
        float v = 0.0f;
        if (q < 64) v = params[P_B1 + q];
        else if (q < 128) v = params[P_B2 + q - 64];
        else if (q < 192) v = params[P_B3 + q - 128];
        else if (q < 198) v = params[P_B4 + q - 192];
        bias[q] = v;
    }
    const uint32_t mbar = sb + TC_MBAR;
    volatile uint32_t* flag = reinterpret_cast<volatile uint32_t*>(sm + TC_FLAG);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(sb + TC_TSLOT), "r"(TC_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + TC_TSLOT);
    const uint32_t tmem_warp = tmem + (uint32_t(32 * warp) << 16);
    uint32_t phase = 0;
    bool failed = false;

    for (long long tile = blockIdx.x; tile * 128 < nrows && !failed; tile += gridDim.x) {
        const long long q = tile * 128 + tid;
        float x[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (q < nrows) src.load(q, norm, x);
        {
            uint4 v;
            v.x = pack_bf16(x[0], x[1]);
            v.y = pack_bf16(x[2], x[3]);
            v.z = pack_bf16(x[4], x[5]);
            v.w = pack_bf16(x[6], x[7]);
            *reinterpret_cast<uint4*>(sm + TC_X0 + tc_row_chunk(tid, 0, 16)) = v;
            *reinterpret_cast<uint4*>(sm + TC_X0 + tc_row_chunk(tid, 1, 16)) = zero4;
        }
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        for (int layer = 0; layer < 4; ++layer) {
            if (tid == 0) {
                tc_fence_after();
                if (layer == 0) {
                    umma_bf16(tmem, umma_desc(sb + TC_X0, 2048, 128), umma_desc(sb + TC_W1, 1024, 128),
                              umma_idesc(64), 0u);
                } else {
                    const uint32_t wb = layer == 1 ? TC_W2 : layer == 2 ? TC_W3 : TC_W4;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint64_t ad = umma_desc(sb + TC_H + 4096 * k, 2048, 128);
                        const uint64_t bd = layer < 3 ? umma_desc(sb + wb + 2048 * k, 1024, 128)
                                                      : umma_desc(sb + wb + 512 * k, 256, 128);
                        umma_bf16(tmem, ad, bd, umma_idesc(layer < 3 ? 64 : 16), k > 0 ? 1u : 0u);
                    }
                }
                umma_commit(mbar);
                *flag = mbar_wait(mbar, phase, first_wait_tries) ? 1u : 0u;
            }
            __syncthreads();
            if (*flag == 0u) {
                failed = true;
                break;
            }
            phase ^= 1u;
            tc_fence_after();
            if (layer < 3) {
                uint32_t r[64];
                tmem_ld64(tmem_warp, r);
                const float* bl = bias + 64 * layer;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    float h[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) h[e] = gelu_f(__uint_as_float(r[8 * c + e]) + bl[8 * c + e]);
                    uint4 v;
                    v.x = pack_bf16(h[0], h[1]);
                    v.y = pack_bf16(h[2], h[3]);
                    v.z = pack_bf16(h[4], h[5]);
                    v.w = pack_bf16(h[6], h[7]);
                    *reinterpret_cast<uint4*>(sm + TC_H + tc_row_chunk(tid, c, 16)) = v;
                }
                proxy_fence();
            } else {
                uint32_t r[16];
                tmem_ld16(tmem_warp, r);
                float z[6];
#pragma unroll
                for (int e = 0; e < 6; ++e) z[e] = __uint_as_float(r[e]) + bias[192 + e];
                if (q < nrows) src.store(q, z, norm);
            }
            tc_fence_before();
            __syncthreads();
        }
    }
    if (failed) {
        // the tensor cores did not signal completion: report, give the MMA a
        // second bounded wait (the full count of tries), then release the
        // tensor memory
        if (tid == 0) {
            if (sim && atomicCAS(&sim->status, 0, E4C_ERR_TIMEOUT) == 0) sim->status_step = sim->step;
            (void)mbar_wait(mbar, phase);
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS)
                     : "memory");
}

// ---------------------------------------------------------------------------
// Training on the 5th-generation tensor cores: one CTA per 128-row tile of a
// mini-batch, thread t the tile's row t, warp w the tensor-memory lanes
// 32w..32w+31.  Every product is a tcgen05.mma (kind::f16, BF16 operands,
// FP32 accumulators in tensor memory, M = 128) issued by one thread, with
// operands in canonical layouts without swizzle:
//   forward   Z_l = H_{l-1} W_l^T    A = H_{l-1} [128][in] K-major, B = W_l [out][in] K-major
//   backward  dH_{l-1} = dZ_l W_l    A = dZ_l [128][out] K-major, B = W_l^T [in][out] K-major
//             dW_l = dZ_l^T H_{l-1}  A = dZ_l, B = H_{l-1}, both read MN-major (the
//                                    tile's rows are the contraction)
//             db_l = dZ_l^T 1        A = dZ_l MN-major, B = a 16 x 128 block of ones
// A K-major operand stored as [rows][k] with 8-row groups SBO = 128 B apart
// and 8-element k chunks LBO apart is, read MN-major, the transposed operand
// with K groups LBO' = 128 B apart and MN groups SBO' = the old LBO apart,
// so the backward pass needs no transposed copies.  M = 128 for the weight
// gradients reads 128 output rows: rows past a layer's outputs come from the
// arrays laid out after dZ (in this CTA's shared memory) and land in
// tensor-memory lanes nobody reads.  The pre-activations Z_1..Z_3 stay in
// tensor memory for the GELU derivatives.  BF16 rounding falls where the
// oracle's mirror puts it: inputs, weights, activations and back-propagated
// output gradients.  The tile's gradients are added to grad with FP32
// atomics.  Loops are kept rolled (tensor-memory loads 16 columns at a time)
// so the kernel's instructions stay in the instruction cache.
// ---------------------------------------------------------------------------
constexpr int TT_W1 = 0;          // W1: 64 rows x 16, LBO 1024
constexpr int TT_W2 = 2048;       // W2: 64 x 64, LBO 1024
constexpr int TT_W3 = 10240;      // W3
constexpr int TT_W4 = 18432;      // W4: 16 rows (6 used) x 64, LBO 256
constexpr int TT_W4T = 20480;     // W4^T: 64 rows x 16 (6 used), LBO 1024
constexpr int TT_W3T = 22528;     // W3^T: 64 x 64
constexpr int TT_W2T = 30720;     // W2^T
constexpr int TT_X0 = 38912;      // inputs: 128 rows x 16, LBO 2048
constexpr int TT_D4 = 43008;      // dZ4: 128 x 16, LBO 2048
constexpr int TT_DZ = 47104;      // dZ3, then dZ2, dZ1: 128 x 64, LBO 2048
constexpr int TT_H1 = 63488;      // activations: 128 x 64, LBO 2048
constexpr int TT_H2 = 79872;
constexpr int TT_H3 = 96256;
constexpr int TT_ONES = 112640;   // 16 x 128 BF16 ones (K-major, LBO 256)
constexpr int TT_BIAS = 116736;   // NBIAS floats
constexpr int TT_MBAR = 117536;   // mbarrier (8 B)
constexpr int TT_TSLOT = 117544;  // tensor-memory address written by tcgen05.alloc
constexpr int TT_FLAG = 117548;   // MMA completion seen by thread 0
constexpr int TT_SMEM = 117552 + 1024;
// An MN-major operand of M = 128 starting at dZ4 (dZ) spans 16 groups of
// 2048 B, to 75776 (79872): inside the arrays above.
static_assert(TT_D4 + 16 * 2048 <= TT_ONES && TT_DZ + 16 * 2048 <= TT_ONES, "MN-major span");
static_assert(TT_BIAS + 4 * NBIAS <= TT_MBAR, "bias");
static_assert(TT_H2 == TT_H1 + 16384 && TT_H3 == TT_H1 + 2 * 16384 && TT_W3 == TT_W2 + 8192 &&
                  TT_W3T == TT_W2T - 8192, "layer strides");
constexpr uint32_t TT_COLS = 512;
// tensor-memory columns: pre-activations, output, data, weight and bias gradients
constexpr uint32_t TM_Z1 = 0, TM_Z4 = 192, TM_DH = 256, TM_DW = 384, TM_DB = 448;
constexpr uint32_t IDESC_A_MN = 1u << 15, IDESC_B_MN = 1u << 16;

// ksteps K = 16 products D (+)= A B^T of K-major operands with LBOs albo, blbo.
__device__ __forceinline__ void umma_k(uint32_t tmem_d, uint32_t a, uint32_t albo, uint32_t b,
                                       uint32_t blbo, int ksteps, uint32_t n) {
    for (int k = 0; k < ksteps; ++k)
        umma_bf16(tmem_d, umma_desc(a + 2 * k * albo, albo, 128),
                  umma_desc(b + 2 * k * blbo, blbo, 128), umma_idesc(n), k > 0 ? 1u : 0u);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
    return static_cast<uint16_t>(pack_bf16(x, 0.0f) & 0xFFFFu);
}

__global__ void __launch_bounds__(128, 1) k_seed_train_tc(const float* __restrict__ params,
                                                          const uint16_t* __restrict__ packed,
                                                          const float* __restrict__ X,
                                                          const float* __restrict__ Y,
                                                          const int* __restrict__ idx, int nbatch,
                                                          float inv_count, int backward,
                                                          float* __restrict__ grad,
                                                          float* __restrict__ loss,
                                                          int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
    unsigned char* sm = smem_raw + pad;
    const uint32_t sb = raw + pad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = blockIdx.x * 128 + tid;
    const bool valid = row < nbatch;
    const int src = valid ? idx[row] : 0;

    // weights (forward and transposed copies) into the canonical layouts
    const uint4* pk = reinterpret_cast<const uint4*>(packed);
    const uint4 zero4 = make_uint4(0u, 0u, 0u, 0u);
    {
        const int r = tid >> 1, c = tid & 1;   // 64 rows x 2 chunks
        *reinterpret_cast<uint4*>(sm + TT_W1 + tc_row_chunk(r, c, 8)) = pk[(OFF_W1 + r * S16 + 8 * c) / 8];
        *reinterpret_cast<uint4*>(sm + TT_W4T + tc_row_chunk(r, c, 8)) = pk[(OFF_W4T + r * S16 + 8 * c) / 8];
    }
#pragma unroll 1
    for (int e = tid; e < 512; e += 128) {   // 64 rows x 8 chunks
        const int r = e >> 3, c = e & 7;
        *reinterpret_cast<uint4*>(sm + TT_W2 + tc_row_chunk(r, c, 8)) = pk[(OFF_W2 + r * S64 + 8 * c) / 8];
        *reinterpret_cast<uint4*>(sm + TT_W3 + tc_row_chunk(r, c, 8)) = pk[(OFF_W3 + r * S64 + 8 * c) / 8];
        *reinterpret_cast<uint4*>(sm + TT_W2T + tc_row_chunk(r, c, 8)) = pk[(OFF_W2T + r * S64 + 8 * c) / 8];
        *reinterpret_cast<uint4*>(sm + TT_W3T + tc_row_chunk(r, c, 8)) = pk[(OFF_W3T + r * S64 + 8 * c) / 8];
    }
    {
        const int r = tid >> 3, c = tid & 7;   // W4: 16 rows (8.. zero) x 8 chunks
        *reinterpret_cast<uint4*>(sm + TT_W4 + tc_row_chunk(r, c, 2)) =
            r < 8 ? pk[(OFF_W4 + r * S64 + 8 * c) / 8] : zero4;
    }
    {
        const uint32_t one2 = 0x3F803F80u;     // two BF16 ones
        const uint4 ones = make_uint4(one2, one2, one2, one2);
#pragma unroll
        for (int q = 0; q < 2; ++q) reinterpret_cast<uint4*>(sm + TT_ONES)[tid + 128 * q] = ones;
    }
    float* bias = reinterpret_cast<float*>(sm + TT_BIAS);
#pragma unroll 1
    for (int q = tid; q < NBIAS; q += 128) {
        float v = 0.0f;
        if (q < 64) v = params[P_B1 + q];
        else if (q < 128) v = params[P_B2 + q - 64];
        else if (q < 192) v = params[P_B3 + q - 128];
        else if (q < 198) v = params[P_B4 + q - 192];
        bias[q] = v;
    }
    // this row's inputs
    {
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = valid ? X[src * 8 + i] : 0.0f;
        uint4 v;
        v.x = pack_bf16(x[0], x[1]); v.y = pack_bf16(x[2], x[3]);
        v.z = pack_bf16(x[4], x[5]); v.w = pack_bf16(x[6], x[7]);
        *reinterpret_cast<uint4*>(sm + TT_X0 + tc_row_chunk(tid, 0, 16)) = v;
        *reinterpret_cast<uint4*>(sm + TT_X0 + tc_row_chunk(tid, 1, 16)) = zero4;
    }
    const uint32_t mbar = sb + TT_MBAR;
    volatile uint32_t* flag = reinterpret_cast<volatile uint32_t*>(sm + TT_FLAG);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(sb + TT_TSLOT), "r"(TT_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + TT_TSLOT);
    const uint32_t tw = tmem + (uint32_t(32 * warp) << 16);
    uint32_t phase = 0;
    bool failed = false;

    // The operands written by the threads are visible to the tensor cores
    // (proxy fence, barrier); thread 0 issues the products and waits (bounded)
    // for their completion; every thread learns the outcome.
    auto sync_mma = [&](auto issue) -> bool {
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            issue();
            umma_commit(mbar);
            *flag = mbar_wait(mbar, phase) ? 1u : 0u;
        }
        __syncthreads();
        if (*flag == 0u) return false;
        phase ^= 1u;
        tc_fence_after();
        return true;
    };

    // ---- forward: Z_l in tensor memory, H_l = GELU(Z_l + b_l) as the next A
#pragma unroll 1
    for (int l = 0; l < 4 && !failed; ++l) {
        const uint32_t a = l == 0 ? TT_X0 : TT_H1 + (l - 1) * 16384;
        const uint32_t b = l == 0 ? TT_W1 : l == 3 ? TT_W4 : TT_W2 + (l - 1) * 8192;
        const uint32_t zc = TM_Z1 + 64 * l;
        failed = !sync_mma([&] {
            umma_k(tmem + zc, sb + a, 2048, sb + b, l == 3 ? 256 : 1024, l == 0 ? 1 : 4,
                   l == 3 ? 16 : 64);
        });
        if (failed || l == 3) break;
        const int dst = TT_H1 + l * 16384;
#pragma unroll 1
        for (int c = 0; c < 8; c += 2) {
            uint32_t r[16];
            tmem_ld16(tw + zc + 8 * c, r);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float g[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    g[e] = gelu_f(__uint_as_float(r[8 * h + e]) + bias[64 * l + 8 * (c + h) + e]);
                uint4 v;
                v.x = pack_bf16(g[0], g[1]); v.y = pack_bf16(g[2], g[3]);
                v.z = pack_bf16(g[4], g[5]); v.w = pack_bf16(g[6], g[7]);
                *reinterpret_cast<uint4*>(sm + dst + tc_row_chunk(tid, c + h, 16)) = v;
            }
        }
    }
    if (!failed) {
        // squared error on the 6 outputs and its derivative, dZ4 as this row of A
        uint32_t r[16];
        tmem_ld16(tw + TM_Z4, r);
        float lsum = 0.0f;
        uint16_t d[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int o = 0; o < 6; ++o) {
            if (valid) {
                const float diff = __uint_as_float(r[o]) + bias[192 + o] - Y[src * 6 + o];
                lsum += diff * diff;
                d[o] = bf16_bits(2.0f * diff * inv_count);
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
        if (lane == 0) atomicAdd(loss, lsum * inv_count);
        uint4 v;
        v.x = uint32_t(d[0]) | (uint32_t(d[1]) << 16);
        v.y = uint32_t(d[2]) | (uint32_t(d[3]) << 16);
        v.z = uint32_t(d[4]) | (uint32_t(d[5]) << 16);
        v.w = 0u;
        *reinterpret_cast<uint4*>(sm + TT_D4 + tc_row_chunk(tid, 0, 16)) = v;
        *reinterpret_cast<uint4*>(sm + TT_D4 + tc_row_chunk(tid, 1, 16)) = zero4;
    }
    // ---- backward: layer l's weight and bias gradients, then dH_{l-1}
#pragma unroll 1
    for (int l = 3; l >= 0 && !failed && backward; --l) {
        const uint32_t dz = l == 3 ? TT_D4 : TT_DZ;
        const uint32_t hp = l == 0 ? TT_X0 : TT_H1 + (l - 1) * 16384;
        const uint32_t nin = l == 0 ? 16 : 64;
        failed = !sync_mma([&] {
            for (int k = 0; k < 8; ++k) {   // K = the tile's 128 rows
                const uint64_t ad = umma_desc(sb + dz + 256 * k, 128, 2048);
                umma_bf16(tmem + TM_DW, ad, umma_desc(sb + hp + 256 * k, 128, 2048),
                          umma_idesc(nin) | IDESC_A_MN | IDESC_B_MN, k > 0 ? 1u : 0u);
                umma_bf16(tmem + TM_DB, ad, umma_desc(sb + TT_ONES + 512 * k, 256, 128),
                          umma_idesc(16) | IDESC_A_MN, k > 0 ? 1u : 0u);
            }
            if (l > 0)
                umma_k(tmem + TM_DH, sb + dz, 2048,
                       sb + (l == 3 ? TT_W4T : TT_W2T - (l - 1) * 8192), 1024, l == 3 ? 1 : 4, 64);
        });
        if (failed) break;
        const int nout = l == 3 ? 6 : 64;
        if (32 * warp < nout) {
            const int o = 32 * warp + lane;
            float* gW = grad + (l == 0 ? P_W1 : l == 1 ? P_W2 : l == 2 ? P_W3 : P_W4);
            float* gB = grad + (l == 0 ? P_B1 : l == 1 ? P_B2 : l == 2 ? P_B3 : P_B4);
            const int nw = l == 0 ? 8 : 64;
            uint32_t r[16];
            tmem_ld16(tw + TM_DB, r);
            if (o < nout) atomicAdd(gB + o, __uint_as_float(r[0]));
#pragma unroll 1
            for (int c = 0; c < nw; c += 16) {
                tmem_ld16(tw + TM_DW + c, r);
                if (o < nout) {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (c + i < nw) atomicAdd(gW + o * nw + c + i, __uint_as_float(r[i]));
                }
            }
        }
        if (l == 0) break;
        // dZ_{l-1} = dH_{l-1} GELU'(Z_{l-1} + b): this row of the next A
        const uint32_t zc = TM_Z1 + 64 * (l - 1);
#pragma unroll 1
        for (int c = 0; c < 8; c += 2) {
            uint32_t rd[16], rz[16];
            tmem_ld16(tw + TM_DH + 8 * c, rd);
            tmem_ld16(tw + zc + 8 * c, rz);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float g[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float z = __uint_as_float(rz[8 * h + e]) + bias[64 * (l - 1) + 8 * (c + h) + e];
                    g[e] = __uint_as_float(rd[8 * h + e]) * gelu_grad_f(z);
                }
                uint4 v;
                v.x = pack_bf16(g[0], g[1]); v.y = pack_bf16(g[2], g[3]);
                v.z = pack_bf16(g[4], g[5]); v.w = pack_bf16(g[6], g[7]);
                *reinterpret_cast<uint4*>(sm + TT_DZ + tc_row_chunk(tid, c + h, 16)) = v;
            }
        }
    }
    if (failed) {
        // the tensor cores did not signal completion: report, give the products
        // a second bounded wait, then release the tensor memory
        if (tid == 0) {
            if (status) atomicCAS(status, 0, E4C_ERR_TIMEOUT);
            (void)mbar_wait(mbar, phase);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TT_COLS)
                     : "memory");
}

// Sums over the valid samples (first feature finite) of the features, the
// transformed targets asinh(d / s) and their squares: acc[0..13] sums,
// acc[14..27] sums of squares, acc[28] count.
__global__ void k_seed_stats(const double* __restrict__ feat, const double* __restrict__ targ,
                             long long n, double sY, double sT, double* __restrict__ acc) {
    __shared__ double red[29][8];
    double loc[29];
    for (int q = 0; q < 29; ++q) loc[q] = 0.0;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
         r += (long long)gridDim.x * blockDim.x) {
        if (!isfinite(feat[r * 8])) continue;
        for (int q = 0; q < 8; ++q) {
            const double v = feat[r * 8 + q];
            loc[q] += v;
            loc[14 + q] += v * v;
        }
        for (int q = 0; q < 6; ++q) {
            const double v = asinh(targ[r * 6 + q] / (q < 5 ? sY : sT));
            loc[8 + q] += v;
            loc[22 + q] += v * v;
        }
        loc[28] += 1.0;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = 0; q < 29; ++q) {
        double v = loc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 29) {
        double v = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        atomicAdd(acc + threadIdx.x, v);
    }
}

// Normalised FP32 training arrays of the valid samples, compacted.
__global__ void k_seed_normalize(const double* __restrict__ feat, const double* __restrict__ targ,
                                 long long n, const double* __restrict__ norm,
                                 float* __restrict__ X, float* __restrict__ Y,
                                 int* __restrict__ count) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
         r += (long long)gridDim.x * blockDim.x) {
        if (!isfinite(feat[r * 8])) continue;
        const int o = atomicAdd(count, 1);
        for (int q = 0; q < 8; ++q)
            X[(long long)o * 8 + q] =
                float((feat[r * 8 + q] - norm[N_MU_IN + q]) / norm[N_SD_IN + q]);
        for (int q = 0; q < 6; ++q) {
            const double v = asinh(targ[r * 6 + q] / norm[q < 5 ? N_SY : N_ST]);
            Y[(long long)o * 6 + q] = float((v - norm[N_MU_OUT + q]) / norm[N_SD_OUT + q]);
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int grid_of(long long n, int threads, int cap) {
    long long g = (n + threads - 1) / threads;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return int(g);
}

int Ctx::seed_alloc_net() {
    SeedNet& s = seed;
    if (s.d_params) return E4C_OK;
    s.d_params = static_cast<float*>(dalloc(4 * P_N * sizeof(float)));
    s.d_packed = static_cast<uint16_t*>(dalloc(PACKED_N * sizeof(uint16_t)));
    s.d_norm = static_cast<double*>(dalloc(64 * sizeof(double)));
    s.d_loss = static_cast<float*>(dalloc(64 * sizeof(float)));
    if (!s.d_params || !s.d_packed || !s.d_norm || !s.d_loss)
        return fail(E4C_ERR_CUDA, "cudaMalloc of the seed network failed");
    s.d_grad = s.d_params + P_N;
    s.d_m = s.d_params + 2 * P_N;
    s.d_v = s.d_params + 3 * P_N;
    E4C_CUDA(cudaMemsetAsync(s.d_params, 0, 4 * P_N * sizeof(float), stream));
    E4C_CUDA(cudaMemsetAsync(s.d_loss, 0, 64 * sizeof(float), stream));
    return E4C_OK;
}

int Ctx::seed_pack() {
    k_seed_pack<<<grid_of(PACKED_N, 256, 148), 256, 0, stream>>>(seed.d_params, seed.d_packed);
    E4C_CUDA(cudaGetLastError());
    return E4C_OK;
}

int Ctx::seed_dataset_reserve(long long n) {
    SeedNet& s = seed;
    if (n <= s.cap) return E4C_OK;
    long long cap = std::max(n, 2 * s.cap);
    double* f = static_cast<double*>(dalloc(size_t(cap) * 8 * sizeof(double)));
    double* t = static_cast<double*>(dalloc(size_t(cap) * 6 * sizeof(double)));
    if (!f || !t) {
        dfree(f);
        dfree(t);
        return fail(E4C_ERR_CUDA, "cudaMalloc of the seed training set failed");
    }
    if (s.n > 0) {
        E4C_CUDA(cudaMemcpyAsync(f, s.d_feat, size_t(s.n) * 8 * sizeof(double),
                                 cudaMemcpyDeviceToDevice, stream));
        E4C_CUDA(cudaMemcpyAsync(t, s.d_targ, size_t(s.n) * 6 * sizeof(double),
                                 cudaMemcpyDeviceToDevice, stream));
    }
    E4C_CUDA(cudaStreamSynchronize(stream));
    dfree(s.d_feat);
    dfree(s.d_targ);
    s.d_feat = f;
    s.d_targ = t;
    s.cap = cap;
    return E4C_OK;
}

int Ctx::seed_guess_reserve(size_t ncell) {
    SeedNet& s = seed;
    if (ncell <= s.guess_cap) return E4C_OK;
    dfree(s.d_guess);
    s.d_guess = static_cast<double*>(dalloc(ncell * 6 * sizeof(double)));
    if (!s.d_guess) {
        s.guess_cap = 0;
        return fail(E4C_ERR_CUDA, "cudaMalloc of the seed guess buffer failed");
    }
    s.guess_cap = ncell;
    return E4C_OK;
}

void Ctx::seed_infer(const BlockView& v, const double* dt, const int* work, const int* nwork) {
    WorkRows rows{};
    rows.b = BlockCells{v.W, v.npad, v.ni, v.nj, v.imin, v.jmin, v.kmin, v.nidim, v.njdim};
    rows.n = (long long)v.ni * v.nj * v.nk;
    rows.work = work;
    rows.nwork = nwork;
    rows.dt_p = dt;
    rows.mol = seed.mol;
    rows.guess = seed.d_guess;
    // the list length is known only on the device: CTAs past its end return
    // before touching tensor memory
    k_seed_infer_tc<WorkRows><<<grid_of(rows.n, 128, 148 * 4), 128, TC_SMEM, stream>>>(
        rows, seed.d_params, seed.d_packed, seed.d_norm, d_sim, seed.first_wait_tries);
}

}  // namespace e4c

using namespace e4c;

extern "C" {

int e4c_seed_collect(const int* h, int nb, double dt, long long nsamples, unsigned long long rng_seed) {
    NvtxRange nvtx_range("e4c_seed_collect");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!c.cfg.reacting || !c.have_thermochem) return fail(E4C_ERR_STATE, "not a reacting configuration");
    if (!h || nb <= 0 || nsamples <= 0 || !(dt > 0.0)) return fail(E4C_ERR_ARG, "bad arguments");
    for (int q = 0; q < nb; ++q)
        if (h[q] < 0 || h[q] >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    // cells needing Newton work over dt in each block
    size_t maxcell = 0;
    for (int q = 0; q < nb; ++q) maxcell = std::max(maxcell, c.blocks[h[q]].ncell);
    int* d_list = static_cast<int*>(c.dalloc(maxcell * sizeof(int) + 64));
    if (!d_list) return fail(E4C_ERR_CUDA, "cudaMalloc failed");
    int* d_count = d_list + maxcell;
    std::vector<long long> hot(nb, 0);
    int* hp = static_cast<int*>(c.host_pinned) + 512;
    for (int q = 0; q < nb; ++q) {
        E4C_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), c.stream));
        launch_seed_active_list(c.blocks[h[q]].v, c.cfg.T_frozen, dt, d_list, d_count, c.stream);
        E4C_CUDA(cudaMemcpyAsync(hp, d_count, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        E4C_CUDA(cudaStreamSynchronize(c.stream));
        hot[q] = hp[0];
    }
    long long total_hot = 0;
    for (long long x : hot) total_hot += x;
    if (total_hot == 0) {   // no cell needs Newton work: nothing to learn from
        c.dfree(d_list);
        return E4C_OK;
    }
    int rc = c.seed_dataset_reserve(c.seed.n + nsamples);
    if (rc != E4C_OK) {
        c.dfree(d_list);
        return rc;
    }
    long long done = 0;
    for (int q = 0; q < nb; ++q) {
        if (hot[q] == 0) continue;
        long long ns = (q == nb - 1) ? nsamples - done : nsamples * hot[q] / total_hot;
        if (ns <= 0) continue;
        E4C_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), c.stream));
        launch_seed_active_list(c.blocks[h[q]].v, c.cfg.T_frozen, dt, d_list, d_count, c.stream);
        launch_seed_collect(c.blocks[h[q]].v, d_list, int(hot[q]), ns, rng_seed + 0x9E37ull * q, dt,
                            c.cfg.T_frozen, c.seed.d_feat + c.seed.n * 8,
                            c.seed.d_targ + c.seed.n * 6, c.stream);
        E4C_CUDA(cudaGetLastError());
        c.seed.n += ns;
        done += ns;
    }
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    c.dfree(d_list);
    return E4C_OK;
}

int e4c_seed_dataset(long long* n) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!n) return fail(E4C_ERR_ARG, "null output");
    *n = c.seed.n;
    return E4C_OK;
}

int e4c_seed_clear(void) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    c.seed.n = 0;
    return E4C_OK;
}

int e4c_seed_train(int epochs, int batch, double lr, unsigned long long rng_seed, double* report) {
    NvtxRange nvtx_range("e4c_seed_train");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (epochs < 1 || batch < 64 || !(lr > 0.0)) return fail(E4C_ERR_ARG, "bad training arguments");
    SeedNet& s = c.seed;
    if (s.n < 256) return fail(E4C_ERR_STATE, "collect at least 256 training pairs first");
    auto t0 = std::chrono::steady_clock::now();
    int rc = c.seed_alloc_net();
    s.adam_t = 0;
    if (rc != E4C_OK) return rc;
    // normalisation from the valid samples
    double* d_acc = static_cast<double*>(c.dalloc(32 * sizeof(double)));
    float* d_X = static_cast<float*>(c.dalloc(size_t(s.n) * 8 * sizeof(float)));
    float* d_Y = static_cast<float*>(c.dalloc(size_t(s.n) * 6 * sizeof(float)));
    int* d_idx = static_cast<int*>(c.dalloc(size_t(s.n) * sizeof(int) + 64));
    if (!d_acc || !d_X || !d_Y || !d_idx) {
        c.dfree(d_acc); c.dfree(d_X); c.dfree(d_Y); c.dfree(d_idx);
        return fail(E4C_ERR_CUDA, "cudaMalloc of the training arrays failed");
    }
    auto cleanup = [&] { c.dfree(d_acc); c.dfree(d_X); c.dfree(d_Y); c.dfree(d_idx); };
    const double sY = 1.0e-9, sT = 1.0e-3;
    E4C_CUDA(cudaMemsetAsync(d_acc, 0, 32 * sizeof(double), c.stream));
    k_seed_stats<<<grid_of(s.n, 256, 148 * 4), 256, 0, c.stream>>>(s.d_feat, s.d_targ, s.n, sY, sT,
                                                                   d_acc);
    double acc[32];
    E4C_CUDA(cudaMemcpyAsync(acc, d_acc, 29 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    const double cnt = acc[28];
    if (cnt < 256) { cleanup(); return fail(E4C_ERR_STATE, "too few valid training pairs"); }
    double norm[E4C_SEED_NNORM];
    for (int q = 0; q < 14; ++q) {
        const double mu = acc[q] / cnt;
        double var = acc[14 + q] / cnt - mu * mu;
        double sd = var > 0.0 ? std::sqrt(var) : 0.0;
        if (!(sd > 1.0e-6)) sd = 1.0;   // a constant input or output
        if (q < 8) { norm[N_MU_IN + q] = mu; norm[N_SD_IN + q] = sd; }
        else { norm[N_MU_OUT + q - 8] = mu; norm[N_SD_OUT + q - 8] = sd; }
    }
    norm[N_SY] = sY;
    norm[N_ST] = sT;
    std::memcpy(s.norm, norm, sizeof(norm));
    E4C_CUDA(cudaMemcpyAsync(s.d_norm, s.norm, sizeof(norm), cudaMemcpyHostToDevice, c.stream));
    E4C_CUDA(cudaMemsetAsync(d_idx + s.n, 0, sizeof(int), c.stream));
    k_seed_normalize<<<grid_of(s.n, 256, 148 * 8), 256, 0, c.stream>>>(
        s.d_feat, s.d_targ, s.n, s.d_norm, d_X, d_Y, d_idx + s.n);
    int nvalid = 0;
    E4C_CUDA(cudaMemcpyAsync(&nvalid, d_idx + s.n, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    const int nval = std::max(64, nvalid / 50);
    const int ntrain = nvalid - nval;
    // initial weights: uniform in +-1/sqrt(fan_in) (weights and biases)
    std::mt19937_64 gen(rng_seed);
    std::vector<float> w(P_N);
    auto init = [&](int off, int count, int fan_in) {
        std::uniform_real_distribution<float> u(-1.0f / std::sqrt(float(fan_in)),
                                                1.0f / std::sqrt(float(fan_in)));
        for (int q = 0; q < count; ++q) w[off + q] = u(gen);
    };
    init(P_W1, 64 * 8 + 64, 8);
    init(P_W2, 64 * 64 + 64, 64);
    init(P_W3, 64 * 64 + 64, 64);
    init(P_W4, 6 * 64 + 6, 64);
    E4C_CUDA(cudaMemcpyAsync(s.d_params, w.data(), P_N * sizeof(float), cudaMemcpyHostToDevice, c.stream));
    E4C_CUDA(cudaMemsetAsync(s.d_grad, 0, 3 * P_N * sizeof(float), c.stream));
    rc = c.seed_pack();
    if (rc != E4C_OK) { cleanup(); return rc; }
    E4C_CUDA(cudaFuncSetAttribute(k_seed_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TT_SMEM));
    // a time-out of the tensor cores is reported here (the word after the
    // normalisation sums, cleared with them)
    int* d_status = reinterpret_cast<int*>(d_acc + 30);
    std::vector<int> perm(ntrain), vidx(nval);
    std::iota(perm.begin(), perm.end(), 0);
    std::iota(vidx.begin(), vidx.end(), ntrain);
    const long long steps_per_epoch = (ntrain + batch - 1) / batch;
    const long long total = steps_per_epoch * epochs;
    long long step = 0;
    double train_loss = 0.0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), gen);
        E4C_CUDA(cudaMemcpyAsync(d_idx, perm.data(), size_t(ntrain) * sizeof(int),
                                 cudaMemcpyHostToDevice, c.stream));
        E4C_CUDA(cudaMemsetAsync(s.d_loss, 0, sizeof(float), c.stream));
        for (long long b = 0; b < steps_per_epoch; ++b) {
            const int off = int(b * batch);
            const int nb = std::min(batch, ntrain - off);
            // cosine decay to 1 % of lr
            const double frac = double(step) / double(total);
            const float lr_t = float(lr * (0.01 + 0.99 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * frac))));
            ++step;
            k_seed_train_tc<<<(nb + 127) / 128, 128, TT_SMEM, c.stream>>>(
                s.d_params, s.d_packed, d_X, d_Y, d_idx + off, nb, 1.0f / float(nb * 6), 1,
                s.d_grad, s.d_loss, d_status);
            ++s.adam_t;
            const float bc1 = float(1.0 - std::pow(0.9, double(s.adam_t)));
            const float bc2 = float(1.0 - std::pow(0.999, double(s.adam_t)));
            k_seed_adam<<<grid_of(P_N, 256, 64), 256, 0, c.stream>>>(
                s.d_params, s.d_grad, s.d_m, s.d_v, P_N, lr_t, 0.9f, 0.999f, 1.0e-8f, bc1, bc2);
            k_seed_pack<<<grid_of(PACKED_N, 256, 148), 256, 0, c.stream>>>(s.d_params, s.d_packed);
            c.launches += 3;
        }
        E4C_CUDA(cudaGetLastError());
        float lsum = 0.0f;
        E4C_CUDA(cudaMemcpyAsync(&lsum, s.d_loss, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
        E4C_CUDA(cudaStreamSynchronize(c.stream));
        train_loss = lsum / double(steps_per_epoch);
    }
    // validation loss (no gradient)
    E4C_CUDA(cudaMemcpyAsync(d_idx, vidx.data(), size_t(nval) * sizeof(int),
                             cudaMemcpyHostToDevice, c.stream));
    E4C_CUDA(cudaMemsetAsync(s.d_loss, 0, sizeof(float), c.stream));
    k_seed_train_tc<<<(nval + 127) / 128, 128, TT_SMEM, c.stream>>>(
        s.d_params, s.d_packed, d_X, d_Y, d_idx, nval, 1.0f / float(nval * 6), 0, s.d_grad,
        s.d_loss, d_status);
    float vloss = 0.0f;
    int status = 0;
    E4C_CUDA(cudaMemcpyAsync(&vloss, s.d_loss, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    E4C_CUDA(cudaGetLastError());
    cleanup();
    if (status != 0)
        return fail(status, "seed training: the tensor cores did not signal completion within "
                            "the wait limit");
    s.have_weights = true;
    c.reset_graphs();
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (report) {
        report[0] = train_loss;
        report[1] = vloss;
        report[2] = ntrain;
        report[3] = nval;
        report[4] = secs;
        report[5] = double(step);
    }
    return E4C_OK;
}

int e4c_seed_get(float* params, double* norm) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!c.seed.have_weights) return fail(E4C_ERR_STATE, "no trained or installed network");
    if (params)
        E4C_CUDA(cudaMemcpyAsync(params, c.seed.d_params, P_N * sizeof(float),
                                 cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    if (norm) std::memcpy(norm, c.seed.norm, sizeof(c.seed.norm));
    return E4C_OK;
}

int e4c_seed_set(const float* params, const double* norm) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!params || !norm) return fail(E4C_ERR_ARG, "null pointer");
    for (int q = 0; q < E4C_SEED_NNORM; ++q)
        if (!std::isfinite(norm[q])) return fail(E4C_ERR_ARG, "non-finite normalisation constant");
    for (int q = 0; q < 6; ++q)
        if (!(norm[N_SD_IN + q] > 0.0) || !(norm[N_SD_OUT + q] > 0.0))
            return fail(E4C_ERR_ARG, "non-positive spread in the normalisation constants");
    int rc = c.seed_alloc_net();
    if (rc != E4C_OK) return rc;
    std::memcpy(c.seed.norm, norm, sizeof(c.seed.norm));
    E4C_CUDA(cudaMemcpyAsync(c.seed.d_params, params, P_N * sizeof(float), cudaMemcpyHostToDevice,
                             c.stream));
    E4C_CUDA(cudaMemcpyAsync(c.seed.d_norm, c.seed.norm, sizeof(c.seed.norm),
                             cudaMemcpyHostToDevice, c.stream));
    rc = c.seed_pack();
    if (rc != E4C_OK) return rc;
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    c.seed.have_weights = true;
    c.reset_graphs();
    return E4C_OK;
}

int e4c_seed_enable(int on) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (on && !c.seed.have_weights) return fail(E4C_ERR_STATE, "no trained or installed network");
    if (on && (!c.cfg.reacting || !c.have_thermochem))
        return fail(E4C_ERR_STATE, "not a reacting configuration");
    if (on) {
        size_t maxcell = 0;
        for (const BlockHost& b : c.blocks) maxcell = std::max(maxcell, b.ncell);
        int rc = c.seed_guess_reserve(std::max<size_t>(maxcell, 1));
        if (rc != E4C_OK) return rc;
    }
    c.seed.enabled = on != 0;
    c.reset_graphs();
    return E4C_OK;
}

int e4c_seed_predict(const double* rows, long long n, double* out) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!c.seed.have_weights) return fail(E4C_ERR_STATE, "no trained or installed network");
    if (!rows || !out || n <= 0) return fail(E4C_ERR_ARG, "bad arguments");
    // rows in, predictions out, and a status word of this call's own (a
    // time-out here does not touch the simulation's status)
    double* d = static_cast<double*>(c.dalloc(size_t(n) * 14 * sizeof(double) + sizeof(SimDev)));
    if (!d) return fail(E4C_ERR_CUDA, "cudaMalloc failed");
    SimDev* st = reinterpret_cast<SimDev*>(d + size_t(n) * 14);
    E4C_CUDA(cudaMemsetAsync(st, 0, sizeof(SimDev), c.stream));
    E4C_CUDA(cudaMemcpyAsync(d, rows, size_t(n) * 8 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    HostRows hr{d, n, d + n * 8};
    k_seed_infer_tc<HostRows><<<grid_of(n, 128, 148 * 4), 128, TC_SMEM, c.stream>>>(
        hr, c.seed.d_params, c.seed.d_packed, c.seed.d_norm, st, c.seed.first_wait_tries);
    c.launches += 1;
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaMemcpyAsync(out, d + n * 8, size_t(n) * 6 * sizeof(double), cudaMemcpyDeviceToHost,
                             c.stream));
    int status = 0;
    E4C_CUDA(cudaMemcpyAsync(&status, &st->status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    c.dfree(d);
    if (status != 0) return fail(status, "seed inference: the tensor cores did not signal "
                                         "completion within the wait limit");
    return E4C_OK;
}

int e4c_seed_set_wait_limit(int first_wait_tries) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    c.seed.first_wait_tries = first_wait_tries < 0 ? kMbarTries : first_wait_tries;
    return E4C_OK;
}

int e4c_seed_loss_grad(const float* x, const float* y, int n, double* loss, float* grad) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!c.seed.have_weights) return fail(E4C_ERR_STATE, "no trained or installed network");
    if (!x || !y || n <= 0 || !loss || !grad) return fail(E4C_ERR_ARG, "bad arguments");
    const size_t bytes = size_t(n) * (8 + 6) * sizeof(float) + size_t(n) * sizeof(int) +
                         P_N * sizeof(float) + 64 + 16;
    char* d = static_cast<char*>(c.dalloc(bytes));
    if (!d) return fail(E4C_ERR_CUDA, "cudaMalloc failed");
    float* dX = reinterpret_cast<float*>(d);
    float* dY = dX + size_t(n) * 8;
    float* dG = dY + size_t(n) * 6;
    float* dL = dG + P_N;
    int* dI = reinterpret_cast<int*>(dL + 4);
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    E4C_CUDA(cudaMemcpyAsync(dX, x, size_t(n) * 8 * sizeof(float), cudaMemcpyHostToDevice, c.stream));
    E4C_CUDA(cudaMemcpyAsync(dY, y, size_t(n) * 6 * sizeof(float), cudaMemcpyHostToDevice, c.stream));
    E4C_CUDA(cudaMemcpyAsync(dI, idx.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice, c.stream));
    int* dS = reinterpret_cast<int*>(dI + n);   // time-out status
    E4C_CUDA(cudaMemsetAsync(dG, 0, (P_N + 4) * sizeof(float), c.stream));
    E4C_CUDA(cudaMemsetAsync(dS, 0, sizeof(int), c.stream));
    E4C_CUDA(cudaFuncSetAttribute(k_seed_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TT_SMEM));
    k_seed_train_tc<<<(n + 127) / 128, 128, TT_SMEM, c.stream>>>(
        c.seed.d_params, c.seed.d_packed, dX, dY, dI, n, 1.0f / float(n * 6), 1, dG, dL, dS);
    c.launches += 1;
    E4C_CUDA(cudaGetLastError());
    float l = 0.0f;
    int status = 0;
    E4C_CUDA(cudaMemcpyAsync(grad, dG, P_N * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaMemcpyAsync(&l, dL, sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaMemcpyAsync(&status, dS, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    *loss = l;
    c.dfree(d);
    if (status != 0)
        return fail(status, "seed training: the tensor cores did not signal completion within "
                            "the wait limit");
    return E4C_OK;
}

}  // extern "C"
