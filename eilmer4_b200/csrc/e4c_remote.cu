// e4c_remote.cu -- faces of fused (uniform) blocks joined to blocks that live
// on another rank, one rank per GPU: the halo exchange of the reference's MPI
// runs (GhostCellFullFaceCopy, src/eilmer/bc/ghost_cell_effect/
// full_face_copy.d: the cells next to the joint packed and sent to the
// partner's rank before every stage, :1134-1255).
//
// Such a face gets a shadow: a block two cells thick across the joint, with
// the face's tangential extents and the block's geometry, whose arrays hold
// the partner's two cell layers next to the joint.  The fused stage kernels
// read a shadow exactly as they read a local partner block (exchange boundary,
// opposite faces, orientation 0), so a domain split across ranks computes
// what the uncut block computes.  The host moves the layers: before each
// stage, e4c_pack_face on the partner's rank writes them into a device buffer
// (the stage's input state, the sound speed of the uploaded state and the
// flag that says whether it is still in use), the buffer crosses NVLink (NCCL
// send/receive), and e4c_unpack_face copies it into the shadow.
#include <cstring>

#include "e4c_internal.h"

namespace e4c {

// Cells of the two layers next to `face` of a block of ni x nj x nk, in the
// shadow's own (i fastest) order, and the extents of that two-thick box.
__host__ __device__ static void shadow_extents(int ni, int nj, int nk, int face, int& si, int& sj, int& sk) {
    si = ni; sj = nj; sk = nk;
    if (face == EAST || face == WEST) si = 2;
    else if (face == NORTH || face == SOUTH) sj = 2;
    else sk = 2;
}

static size_t slab_bytes(size_t n, size_t rsz) { return 5 * n * rsz + n * sizeof(double) + 8; }

template <typename R>
__global__ void k_pack_face(FusedDesc d, int face, int stage, unsigned char* dst) {
    int si, sj, sk;
    shadow_extents(d.ni, d.nj, d.nk, face, si, sj, sk);
    const long long n = (long long)si * sj * sk;
    const size_t nc = size_t(d.ni) * d.nj * d.nk;
    const R* W = static_cast<const R*>(stage == 1 ? d.WA : d.WB);
    R* dW = reinterpret_cast<R*>(dst);
    double* dA = reinterpret_cast<double*>(dst + 5 * size_t(n) * sizeof(R));
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = int(t % si), j = int((t / si) % sj), k = int(t / ((long long)si * sj));
        // the shadow's index along the joint counts away from the partner:
        // on an east (north, top) face the layers are the block's last two
        if (face == EAST) i += d.ni - 2;
        else if (face == NORTH) j += d.nj - 2;
        else if (face == TOP) k += d.nk - 2;
        const size_t c = (size_t(k) * d.nj + j) * d.ni + i;
#pragma unroll
        for (int f = 0; f < 5; ++f) dW[f * n + t] = W[f * nc + c];
        dA[t] = d.A0[c];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int* flag = reinterpret_cast<int*>(dst + 5 * size_t(n) * sizeof(R) + size_t(n) * 8);
        flag[0] = *d.use_a0;
        flag[1] = 0;
    }
}

}  // namespace e4c

using namespace e4c;

static int remote_of(int h, int face, RemoteFace** out) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    if (face < 0 || face > 5) return fail(E4C_ERR_ARG, "bad face");
    const int r = c.blocks[h].remote[face];
    if (r < 0) return fail(E4C_ERR_ARG, "the face is not joined to another rank");
    *out = &c.remote[r];
    return E4C_OK;
}

extern "C" {

int e4c_connect_remote(int h, int face) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    if (face < 0 || face > 5) return fail(E4C_ERR_ARG, "bad face");
    BlockHost& b = c.blocks[h];
    if (!b.fused)
        return fail(E4C_ERR_UNSUPPORTED, "faces joined to another rank are on the fused "
                                         "(uniform 3-D block) path only");
    if (c.cfg.flux_calculator == E4C_FLUX_ADAPTIVE_HANEL_AUSMDV)
        return fail(E4C_ERR_UNSUPPORTED, "the exchanged layers carry no shock flags: "
                                         "joints to another rank take the non-adaptive fluxes");
    if (b.remote[face] >= 0 || b.ex_block[face] >= 0)
        return fail(E4C_ERR_ARG, "the face is joined already");
    RemoteFace r;
    r.h = h;
    r.face = face;
    FusedDesc d = b.f;   // the block's geometry constants and frames
    int si, sj, sk;
    shadow_extents(b.f.ni, b.f.nj, b.f.nk, face, si, sj, sk);
    d.ni = si; d.nj = sj; d.nk = sk;
    d.tiles_i = d.tiles_j = d.kchunks = 0;   // no work items
    const size_t n = size_t(si) * sj * sk;
    const size_t rsz = (c.cfg.precision == E4C_PREC_FP32_FLUX) ? sizeof(float) : sizeof(double);
    r.bytes = slab_bytes(n, rsz);
    r.buf = c.dalloc(r.bytes);
    if (!r.buf) return fail(E4C_ERR_CUDA, "cudaMalloc of a shadow failed");
    cudaError_t e = cudaMemsetAsync(r.buf, 0, r.bytes, c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    unsigned char* p = static_cast<unsigned char*>(r.buf);
    d.WA = d.WB = p;
    d.A0 = reinterpret_cast<const double*>(p + 5 * n * rsz);
    d.use_a0 = reinterpret_cast<int*>(p + 5 * n * rsz + n * sizeof(double));
    d.U0 = nullptr;
    d.S[0] = d.S[1] = nullptr;
    d.dUdt0 = nullptr;
    d.acc = nullptr;
    for (int w = 0; w < 6; ++w) { d.bc[w] = E4C_BC_WALL_WITH_SLIP; d.ex[w] = -1; }
    r.d = d;
    b.remote[face] = int(c.remote.size());
    b.f.bc[face] = E4C_BC_EXCHANGE;
    b.v.bc[face] = E4C_BC_EXCHANGE;
    c.remote.push_back(r);
    c.descs_valid = false;
    c.reset_graphs();
    e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "e4c_connect_remote");
    return E4C_OK;
}

int e4c_face_slab_bytes(int h, int face, long long* bytes) {
    RemoteFace* r = nullptr;
    int rc = remote_of(h, face, &r);
    if (rc != E4C_OK) return rc;
    if (!bytes) return fail(E4C_ERR_ARG, "null output");
    *bytes = (long long)r->bytes;
    return E4C_OK;
}

int e4c_pack_face(int h, int face, int stage, void* dev_dst) {
    NvtxRange nvtx_range("e4c_pack_face");
    RemoteFace* r = nullptr;
    int rc = remote_of(h, face, &r);
    if (rc != E4C_OK) return rc;
    if (!dev_dst) return fail(E4C_ERR_ARG, "null buffer");
    if (stage != 1 && stage != 2) return fail(E4C_ERR_ARG, "stage must be 1 or 2");
    Ctx& c = g_ctx;
    const FusedDesc& d = c.blocks[h].f;
    int si, sj, sk;
    shadow_extents(d.ni, d.nj, d.nk, face, si, sj, sk);
    const long long n = (long long)si * sj * sk;
    int g = int((n + 255) / 256);
    if (g > 148 * 8) g = 148 * 8;
    unsigned char* dst = static_cast<unsigned char*>(dev_dst);
    if (c.cfg.precision == E4C_PREC_FP32_FLUX)
        k_pack_face<float><<<g, 256, 0, c.stream>>>(d, face, stage, dst);
    else
        k_pack_face<double><<<g, 256, 0, c.stream>>>(d, face, stage, dst);
    c.launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "e4c_pack_face");
    return E4C_OK;
}

int e4c_unpack_face(int h, int face, const void* dev_src) {
    NvtxRange nvtx_range("e4c_unpack_face");
    RemoteFace* r = nullptr;
    int rc = remote_of(h, face, &r);
    if (rc != E4C_OK) return rc;
    if (!dev_src) return fail(E4C_ERR_ARG, "null buffer");
    Ctx& c = g_ctx;
    cudaError_t e = cudaMemcpyAsync(r->buf, dev_src, r->bytes, cudaMemcpyDeviceToDevice, c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "e4c_unpack_face");
    return E4C_OK;
}

}  // extern "C"
