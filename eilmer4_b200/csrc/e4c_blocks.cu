// e4c_blocks.cu -- block construction and the per-step launch sequence.
#include <cstring>
#include <vector>

#include "e4c_internal.h"

namespace e4c {

#define E4C_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

int Ctx::ensure_dtacc(int nb) {
    if (nb <= dtacc_cap) return E4C_OK;
    int cap = nb < 64 ? 64 : nb;
    d_dtacc = static_cast<unsigned long long*>(dalloc(size_t(3) * cap * sizeof(unsigned long long)));
    if (!d_dtacc) return fail(E4C_ERR_CUDA, "cudaMalloc of dt accumulators failed");
    dtacc_cap = cap;
    reset_graphs();
    return E4C_OK;
}

int Ctx::build_block(int ni, int nj, int nk, const double* vtx, const int* bc,
                     const double* inflow, BlockHost& out) {
    const int dim = cfg.dimensions;
    BlockView v{};
    v.dim = dim;
    v.ni = ni; v.nj = nj; v.nk = (dim == 3) ? nk : 1;
    v.nidim = ni + 4; v.njdim = nj + 4; v.nkdim = (dim == 3) ? nk + 4 : 1;
    v.imin = 2; v.imax = v.imin + ni - 1;
    v.jmin = 2; v.jmax = v.jmin + nj - 1;
    if (dim == 3) { v.kmin = 2; v.kmax = v.kmin + nk - 1; }
    else { v.kmin = 0; v.kmax = 0; }
    v.npad = size_t(v.nidim) * v.njdim * v.nkdim;
    v.nsp = 1;
    v.nv = 5;
    for (int q = 0; q < 6; ++q) v.bc[q] = bc[q];
    for (int q = 0; q < 8; ++q) v.inflow[q] = inflow[q];
    const size_t np = v.npad;
    const size_t nw = W_NBASE;
    const size_t total = nw * np + 2 * size_t(v.nv) * np + 3 * size_t(v.nv) * np + 4 * np + 30 * np;
    double* slab = static_cast<double*>(dalloc(total * sizeof(double)));
    if (!slab) return fail(E4C_ERR_CUDA, "cudaMalloc of block storage failed");
    E4C_CUDA(cudaMemsetAsync(slab, 0, total * sizeof(double), stream));
    double* p = slab;
    v.W = p; p += nw * np;
    v.U0 = p; p += v.nv * np;
    v.dUdt0 = p; p += v.nv * np;
    v.Fi = p; p += v.nv * np;
    v.Fj = p; p += v.nv * np;
    v.Fk = p; p += v.nv * np;
    v.cgeom = p; p += 4 * np;
    v.fgi = p; p += 10 * np;
    v.fgj = p; p += 10 * np;
    v.fgk = p; p += 10 * np;
    // geometry from the vertices (compute_primary_cell_geometric_data)
    const size_t nvtx = size_t(ni + 1) * (nj + 1) * ((dim == 3) ? nk + 1 : 1);
    double* d_vtx = nullptr;
    E4C_CUDA(cudaMalloc(&d_vtx, nvtx * 3 * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(d_vtx, vtx, nvtx * 3 * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        launch_geometry(v, d_vtx, stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_vtx);
    if (e != cudaSuccess) return cuda_fail(e, "block geometry");
    out.v = v;
    out.ncell = size_t(ni) * nj * v.nk;
    out.nprim_vars = 8;
    out.fused = false;
    // staging area for uploads and downloads (primitive + conserved)
    const size_t need = (out.nprim_vars + size_t(v.nv)) * out.ncell * sizeof(double);
    if (need > staging_bytes) {
        double* s = static_cast<double*>(dalloc(need));
        if (!s) return fail(E4C_ERR_CUDA, "cudaMalloc of staging buffer failed");
        d_staging = s;
        staging_bytes = need;
    }
    return E4C_OK;
}

int Ctx::run_step(const std::vector<int>& hs, bool dt_check) {
    auto enqueue = [&]() {
        if (dt_check) enqueue_dt(hs, &d_sim->dt_global, -1, -1, d_sim, nullptr);
        enqueue_gasdynamic(hs);
    };
    if (!cfg.use_graphs) {
        enqueue();
        E4C_CUDA(cudaGetLastError());
        return E4C_OK;
    }
    GraphSlot& gs = graphs[dt_check ? 1 : 0];
    if (!gs.exec) {
        cudaGraph_t graph = nullptr;
        E4C_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const long long before = launches;
        enqueue();
        gs.nkernels = launches - before;
        launches = before;  // captured launches run only when the graph is replayed
        cudaError_t e = cudaStreamEndCapture(stream, &graph);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&gs.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            gs.exec = nullptr;
            return cuda_fail(e, "cudaGraphInstantiate");
        }
    }
    E4C_CUDA(cudaGraphLaunch(gs.exec, stream));
    launches += gs.nkernels;
    return E4C_OK;
}

// The fused uniform path is not selected yet; these are never reached.
void Ctx::fused_stage(const BlockHost&, int, int) {}
void Ctx::fused_dt(const BlockHost&, SimDev*, const double*, unsigned long long*) {}
void Ctx::fused_upload(BlockHost&, const double*) {}
void Ctx::fused_download(const BlockHost&, double*, double*) {}

}  // namespace e4c
