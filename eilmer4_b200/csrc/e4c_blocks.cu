// e4c_blocks.cu -- block construction, the fused-path bookkeeping and the
// per-step launch sequence.
#include <algorithm>
#include <cstring>
#include <vector>

#include "e4c_internal.h"

namespace e4c {

#define E4C_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

void Ctx::dfree(void* p) {
    auto it = std::find(allocations.begin(), allocations.end(), p);
    if (it != allocations.end()) {
        cudaFree(p);
        allocations.erase(it);
    }
}

int Ctx::ensure_dtacc(int nb) {
    if (nb <= dtacc_cap) return E4C_OK;
    int cap = nb < 64 ? 64 : nb;
    d_dtacc = static_cast<unsigned long long*>(dalloc(size_t(3) * cap * sizeof(unsigned long long)));
    d_hlist = static_cast<int*>(dalloc(size_t(2) * cap * sizeof(int)));  // [all blocks | scratch]
    if (!d_dtacc || !d_hlist) return fail(E4C_ERR_CUDA, "cudaMalloc of dt accumulators failed");
    dtacc_cap = cap;
    hlist_cap = cap;
    descs_valid = false;
    reset_graphs();
    return E4C_OK;
}

// Copy a list of block handles to the scratch half of d_hlist (synchronously,
// so the pinned staging slot can be reused at once).
int Ctx::set_hlist(const std::vector<int>& hs) {
    int* hp = static_cast<int*>(host_pinned) + 256;  // a scratch slot past the scalars
    if (hs.size() > 512) return fail(E4C_ERR_ARG, "too many blocks in one call");
    for (size_t q = 0; q < hs.size(); ++q) hp[q] = hs[q];
    E4C_CUDA(cudaMemcpyAsync(d_hlist + hlist_cap, hp, hs.size() * sizeof(int),
                             cudaMemcpyHostToDevice, stream));
    E4C_CUDA(cudaStreamSynchronize(stream));
    return E4C_OK;
}

bool Ctx::uses_all_fused(const std::vector<int>& hs) const {
    int n = 0;
    for (int h : hs)
        if (blocks[h].fused) ++n;
    return n == 0 || n == nfused;
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
    v.nsp = (cfg.gas_model == E4C_GAS_THERM_PERF_5SP_AIR) ? 5 : 1;
    v.nv = 5 + (v.nsp > 1 ? v.nsp : 0);
    for (int q = 0; q < 6; ++q) v.bc[q] = bc[q];
    for (int q = 0; q < 8 + (v.nsp > 1 ? v.nsp : 0); ++q) v.inflow[q] = inflow[q];
    const size_t np = v.npad;
    // geometry arrays first (needed on either path), then the general-path state
    const size_t ngeom = 4 * np + 30 * np;
    const size_t nw = W_NBASE + (v.nsp > 1 ? size_t(v.nsp) : 0);
    const size_t nstate = nw * np + 2 * size_t(v.nv) * np + 3 * size_t(v.nv) * np +
                          (cfg.reacting ? np : 0);
    double* geom = static_cast<double*>(dalloc(ngeom * sizeof(double)));
    if (!geom) return fail(E4C_ERR_CUDA, "cudaMalloc of block geometry failed");
    E4C_CUDA(cudaMemsetAsync(geom, 0, ngeom * sizeof(double), stream));
    double* p = geom;
    v.cgeom = p; p += 4 * np;
    v.fgi = p; p += 10 * np;
    v.fgj = p; p += 10 * np;
    v.fgk = p; p += 10 * np;
    // geometry from the vertices (compute_primary_cell_geometric_data)
    const size_t nvtx = size_t(ni + 1) * (nj + 1) * ((dim == 3) ? nk + 1 : 1);
    double* d_vtx = nullptr;
    E4C_CUDA(cudaMalloc(&d_vtx, nvtx * 3 * sizeof(double) + 64));
    int* d_flag = reinterpret_cast<int*>(d_vtx + nvtx * 3);
    cudaError_t e = cudaMemcpyAsync(d_vtx, vtx, nvtx * 3 * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flag, 0, 2 * sizeof(int), stream);
    if (e == cudaSuccess) {
        launch_geometry(v, d_vtx, stream);
        launch_check_uniform(v, d_flag, stream);
        e = cudaGetLastError();
    }
    int flags[2] = {1, 1};
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, d_flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_vtx);
    if (e != cudaSuccess) return cuda_fail(e, "block geometry");

    out.ncell = size_t(ni) * nj * v.nk;
    out.nprim_vars = nw;
    v.axis_frames = (flags[1] == 0) ? 1 : 0;
    const bool uniform = (flags[0] == 0);
    out.simple_flux = false;
    for (int q = 0; q < 6; ++q) out.simple_flux = out.simple_flux || bc[q] == E4C_BC_OUTFLOW_SIMPLE_FLUX;
    out.linear_bc = false;
    for (int q = 0; q < 6; ++q) out.linear_bc = out.linear_bc || bc[q] == E4C_BC_OUTFLOW_EXTRAPOLATE_LINEAR;
    // the fused kernel carries the ausmdv and hllc fluxes (no shock flags)
    // and the ghost-cell boundaries (no flux computed in a boundary)
    // (the Hanel and adaptive fluxes on the FP64 form only)
    const bool fused_flux = cfg.flux_calculator <= E4C_FLUX_HLLC ||
                            (cfg.precision != E4C_PREC_FP32_FLUX &&
                             cfg.flux_calculator <= E4C_FLUX_ADAPTIVE_HANEL_AUSMDV);
    out.fused = uniform && dim == 3 && cfg.gasdynamic_update_scheme == E4C_UPDATE_PC && v.nsp == 1 &&
                fused_flux && !out.simple_flux && !out.linear_bc;
    if (cfg.precision == E4C_PREC_FP32_FLUX && !out.fused)
        return fail(E4C_ERR_UNSUPPORTED,
                    "the FP32-flux form needs a 3-D block with uniform geometry and the "
                    "predictor-corrector scheme");
    if (out.fused) {
        // uniform constants: the first interior cell and its west/south/bottom faces
        FusedDesc& f = out.f;
        std::memset(&f, 0, sizeof(f));
        f.ni = ni; f.nj = nj; f.nk = nk;
        for (int q = 0; q < 6; ++q) f.bc[q] = bc[q];
        const size_t c0 = (size_t(v.kmin) * v.njdim + v.jmin) * v.nidim + v.imin;
        double g[4], fg[3][10];
        for (int q = 0; q < 4; ++q)
            E4C_CUDA(cudaMemcpy(&g[q], v.cgeom + q * np + c0, sizeof(double), cudaMemcpyDeviceToHost));
        const double* fgs[3] = {v.fgi, v.fgj, v.fgk};
        for (int d = 0; d < 3; ++d)
            for (int q = 0; q < 10; ++q)
                E4C_CUDA(cudaMemcpy(&fg[d][q], fgs[d] + q * np + c0, sizeof(double),
                                    cudaMemcpyDeviceToHost));
        f.vol = g[0];
        // the fused kernel applies the face frames as permutations: require
        // n, t1, t2 = (x,y,z), (y,z,x), (z,x,y) for the i, j, k faces
        bool axis = true;
        for (int d = 0; d < 3; ++d)
            for (int q = 0; q < 3; ++q) {
                const double en = (q == d) ? 1.0 : 0.0;
                const double e1 = (q == (d + 1) % 3) ? 1.0 : 0.0;
                const double e2 = (q == (d + 2) % 3) ? 1.0 : 0.0;
                if (fg[d][q] != en || fg[d][3 + q] != e1 || fg[d][6 + q] != e2) axis = false;
            }
        for (int d = 0; d < 3; ++d) {
            f.len[d] = g[1 + d];
            f.area[d] = fg[d][9];
            for (int q = 0; q < 3; ++q) {
                f.fn[d][q] = fg[d][q];
                f.ft1[d][q] = fg[d][3 + q];
                f.ft2[d][q] = fg[d][6 + q];
            }
        }
        if (!axis) {
            if (cfg.precision == E4C_PREC_FP32_FLUX)
                return fail(E4C_ERR_UNSUPPORTED, "the FP32-flux form needs an axis-aligned Cartesian block");
            out.fused = false;
        }
        // inflow FlowState: rho, vx, vy, vz, u, a
        f.inflow[0] = inflow[0]; f.inflow[1] = inflow[1]; f.inflow[2] = inflow[2];
        f.inflow[3] = inflow[3]; f.inflow[4] = inflow[6]; f.inflow[5] = inflow[7];
    }
    if (out.fused) {
        FusedDesc& f = out.f;
        dfree(geom);
        const size_t nc = out.ncell;
        const size_t rsz = (cfg.precision == E4C_PREC_FP32_FLUX) ? sizeof(float) : sizeof(double);
        // (+ two bytes per cell: the adaptive flux's shock flags, both stages)
        const size_t nbytes = 2 * 5 * nc * rsz + (1 + 10) * nc * sizeof(double) + 256 + 2 * nc;
        char* s = static_cast<char*>(dalloc(nbytes));
        if (!s) return fail(E4C_ERR_CUDA, "cudaMalloc of fused block storage failed");
        E4C_CUDA(cudaMemsetAsync(s, 0, nbytes, stream));
        double* dp = reinterpret_cast<double*>(s);
        f.U0 = dp; dp += 5 * nc;
        f.dUdt0 = dp; dp += 5 * nc;
        f.A0 = dp; dp += nc;
        f.use_a0 = reinterpret_cast<int*>(dp); dp += 32;
        char* rp = reinterpret_cast<char*>(dp);
        f.WA = rp; rp += 5 * nc * rsz;
        f.WB = rp; rp += 5 * nc * rsz;
        f.S[0] = reinterpret_cast<unsigned char*>(rp);
        f.S[1] = f.S[0] + nc;
        v.W = v.U0 = v.dUdt0 = v.Fi = v.Fj = v.Fk = nullptr;
        v.cgeom = v.fgi = v.fgj = v.fgk = nullptr;
        max_cells_fused = std::max(max_cells_fused, int(nc));
    } else {
        double* slab = static_cast<double*>(dalloc(nstate * sizeof(double)));
        if (!slab) return fail(E4C_ERR_CUDA, "cudaMalloc of block storage failed");
        E4C_CUDA(cudaMemsetAsync(slab, 0, nstate * sizeof(double), stream));
        double* q = slab;
        v.W = q; q += nw * np;
        v.U0 = q; q += v.nv * np;
        v.dUdt0 = q; q += v.nv * np;
        v.Fi = q; q += v.nv * np;
        v.Fj = q; q += v.nv * np;
        v.Fk = q; q += v.nv * np;
        v.dt_chem = cfg.reacting ? q : nullptr;  // zero: no suggestion yet, as dt_chem = -1
        // shock flags, false at the start (FlowState.S)
        v.S = static_cast<int*>(dalloc(np * sizeof(int)));
        if (!v.S) return fail(E4C_ERR_CUDA, "cudaMalloc of shock flags failed");
        E4C_CUDA(cudaMemsetAsync(v.S, 0, np * sizeof(int), stream));
        if (!v.axis_frames) {
            v.Vrt = static_cast<double*>(dalloc(6 * np * sizeof(double)));
            if (!v.Vrt) return fail(E4C_ERR_CUDA, "cudaMalloc of round-trip velocities failed");
            E4C_CUDA(cudaMemsetAsync(v.Vrt, 0, 6 * np * sizeof(double), stream));
        }
    }
    out.v = v;
    // staging area for uploads and downloads (primitive + conserved)
    const size_t need = (out.nprim_vars + size_t(v.nv)) * out.ncell * sizeof(double);
    if (need > staging_bytes) {
        double* st = static_cast<double*>(dalloc(need));
        if (!st) return fail(E4C_ERR_CUDA, "cudaMalloc of staging buffer failed");
        dfree(d_staging);
        d_staging = st;
        staging_bytes = need;
    }
    descs_valid = false;
    return E4C_OK;
}

// (Re)build the device descriptor array of the fused blocks and the
// persistent grid of the fused stage kernel.
int Ctx::prepare_fused() {
    if (descs_valid) return E4C_OK;
    int rc = ensure_dtacc(int(blocks.size()));
    if (rc != E4C_OK) return rc;
    {
        // the "all blocks" handle list
        int* hp = static_cast<int*>(host_pinned) + 256;
        for (size_t q = 0; q < blocks.size(); ++q) hp[q] = int(q);
        E4C_CUDA(cudaMemcpyAsync(d_hlist, hp, blocks.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 stream));
        E4C_CUDA(cudaStreamSynchronize(stream));
    }
    std::vector<FusedDesc> ds;
    long long items = 0;
    std::vector<int> desc_of(blocks.size(), -1);
    int nreal = 0;
    for (size_t h = 0; h < blocks.size(); ++h)
        if (blocks[h].fused) desc_of[h] = nreal++;
    for (size_t h = 0; h < blocks.size(); ++h) {
        BlockHost& b = blocks[h];
        if (!b.fused) continue;
        FusedDesc& f = b.f;
        for (int w = 0; w < 6; ++w) {
            f.ex[w] = b.ex_block[w] >= 0 ? desc_of[b.ex_block[w]] : -1;
            // a partner on another rank: its shadow descriptor, after the
            // real ones (e4c_remote.cu)
            if (b.remote[w] >= 0) f.ex[w] = nreal + b.remote[w];
        }
        f.tiles_i = (f.ni + tile_ti - 1) / tile_ti;
        f.tiles_j = (f.nj + tile_tj - 1) / tile_tj;
        f.kchunks = (f.nk + tile_kc - 1) / tile_kc;
        f.item0 = items;
        f.acc = d_dtacc + 3 * h;
        items += (long long)f.tiles_i * f.tiles_j * f.kchunks;
        ds.push_back(f);
    }
    nfused = int(ds.size());
    fused_items = items;
    // shadows of remote partners: no work items (item0 past the last item, so
    // no CTA finds them), only read across the joints
    for (const RemoteFace& r : remote) {
        FusedDesc sd = r.d;
        sd.item0 = items;
        ds.push_back(sd);
    }
    const int ndesc = int(ds.size());
    if (nfused > 0) {
        if (ndesc > descs_cap) {
            dfree(d_descs);
            d_descs = static_cast<FusedDesc*>(dalloc(sizeof(FusedDesc) * std::max(ndesc, 64)));
            if (!d_descs) return fail(E4C_ERR_CUDA, "cudaMalloc of block descriptors failed");
            descs_cap = std::max(ndesc, 64);
        }
        E4C_CUDA(cudaMemcpyAsync(d_descs, ds.data(), sizeof(FusedDesc) * ndesc,
                                 cudaMemcpyHostToDevice, stream));
        // work items ordered by cost, costliest first (longest-processing-time
        // order for the CTAs that take them from a counter): the cells a tile
        // updates times its k-chunk length plus the four prologue planes
        std::vector<std::pair<long long, int>> cost;
        cost.reserve(size_t(items));
        for (const FusedDesc& f : ds) {
            for (int tj = 0; tj < f.tiles_j; ++tj)
                for (int ti = 0; ti < f.tiles_i; ++ti)
                    for (int kc = 0; kc < f.kchunks; ++kc) {
                        const long long ci = std::min(tile_ti, f.ni - ti * tile_ti);
                        const long long cj = std::min(tile_tj, f.nj - tj * tile_tj);
                        const long long ck = std::min(tile_kc, f.nk - kc * tile_kc);
                        const long long item =
                            f.item0 + (long long)(tj * f.tiles_i + ti) * f.kchunks + kc;
                        cost.push_back({-(ci * cj * (ck + 4)), int(item)});
                    }
        }
        std::stable_sort(cost.begin(), cost.end());
        if (items > item_order_cap) {
            dfree(d_item_order);
            d_item_order = static_cast<int*>(dalloc(sizeof(int) * size_t(items)));
            if (!d_item_order) {
                item_order_cap = 0;
                return fail(E4C_ERR_CUDA, "cudaMalloc of the work-item order failed");
            }
            item_order_cap = items;
        }
        std::vector<int> order(cost.size());
        for (size_t q = 0; q < cost.size(); ++q) order[q] = cost[q].second;
        E4C_CUDA(cudaMemcpyAsync(d_item_order, order.data(), sizeof(int) * order.size(),
                                 cudaMemcpyHostToDevice, stream));
        E4C_CUDA(cudaStreamSynchronize(stream));
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cfg.device);
        const int per_sm = (cfg.precision == E4C_PREC_FP32_FLUX)
                               ? f32::fused_occupancy(cfg.flux_calculator, tile_ti, tile_tj)
                               : f64::fused_occupancy(cfg.flux_calculator, tile_ti, tile_tj);
        if (per_sm <= 0) return fail(E4C_ERR_UNSUPPORTED, "fused tile shape does not fit on the device");
        long long g = (long long)nsm * per_sm;
        fused_grid = int(std::min<long long>(g, items));
    }
    descs_valid = true;
    reset_graphs();
    return E4C_OK;
}

void Ctx::fused_stage_all(int stage) {
    FusedLaunch L{d_descs, nfused, fused_items, tile_kc, tile_ti, tile_tj, fused_grid, d_item_order};
    if (cfg.precision == E4C_PREC_FP32_FLUX) f32::fused_stage(L, d_sim, gas, fopts, stage, stream);
    else f64::fused_stage(L, d_sim, gas, fopts, stage, stream);
}

void Ctx::fused_dt_all(SimDev* sim, const double* dt_current) {
    int gx = (max_cells_fused + 255) / 256;
    if (gx > 148 * 8) gx = 148 * 8;
    if (gx < 1) gx = 1;
    if (cfg.precision == E4C_PREC_FP32_FLUX)
        f32::fused_dt(d_descs, nfused, gx, sim, gas, cfg.cfl_value, dt_current, stream);
    else
        f64::fused_dt(d_descs, nfused, gx, sim, gas, cfg.cfl_value, dt_current, stream);
}

int Ctx::fused_upload(BlockHost& b, const double* prim) {
    FusedDesc& f = b.f;
    if (cfg.precision == E4C_PREC_FP32_FLUX) f32::fused_upload(prim, b.ncell, f.WA, const_cast<double*>(f.A0), f.U0, stream);
    else f64::fused_upload(prim, b.ncell, f.WA, const_cast<double*>(f.A0), f.U0, stream);
    const int one = 1;
    E4C_CUDA(cudaMemcpyAsync(f.use_a0, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    return E4C_OK;
}

int Ctx::fused_upload_cons(BlockHost& b, const double* cons) {
    FusedDesc& f = b.f;
    if (cfg.precision == E4C_PREC_FP32_FLUX) f32::fused_upload_cons(cons, b.ncell, f.WA, f.U0, d_sim, gas, stream);
    else f64::fused_upload_cons(cons, b.ncell, f.WA, f.U0, d_sim, gas, stream);
    const int zero = 0;
    E4C_CUDA(cudaMemcpyAsync(f.use_a0, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
    return E4C_OK;
}

// Conserved state already on the device (dense, v * ncell + cell) -> the
// block's state, decoded on the device.
int Ctx::upload_cons(BlockHost& b, const double* dev_cons) {
    if (b.v.nsp != 1)
        return fail(E4C_ERR_UNSUPPORTED,
                    "a conserved-state upload decodes the ideal gas only (the mixture's "
                    "temperature iteration needs a starting temperature)");
    if (b.fused) return fused_upload_cons(b, dev_cons);
    launch_upload_cons(b.v, dev_cons, d_sim, gas, stream);
    if (b.linear_bc) launch_ghost_defaults(b.v, gas, stream);
    return E4C_OK;
}

void Ctx::fused_download(const BlockHost& b, double* prim, double* cons) {
    const FusedDesc& f = b.f;
    if (cfg.precision == E4C_PREC_FP32_FLUX)
        f32::fused_download(f.WA, f.A0, f.use_a0, f.U0, b.ncell, gas, prim, cons, stream);
    else
        f64::fused_download(f.WA, f.A0, f.use_a0, f.U0, b.ncell, gas, prim, cons, stream);
}

int Ctx::run_step(const std::vector<int>& hs, bool dt_check) {
    auto enqueue = [&]() {
        if (dt_check) enqueue_dt(hs, d_hlist, &d_sim->dt_global, -1, -1, d_sim, nullptr);
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

}  // namespace e4c
