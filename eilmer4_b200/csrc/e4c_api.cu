// e4c_api.cu -- the extern "C" ABI of libe4cuda (declared in include/e4cuda.h).
//
// Host side of the library: one context, block storage, the device-side time
// loop of integrate_in_time (src/eilmer/simcore.d:791-1110) recorded as CUDA
// graphs, and the error conventions of src/gas/gas_cwrap.d (int handles,
// 0 / negative return codes, never throwing across the ABI).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/e4cuda.h"
#include "e4c_internal.h"
#include "e4c_kernels.h"

namespace e4c {

Ctx g_ctx;

int fail(int code, const std::string& msg) {
    g_ctx.last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return fail(E4C_ERR_CUDA, m);
}

#define E4C_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

void* Ctx::dalloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    allocations.push_back(p);
    return p;
}

void Ctx::reset_graphs() {
    for (auto& gx : graphs) {
        if (gx.exec) cudaGraphExecDestroy(gx.exec);
        gx.exec = nullptr;
    }
}

void Ctx::release() {
    reset_graphs();
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : allocations) cudaFree(p);
    allocations.clear();
    if (host_pinned) cudaFreeHost(host_pinned);
    host_pinned = nullptr;
    if (h2d_stream) cudaStreamSynchronize(h2d_stream);
    if (d2h_stream) cudaStreamSynchronize(d2h_stream);
    for (cudaEvent_t* e : {&ev_in_copied, &ev_in_consumed, &ev_out_ready, &ev_out_copied}) {
        if (*e) cudaEventDestroy(*e);
        *e = nullptr;
    }
    if (h2d_stream) cudaStreamDestroy(h2d_stream);
    if (d2h_stream) cudaStreamDestroy(d2h_stream);
    h2d_stream = d2h_stream = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    blocks.clear();
    // every device pointer above is now dangling: forget them all
    d_descs = nullptr;
    descs_cap = 0;
    d_item_order = nullptr;
    item_order_cap = 0;
    nfused = 0;
    fused_items = 0;
    descs_valid = false;
    max_cells_fused = 0;
    d_hlist = nullptr;
    hlist_cap = 0;
    d_sim = nullptr;
    d_scalars = nullptr;
    d_chem_stats = nullptr;
    d_chem_work = nullptr;
    d_chem_nwork = nullptr;
    chem_work_cap = 0;
    seed = SeedNet{};
    d_dtacc = nullptr;
    dtacc_cap = 0;
    noalloc_scratch = nullptr;
    remote.clear();
    d_staging = nullptr;
    staging_bytes = 0;
    d_stage_in = d_stage_out = nullptr;
    stage_io_bytes = 0;
    initialised = false;
}

void Profiler::begin(cudaStream_t s, int c) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    ev.push_back(a);
    ev.push_back(b);
    cls.push_back(c);
}

void Profiler::end(cudaStream_t s) { cudaEventRecord(ev.back(), s); }

// Every kernel launch goes through this bracket: it counts the launch and,
// while profiling, times it by class with events on the library stream.
template <typename F>
static inline void launch_as(Ctx& c, int cls, int nkernels, F&& f) {
    c.launches += nkernels;
    if (c.prof.on) c.prof.begin(c.stream, cls);
    f();
    if (c.prof.on) c.prof.end(c.stream);
}

// One stage over the given blocks (simcore.d:2325-2493 / 2529-2730).  All
// fused blocks go through one launch of the fused stage kernel.
void Ctx::enqueue_stage(const std::vector<int>& hs, int stage, int final_stage) {
    launch_as(*this, E4C_KCLASS_OTHER, 1, [&] { launch_reset_bad(d_sim, stream); });
    bool any_fused = false;
    for (int h : hs) any_fused = any_fused || blocks[h].fused;
    if (any_fused) launch_as(*this, E4C_KCLASS_STAGE, 1, [&] { fused_stage_all(stage); });
    for (int h : hs) {
        const BlockHost& b = blocks[h];
        if (!b.fused) launch_as(*this, E4C_KCLASS_BC, 1, [&] { launch_bc(b.v, d_sim, stream); });
        if (b.linear_bc)
            launch_as(*this, E4C_KCLASS_BC, 1, [&] { launch_bc_linear(b.v, d_sim, gas, stream); });
    }
    // simcore.d:2354-2358: shock points after every block's ghost cells
    if (cfg.flux_calculator == E4C_FLUX_ADAPTIVE_HANEL_AUSMDV) {
        for (int h : hs) {
            const BlockHost& b = blocks[h];
            if (!b.fused)
                launch_as(*this, E4C_KCLASS_BC, 1,
                          [&] { launch_shock(b.v, d_sim, fopts.compression_tol, stream); });
        }
    }
    // every face direction of a block in one launch
    for (int h : hs) {
        const BlockHost& b = blocks[h];
        if (b.fused) continue;
        if (b.v.Vrt && fopts.order2 && fopts.local_frame)
            launch_as(*this, E4C_KCLASS_FLUX, 1, [&] { launch_replay_base(b.v, d_sim, stream); });
        launch_as(*this, E4C_KCLASS_FLUX, 1, [&] { launch_flux(b.v, d_sim, fopts, -1, stream); });
    }
    // applyPostConvFluxAction of every block (simcore.d:2373-2377)
    for (int h : hs) {
        const BlockHost& b = blocks[h];
        if (b.fused || !b.simple_flux) continue;
        launch_as(*this, E4C_KCLASS_BC, 1, [&] { launch_bc_flux(b.v, d_sim, fopts, stream); });
    }
    for (int h : hs) {
        const BlockHost& b = blocks[h];
        if (b.fused) continue;
        launch_as(*this, E4C_KCLASS_UPDATE, 1,
                  [&] { launch_update(b.v, d_sim, gas, stage, final_stage, stream); });
    }
    launch_as(*this, E4C_KCLASS_OTHER, 1,
              [&] { launch_stage_check(d_sim, cfg.max_invalid_cells, stream); });
}

void Ctx::enqueue_chemistry(const std::vector<int>& hs, const double* dt) {
    for (int h : hs) {
        const BlockHost& b = blocks[h];
        cudaMemsetAsync(d_chem_nwork, 0, sizeof(int), stream);
        launch_as(*this, E4C_KCLASS_CHEM, 1, [&] {
            launch_chem(b.v, d_sim, cfg.T_frozen, dt, nreac, d_chem_work, d_chem_nwork,
                        d_chem_stats, stream);
        });
        const double* guess = nullptr;
        if (seed.enabled && seed.d_guess && b.ncell <= seed.guess_cap) {
            launch_as(*this, E4C_KCLASS_SEED, 1,
                      [&] { seed_infer(b.v, dt, d_chem_work, d_chem_nwork); });
            guess = seed.d_guess;
        }
        launch_as(*this, E4C_KCLASS_CHEM_WORK, 1, [&] {
            launch_chem_work(b.v, d_sim, cfg.T_frozen, dt, nreac, d_chem_work, d_chem_nwork,
                             guess, d_chem_stats, stream);
        });
    }
}

int Ctx::ensure_chem_work(size_t ncell) {
    if (ncell <= chem_work_cap) return E4C_OK;
    dfree(d_chem_work);
    d_chem_work = static_cast<int*>(dalloc((ncell + 16) * sizeof(int)));
    if (!d_chem_work) {
        chem_work_cap = 0;
        d_chem_nwork = nullptr;
        return fail(E4C_ERR_CUDA, "cudaMalloc of the chemistry work list failed");
    }
    d_chem_nwork = d_chem_work + ncell;
    chem_work_cap = ncell;
    return E4C_OK;
}

void Ctx::enqueue_gasdynamic(const std::vector<int>& hs) {
    const int nstages = (cfg.gasdynamic_update_scheme == E4C_UPDATE_PC) ? 2 : 1;
    for (int s = 1; s <= nstages; ++s) enqueue_stage(hs, s, s == nstages);
    // chemistry_step(dt_global) after the gas-dynamic increment (simcore.d:903-907)
    if (cfg.reacting) enqueue_chemistry(hs, &d_sim->dt_global);
    launch_as(*this, E4C_KCLASS_OTHER, 1, [&] { launch_end_step(d_sim, stream); });
}

// dt control over the given blocks; accumulators are indexed by handle and
// d_hl lists the handles of hs on the device.
void Ctx::enqueue_dt(const std::vector<int>& hs, const int* d_hl, const double* dt_current,
                     int check_cfl, int step0, SimDev* sim, double* out) {
    launch_as(*this, E4C_KCLASS_OTHER, 1,
              [&] { launch_dt_reset(d_dtacc, int(blocks.size()), stream); });
    bool any_fused = false;
    for (int h : hs) {
        const BlockHost& b = blocks[h];
        if (b.fused) { any_fused = true; continue; }
        launch_as(*this, E4C_KCLASS_DT, 1, [&] {
            launch_dt(b.v, sim, cfg.cfl_value, dt_current, d_dtacc + 3 * h, stream);
        });
    }
    if (any_fused) launch_as(*this, E4C_KCLASS_DT, 1, [&] { fused_dt_all(sim, dt_current); });
    const double cfl_allow = (cfg.gasdynamic_update_scheme == E4C_UPDATE_PC) ? 1.2 : 0.9;
    launch_as(*this, E4C_KCLASS_OTHER, 1, [&] {
        launch_dt_finalize(sim, d_dtacc, d_hl, int(hs.size()), cfl_allow, cfg.dt_init, cfg.dt_max,
                           check_cfl, step0, out, out ? out + 1 : nullptr, stream);
    });
}

std::vector<int> Ctx::all_blocks() const {
    std::vector<int> hs(blocks.size());
    for (size_t q = 0; q < blocks.size(); ++q) hs[q] = int(q);
    return hs;
}

}  // namespace e4c

using namespace e4c;

extern "C" {

static int read_sim(SimDev& s);
static int status_error(const SimDev& s);

int e4c_config_default(e4c_config* c) {
    if (!c) return fail(E4C_ERR_ARG, "e4c_config_default: null config");
    std::memset(c, 0, sizeof(*c));
    c->dimensions = 2;
    c->flux_calculator = E4C_FLUX_ADAPTIVE_HANEL_AUSMDV;  // globalconfig.d:533
    c->interpolation_order = 2;
    c->apply_limiter = 1;
    c->extrema_clipping = 1;
    c->interpolate_in_local_frame = 1;
    c->gasdynamic_update_scheme = E4C_UPDATE_PC;
    c->cfl_value = 0.5;
    c->dt_init = 1.0e-3;
    c->dt_max = 1.0e-3;
    c->cfl_count = 10;
    c->max_invalid_cells = 0;
    c->gas_model = E4C_GAS_IDEAL;
    c->ideal_mol_mass = 0.02896;
    c->ideal_gamma = 1.4;
    c->reacting = 0;
    c->T_frozen = 300.0;
    c->precision = E4C_PREC_FP64;
    c->device = 0;
    c->use_graphs = 1;
    c->shear_tolerance = 0.20;        // globalconfig.d:585
    c->compression_tolerance = -0.30; // globalconfig.d:600
    c->chem_newton_iterations = 12;
    return E4C_OK;
}

int e4c_init(const e4c_config* cfg) {
    if (!cfg) return fail(E4C_ERR_ARG, "e4c_init: null config");
    if (g_ctx.initialised) g_ctx.release();
    if (cfg->dimensions != 2 && cfg->dimensions != 3)
        return fail(E4C_ERR_UNSUPPORTED, "dimensions must be 2 or 3");
    if (cfg->flux_calculator < E4C_FLUX_AUSMDV || cfg->flux_calculator > E4C_FLUX_ADAPTIVE_HANEL_AUSMDV)
        return fail(E4C_ERR_UNSUPPORTED,
                    "flux_calculator must be ausmdv, hllc, hanel or adaptive_hanel_ausmdv");
    if (cfg->interpolation_order != 1 && cfg->interpolation_order != 2)
        return fail(E4C_ERR_UNSUPPORTED, "interpolation_order must be 1 or 2");
    if (cfg->gasdynamic_update_scheme != E4C_UPDATE_EULER &&
        cfg->gasdynamic_update_scheme != E4C_UPDATE_PC)
        return fail(E4C_ERR_UNSUPPORTED, "gasdynamic_update_scheme must be euler or predictor-corrector");
    if (cfg->gas_model != E4C_GAS_IDEAL && cfg->gas_model != E4C_GAS_THERM_PERF_5SP_AIR)
        return fail(E4C_ERR_UNSUPPORTED, "unknown gas model");
    if (cfg->precision != E4C_PREC_FP64 && cfg->precision != E4C_PREC_FP32_FLUX)
        return fail(E4C_ERR_UNSUPPORTED, "unknown precision");
    if (cfg->reacting && cfg->gas_model != E4C_GAS_THERM_PERF_5SP_AIR)
        return fail(E4C_ERR_UNSUPPORTED, "reacting flow needs the thermally perfect mixture");
    if (cfg->gas_model != E4C_GAS_IDEAL && cfg->precision != E4C_PREC_FP64)
        return fail(E4C_ERR_UNSUPPORTED, "the FP32-flux form is for the ideal gas");
    if (cfg->cfl_count < 1) return fail(E4C_ERR_ARG, "cfl_count must be >= 1");
    if (cfg->chem_newton_iterations < 0 || cfg->chem_newton_iterations > 100)
        return fail(E4C_ERR_ARG, "chem_newton_iterations must be in 0..100");
    if (cfg->chem_method != E4C_CHEM_POINT_IMPLICIT && cfg->chem_method != E4C_CHEM_RKF)
        return fail(E4C_ERR_UNSUPPORTED, "chem_method must be point-implicit or rkf");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(E4C_ERR_CUDA, "no CUDA device available");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(E4C_ERR_ARG, "bad device ordinal");
    E4C_CUDA(cudaSetDevice(cfg->device));
    Ctx& c = g_ctx;
    c.cfg = *cfg;
    {
        // the allocation-free dt control's scratch array, on this device
        int rc = noalloc_setup(&c.noalloc_scratch);
        if (rc != E4C_OK) return rc;
    }
    c.gas.Rgas = 8.31451 / cfg->ideal_mol_mass;  // ideal_gas.d:66-69
    c.gas.gamma = cfg->ideal_gamma;
    c.gas.Cv = c.gas.Rgas / (c.gas.gamma - 1.0);
    c.gas.Cvinv = 1.0 / c.gas.Cv;
    c.gas.Cp = c.gas.Rgas * c.gas.gamma / (c.gas.gamma - 1.0);
    c.fopts.flux = cfg->flux_calculator;
    c.fopts.order2 = cfg->interpolation_order > 1;
    c.fopts.limiter = cfg->apply_limiter != 0;
    c.fopts.clip = cfg->extrema_clipping != 0;
    c.fopts.local_frame = cfg->interpolate_in_local_frame != 0;
    c.fopts.gas = c.gas;
    c.fopts.shear_tol = cfg->shear_tolerance;
    c.fopts.compression_tol = cfg->compression_tolerance;
    c.fopts.row_run_i = 0;
    c.fopts.row_run_jk = 0;
    E4C_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    E4C_CUDA(cudaStreamCreateWithFlags(&c.h2d_stream, cudaStreamNonBlocking));
    E4C_CUDA(cudaStreamCreateWithFlags(&c.d2h_stream, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&c.ev_in_copied, &c.ev_in_consumed, &c.ev_out_ready, &c.ev_out_copied})
        E4C_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    c.d_sim = static_cast<SimDev*>(c.dalloc(sizeof(SimDev) + 64));
    c.d_dtacc = nullptr;
    c.dtacc_cap = 0;
    c.d_scalars = static_cast<double*>(c.dalloc(8 * sizeof(double)));
    c.d_chem_stats = static_cast<unsigned long long*>(c.dalloc(4 * sizeof(unsigned long long)));
    if (!c.d_sim || !c.d_scalars || !c.d_chem_stats) return fail(E4C_ERR_CUDA, "cudaMalloc failed");
    E4C_CUDA(cudaMemsetAsync(c.d_chem_stats, 0, 4 * sizeof(unsigned long long), c.stream));
    E4C_CUDA(cudaMallocHost(&c.host_pinned, 4096));
    SimDev s0{};
    s0.dt_global = cfg->dt_init;  // simcore.d:562
    s0.max_time = 1.0e300;
    E4C_CUDA(cudaMemcpyAsync(c.d_sim, &s0, sizeof(SimDev), cudaMemcpyHostToDevice, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    c.host_step = 0;
    c.host_step_valid = false;
    c.have_thermochem = false;
    c.nreac = 0;
    c.initialised = true;
    return E4C_OK;
}

int e4c_finalize(void) {
    if (g_ctx.initialised) g_ctx.release();
    return E4C_OK;
}

int e4c_set_thermochem(const e4c_thermochem* tc) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!tc) return fail(E4C_ERR_ARG, "null thermochem");
    if (c.cfg.gas_model != E4C_GAS_THERM_PERF_5SP_AIR)
        return fail(E4C_ERR_STATE, "the configured gas model is not the thermally perfect mixture");
    if (tc->nsp != 5 || tc->nreac != 5)
        return fail(E4C_ERR_UNSUPPORTED, "this build carries 5 species and 5 reactions");
    for (int i = 0; i < tc->nsp; ++i)
        if (tc->nseg[i] < 2 || tc->nseg[i] > E4C_MAXSEG || !(tc->M[i] > 0.0))
            return fail(E4C_ERR_ARG, "bad species thermo data");
    if (!c.blocks.empty()) return fail(E4C_ERR_STATE, "set the mixture before creating blocks");
    if (set_thermochem_constants(*tc) != 0) return fail(E4C_ERR_CUDA, "copy of the mixture failed");
    if (set_chem_newton_iterations(c.cfg.chem_newton_iterations) != 0)
        return fail(E4C_ERR_CUDA, "copy of the chemistry settings failed");
    if (set_chem_method(c.cfg.chem_method) != 0)
        return fail(E4C_ERR_CUDA, "setting the chemistry method failed");
    c.have_thermochem = true;
    c.nreac = tc->nreac;
    for (int i = 0; i < 5; ++i) c.seed.mol.M[i] = tc->M[i];
    return E4C_OK;
}

int e4c_chemistry_step(const int* h, int nb, double dt) {
    NvtxRange nvtx_range("e4c_chemistry_step");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!c.cfg.reacting || !c.have_thermochem) return fail(E4C_ERR_STATE, "not a reacting configuration");
    if (!h || nb <= 0) return fail(E4C_ERR_ARG, "no blocks given");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(E4C_ERR_ARG, "dt must be positive and finite");
    std::vector<int> hs(h, h + nb);
    for (int x : hs)
        if (x < 0 || x >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    double* hp = static_cast<double*>(c.host_pinned);
    hp[9] = dt;
    E4C_CUDA(cudaMemcpyAsync(c.d_scalars + 4, hp + 9, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    launch_begin_run(c.d_sim, 1.0e300, c.stream);
    c.enqueue_chemistry(hs, c.d_scalars + 4);
    E4C_CUDA(cudaGetLastError());
    SimDev s;
    int rc = read_sim(s);
    if (rc != E4C_OK) return rc;
    if (s.status != 0) return status_error(s);
    return E4C_OK;
}

int e4c_chemistry_counters(long long* out, int reset) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!out) return fail(E4C_ERR_ARG, "null output");
    unsigned long long* hp = static_cast<unsigned long long*>(c.host_pinned) + 32;
    E4C_CUDA(cudaMemcpyAsync(hp, c.d_chem_stats, 4 * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, c.stream));
    if (reset)
        E4C_CUDA(cudaMemsetAsync(c.d_chem_stats, 0, 4 * sizeof(unsigned long long), c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    for (int q = 0; q < 4; ++q) out[q] = (long long)hp[q];
    return E4C_OK;
}

int e4c_block_create(int ni, int nj, int nk, const double* vtx_xyz, const int* bc_type,
                     const double* inflow_prim) {
    NvtxRange nvtx_range("e4c_block_create");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "e4c_block_create before e4c_init");
    if (c.cfg.gas_model == E4C_GAS_THERM_PERF_5SP_AIR && !c.have_thermochem)
        return fail(E4C_ERR_STATE, "call e4c_set_thermochem before creating blocks");
    if (!vtx_xyz || !bc_type || !inflow_prim) return fail(E4C_ERR_ARG, "null pointer");
    const int dim = c.cfg.dimensions;
    if (dim == 2) nk = 1;
    if (ni < 2 || nj < 2 || (dim == 3 && nk < 2))
        return fail(E4C_ERR_ARG, "a block needs at least 2 cells in each active direction");
    for (int q = 0; q < 6; ++q)
        if (bc_type[q] < 0 || bc_type[q] > E4C_BC_OUTFLOW_EXTRAPOLATE_LINEAR || bc_type[q] == E4C_BC_EXCHANGE)
            return fail(E4C_ERR_UNSUPPORTED, "unknown boundary type");
    BlockHost b;
    int rc = c.build_block(ni, nj, nk, vtx_xyz, bc_type, inflow_prim, b);
    if (rc != E4C_OK) return rc;
    if (c.cfg.reacting) {
        rc = c.ensure_chem_work(b.ncell);
        if (rc != E4C_OK) return rc;
    }
    c.blocks.push_back(b);
    c.blocks.back().v.block_id = int(c.blocks.size()) - 1;
    c.reset_graphs();
    return int(c.blocks.size()) - 1;
}

int e4c_connect_blocks(int ha, int fa, int hb, int fb, int orientation) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    const int nb = int(c.blocks.size());
    if (ha < 0 || ha >= nb || hb < 0 || hb >= nb || ha == hb)
        return fail(E4C_ERR_ARG, "bad block handles");
    if (fa < 0 || fa > 5 || fb < 0 || fb > 5) return fail(E4C_ERR_ARG, "bad face");
    BlockHost& A = c.blocks[ha];
    BlockHost& B = c.blocks[hb];
    const bool three_d = c.cfg.dimensions == 3;
    if (!three_d && (fa >= 4 || fb >= 4)) return fail(E4C_ERR_ARG, "no top/bottom faces in 2-D");
    if (orientation < 0 || orientation > 3 || (!three_d && orientation != 0))
        return fail(E4C_ERR_ARG, "orientation must be 0..3 (0 in 2-D)");
    const BlockView &va = A.v, &vb = B.v;
    // the cells of the two faces along their (p, q) indices (ffc_partner)
    auto face_extents = [](const BlockView& v, int f, int& P, int& Q) {
        P = (f == EAST || f == WEST) ? v.nj : v.ni;
        Q = (f == TOP || f == BOTTOM) ? v.nj : v.nk;
    };
    int Pa, Qa, Pb, Qb;
    face_extents(va, fa, Pa, Qa);
    face_extents(vb, fb, Pb, Qb);
    const bool same = (orientation & 1) ? (Pa == Qb && Qa == Pb) : (Pa == Pb && Qa == Qb);
    if (!same) return fail(E4C_ERR_ARG, "the joined faces differ in size");
    static const int opposite[6] = {SOUTH, WEST, NORTH, EAST, BOTTOM, TOP};
    if (A.fused != B.fused)
        return fail(E4C_ERR_UNSUPPORTED, "a uniform (fused) block joins only another uniform block");
    if (A.fused) {
        if (opposite[fa] != fb || orientation != 0)
            return fail(E4C_ERR_UNSUPPORTED, "uniform (fused) blocks join opposite faces at "
                                             "orientation 0 only (their frames are the axes)");
        const FusedDesc &x = A.f, &y = B.f;
        bool eq = x.vol == y.vol;
        for (int q = 0; q < 3; ++q) {
            eq = eq && x.len[q] == y.len[q] && x.area[q] == y.area[q];
            for (int r = 0; r < 3; ++r)
                eq = eq && x.fn[q][r] == y.fn[q][r] && x.ft1[q][r] == y.ft1[q][r] &&
                     x.ft2[q][r] == y.ft2[q][r];
        }
        if (!eq) return fail(E4C_ERR_UNSUPPORTED, "joined uniform blocks must have identical cell geometry");
        A.f.bc[fa] = E4C_BC_EXCHANGE;
        B.f.bc[fb] = E4C_BC_EXCHANGE;
    }
    A.ex_block[fa] = hb;
    B.ex_block[fb] = ha;
    A.v.bc[fa] = E4C_BC_EXCHANGE;
    B.v.bc[fb] = E4C_BC_EXCHANGE;
    if (!A.fused) {
        auto src = [orientation](const BlockView& o, int face) {
            ExchangeSrc e{};
            e.W = o.W;
            e.cgeom = o.cgeom;
            e.S = o.S;
            e.npad = o.npad;
            e.nidim = o.nidim;
            e.njdim = o.njdim;
            e.ni = o.ni;
            e.nj = o.nj;
            e.nk = o.nk;
            e.face = face;
            e.orient = orientation;
            e.kmin = o.kmin;
            return e;
        };
        A.v.ex[fa] = src(B.v, fb);
        B.v.ex[fb] = src(A.v, fa);
        launch_exchange_geometry(A.v, fa, c.stream);
        launch_exchange_geometry(B.v, fb, c.stream);
        c.launches += 2;
        E4C_CUDA(cudaGetLastError());
        E4C_CUDA(cudaStreamSynchronize(c.stream));
    }
    c.descs_valid = false;
    c.reset_graphs();
    return E4C_OK;
}

int e4c_block_upload(int h, const double* prim) {
    NvtxRange nvtx_range("e4c_block_upload");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size()) || !prim) return fail(E4C_ERR_ARG, "bad handle or pointer");
    BlockHost& b = c.blocks[h];
    size_t bytes = b.nprim_vars * b.ncell * sizeof(double);
    E4C_CUDA(cudaMemcpyAsync(c.d_staging, prim, bytes, cudaMemcpyHostToDevice, c.stream));
    if (b.fused) {
        int rc = c.fused_upload(b, c.d_staging);
        if (rc != E4C_OK) return rc;
    } else {
        launch_upload(b.v, c.d_staging, c.stream);
        if (b.linear_bc) launch_ghost_defaults(b.v, c.gas, c.stream);
    }
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    return E4C_OK;
}

int e4c_block_upload_cons(int h, const double* cons) {
    NvtxRange nvtx_range("e4c_block_upload_cons");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size()) || !cons) return fail(E4C_ERR_ARG, "bad handle or pointer");
    BlockHost& b = c.blocks[h];
    if (b.v.nsp != 1) return c.upload_cons(b, nullptr);
    const size_t bytes = 5 * b.ncell * sizeof(double);
    E4C_CUDA(cudaMemcpyAsync(c.d_staging, cons, bytes, cudaMemcpyHostToDevice, c.stream));
    int rc = c.upload_cons(b, c.d_staging);
    if (rc != E4C_OK) return rc;
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    SimDev st;
    rc = read_sim(st);
    if (rc != E4C_OK) return rc;
    if (st.status != 0) return status_error(st);
    return E4C_OK;
}

int e4c_block_download(int h, double* prim, double* cons) {
    NvtxRange nvtx_range("e4c_block_download");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad handle");
    BlockHost& b = c.blocks[h];
    double* dp = c.d_staging;
    double* dc = c.d_staging + b.nprim_vars * b.ncell;
    if (b.fused) c.fused_download(b, prim ? dp : nullptr, cons ? dc : nullptr);
    else launch_download(b.v, prim ? dp : nullptr, cons ? dc : nullptr, c.stream);
    E4C_CUDA(cudaGetLastError());
    if (prim)
        E4C_CUDA(cudaMemcpyAsync(prim, dp, b.nprim_vars * b.ncell * sizeof(double),
                                 cudaMemcpyDeviceToHost, c.stream));
    if (cons)
        E4C_CUDA(cudaMemcpyAsync(cons, dc, b.v.nv * b.ncell * sizeof(double),
                                 cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    return E4C_OK;
}

static int dt_chem_io(int h, double* host, int to_host) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size()) || !host) return fail(E4C_ERR_ARG, "bad handle or pointer");
    BlockHost& b = c.blocks[h];
    if (!b.v.dt_chem) return fail(E4C_ERR_STATE, "the block carries no chemistry step (not reacting)");
    const size_t bytes = b.ncell * sizeof(double);
    if (to_host) {
        launch_dt_chem_copy(b.v, c.d_staging, 1, c.stream);
        c.launches += 1;
        E4C_CUDA(cudaGetLastError());
        E4C_CUDA(cudaMemcpyAsync(host, c.d_staging, bytes, cudaMemcpyDeviceToHost, c.stream));
    } else {
        E4C_CUDA(cudaMemcpyAsync(c.d_staging, host, bytes, cudaMemcpyHostToDevice, c.stream));
        launch_dt_chem_copy(b.v, c.d_staging, 0, c.stream);
        c.launches += 1;
        E4C_CUDA(cudaGetLastError());
    }
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    return E4C_OK;
}

int e4c_block_get_dt_chem(int h, double* dt_chem) { return dt_chem_io(h, dt_chem, 1); }

int e4c_block_set_dt_chem(int h, const double* dt_chem) {
    return dt_chem_io(h, const_cast<double*>(dt_chem), 0);
}

int Ctx::ensure_stage_io(size_t bytes) {
    if (bytes <= stage_io_bytes) return E4C_OK;
    // the previous buffers may still be in use by queued transfers
    if (h2d_stream) cudaStreamSynchronize(h2d_stream);
    if (d2h_stream) cudaStreamSynchronize(d2h_stream);
    cudaStreamSynchronize(stream);
    dfree(d_stage_in);
    dfree(d_stage_out);
    d_stage_in = static_cast<double*>(dalloc(bytes));
    d_stage_out = static_cast<double*>(dalloc(bytes));
    if (!d_stage_in || !d_stage_out) {
        dfree(d_stage_in);
        dfree(d_stage_out);
        d_stage_in = d_stage_out = nullptr;
        stage_io_bytes = 0;
        return fail(E4C_ERR_CUDA, "cudaMalloc of the transfer staging buffers failed");
    }
    stage_io_bytes = bytes;
    return E4C_OK;
}

int e4c_block_upload_async(int h, const double* prim) {
    NvtxRange nvtx_range("e4c_block_upload_async");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size()) || !prim) return fail(E4C_ERR_ARG, "bad handle or pointer");
    BlockHost& b = c.blocks[h];
    int rc = c.ensure_stage_io((b.nprim_vars + size_t(b.v.nv)) * b.ncell * sizeof(double));
    if (rc != E4C_OK) return rc;
    const size_t bytes = b.nprim_vars * b.ncell * sizeof(double);
    // the copy waits until the previous upload's conversion has read the buffer
    E4C_CUDA(cudaStreamWaitEvent(c.h2d_stream, c.ev_in_consumed, 0));
    E4C_CUDA(cudaMemcpyAsync(c.d_stage_in, prim, bytes, cudaMemcpyHostToDevice, c.h2d_stream));
    E4C_CUDA(cudaEventRecord(c.ev_in_copied, c.h2d_stream));
    E4C_CUDA(cudaStreamWaitEvent(c.stream, c.ev_in_copied, 0));
    if (b.fused) {
        rc = c.fused_upload(b, c.d_stage_in);
        if (rc != E4C_OK) return rc;
    } else {
        launch_upload(b.v, c.d_stage_in, c.stream);
        if (b.linear_bc) launch_ghost_defaults(b.v, c.gas, c.stream);
    }
    c.launches += 1;
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaEventRecord(c.ev_in_consumed, c.stream));
    return E4C_OK;
}

int e4c_block_upload_cons_async(int h, const double* cons) {
    NvtxRange nvtx_range("e4c_block_upload_cons_async");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size()) || !cons) return fail(E4C_ERR_ARG, "bad handle or pointer");
    BlockHost& b = c.blocks[h];
    if (b.v.nsp != 1) return c.upload_cons(b, nullptr);
    int rc = c.ensure_stage_io((b.nprim_vars + size_t(b.v.nv)) * b.ncell * sizeof(double));
    if (rc != E4C_OK) return rc;
    const size_t bytes = 5 * b.ncell * sizeof(double);
    E4C_CUDA(cudaStreamWaitEvent(c.h2d_stream, c.ev_in_consumed, 0));
    E4C_CUDA(cudaMemcpyAsync(c.d_stage_in, cons, bytes, cudaMemcpyHostToDevice, c.h2d_stream));
    E4C_CUDA(cudaEventRecord(c.ev_in_copied, c.h2d_stream));
    E4C_CUDA(cudaStreamWaitEvent(c.stream, c.ev_in_copied, 0));
    rc = c.upload_cons(b, c.d_stage_in);
    if (rc != E4C_OK) return rc;
    c.launches += 1;
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaEventRecord(c.ev_in_consumed, c.stream));
    return E4C_OK;
}

int e4c_block_download_async(int h, double* prim, double* cons) {
    NvtxRange nvtx_range("e4c_block_download_async");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (h < 0 || h >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad handle");
    BlockHost& b = c.blocks[h];
    int rc = c.ensure_stage_io((b.nprim_vars + size_t(b.v.nv)) * b.ncell * sizeof(double));
    if (rc != E4C_OK) return rc;
    double* dp = c.d_stage_out;
    double* dc = c.d_stage_out + b.nprim_vars * b.ncell;
    // the conversion waits until the previous download has been copied out
    E4C_CUDA(cudaStreamWaitEvent(c.stream, c.ev_out_copied, 0));
    if (b.fused) c.fused_download(b, prim ? dp : nullptr, cons ? dc : nullptr);
    else launch_download(b.v, prim ? dp : nullptr, cons ? dc : nullptr, c.stream);
    c.launches += 1;
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaEventRecord(c.ev_out_ready, c.stream));
    E4C_CUDA(cudaStreamWaitEvent(c.d2h_stream, c.ev_out_ready, 0));
    if (prim)
        E4C_CUDA(cudaMemcpyAsync(prim, dp, b.nprim_vars * b.ncell * sizeof(double),
                                 cudaMemcpyDeviceToHost, c.d2h_stream));
    if (cons)
        E4C_CUDA(cudaMemcpyAsync(cons, dc, b.v.nv * b.ncell * sizeof(double),
                                 cudaMemcpyDeviceToHost, c.d2h_stream));
    E4C_CUDA(cudaEventRecord(c.ev_out_copied, c.d2h_stream));
    return E4C_OK;
}

int e4c_transfers_wait(void) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    E4C_CUDA(cudaStreamSynchronize(c.h2d_stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.d2h_stream));
    return E4C_OK;
}

static int check_handles(const int* h, int nb, std::vector<int>& hs) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!h || nb <= 0) return fail(E4C_ERR_ARG, "no blocks given");
    hs.assign(h, h + nb);
    for (int x : hs)
        if (x < 0 || x >= int(c.blocks.size())) return fail(E4C_ERR_ARG, "bad block handle");
    int rc = c.prepare_fused();
    if (rc != E4C_OK) return rc;
    if (!c.uses_all_fused(hs))
        return fail(E4C_ERR_ARG, "blocks on the fused uniform path advance together: "
                                 "pass all of them or none");
    return c.set_hlist(hs);
}

int e4c_dt_allow(const int* h, int nb, double dt_current, int check_cfl, double* dt_allow,
                 double* cfl_max) {
    NvtxRange nvtx_range("e4c_dt_allow");
    std::vector<int> hs;
    int rc = check_handles(h, nb, hs);
    if (rc != E4C_OK) return rc;
    if (!dt_allow || !cfl_max) return fail(E4C_ERR_ARG, "null output");
    Ctx& c = g_ctx;
    double* hp = static_cast<double*>(c.host_pinned);
    hp[0] = dt_current;
    E4C_CUDA(cudaMemcpyAsync(c.d_scalars, hp, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    c.enqueue_dt(hs, c.d_hlist + c.hlist_cap, c.d_scalars, check_cfl ? 1 : 0, 0, nullptr,
                 c.d_scalars + 2);
    E4C_CUDA(cudaGetLastError());
    E4C_CUDA(cudaMemcpyAsync(hp + 2, c.d_scalars + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                             c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    *dt_allow = hp[2];
    *cfl_max = hp[3];
    return E4C_OK;
}

static int read_sim(SimDev& s) {
    Ctx& c = g_ctx;
    E4C_CUDA(cudaMemcpyAsync(c.host_pinned, c.d_sim, sizeof(SimDev), cudaMemcpyDeviceToHost, c.stream));
    E4C_CUDA(cudaStreamSynchronize(c.stream));
    std::memcpy(&s, c.host_pinned, sizeof(SimDev));
    return E4C_OK;
}

static int status_error(const SimDev& s) {
    char msg[160];
    const char* what = "device error";
    switch (s.status) {
        case E4C_ERR_BAD_CELLS: what = "Too many bad cells"; break;
        case E4C_ERR_BAD_MASS: what = "Bad cell with negative mass"; break;
        case E4C_ERR_THERMO: what = "Bad cell with failed thermodynamic update"; break;
        case E4C_ERR_CHEM: what = "chemistry update failed"; break;
        case E4C_ERR_TIMEOUT: what = "device wait timed out"; break;
    }
    std::snprintf(msg, sizeof(msg), "%s at step %d (%d invalid cells)", what, s.status_step,
                  s.bad_cells);
    return fail(s.status, msg);
}

int e4c_gasdynamic_step(const int* h, int nb, double dt, int* bad_cells) {
    NvtxRange nvtx_range("e4c_gasdynamic_step");
    g_ctx.host_step_valid = false;
    std::vector<int> hs;
    int rc = check_handles(h, nb, hs);
    if (rc != E4C_OK) return rc;
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(E4C_ERR_ARG, "dt must be positive and finite");
    Ctx& c = g_ctx;
    if (!c.remote.empty())
        return fail(E4C_ERR_STATE, "blocks joined to other ranks advance one stage at a time "
                                   "(e4c_stage, with the face exchange between stages)");
    // The host owns dt: write it as SimState.dt_global, clear a stale finish flag.
    launch_begin_run(c.d_sim, 1.0e300, c.stream);
    double* hp = static_cast<double*>(c.host_pinned);
    hp[8] = dt;
    E4C_CUDA(cudaMemcpyAsync(&c.d_sim->dt_global, hp + 8, sizeof(double), cudaMemcpyHostToDevice,
                             c.stream));
    c.enqueue_gasdynamic(hs);
    E4C_CUDA(cudaGetLastError());
    SimDev s;
    rc = read_sim(s);
    if (rc != E4C_OK) return rc;
    if (bad_cells) *bad_cells = s.bad_cells;
    if (s.status != 0) return status_error(s);
    return E4C_OK;
}

int e4c_stage(const int* h, int nb, int stage, double dt, int* bad_cells) {
    NvtxRange nvtx_range("e4c_stage");
    g_ctx.host_step_valid = false;
    std::vector<int> hs;
    int rc = check_handles(h, nb, hs);
    if (rc != E4C_OK) return rc;
    Ctx& c = g_ctx;
    const int nstages = (c.cfg.gasdynamic_update_scheme == E4C_UPDATE_PC) ? 2 : 1;
    if (stage < 1 || stage > nstages) return fail(E4C_ERR_ARG, "no such stage in this scheme");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(E4C_ERR_ARG, "dt must be positive and finite");
    if (stage == 1) {
        // the host owns dt: SimState.dt_global for the whole step
        launch_begin_run(c.d_sim, 1.0e300, c.stream);
        double* hp = static_cast<double*>(c.host_pinned);
        hp[8] = dt;
        E4C_CUDA(cudaMemcpyAsync(&c.d_sim->dt_global, hp + 8, sizeof(double),
                                 cudaMemcpyHostToDevice, c.stream));
    }
    c.enqueue_stage(hs, stage, stage == nstages);
    if (stage == nstages) {
        // chemistry_step(dt_global) after the gas-dynamic increment, then the
        // step's end (as e4c_gasdynamic_step)
        if (c.cfg.reacting) c.enqueue_chemistry(hs, &c.d_sim->dt_global);
        launch_end_step(c.d_sim, c.stream);
        c.launches += 1;
    }
    E4C_CUDA(cudaGetLastError());
    SimDev s;
    rc = read_sim(s);
    if (rc != E4C_OK) return rc;
    if (bad_cells) *bad_cells = s.bad_cells;
    if (s.status != 0) return status_error(s);
    return E4C_OK;
}

int e4c_integrate(int nsteps, double max_time, e4c_run_info* info) {
    NvtxRange nvtx_range("e4c_integrate");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!c.remote.empty())
        return fail(E4C_ERR_STATE, "blocks joined to other ranks advance one stage at a time "
                                   "(e4c_stage, with the face exchange between stages)");
    if (c.blocks.empty()) return fail(E4C_ERR_STATE, "no blocks");
    if (nsteps < 0) return fail(E4C_ERR_ARG, "negative step count");
    std::vector<int> hs = c.all_blocks();
    int rc = c.prepare_fused();
    if (rc != E4C_OK) return rc;
    SimDev s0;
    rc = read_sim(s0);
    if (rc != E4C_OK) return rc;
    launch_begin_run(c.d_sim, max_time, c.stream);
    const int step_start = s0.step;
    for (int q = 0; q < nsteps; ++q) {
        const int step = step_start + q;
        const bool dt_check = (step % c.cfg.cfl_count) == 0;  // simcore.d:1350-1352
        rc = c.run_step(hs, dt_check);
        if (rc != E4C_OK) return rc;
    }
    E4C_CUDA(cudaGetLastError());
    SimDev s;
    rc = read_sim(s);
    if (rc != E4C_OK) return rc;
    c.host_step = s.step;
    c.host_step_valid = true;
    if (info) {
        info->steps_taken = s.step - step_start;
        info->time = s.time;
        info->dt_global = s.dt_global;
        info->status = s.status;
        info->status_step = s.status_step;
        info->bad_cells = s.bad_cells;
    }
    if (s.status != 0) return status_error(s);
    return E4C_OK;
}

int e4c_integrate_async(int nsteps, double max_time) {
    NvtxRange nvtx_range("e4c_integrate_async");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (c.blocks.empty()) return fail(E4C_ERR_STATE, "no blocks");
    if (nsteps < 0) return fail(E4C_ERR_ARG, "negative step count");
    std::vector<int> hs = c.all_blocks();
    int rc = c.prepare_fused();
    if (rc != E4C_OK) return rc;
    if (!c.host_step_valid) {
        SimDev s0;
        rc = read_sim(s0);
        if (rc != E4C_OK) return rc;
        c.host_step = s0.step;
        c.host_step_valid = true;
    }
    launch_begin_run(c.d_sim, max_time, c.stream);
    for (int q = 0; q < nsteps; ++q) {
        const bool dt_check = ((c.host_step + q) % c.cfg.cfl_count) == 0;  // simcore.d:1350-1352
        rc = c.run_step(hs, dt_check);
        if (rc != E4C_OK) return rc;
    }
    c.host_step += nsteps;
    E4C_CUDA(cudaGetLastError());
    return E4C_OK;
}

int e4c_sim_state(double* time, double* dt_global, int* step) {
    if (!g_ctx.initialised) return fail(E4C_ERR_STATE, "not initialised");
    SimDev s;
    int rc = read_sim(s);
    if (rc != E4C_OK) return rc;
    if (time) *time = s.time;
    if (dt_global) *dt_global = s.dt_global;
    if (step) *step = s.step;
    return E4C_OK;
}

int e4c_synchronize(void) {
    if (!g_ctx.initialised) return fail(E4C_ERR_STATE, "not initialised");
    E4C_CUDA(cudaStreamSynchronize(g_ctx.stream));
    return E4C_OK;
}

void* e4c_stream(void) { return g_ctx.initialised ? static_cast<void*>(g_ctx.stream) : nullptr; }

long long e4c_kernel_launches(void) { return g_ctx.launches; }

int e4c_profile_steps(int nsteps, double* ms, int* launches) {
    NvtxRange nvtx_range("e4c_profile_steps");
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (c.blocks.empty()) return fail(E4C_ERR_STATE, "no blocks");
    if (!ms || !launches || nsteps < 0) return fail(E4C_ERR_ARG, "bad arguments");
    std::vector<int> hs = c.all_blocks();
    int rc = c.prepare_fused();
    if (rc != E4C_OK) return rc;
    SimDev s0;
    rc = read_sim(s0);
    if (rc != E4C_OK) return rc;
    launch_begin_run(c.d_sim, 1.0e300, c.stream);
    c.prof.on = true;
    for (int q = 0; q < nsteps; ++q) {
        const bool dt_check = ((s0.step + q) % c.cfg.cfl_count) == 0;
        if (dt_check) c.enqueue_dt(hs, c.d_hlist, &c.d_sim->dt_global, -1, -1, c.d_sim, nullptr);
        c.enqueue_gasdynamic(hs);
    }
    c.prof.on = false;
    cudaError_t e = cudaStreamSynchronize(c.stream);
    for (int k = 0; k < E4C_NKCLASS; ++k) { ms[k] = 0.0; launches[k] = 0; }
    for (size_t q = 0; q < c.prof.cls.size(); ++q) {
        float t = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&t, c.prof.ev[2 * q], c.prof.ev[2 * q + 1]);
        ms[c.prof.cls[q]] += t;
        launches[c.prof.cls[q]] += 1;
    }
    for (cudaEvent_t x : c.prof.ev) cudaEventDestroy(x);
    c.prof.ev.clear();
    c.prof.cls.clear();
    if (e != cudaSuccess) return cuda_fail(e, "profiled steps");
    SimDev s;
    rc = read_sim(s);
    if (rc != E4C_OK) return rc;
    if (s.status != 0) return status_error(s);
    return E4C_OK;
}

static int read_sim(SimDev& s);

static bool tile_available(int ti, int tj) {
    const int tiles[][2] = {{32, 8}, {32, 4}, {16, 8}, {64, 4}, {16, 16}, {32, 16}};
    for (auto& t : tiles)
        if (t[0] == ti && t[1] == tj) return true;
    return false;
}

int e4c_set_tile(int ti, int tj, int kc) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (!tile_available(ti, tj) || kc < 1) return fail(E4C_ERR_ARG, "tile shape not available");
    c.tile_ti = ti;
    c.tile_tj = tj;
    c.tile_kc = kc;
    c.descs_valid = false;
    c.reset_graphs();
    return E4C_OK;
}

int e4c_set_flux_runs(int i_faces, int jk_faces) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (i_faces < 0 || jk_faces < 0 || (i_faces == 0) != (jk_faces == 0) || i_faces > 4096 ||
        jk_faces > 4096)
        return fail(E4C_ERR_ARG, "flux run lengths: both 0, or both in 1..4096");
    c.fopts.row_run_i = i_faces;
    c.fopts.row_run_jk = jk_faces;
    c.reset_graphs();
    return E4C_OK;
}

int e4c_get_tile(int* ti, int* tj, int* kc) {
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (ti) *ti = c.tile_ti;
    if (tj) *tj = c.tile_tj;
    if (kc) *kc = c.tile_kc;
    return E4C_OK;
}

int e4c_autotune(int nsteps, int* ti, int* tj, int* kc, double* ms_per_step) {
    NvtxRange nvtx_range("e4c_autotune");
    g_ctx.host_step_valid = false;
    Ctx& c = g_ctx;
    if (!c.initialised) return fail(E4C_ERR_STATE, "not initialised");
    if (c.blocks.empty()) return fail(E4C_ERR_STATE, "no blocks");
    if (nsteps < 1) return fail(E4C_ERR_ARG, "nsteps must be >= 1");
    int rc = c.prepare_fused();
    if (rc != E4C_OK) return rc;
    if (c.nfused == 0) {
        if (ti) *ti = c.tile_ti;
        if (tj) *tj = c.tile_tj;
        if (kc) *kc = c.tile_kc;
        if (ms_per_step) *ms_per_step = 0.0;
        return E4C_OK;
    }
    // snapshot everything a step changes: the primitive and conserved state of
    // every block, the initial-sound-speed flags and the device clock
    struct Saved { void* dst; const void* src; size_t bytes; };
    std::vector<Saved> saved;
    const size_t rsz = (c.cfg.precision == E4C_PREC_FP32_FLUX) ? sizeof(float) : sizeof(double);
    for (BlockHost& b : c.blocks) {
        if (b.fused) {
            saved.push_back({nullptr, b.f.WA, 5 * b.ncell * rsz});
            saved.push_back({nullptr, b.f.U0, 5 * b.ncell * sizeof(double)});
            saved.push_back({nullptr, b.f.use_a0, sizeof(int)});
        } else {
            saved.push_back({nullptr, b.v.W, W_NBASE * b.v.npad * sizeof(double)});
            saved.push_back({nullptr, b.v.U0, size_t(b.v.nv) * b.v.npad * sizeof(double)});
        }
    }
    saved.push_back({nullptr, c.d_sim, sizeof(SimDev)});
    size_t total = 0;
    for (auto& x : saved) total += (x.bytes + 255) & ~size_t(255);
    char* backup = nullptr;
    E4C_CUDA(cudaMalloc(&backup, total));
    size_t off = 0;
    for (auto& x : saved) {
        x.dst = backup + off;
        off += (x.bytes + 255) & ~size_t(255);
        E4C_CUDA(cudaMemcpyAsync(x.dst, x.src, x.bytes, cudaMemcpyDeviceToDevice, c.stream));
    }
    auto restore = [&]() {
        for (auto& x : saved)
            cudaMemcpyAsync(const_cast<void*>(x.src), x.dst, x.bytes, cudaMemcpyDeviceToDevice,
                            c.stream);
    };
    const int tiles[][2] = {{32, 8}, {32, 4}, {16, 8}, {64, 4}, {16, 16}, {32, 16}};
    const int kcs[] = {16, 32, 64, 128};
    int best_ti = c.tile_ti, best_tj = c.tile_tj, best_kc = c.tile_kc;
    double best = 1.0e300;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<int> hs = c.all_blocks();
    const bool graphs = c.cfg.use_graphs != 0;
    c.cfg.use_graphs = 0;
    for (auto& t : tiles) {
        for (int k : kcs) {
            c.tile_ti = t[0]; c.tile_tj = t[1]; c.tile_kc = k;
            c.descs_valid = false;
            if (c.prepare_fused() != E4C_OK) { c.last_error.clear(); continue; }
            restore();
            launch_begin_run(c.d_sim, 1.0e300, c.stream);
            // one untimed step with the dt control (as at the start of a run),
            // then the timed ones
            c.run_step(hs, true);
            cudaEventRecord(e0, c.stream);
            for (int q = 0; q < nsteps; ++q) c.run_step(hs, false);
            cudaEventRecord(e1, c.stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            SimDev st;
            if (read_sim(st) != E4C_OK) break;
            if (st.status != 0) continue;  // a trial that failed says nothing about speed
            if (ms / nsteps < best) {
                best = ms / nsteps;
                best_ti = t[0]; best_tj = t[1]; best_kc = k;
            }
        }
    }
    c.cfg.use_graphs = graphs ? 1 : 0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    restore();
    cudaError_t e = cudaStreamSynchronize(c.stream);
    cudaFree(backup);
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    c.tile_ti = best_ti; c.tile_tj = best_tj; c.tile_kc = best_kc;
    c.descs_valid = false;
    rc = c.prepare_fused();
    if (rc != E4C_OK) return rc;
    if (ti) *ti = best_ti;
    if (tj) *tj = best_tj;
    if (kc) *kc = best_kc;
    if (ms_per_step) *ms_per_step = best;
    return E4C_OK;
}

int e4c_last_error(char* buf, int len) {
    if (!buf || len <= 0) return E4C_ERR_ARG;
    std::strncpy(buf, g_ctx.last_error.c_str(), size_t(len) - 1);
    buf[len - 1] = '\0';
    return E4C_OK;
}

}  // extern "C"
