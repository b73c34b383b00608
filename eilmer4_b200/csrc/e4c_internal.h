// e4c_internal.h -- library context and block storage (internal to libe4cuda).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>
#include <vector>

#include "../../include/e4cuda.h"
#include "e4c_kernels.h"
#include "e4c_types.h"

namespace e4c {

// A named NVTX range for the duration of a C-ABI call (seen by Nsight
// Systems and other NVTX tools; a no-op when none is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct BlockHost {
    BlockView v{};          // general path (device arrays unset on the fused path)
    size_t ncell = 0;
    size_t nprim_vars = 8;
    bool fused = false;
    bool simple_flux = false;   // has an OutFlowBC_SimpleFlux boundary
    bool linear_bc = false;     // has an x_order 1 extrapolation boundary
    FusedDesc f{};          // fused path: storage and uniform geometry
    int ex_block[6] = {-1, -1, -1, -1, -1, -1};   // partner handle of an exchange boundary
    int remote[6] = {-1, -1, -1, -1, -1, -1};     // shadow of a partner on another rank
};

// A face of a fused block joined to a block on another rank (e4c_remote.cu):
// the partner's two cell layers next to the joint, as a two-cell-thick
// block the fused loader reads across the joint like a local partner.  Its
// storage (`buf`) is the packed layout e4c_pack_face writes:
// [5 x n primitive values, precision-typed][n doubles: A0][8 bytes: use_a0].
struct RemoteFace {
    int h = -1, face = -1;
    FusedDesc d{};
    void* buf = nullptr;
    size_t bytes = 0;
};

// The learned chemistry seed (e4c_seed.cu): network, training set, guesses.
struct SeedNet {
    float* d_params = nullptr;     // FP32 master parameters
    float* d_grad = nullptr;       // gradient, Adam moments (same layout)
    float* d_m = nullptr;
    float* d_v = nullptr;
    uint16_t* d_packed = nullptr;  // BF16 image used by the tensor-core kernels
    double* d_norm = nullptr;
    float* d_loss = nullptr;
    double norm[E4C_SEED_NNORM] = {};
    bool have_weights = false;
    bool enabled = false;
    int adam_t = 0;
    double* d_feat = nullptr;      // training pairs: features [n][8], targets [n][6]
    double* d_targ = nullptr;
    long long n = 0, cap = 0;
    double* d_guess = nullptr;     // per-cell guesses of the chemistry step [6][ncell]
    size_t guess_cap = 0;
    SeedMolar mol{};
    // tries of the inference kernel's first wait for the tensor cores (the
    // second wait after a time-out always takes the full count)
    int first_wait_tries = 1 << 20;
};

struct GraphSlot {
    cudaGraphExec_t exec = nullptr;
    long long nkernels = 0;   // kernel nodes in the graph
};

// Event bracketing of kernel classes while profiling (e4c_profile_steps).
struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> ev;       // pairs (start, stop)
    std::vector<int> cls;              // class of each pair
    void begin(cudaStream_t s, int c);
    void end(cudaStream_t s);
};

struct Ctx {
    bool initialised = false;
    e4c_config cfg{};
    GasConsts gas{};
    FluxOpts fopts{};
    cudaStream_t stream = nullptr;
    SimDev* d_sim = nullptr;
    unsigned long long* d_dtacc = nullptr;
    int dtacc_cap = 0;
    double* d_scalars = nullptr;
    double* d_staging = nullptr;
    size_t staging_bytes = 0;
    // asynchronous transfers: copy streams, staging buffers and ordering events
    cudaStream_t h2d_stream = nullptr;
    cudaStream_t d2h_stream = nullptr;
    double* d_stage_in = nullptr;
    double* d_stage_out = nullptr;
    size_t stage_io_bytes = 0;
    cudaEvent_t ev_in_copied = nullptr, ev_in_consumed = nullptr;
    cudaEvent_t ev_out_ready = nullptr, ev_out_copied = nullptr;
    void* host_pinned = nullptr;
    std::vector<void*> allocations;
    std::vector<BlockHost> blocks;
    GraphSlot graphs[2];    // [0] plain step, [1] step with dt check
    int host_step = 0;           // device step count as the host last knew it
    bool host_step_valid = false;
    bool have_thermochem = false;
    int nreac = 0;
    // chemistry counters: reacting cells, Newton iterations, recovered cells
    unsigned long long* d_chem_stats = nullptr;
    // chemistry work list (cells needing Newton work) and its length
    int* d_chem_work = nullptr;
    int* d_chem_nwork = nullptr;
    size_t chem_work_cap = 0;
    SeedNet seed;
    // fused path: descriptors of every fused block, rebuilt when blocks change
    FusedDesc* d_descs = nullptr;
    int descs_cap = 0;
    int* d_item_order = nullptr;    // fused work items, costliest first
    long long item_order_cap = 0;
    int nfused = 0;
    long long fused_items = 0;
    bool descs_valid = false;
    int tile_ti = 32, tile_tj = 8, tile_kc = 32;
    int fused_grid = 0;
    int max_cells_fused = 0;
    // device list of block handles for the dt reduction
    int* d_hlist = nullptr;
    int hlist_cap = 0;
    long long launches = 0;   // kernels enqueued (graph replays add their node count)
    // faces joined to blocks on other ranks (their shadow descriptors)
    std::vector<RemoteFace> remote;
    // device address of the allocation-free dt control's scratch array on
    // this context's device (resolved by e4c_init)
    void* noalloc_scratch = nullptr;
    Profiler prof;
    std::string last_error;

    void* dalloc(size_t bytes);
    void dfree(void* p);
    int prepare_fused();
    int set_hlist(const std::vector<int>& hs);
    bool uses_all_fused(const std::vector<int>& hs) const;
    void release();
    void reset_graphs();
    int build_block(int ni, int nj, int nk, const double* vtx, const int* bc,
                    const double* inflow, BlockHost& out);
    int ensure_dtacc(int nb);
    int run_step(const std::vector<int>& hs, bool dt_check);
    void enqueue_stage(const std::vector<int>& hs, int stage, int final_stage);
    void enqueue_gasdynamic(const std::vector<int>& hs);
    void enqueue_chemistry(const std::vector<int>& hs, const double* dt);
    // learned chemistry seed
    int seed_alloc_net();
    int seed_pack();
    int seed_dataset_reserve(long long n);
    int seed_guess_reserve(size_t ncell);
    void seed_infer(const BlockView& v, const double* dt, const int* work, const int* nwork);
    int ensure_chem_work(size_t ncell);
    int ensure_stage_io(size_t bytes);
    void enqueue_dt(const std::vector<int>& hs, const int* d_hl, const double* dt_current,
                    int check_cfl, int step0, SimDev* sim, double* out);
    std::vector<int> all_blocks() const;
    // fused uniform path
    void fused_stage_all(int stage);
    void fused_dt_all(SimDev* sim, const double* dt_current);
    int fused_upload(BlockHost& b, const double* prim);
    int fused_upload_cons(BlockHost& b, const double* cons);
    int upload_cons(BlockHost& b, const double* dev_cons);
    void fused_download(const BlockHost& b, double* prim, double* cons);
};

extern Ctx g_ctx;
// e4c_noalloc.cu: the scratch array's device address on the current device
int noalloc_setup(void** out);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

}  // namespace e4c
