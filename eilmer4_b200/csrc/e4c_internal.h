// e4c_internal.h -- library context and block storage (internal to libe4cuda).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/e4cuda.h"
#include "e4c_kernels.h"
#include "e4c_types.h"

namespace e4c {

// Constants of a block whose geometry is exactly uniform and axis aligned
// (every cell and every face of a direction has the same bits).
struct UniformGeom {
    double vol;
    double len[3];          // iLength, jLength, kLength
    double area[3];         // face area per direction
    double n[3][3], t1[3][3], t2[3][3];  // face frame per direction
};

// Device view of a block on the fused uniform path (e4c_fused.cu).
struct FusedView {
    int ni, nj, nk;
    int bc[6];
    size_t ncell;           // ni*nj*nk, interior only, i fastest
    // primitive state rho, vx, vy, vz, u (FP64) -- 5 x ncell
    double* W;
    // sound speed as uploaded; used until the first decode, then unused
    double* a0;
    int use_a0;
    // primitive state in FP32 for the FP32-flux form -- 5 x ncell
    float* Wf;
    double* U0;             // 5 x ncell
    double* dUdt0;          // 5 x ncell
    double* Wn;             // second primitive buffer (ping-pong), 5 x ncell
    float* Wfn;
    UniformGeom g;
    double inflow[8];
};

struct BlockHost {
    BlockView v{};
    size_t ncell = 0;
    size_t nprim_vars = 8;
    bool fused = false;
    FusedView f{};
    int wsel = 0;           // which primitive buffer holds the current state (fused path)
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
    void* host_pinned = nullptr;
    std::vector<void*> allocations;
    std::vector<BlockHost> blocks;
    GraphSlot graphs[2];    // [0] plain step, [1] step with dt check
    int host_step = 0;
    long long launches = 0;   // kernels enqueued (graph replays add their node count)
    Profiler prof;
    std::string last_error;

    void* dalloc(size_t bytes);
    void release();
    void reset_graphs();
    int build_block(int ni, int nj, int nk, const double* vtx, const int* bc,
                    const double* inflow, BlockHost& out);
    int ensure_dtacc(int nb);
    int run_step(const std::vector<int>& hs, bool dt_check);
    void enqueue_stage(const std::vector<int>& hs, int stage, int final_stage);
    void enqueue_gasdynamic(const std::vector<int>& hs);
    void enqueue_dt(const std::vector<int>& hs, const double* dt_current, int check_cfl, int step0,
                    SimDev* sim, double* out);
    std::vector<int> all_blocks() const;
    // fused uniform path
    void fused_stage(const BlockHost& b, int stage, int final_stage);
    void fused_dt(const BlockHost& b, SimDev* sim, const double* dt_current,
                  unsigned long long* acc);
    void fused_upload(BlockHost& b, const double* prim);
    void fused_download(const BlockHost& b, double* prim, double* cons);
};

extern Ctx g_ctx;
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

}  // namespace e4c
