/*
 * e4cuda.h -- C ABI of libe4cuda, the B200 (sm_100a) explicit structured-block
 * gas-dynamic update for the Eilmer4 solver.
 *
 * The D host keeps its time loop, I/O and configuration; under a
 * version(e4cuda) build the calls below replace, one for one:
 *
 *   e4c_init / e4c_finalize      GlobalConfig set-up and tear-down around
 *                                init_simulation (src/eilmer/simcore.d:180) and
 *                                finalize_simulation (simcore.d:3426)
 *   e4c_block_create             SFluidBlock construction + geometry,
 *                                compute_primary_cell_geometric_data
 *                                (src/eilmer/sfluidblock.d:94-126, 650-842)
 *                                and the boundary-condition set-up of
 *                                bc.lua:528-551 (WallBC_WithSlip),
 *                                :974-994 (InFlowBC_Supersonic),
 *                                :1103-1121 (OutFlowBC_SimpleExtrapolate)
 *   e4c_block_upload             read_solution + encode_conserved per block
 *                                (simcore.d:305-322, sfluidblock.d:1778,
 *                                src/eilmer/fvcell.d:494)
 *   e4c_block_download           the state the host writes with
 *                                write_solution_files (simcore.d:637)
 *   e4c_dt_allow                 FluidBlock.determine_time_step_size over the
 *                                given blocks (src/eilmer/fluidblock.d:776-862)
 *   e4c_gasdynamic_step          gasdynamic_explicit_increment_with_fixed_grid
 *                                (simcore.d:2303-2952)
 *   e4c_integrate                the integrate_in_time loop (simcore.d:791-1110)
 *                                restricted to dt control + gas dynamics,
 *                                run on the device as CUDA graphs
 *
 * Conventions (after the gas_cwrap.d C ABI, src/gas/gas_cwrap.d:35-67):
 * integer handles, plain pointers to host arrays borrowed for the duration
 * of the call, return 0 on success and a negative E4C_ERR_* code on failure;
 * e4c_last_error() gives the message.  The library never throws across the
 * ABI, never aborts the process and never traps on the device.  It is not
 * thread-safe: call it from one host thread.  All device memory belongs to
 * the library (allocated at block creation, freed at e4c_finalize).
 *
 * Host arrays:
 *   vertices    (ni+1)*(nj+1)*(nk+1) points, xyz each, i fastest (one k layer in 2-D)
 *   primitive   SoA over interior cells (i fastest), variables
 *               rho, vel.x, vel.y, vel.z, p, T, u, a [, massf[nsp]]
 *   conserved   SoA: mass, x-, y-, z-momentum, total energy [, rho*massf[nsp]]
 */
#ifndef E4CUDA_H
#define E4CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define E4C_OK 0
#define E4C_ERR_ARG (-1)          /* bad argument or handle */
#define E4C_ERR_CUDA (-2)         /* a CUDA runtime call failed */
#define E4C_ERR_UNSUPPORTED (-3)  /* configuration outside the implemented path */
#define E4C_ERR_BAD_CELLS (-4)    /* more invalid cells than max_invalid_cells (simcore.d:2480-2493) */
#define E4C_ERR_BAD_MASS (-5)     /* non-positive density in decode (fvcell.d:570-590) */
#define E4C_ERR_THERMO (-6)       /* thermodynamic update failed (fvcell.d:654-720) */
#define E4C_ERR_CHEM (-7)         /* chemistry update failed (chemistry_update.d:213-270) */
#define E4C_ERR_TIMEOUT (-8)      /* a bounded device wait ran out */
#define E4C_ERR_STATE (-9)        /* call out of order (no e4c_init, no blocks, ...) */

/* Boundary conditions (bc.lua names). */
#define E4C_BC_WALL_WITH_SLIP 0
#define E4C_BC_INFLOW_SUPERSONIC 1
#define E4C_BC_OUTFLOW_SIMPLE_EXTRAPOLATE 2
#define E4C_BC_EXCHANGE 3      /* set by e4c_connect_blocks only */
/* OutFlowBC_SimpleFlux (bc.lua:1124-1146): extrapolated ghost cells and the
 * boundary-face flux from the interior cell (boundary_flux_effect.d:367-546) */
#define E4C_BC_OUTFLOW_SIMPLE_FLUX 4
/* OutFlowBC_SimpleExtrapolate{xOrder=1} (bc.lua:1108-1120): ExtrapolateCopy
 * with x_order 1 (extrapolate_copy.d:206-258 and alike for each face), each
 * ghost layer extrapolated linearly from the two cells before it in rho, u,
 * mass fractions and velocity, T and p from update_thermo_from_rhou, the
 * sound speed and shock flag left as they were (from a ghost cell's initial
 * FlowState: 100 kPa, 300 K, at rest, the first species, set at upload, as
 * fvcell.d:168-170 constructs every cell).  General path only. */
#define E4C_BC_OUTFLOW_EXTRAPOLATE_LINEAR 5

/* flux_calculator (src/eilmer/fvcore.d:184-228, plus the new "hllc"). */
#define E4C_FLUX_AUSMDV 0
#define E4C_FLUX_HLLC 1
#define E4C_FLUX_HANEL 2                  /* fluxcalc.d:532-629 */
#define E4C_FLUX_ADAPTIVE_HANEL_AUSMDV 3  /* fluxcalc.d:824-838, the reference's default;
                                             turns on the shock detector */

/* gasdynamic_update_scheme (fvcore.d:29-110). */
#define E4C_UPDATE_EULER 0
#define E4C_UPDATE_PC 1

/* Arithmetic of the reconstruction and flux. */
#define E4C_PREC_FP64 0       /* all FP64, same operation order as the reference */
#define E4C_PREC_FP32_FLUX 1  /* FP32 reconstruction/flux, FP64 accumulation + decode */

/* Gas models. */
#define E4C_GAS_IDEAL 0
#define E4C_GAS_THERM_PERF_5SP_AIR 1

typedef struct e4c_config {
    int dimensions;                 /* "dimensions" (globalconfig.d:1260) */
    int flux_calculator;            /* "flux_calculator" (globalconfig.d:1329) */
    int interpolation_order;        /* "interpolation_order" (globalconfig.d:1330) */
    int apply_limiter;              /* "apply_limiter" (globalconfig.d:1338) */
    int extrema_clipping;           /* "extrema_clipping" (globalconfig.d:568) */
    int interpolate_in_local_frame; /* "interpolate_in_local_frame" (globalconfig.d:569) */
    int gasdynamic_update_scheme;   /* "gasdynamic_update_scheme" (globalconfig.d:1281) */
    double cfl_value;               /* control "cfl_value" */
    double dt_init;                 /* control "dt_init" */
    double dt_max;                  /* control "dt_max" */
    int cfl_count;                  /* control "cfl_count" */
    int max_invalid_cells;          /* "max_invalid_cells" (globalconfig.d:519) */
    int gas_model;                  /* E4C_GAS_* */
    double ideal_mol_mass;          /* IdealGas.mMass (kg/mol) */
    double ideal_gamma;             /* IdealGas.gamma */
    int reacting;                   /* "reacting" (globalconfig.d:1502) */
    double T_frozen;                /* "T_frozen" (globalconfig.d:692) */
    int precision;                  /* E4C_PREC_* */
    int device;                     /* CUDA device ordinal */
    int use_graphs;                 /* capture e4c_integrate steps in CUDA graphs */
    double shear_tolerance;         /* "shear_tolerance" (globalconfig.d:585), adaptive flux */
    double compression_tolerance;   /* "compression_tolerance" (globalconfig.d:600), shock detector */
    int chem_newton_iterations;     /* Newton iterations of the whole-interval point-implicit
                                       chemistry step before opCall's sub-cycling takes over
                                       (default 12; 0 sends every cell that needs Newton work
                                       to the sub-cycling) */
    int chem_method;                /* E4C_CHEM_POINT_IMPLICIT (default) or E4C_CHEM_RKF: the
                                       reference's odeStep.method 'rkf' (ChemistryUpdate.opCall's
                                       sub-cycling with RKFStep, chemistry_update.d:119-307,
                                       362-461) */
} e4c_config;

#define E4C_CHEM_POINT_IMPLICIT 0
#define E4C_CHEM_RKF 1

typedef struct e4c_run_info {
    int steps_taken;
    double time;
    double dt_global;
    int status;                     /* 0 or the first E4C_ERR_* seen on the device */
    int status_step;                /* step at which status was set */
    int bad_cells;                  /* invalid cells in the last stage */
} e4c_run_info;

/* Thermally perfect mixture and finite-rate mechanism (the data a gas-model
 * file and a reaction file carry): NASA Glenn/CEA 9-coefficient curves with
 * blend ranges per species (src/gas/thermo/cea_thermo_curves.d), modified
 * Arrhenius forward/backward rate constants in SI units
 * (src/kinetics/rate_constant.d:71-75, reaction.lua:20-36), integer
 * stoichiometric coefficients, third-body efficiencies and the rate-constant
 * temperature limits (reaction_mechanism.d:47-57). */
#define E4C_MAXSP 8
#define E4C_MAXSEG 4
#define E4C_MAXR 8
typedef struct e4c_thermochem {
    int nsp;
    double M[E4C_MAXSP];
    int nseg[E4C_MAXSP];
    double T_break[E4C_MAXSP][E4C_MAXSEG + 1];
    double T_blend[E4C_MAXSP][E4C_MAXSEG];
    double coeffs[E4C_MAXSP][E4C_MAXSEG][9];
    int nreac;
    double A_f[E4C_MAXR], n_f[E4C_MAXR], C_f[E4C_MAXR];
    double A_b[E4C_MAXR], n_b[E4C_MAXR], C_b[E4C_MAXR];
    int nu_r[E4C_MAXR][E4C_MAXSP];
    int nu_p[E4C_MAXR][E4C_MAXSP];
    int third_body[E4C_MAXR];
    double eff[E4C_MAXR][E4C_MAXSP];
    double T_lower, T_upper;
} e4c_thermochem;

/* Fill cfg with the reference defaults (globalconfig.d:440-734). */
int e4c_config_default(e4c_config* cfg);

/* Select the device, check the configuration, create the context. */
int e4c_init(const e4c_config* cfg);

/* Install the thermally perfect mixture and mechanism (gas_model
 * E4C_GAS_THERM_PERF_5SP_AIR; call after e4c_init, before creating blocks).
 * Replaces the gas-model construction of src/gas/therm_perf_gas.d and the
 * ChemistryUpdate set-up of src/kinetics/chemistry_update.d:35-117. */
int e4c_set_thermochem(const e4c_thermochem* tc);

/* One chemistry update of every cell of the blocks over dt (chemistry_step,
 * src/eilmer/simcore.d:1489-1505, i.e. FVCell.thermochemical_increment per
 * cell); e4c_integrate calls it after each gas-dynamic step when reacting.
 * Each cell hotter than T_frozen takes one point-implicit (backward-Euler)
 * step over dt, solved by Newton iteration with the analytic Jacobian; when
 * that iteration does not converge, ChemistryUpdate.opCall's sub-cycling
 * (src/kinetics/chemistry_update.d:119-307) with error-controlled
 * point-implicit sub-steps takes over for that cell.  dt must be positive and
 * finite (E4C_ERR_ARG otherwise). */
int e4c_chemistry_step(const int* h, int nb, double dt);

/* Chemistry counters accumulated since e4c_init or the last reset: out[0]
 * reacting cells updated (hotter than T_frozen), out[1] Newton iterations,
 * out[2] cells that needed the sub-cycled recovery, out[3] cells whose start
 * state did not already satisfy the convergence test (the Newton-active
 * cells).  reset != 0 zeroes them after reading.  No counterpart in the
 * reference (diagnostics of the point-implicit update). */
int e4c_chemistry_counters(long long* out, int reset);

/* ---- Learned chemistry seed (no counterpart in the reference) ----------
 * A small multilayer perceptron, input (log T, log p, Y[5], log dt), three
 * hidden layers of 64 GELU units, output the change of the five mass
 * fractions and of T over dt, with BF16 weights run on the tensor cores
 * (FP32 accumulation).  When enabled, each chemistry update first evaluates
 * it for every cell and starts the point-implicit Newton iteration from the
 * predicted end concentrations (or from the start state, whichever has the
 * smaller residual), and the temperature Newton iteration from the predicted
 * end temperature.  The converged result is that of the plain update to
 * within the Newton tolerances; the plain update is also the fallback. */
#define E4C_SEED_NPARAM 9286   /* FP32 parameters: W1[64][8] b1 W2[64][64] b2 W3 b3 W4[6][64] b4 */
#define E4C_SEED_NNORM 30      /* mu_in[8] sd_in[8] mu_out[6] sd_out[6] sY sT */

/* Add nsamples training pairs to the library's training set: cells drawn
 * uniformly from the blocks' Newton-active cells (hotter than T_frozen, start
 * state not already converged over dt; current state), steps dt * f with
 * log f uniform in [log 1/4, log 4], each advanced by the plain chemistry
 * update on the device.  Adds nothing when no cell is active. */
int e4c_seed_collect(const int* h, int nb, double dt, long long nsamples, unsigned long long seed);
int e4c_seed_dataset(long long* n);
int e4c_seed_clear(void);

/* Train the network on the collected pairs with the library's forward and
 * backward tensor-core kernels and Adam (cosine learning-rate decay to 1 % of
 * lr), 2 % of the pairs held out.  report (optional, 6 doubles): final
 * training loss, validation loss, training pairs, validation pairs, seconds,
 * optimiser steps. */
int e4c_seed_train(int epochs, int batch, double lr, unsigned long long seed, double* report);

/* Read or install the network: params[E4C_SEED_NPARAM], norm[E4C_SEED_NNORM]. */
int e4c_seed_get(float* params, double* norm);
int e4c_seed_set(const float* params, const double* norm);

/* Use (on != 0) or stop using the network in the chemistry updates. */
int e4c_seed_enable(int on);

/* Network output for n rows (T, p, Y[5], dt): out[n][6] = predicted dY[5], dT
 * (the inference kernel of the chemistry step, on host data). */
int e4c_seed_predict(const double* rows, long long n, double* out);

/* Loss and gradient of the training kernel on n normalised rows x[n][8],
 * targets y[n][6]: loss = mean of the squared errors, grad[E4C_SEED_NPARAM]. */
int e4c_seed_loss_grad(const float* x, const float* y, int n, double* loss, float* grad);

/* Failure-detection hook (no counterpart in the reference): the number of
 * tries of the seed inference kernel's first bounded wait for the tensor
 * cores (negative: the default, about one million).  With 0 the first wait
 * gives up at once, so the kernel takes its time-out path -- report
 * E4C_ERR_TIMEOUT, wait again with the full count for the multiply it
 * issued, release its tensor memory -- on a healthy device. */
int e4c_seed_set_wait_limit(int first_wait_tries);

/* Free every device buffer and graph; the context may be re-initialised. */
int e4c_finalize(void);

/* Create a structured block; returns a handle >= 0 or an error code.
 * bc_type[6] in the order north, east, south, west, top, bottom.
 * inflow_prim is one primitive FlowState used by inflow boundaries. */
int e4c_block_create(int ni, int nj, int nk, const double* vtx_xyz, const int* bc_type,
                     const double* inflow_prim);

/* Join face face_a of block ha to face face_b of block hb
 * (GhostCellFullFaceCopy, src/eilmer/bc/ghost_cell_effect/full_face_copy.d,
 * set up by the reference's FluidBlockArray / connectBlocks in prep): any
 * pair of faces at orientation 0..3 in 3-D (0 in 2-D), with the reference's
 * cell mapping for each face pair and orientation (full_face_copy.d:142-1083;
 * both blocks carry the same orientation, as connectBlocks sets them) and
 * matching face sizes (swapped by orientations 1 and 3).  Both blocks are on
 * the same path: both general, or both fused with identical uniform geometry,
 * in which case only opposite faces at orientation 0 join (a fused block's
 * index axes are the coordinate axes).  Both faces become exchange
 * boundaries: the ghost cells take the partner's cell geometry now (volume
 * and the i, j, k lengths as the partner holds them, CopyDataOption.grid)
 * and its flow state at the start of every stage.  Call after creating the
 * blocks, before stepping. */
int e4c_connect_blocks(int ha, int face_a, int hb, int face_b, int orientation);

/* Upload a block's primitive state and encode its conserved quantities. */
int e4c_block_upload(int h, const double* prim);

/* Upload a block's conserved state (rho, rho*v, E as SoA, ideal gas) and
 * decode it on the device as the end of a stage does (decode_conserved,
 * fvcell.d:563-732): a host that hands the conserved state back and forth
 * between steps continues bit for bit as an uninterrupted run (a primitive
 * upload re-encodes U).  The mixture returns E4C_ERR_UNSUPPORTED (its
 * temperature iteration needs a starting temperature).  A non-positive
 * density returns E4C_ERR_BAD_MASS and leaves the simulation in that error. */
int e4c_block_upload_cons(int h, const double* cons);

/* Download the primitive and/or conserved state (either pointer may be NULL). */
int e4c_block_download(int h, double* prim, double* cons);

/* Per-cell chemistry step suggestion (dt_chem, the reference's
 * FVCell.dt_chem, fvcell.d:1510-1621) of a reacting block's interior cells,
 * i fastest: read for a flow file's dt_chem column, written back from one
 * on restart (sfluidblock.d:1778-1956). */
int e4c_block_get_dt_chem(int h, double* dt_chem);
int e4c_block_set_dt_chem(int h, const double* dt_chem);

/* Asynchronous forms of e4c_block_upload / e4c_block_download (no
 * counterpart in the reference, whose host and solver share memory).  The
 * host-to-device and device-to-host copies run on two copy streams of their
 * own, ordered by events against the computation, so that one step's
 * download overlaps the next step's upload.  The host buffers must be
 * page-locked (cudaHostAlloc / pinned) for the copies to be asynchronous and
 * must not be touched until e4c_transfers_wait returns.  A download reads the
 * state left by all work queued before it; an upload is seen by all work
 * queued after it. */
int e4c_block_upload_async(int h, const double* prim);
int e4c_block_upload_cons_async(int h, const double* cons);
int e4c_block_download_async(int h, double* prim, double* cons);
int e4c_transfers_wait(void);

/* Allowable time step over the blocks, as FluidBlock.determine_time_step_size
 * followed by the min/max reduction over blocks (simcore.d:1362-1386);
 * check_cfl corresponds to SimState.step > 0. */
int e4c_dt_allow(const int* h, int nb, double dt_current, int check_cfl, double* dt_allow,
                 double* cfl_max);

/* One explicit gas-dynamic step of size dt over the blocks; returns the
 * invalid-cell count of the last stage in *bad_cells.  dt must be positive and
 * finite (E4C_ERR_ARG otherwise; nothing is queued). */
int e4c_gasdynamic_step(const int* h, int nb, double dt, int* bad_cells);

/* One stage of the explicit gas-dynamic step (stage 1 or 2 of the
 * predictor-corrector scheme, 1 of Euler) over the blocks, with dt given on
 * stage 1; the last stage also runs the chemistry (reacting flow) and ends the
 * step.  Two calls give what e4c_gasdynamic_step gives.  For blocks joined to
 * other ranks, whose ghost cells must be exchanged before each stage
 * (simcore.d:2303-2952 calls exchange_ghost_cell_boundary_data before each
 * stage's fluxes, simcore.d:1599). */
int e4c_stage(const int* h, int nb, int stage, double dt, int* bad_cells);

/* Blocks on several ranks, one rank per GPU (the reference's MPI runs: the
 * full-face exchange of full_face_copy.d:1134-1255 between ranks, the dt MIN
 * and bad-cell MAX reductions of simcore.d:1399-1401, 2489 left to the host).
 * e4c_connect_remote joins face `face` of block h (fused uniform 3-D blocks
 * only) to a block on another rank: an opposite face of the same tangential
 * extents and cell geometry, orientation 0.  Before each stage the host calls
 * e4c_pack_face on the partner's rank (the partner's two cell layers next to
 * the joint, from its state at the start of that stage, into a device buffer
 * of e4c_face_slab_bytes bytes), moves the buffer to this rank and calls
 * e4c_unpack_face.  Blocks with such faces advance with e4c_stage (e4c_integrate
 * and e4c_gasdynamic_step return E4C_ERR_STATE). */
int e4c_connect_remote(int h, int face);
int e4c_face_slab_bytes(int h, int face, long long* bytes);
int e4c_pack_face(int h, int face, int stage, void* dev_dst);
int e4c_unpack_face(int h, int face, const void* dev_src);

/* Run the time loop over all blocks for nsteps steps or until max_time:
 * dt control every cfl_count steps, dt_init at step 0, x1.5 growth cap and
 * dt_max, then the gas-dynamic step.  The loop stays on the device. */
int e4c_integrate(int nsteps, double max_time, e4c_run_info* info);

/* e4c_integrate without waiting: the steps are queued on the library stream
 * and the call returns at once (no counterpart in the reference).  The dt
 * control cadence follows the host's count of queued steps, so it matches
 * e4c_integrate as long as every queued step runs (max_time not reached);
 * errors are reported by the next e4c_integrate (e.g. with nsteps = 0). */
int e4c_integrate_async(int nsteps, double max_time);

/* Simulation time, dt_global and step counter of the device-side loop. */
int e4c_sim_state(double* time, double* dt_global, int* step);

/* Wait for all queued device work. */
int e4c_synchronize(void);

/* The cudaStream_t the library enqueues all its work on (for event timing). */
void* e4c_stream(void);

/* Number of kernels the library has enqueued so far; a graph replay counts
 * every kernel node it contains. */
long long e4c_kernel_launches(void);

/* Kernel classes timed by e4c_profile_steps. */
#define E4C_KCLASS_DT 0        /* signal frequency + dt reduction */
#define E4C_KCLASS_BC 1        /* ghost-cell fill (general path) */
#define E4C_KCLASS_FLUX 2      /* reconstruction + flux (general path) */
#define E4C_KCLASS_UPDATE 3    /* cell update + decode (general path) */
#define E4C_KCLASS_STAGE 4     /* fused stage kernel (uniform path) */
#define E4C_KCLASS_OTHER 5     /* bookkeeping kernels */
#define E4C_KCLASS_CHEM 6      /* chemistry cell update */
#define E4C_KCLASS_SEED 7      /* learned chemistry seed (inference) */
#define E4C_KCLASS_CHEM_WORK 8 /* chemistry pass 2: the cells needing Newton work */
#define E4C_NKCLASS 9

/* Run nsteps time steps without graphs, timing each kernel class with CUDA
 * events on the library stream: ms[c] = total milliseconds of class c and
 * launches[c] = its launch count (arrays of E4C_NKCLASS). */
int e4c_profile_steps(int nsteps, double* ms, int* launches);

/* Tile shape of the fused stage kernel used for blocks with uniform
 * Cartesian geometry: ti x tj cells per CTA in the i-j plane, marching kc
 * planes in k.  Available (ti, tj): (32,8), (32,4), (16,8), (64,4), (16,16),
 * (32,16). */
int e4c_set_tile(int ti, int tj, int kc);
int e4c_get_tile(int* ti, int* tj, int* kc);

/* Faces per thread of the row-walking flux kernel that 3-D ideal-gas blocks
 * with general (curvilinear) face frames use: i_faces consecutive i faces,
 * jk_faces consecutive j or k faces.  Both 0 (the default): 8 and 32, halved
 * on small blocks until the launch fills the GPU.  Results do not depend on
 * the lengths (every length gives the same bits); they only set the speed. */
int e4c_set_flux_runs(int i_faces, int jk_faces);

/* Autotuner: time nsteps steps with every available tile shape and k-chunk
 * length on the current blocks, keep the fastest, and restore the flow state
 * and simulation clock exactly as they were before the trials.  Returns the
 * chosen shape and its milliseconds per step. */
int e4c_autotune(int nsteps, int* ti, int* tj, int* kc, double* ms_per_step);

/* Most blocks one e4c_dt_allow_noalloc call can reduce over. */
#define E4C_NOALLOC_MAX_BLOCKS 1024

/* e4c_dt_allow without any device allocation.  No counterpart in the
 * reference: it exists for hosts that cannot let a library call cudaMalloc
 * inside their time loop -- a host that has given the whole GPU memory to its
 * own pool or works to a fixed memory budget, where an allocation may fail or
 * fragment the pool.  e4c_dt_allow may allocate its per-block accumulators on
 * first use; this variant keeps its scratch (accumulators, block list, inputs
 * and results, about 28 KB) in one fixed-size device array that lives in the
 * library for as long as it is loaded, so it reduces over at most
 * E4C_NOALLOC_MAX_BLOCKS blocks per call and returns E4C_ERR_ARG beyond that.
 * Same inputs, outputs and results as e4c_dt_allow (it runs the same
 * kernels).  e4c_init looks up the array's device address on the library's
 * device, which also reserves the array there, so no call does either later;
 * the call returns E4C_ERR_STATE if another device is current.  The array is
 * shared by all calls and keeps the last call's contents (each call resets
 * the accumulators it uses): calls that overlap on the GPU race (the library
 * is single-threaded and uses one stream). */
int e4c_dt_allow_noalloc(const int* h, int nb, double dt_current, int check_cfl,
                         double* dt_allow, double* cfl_max);

/* Copy the message of the last error into buf (always NUL-terminated). */
int e4c_last_error(char* buf, int len);

#ifdef __cplusplus
}
#endif
#endif
