/*
 * e4_oracle.h -- C API of the CPU FP64 oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++ restatement of the
 * Eilmer4 explicit structured-block update (the D code under src/eilmer,
 * src/gas, src/geom, src/kinetics of the reference).  It exists to check the
 * CUDA library and to time a CPU baseline.  Only tests/, the smoke() entry
 * point and the bench's CPU-baseline leg may load it; the product path never
 * does.
 *
 * Conventions follow the reference:
 *   - cells of a structured block are indexed (i,j,k), i fastest;
 *   - boundary order is north, east, south, west, top, bottom
 *     (src/eilmer/fvcore.d Face enum);
 *   - primitive arrays are SoA over interior cells with the variable order
 *     rho, vel.x, vel.y, vel.z, p, T, u, a, massf[0..nsp-1];
 *   - conserved arrays are SoA with the order mass, xmom, ymom, zmom,
 *     total_energy, rho*massf[0..nsp-1] (only when nsp > 1).
 */
#ifndef E4_ORACLE_H
#define E4_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { E4O_BC_SLIP_WALL = 0, E4O_BC_INFLOW_SUPERSONIC = 1, E4O_BC_OUTFLOW_EXTRAPOLATE = 2,
       E4O_BC_EXCHANGE = 3, E4O_BC_OUTFLOW_SIMPLE_FLUX = 4,
       E4O_BC_OUTFLOW_EXTRAPOLATE_LINEAR = 5 /* OutFlowBC_SimpleExtrapolate{xOrder=1} */ };
enum { E4O_FLUX_AUSMDV = 0, E4O_FLUX_HLLC = 1, E4O_FLUX_HANEL = 2, E4O_FLUX_ADAPTIVE_HANEL_AUSMDV = 3 };
enum { E4O_UPDATE_EULER = 0, E4O_UPDATE_PC = 1 };
enum { E4O_GAS_IDEAL = 0, E4O_GAS_THERM_PERF_5SP_AIR = 1 };

typedef struct e4o_config {
    int dimensions;                 /* 2 or 3 */
    int flux_calculator;            /* E4O_FLUX_* */
    int interpolation_order;        /* 1 or 2 */
    int apply_limiter;
    int extrema_clipping;
    int interpolate_in_local_frame;
    int update_scheme;              /* E4O_UPDATE_* */
    double cfl_value;
    double dt_init;
    double dt_max;
    int cfl_count;
    int max_invalid_cells;
    int gas_model;                  /* E4O_GAS_* */
    double ideal_mol_mass;          /* kg/mol (ideal gas) */
    double ideal_gamma;
    int reacting;                   /* finite-rate chemistry after each step */
    double T_frozen;
    int n_threads;                  /* OpenMP threads; <=0 means all */
    double shear_tolerance;         /* adaptive flux: globalconfig.d:585 */
    double compression_tolerance;   /* shock detector: globalconfig.d:600 */
    int chem_newton_iterations;     /* whole-interval point-implicit step (default 12) */
    int chem_method;                /* 0: point-implicit step with opCall's sub-cycled recovery;
                                       1: the reference's odeStep.method 'rkf' (opCall with RKF
                                       sub-steps, chemistry_update.d:119-307, 362-461) */
} e4o_config;

/* Thermally perfect mixture and reaction mechanism (plain arrays).
 * Species thermo: NASA Glenn/CEA 9-coefficient curves with blending
 * (src/gas/thermo/cea_thermo_curves.d).  Reactions: modified Arrhenius
 * forward and backward rate constants in SI units, integer stoichiometric
 * coefficients, optional third body with efficiencies. */
#define E4O_MAXSP 8
#define E4O_MAXSEG 4
#define E4O_MAXR 8
typedef struct e4o_thermochem {
    int nsp;
    double M[E4O_MAXSP];
    int nseg[E4O_MAXSP];
    double T_break[E4O_MAXSP][E4O_MAXSEG + 1];
    double T_blend[E4O_MAXSP][E4O_MAXSEG];
    double coeffs[E4O_MAXSP][E4O_MAXSEG][9];
    int nreac;
    double A_f[E4O_MAXR], n_f[E4O_MAXR], C_f[E4O_MAXR];
    double A_b[E4O_MAXR], n_b[E4O_MAXR], C_b[E4O_MAXR];
    int nu_r[E4O_MAXR][E4O_MAXSP];
    int nu_p[E4O_MAXR][E4O_MAXSP];
    int third_body[E4O_MAXR];
    double eff[E4O_MAXR][E4O_MAXSP];
    double T_lower, T_upper;
} e4o_thermochem;

void e4o_default_config(e4o_config* cfg);

void* e4o_sim_new(const e4o_config* cfg);
void e4o_sim_free(void* sim);

/* Add a structured block.  vtx holds (ni+1)*(nj+1)*(nk+1) points, 3 doubles
 * each, i fastest (nk=1 and one vertex layer for 2D).  bc[6] uses the
 * boundary order north, east, south, west, top, bottom.  inflow is a
 * primitive FlowState (rho,vx,vy,vz,p,T,u,a,massf...) used by inflow BCs.
 * Returns the block index, or a negative error code. */
int e4o_add_block(void* sim, int ni, int nj, int nk, const double* vtx,
                  const int* bc, const double* inflow);

/* Connect face fa of block a to face fb of block b (GhostCellFullFaceCopy,
 * src/eilmer/bc/ghost_cell_effect/full_face_copy.d): opposite faces
 * (east-west, north-south, top-bottom), orientation 0, equal face sizes.
 * Both faces become exchange boundaries; the ghost cells take the partner's
 * cell geometry now and its flow state at every stage. */
int e4o_connect_blocks(void* sim, int a, int fa, int b, int fb, int orientation);
/* The active (from 0) indices of the partner cell that fills ghost layer
 * `depth` behind cell (p, q) of face fa, for a joint with the partner's face
 * fb at orientation r (full_face_copy.d:142-1083); partner extents ni, nj, nk. */
void e4o_ffc_map(int fa, int fb, int r, int p, int q, int depth, int ni, int nj, int nk,
                 int* out3);

/* Set the interior flow state from a primitive SoA array and encode the
 * conserved quantities (src/eilmer/fvcell.d encode_conserved). */
int e4o_set_flow(void* sim, int blk, const double* prim);

/* Read back the primitive and conserved arrays of a block (either may be NULL). */
int e4o_get_flow(void* sim, int blk, double* prim, double* cons);

/* Geometry of a block: cell volume, iLength, jLength, kLength per interior
 * cell (4 x ncell SoA) and, per face direction d (0=i,1=j,2=k), for every
 * face of that direction: n(3), t1(3), t2(3), area -> 10 doubles per face,
 * face arrays laid out as the padded-index faces the reference iterates. */
int e4o_get_cell_geometry(void* sim, int blk, double* out);

/* Advance nsteps time steps (or until max_time), replaying
 * src/eilmer/simcore.d integrate_in_time.  Returns 0 or a negative error. */
int e4o_run(void* sim, int nsteps, double max_time);

/* A face whose partner lives on another rank (full_face_copy.d MPI
 * exchange): its ghost cells keep what e4o_unpack_face writes.  Values per
 * packed face (2 layers x face cells x fields), the packing of the two cell
 * layers next to a face, and their unpacking into a remote face's ghosts. */
int e4o_set_remote(void* sim, int blk, int face);
int e4o_face_values(void* sim, int blk, int face);
int e4o_pack_face(void* sim, int blk, int face, double* out);
int e4o_unpack_face(void* sim, int blk, int face, const double* in);

/* This rank's min dt_allow / max CFL over its blocks (simcore.d:1362-1386);
 * dt_global set by the caller; one stage of the gas-dynamic increment (the
 * last stage ends the step). */
int e4o_dt_allow(void* sim, double dt_current, int check_cfl, double* dt_allow, double* cfl_max);
void e4o_set_dt_global(void* sim, double dt);
int e4o_stage(void* sim, int stage);

double e4o_time(void* sim);
double e4o_dt_global(void* sim);
int e4o_step_count(void* sim);
int e4o_last_bad_cells(void* sim);
const char* e4o_last_error(void* sim);

/* Install the thermally perfect mixture / mechanism (before adding blocks). */
int e4o_set_thermochem(void* sim, const e4o_thermochem* tc);

/* Thermally perfect gas state updates on one state (golden-vector tests):
 * mode 0: from (p, T) -> rho, u;  1: from (rho, u) -> p, T (T holds the
 * starting guess on entry);  2: from (rho, T) -> p, u.  a is the frozen
 * sound speed.  Returns 0 or a negative error. */
int e4o_tp_update(const e4o_thermochem* tc, int mode, const double* massf, double* rho,
                  double* p, double* T, double* u, double* a);

/* One chemistry update of one cell (constant rho, u): returns new mass
 * fractions, T, u, p and the suggested chemistry step in *dt_chem. */
int e4o_chem_cell(const e4o_thermochem* tc, double T_frozen, double dt, double rho,
                  double* T, double* u, double* p, double* massf, double* dt_chem);

/* Newton iterations of the whole-interval point-implicit step used by the
 * single-cell entry points above (default 12; a simulation uses its own
 * configuration's value). */
int e4o_set_chem_newton_iterations(int n);
/* Chemistry method of the single-cell entry points (chem_method above). */
int e4o_set_chem_method(int m);
/* One RKF step (chemistry_update.d:362-461, tolerance 1e-3) of the
 * mechanism's rate equations at temperature T from conc0 over h: concOut, the
 * suggested next step; returns 0 on a successful step, 1 on a failed one. */
int e4o_rkf_step(const e4o_thermochem* tc, double T, const double* conc0, double h,
                 double* concOut, double* h_suggest);

/* The chemistry update alone (ChemistryUpdate.opCall with the point-implicit
 * step) at constant rho and T: new mass fractions, no temperature update. */
int e4o_chem_update(const e4o_thermochem* tc, double dt, double rho, double T, double* massf,
                    double* dt_chem);

/* The reference's Newton-solver unit-test problems (which = 0 or 1). */
int e4o_newton_test(int which, double* root);

/* Production and loss rates (mol/m^3/s) of every species at temperature T and
 * concentrations c (mol/m^3). */
int e4o_rates(const e4o_thermochem* tc, double T, const double* c, double* q, double* L);

/* The host side of the reference's GPU chemistry (GPUChem, cuda_gpu_chem.d)
 * around its alpha-QSS kernel, for n cells in SoA arrays (species or reaction
 * outer): prepare gives the kernel's inputs, finish applies its outputs. */
int e4o_gpuchem_prepare(const e4o_thermochem* tc, int n, const double* rho, const double* T,
                        const double* massf, const double* dt_chem, double* conc, double* kf,
                        double* kb, double* h);
int e4o_gpuchem_finish(const e4o_thermochem* tc, int n, const double* conc, const double* h,
                       const double* rho, double* T, double* u, double* p, double* massf,
                       double* dt_chem);

/* Low-level pieces exposed for golden-vector tests. */
int e4o_ideal_gas_pT(double mol_mass, double gamma, double p, double T,
                     double* rho, double* u, double* a);

#ifdef __cplusplus
}
#endif
#endif
