/*
 * e4_oracle_internal.h -- data structures of the CPU FP64 oracle.
 * TEST INFRASTRUCTURE ONLY (see e4_oracle.cpp).
 *
 * The structures mirror the reference's object model: a structured block is
 * a padded (i,j,k) array of cells with two ghost layers, and three padded
 * face arrays (src/eilmer/sfluidblock.d:94-126, 205-262, 420-436).
 */
#ifndef E4_ORACLE_INTERNAL_H
#define E4_ORACLE_INTERNAL_H

#include <string>
#include <vector>

#include "e4_oracle.h"

enum {
    E4O_ERR_ARG = -1,
    E4O_ERR_BAD_MASS = -2,
    E4O_ERR_THERMO = -3,
    E4O_ERR_BAD_CELLS = -4,
    E4O_ERR_CHEM = -5,
};

namespace e4o {

constexpr double R_universal = 8.31451;  // src/gas/physical_constants.d:13
constexpr int NSPMAX = 8;

struct Vec3 {
    double x = 0.0, y = 0.0, z = 0.0;
};

struct GasState {  // src/gas/gas_state.d:18 (single temperature)
    double rho = 0.0, p = 0.0, T = 0.0, u = 0.0, a = 0.0;
    double massf[NSPMAX] = {1.0};
};

struct FlowState {  // src/eilmer/flowstate.d:30
    GasState gas;
    Vec3 vel;
    int S = 0;         // shock flag (copied with the state, flowstate.d:177-193)
};

struct Cell {  // the parts of src/eilmer/fvcell.d used on the hot path
    FlowState fs;
    double U[3][5 + NSPMAX] = {};
    double dUdt[2][5 + NSPMAX] = {};
    double vol = 0.0, iLen = 0.0, jLen = 0.0, kLen = 0.0;
    double dt_chem = -1.0;
    bool data_is_bad = false;
};

struct Face {  // src/eilmer/fvinterface.d
    Vec3 n, t1, t2;
    double area = 0.0;
    double F[5 + NSPMAX] = {};
};

struct Block {
    int dim = 2, ni = 0, nj = 0, nk = 1;
    int nidim = 0, njdim = 0, nkdim = 0;
    int imin = 0, imax = 0, jmin = 0, jmax = 0, kmin = 0, kmax = 0;
    std::vector<Cell> cells;
    std::vector<Face> ifi, ifj, ifk;
    std::vector<Vec3> vtx;
    int bc[6] = {0, 0, 0, 0, 0, 0};
    int ex_block[6] = {-1, -1, -1, -1, -1, -1};   // partner block of an exchange boundary
    int ex_face[6] = {-1, -1, -1, -1, -1, -1};    // the partner's joined face
    int ex_orient[6] = {0, 0, 0, 0, 0, 0};         // orientation of the joint
    FlowState inflow;
    bool axis_frames = true;

    void init(int dim_, int ni_, int nj_, int nk_) {
        dim = dim_; ni = ni_; nj = nj_; nk = (dim == 3) ? nk_ : 1;
        nidim = ni + 4; njdim = nj + 4; nkdim = (dim == 3) ? nk + 4 : 1;
        imin = 2; imax = imin + ni - 1;
        jmin = 2; jmax = jmin + nj - 1;
        if (dim == 3) { kmin = 2; kmax = kmin + nk - 1; }
        else { kmin = 0; kmax = 0; }
        size_t n = size_t(nidim) * njdim * nkdim;
        cells.assign(n, Cell());
        ifi.assign(n, Face()); ifj.assign(n, Face()); ifk.assign(n, Face());
        // Vertices need one more layer in each active direction.
        vtx.assign(size_t(nidim + 1) * (njdim + 1) * (nkdim + 1), Vec3());
    }
    // to_single_index, sfluidblock.d:205
    size_t idx(int i, int j, int k) const { return (size_t(k) * njdim + j) * nidim + i; }
    Cell& cell(int i, int j, int k) { return cells[idx(i, j, k)]; }
    size_t ncell() const { return size_t(ni) * nj * nk; }
    void compute_geometry();
};

struct GasModel {
    int kind = E4O_GAS_IDEAL;
    int nsp = 1;
    // ideal gas
    double Rgas = 0.0, gamma = 1.4, Cv = 0.0, Cvinv = 0.0, Cp = 0.0;
    // thermally perfect mixture and mechanism (installed by e4o_set_thermochem)
    e4o_thermochem tc{};
    void init_ideal(double mol_mass, double gamma);
    void init_therm_perf_air5();
    bool update_thermo_from_pT(GasState& Q) const;
    bool update_thermo_from_rhou(GasState& Q) const;
    bool update_thermo_from_rhoT(GasState& Q) const;
    bool update_sound_speed(GasState& Q) const;
    bool tp_update_thermo_from_pT(GasState& Q) const;
    bool tp_update_thermo_from_rhou(GasState& Q) const;
    bool tp_update_thermo_from_rhoT(GasState& Q) const;
    bool tp_update_sound_speed(GasState& Q) const;
};

struct Sim {
    e4o_config cfg{};
    GasModel gm;
    int nsp_cons = 0;
    std::vector<Block*> blocks;
    double time = 0.0;
    double dt_global = 0.0;
    int step = 0;
    bool dt_initialised = false;
    bool mutate_in_place = false;
    int last_bad_cells = 0;
    double last_cfl_max = 0.0;
    std::string error;

    ~Sim() { for (Block* b : blocks) delete b; }

    void unpack_prim(const double* prim, size_t n, size_t q, FlowState& fs) const {
        fs.gas.rho = prim[0 * n + q];
        fs.vel.x = prim[1 * n + q]; fs.vel.y = prim[2 * n + q]; fs.vel.z = prim[3 * n + q];
        fs.gas.p = prim[4 * n + q]; fs.gas.T = prim[5 * n + q];
        fs.gas.u = prim[6 * n + q]; fs.gas.a = prim[7 * n + q];
        for (int s = 0; s < gm.nsp; ++s) fs.gas.massf[s] = (gm.nsp > 1) ? prim[(8 + s) * n + q] : 1.0;
    }
    void pack_prim(const FlowState& fs, double* prim, size_t n, size_t q) const {
        prim[0 * n + q] = fs.gas.rho;
        prim[1 * n + q] = fs.vel.x; prim[2 * n + q] = fs.vel.y; prim[3 * n + q] = fs.vel.z;
        prim[4 * n + q] = fs.gas.p; prim[5 * n + q] = fs.gas.T;
        prim[6 * n + q] = fs.gas.u; prim[7 * n + q] = fs.gas.a;
        if (gm.nsp > 1)
            for (int s = 0; s < gm.nsp; ++s) prim[(8 + s) * n + q] = fs.gas.massf[s];
    }

    // gas dynamics
    void ausmdv(const FlowState& L, const FlowState& R, double* F) const;
    void hllc(const FlowState& L, const FlowState& R, double* F) const;
    void hanel(const FlowState& L, const FlowState& R, double* F) const;
    void detect_shock_points(Block& b);
    void interface_flux(FlowState& L, FlowState& R, Face& f) const;
    bool scale_mass_fractions(double* massf) const;
    void interp_l2r2(Face& f, Cell& cL1, Cell& cL0, Cell& cR0, Cell& cR1, double lenL1,
                     double lenL0, double lenR0, double lenR1, FlowState& Lft,
                     FlowState& Rght) const;
    void face_flux(Block& b, Face& f, Cell& cL1, Cell& cL0, Cell& cR0, Cell& cR1, int dir) const;
    void convective_flux(Block& b);
    void simple_outflow_flux(Block& b);
    int apply_bcs(Block& b);
    void reset_linear_ghosts(Block& b);
    void encode_conserved(Cell& c, int ftl) const;
    int decode_conserved(Cell& c, int ftl) const;
    void time_derivatives(Block& b, Cell& c, int i, int j, int k, int ftl) const;
    void stage_update(Cell& c, int stage, double dt) const;
    int stage_cells(Block& b, int stage, double dt);
    double signal_frequency(Block& b, Cell& c, int i, int j, int k) const;
    void block_dt(Block& b, double dt_current, bool check_cfl, double& dt_allow, double& cfl_max);
    void determine_time_step_size();
    int gasdynamic_stage(int stage);
    void finish_gasdynamic_step();
    int gasdynamic_increment();
    int end_step();
    int chemistry_step(double dt);
    int run(int nsteps, double max_time);
};

}  // namespace e4o

#endif
