// e4c_types.h -- plain structures shared by the host side of libe4cuda and
// its kernels.  No CUDA or torch types appear here, so the host translation
// units can include it with a plain C++ compiler.
#pragma once

#include <cstddef>
#include <cstdint>

namespace e4c {

// Ideal-gas constants (src/gas/ideal_gas.d:66-69).
struct GasConsts {
    double Rgas, gamma, Cv, Cvinv, Cp;
};

// Boundary order north, east, south, west, top, bottom (src/eilmer/fvcore.d).
enum Bnd { NORTH = 0, EAST = 1, SOUTH = 2, WEST = 3, TOP = 4, BOTTOM = 5 };

// Number of primitive fields kept per padded cell on the general path:
// rho, vel.x, vel.y, vel.z, p, T, u, a (then mass fractions).
enum PrimField { W_RHO = 0, W_VX, W_VY, W_VZ, W_P, W_T, W_U, W_A, W_NBASE };

// The partner of an exchange boundary on the general path (full-face copy,
// opposite faces, orientation 0): its padded primitive arrays and cell
// geometry; padded indices start at 2 in every active direction.
struct ExchangeSrc {
    const double* W;
    const double* cgeom;
    const int* S;
    size_t npad;
    int nidim, njdim;
    int imax, jmax, kmax;
    int pad_;
};

// Device view of one structured block on the general-geometry path.  All
// arrays use the reference's padded (i,j,k) index with two ghost layers,
// (k*njdim + j)*nidim + i (src/eilmer/sfluidblock.d:205).
struct BlockView {
    int dim;
    int ni, nj, nk;                 // interior cells
    int nidim, njdim, nkdim;        // padded extents
    int imin, imax, jmin, jmax, kmin, kmax;
    size_t npad;                    // nidim*njdim*nkdim
    int nsp;                        // species in the primitive state (1 for ideal gas)
    int nv;                         // conserved components (5 [+nsp])
    int bc[6];
    // primitive state, (W_NBASE + nsp) arrays of npad
    double* W;
    // conserved state at the start of the step, and dUdt of stage 1 (nv x npad)
    double* U0;
    double* dUdt0;
    // face fluxes per direction (nv x npad)
    double* Fi;
    double* Fj;
    double* Fk;
    // geometry: cells (vol, iLen, jLen, kLen) x npad; faces per direction
    // (n.xyz, t1.xyz, t2.xyz, area) x npad
    double* cgeom;
    double* fgi;
    double* fgj;
    double* fgk;
    // inflow FlowState (rho, vx, vy, vz, p, T, u, a, massf...)
    double inflow[8 + 8];
    int block_id;
    int axis_frames;                // every face frame is made of signed unit axes
    double* dt_chem;                // per-cell chemistry step suggestion (reacting blocks)
    ExchangeSrc ex[6];              // partners of exchange boundaries (bc == 3)
    int* S;                         // shock flag per padded cell (adaptive flux)
    // blocks with general face frames: velocity (x, y, z) of each interior
    // cell after the in-place round trips of its i faces, then of its i and j
    // faces (6 x npad; null for blocks whose frames are signed unit axes)
    double* Vrt;
};

// Device-resident simulation state (one per library context).
struct SimDev {
    double dt_global;
    double time;
    double max_time;                // the loop stops once time >= max_time
    int step;
    int status;                     // first error code seen, 0 if none
    int status_step;                // step at which it was seen
    int bad_cells;                  // invalid cells counted in the last stage
    int finished;                   // set when time >= max_time
    int pad_;
    unsigned int item_next[2];      // work-item counters of the fused stages 1 and 2
    unsigned int pad2_[2];
};

// Per-block descriptor of the fused uniform path (device array, one entry per
// fused block).  Geometry constants are those every cell and face of the
// block shares; arrays are SoA over interior cells, i fastest.
struct FusedDesc {
    int ni, nj, nk;
    int tiles_i, tiles_j, kchunks;
    long long item0;            // first work item of this block
    int bc[6];
    int* use_a0;                // -> 1 while the uploaded sound speed is still in use
    void* WA;                   // primitive state rho, vx, vy, vz, u (5 x ncell), R-typed
    void* WB;                   // second buffer: stage 1 writes it, stage 2 reads it
    const double* A0;           // uploaded sound speed (ncell)
    double* U0;                 // conserved state (5 x ncell)
    double* dUdt0;              // stage-1 derivative (5 x ncell)
    unsigned long long* acc;    // dt accumulators of this block (3)
    double vol;
    double len[3];
    double area[3];
    double fn[3][3], ft1[3][3], ft2[3][3];
    double inflow[6];           // rho, vx, vy, vz, u, a
    int ex[6];                  // descriptor index of the partner of an exchange boundary
};

// Molar masses of the five species, for the chemistry seed's guesses.
struct SeedMolar {
    double M[5];
};

}  // namespace e4c
