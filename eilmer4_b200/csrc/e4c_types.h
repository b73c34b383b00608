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

// The partner of an exchange boundary on the general path (full-face copy):
// its padded primitive arrays and cell geometry, its joined face and the
// joint's orientation, its active extents and the padded index of its first
// active cell along k (2 in 3-D, 0 in 2-D; 2 along i and j).
struct ExchangeSrc {
    const double* W;
    const double* cgeom;
    const int* S;
    size_t npad;
    int nidim, njdim;
    int ni, nj, nk;
    int face, orient, kmin;
};

#ifdef __CUDACC__
#define E4C_HD __host__ __device__
#else
#define E4C_HD
#endif

// The cell of the partner block that sits `depth` layers behind the joint
// (0: the layer next to it) across from cell (p, q) of face fa, for a joint
// of face fa with the partner's face fb at orientation r: the mapping of
// GhostCellFullFaceCopy.set_up_cell_mapping (src/eilmer/bc/ghost_cell_effect/
// full_face_copy.d:142-1083), written as one rule instead of its 144 cases.
// A face's cells are indexed (p, q): north and south faces (i, k), east and
// west (j, k), top and bottom (i, j); 2-D blocks have q = 0 and orientation 0.
// Faces fall into two classes, {north, west, bottom} and {east, south, top};
// from a face of the second class the orientation counts the other way
// round (r -> 4 - r); then joints within one class and joints across the
// classes each follow four orientation cases.  Both blocks of a joint carry
// the same orientation (connectBlocks, src/eilmer/prep.lua), and the rule
// maps back with it.  Returns the partner's active indices (from 0).
E4C_HD inline void ffc_partner(int fa, int fb, int r, int p, int q, int depth, int ni, int nj,
                               int nk, int& si, int& sj, int& sk) {
    const bool xa = fa == NORTH || fa == WEST || fa == BOTTOM;
    const bool xb = fb == NORTH || fb == WEST || fb == BOTTOM;
    const int P = (fb == EAST || fb == WEST) ? nj : ni;   // extents of fb's (p, q)
    const int Q = (fb == TOP || fb == BOTTOM) ? nj : nk;
    if (!xa) r = (4 - r) & 3;
    int pb, qb;
    if (xa == xb) {
        switch (r) {
            case 0: pb = P - 1 - p; qb = q; break;
            case 1: pb = q; qb = p; break;
            case 2: pb = p; qb = Q - 1 - q; break;
            default: pb = P - 1 - q; qb = Q - 1 - p; break;
        }
    } else {
        switch (r) {
            case 0: pb = p; qb = q; break;
            case 1: pb = P - 1 - q; qb = p; break;
            case 2: pb = P - 1 - p; qb = Q - 1 - q; break;
            default: pb = q; qb = Q - 1 - p; break;
        }
    }
    switch (fb) {
        case NORTH: si = pb; sk = qb; sj = nj - 1 - depth; break;
        case SOUTH: si = pb; sk = qb; sj = depth; break;
        case EAST: sj = pb; sk = qb; si = ni - 1 - depth; break;
        case WEST: sj = pb; sk = qb; si = depth; break;
        case TOP: si = pb; sj = qb; sk = nk - 1 - depth; break;
        default: si = pb; sj = qb; sk = depth; break;
    }
}

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
    // shock flags of the adaptive flux (ncell each): stage 1 writes S[0] and
    // takes the ghost cells' flags from S[1] (the previous stage's), stage 2
    // the other way round
    unsigned char* S[2];
};

// Molar masses of the five species, for the chemistry seed's guesses.
struct SeedMolar {
    double M[5];
};

}  // namespace e4c
