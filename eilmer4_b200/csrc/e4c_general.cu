// e4c_general.cu -- FP64 kernels of the general-geometry path.
//
// Compiled with -fmad=false: every multiply and add is rounded on its own,
// as in the reference's D code, so the results match the reference algorithm
// bit for bit (tests compare against the FP64 CPU oracle with ==).
//
// One face flux per thread (per direction), one cell update per thread.
// Works for any structured grid, including curvilinear 2-D grids; the uniform
// Cartesian 3-D case has its own fused kernel in e4c_fused.cu.
#include <cfloat>

#include "e4c_cells.cuh"

namespace e4c {

// ---------------------------------------------------------------------------
// Geometry (src/geom/elements/properties.d, src/eilmer/fvinterface.d:265-317)
// ---------------------------------------------------------------------------
struct Vd {
    double x, y, z;
};
__device__ __forceinline__ Vd vload(const double* v, const BlockView& b, int i, int j, int k) {
    // vertex of padded indices (i,j,k); the array is unpadded, i fastest
    const int nvi = b.ni + 1, nvj = b.nj + 1;
    size_t q = 3 * ((size_t(k - b.kmin) * nvj + (j - b.jmin)) * nvi + (i - b.imin));
    return {v[q], v[q + 1], v[q + 2]};
}
__device__ __forceinline__ void vcross(Vd& v3, const Vd& v1, const Vd& v2) {
    v3.x = v1.y * v2.z - v2.y * v1.z;  // vector3.d:604-609
    v3.y = v2.x * v1.z - v1.x * v2.z;
    v3.z = v1.x * v2.y - v2.x * v1.y;
}
__device__ __forceinline__ void vnormalize(Vd& v) {
    double mag = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);  // vector3.d:386-404
    if (mag > 0.0) { v.x /= mag; v.y /= mag; v.z /= mag; }
    else { v.x = v.y = v.z = 0.0; }
    if (fabs(v.x) < 1.0e-30) v.x = 0.0;
    if (fabs(v.y) < 1.0e-30) v.y = 0.0;
    if (fabs(v.z) < 1.0e-30) v.z = 0.0;
}
__device__ void quad_props(const Vd& p0, const Vd& p1, const Vd& p2, const Vd& p3, double* out) {
    // quad_properties, properties.d:97-141
    double p01x = p1.x - p0.x + p2.x - p3.x;
    double p01y = p1.y - p0.y + p2.y - p3.y;
    double p01z = p1.z - p0.z + p2.z - p3.z;
    double p03x = p3.x - p0.x + p2.x - p1.x;
    double p03y = p3.y - p0.y + p2.y - p1.y;
    double p03z = p3.z - p0.z + p2.z - p1.z;
    double vax = p01y * p03z - p01z * p03y;
    double vay = p01z * p03x - p01x * p03z;
    double vaz = p01x * p03y - p01y * p03x;
    vax *= 0.25; vay *= 0.25; vaz *= 0.25;
    double area = sqrt(vax * vax + vay * vay + vaz * vaz);
    Vd n, t1, t2;
    if (area > 1.0e-20) {
        n = {vax / area, vay / area, vaz / area};
        t1 = {p01x, p01y, p01z};
        vnormalize(t1);
        vcross(t2, n, t1);
        vnormalize(t2);
    } else {
        n = {1.0, 0.0, 0.0}; t1 = {0.0, 1.0, 0.0}; t2 = {0.0, 0.0, 1.0};
    }
    out[0] = n.x; out[1] = n.y; out[2] = n.z;
    out[3] = t1.x; out[4] = t1.y; out[5] = t1.z;
    out[6] = t2.x; out[7] = t2.y; out[8] = t2.z;
    out[9] = area;
}
__device__ void face2d_props(const Vd& A, const Vd& B, double* out) {
    // FVInterface.update_2D_geometric_data, fvinterface.d:265-297 (planar)
    double LAB = sqrt((B.x - A.x) * (B.x - A.x) + (B.y - A.y) * (B.y - A.y));
    Vd n, t1, t2;
    double area;
    if (LAB > 1.0e-12) {
        n = {(B.y - A.y) / LAB, -(B.x - A.x) / LAB, 0.0};
        t2 = {0.0, 0.0, 1.0};
        vcross(t1, n, t2);
        area = LAB;
    } else {
        n = {1.0, 0.0, 0.0}; t2 = {0.0, 0.0, 1.0}; t1 = {0.0, 1.0, 0.0};
        area = 0.0;
    }
    out[0] = n.x; out[1] = n.y; out[2] = n.z;
    out[3] = t1.x; out[4] = t1.y; out[5] = t1.z;
    out[6] = t2.x; out[7] = t2.y; out[8] = t2.z;
    out[9] = area;
}
__device__ double tet_volume(const Vd& p0, const Vd& p1, const Vd& p2, const Vd& p3) {
    // tetrahedron_volume, properties.d:293-304
    double dx01 = p1.x - p0.x, dy01 = p1.y - p0.y, dz01 = p1.z - p0.z;
    double dx02 = p2.x - p0.x, dy02 = p2.y - p0.y, dz02 = p2.z - p0.z;
    double cx = dy01 * dz02 - dz01 * dy02;
    double cy = dz01 * dx02 - dx01 * dz02;
    double cz = dx01 * dy02 - dy01 * dx02;
    double dx03 = p3.x - p0.x, dy03 = p3.y - p0.y, dz03 = p3.z - p0.z;
    return (dx03 * cx + dy03 * cy + dz03 * cz) / 6.0;
}
__device__ double pyr_volume(const Vd& p0, const Vd& p1, const Vd& p2, const Vd& p3, const Vd& p4) {
    // pyramid_properties, properties.d:390-419 (volume only)
    Vd pmB{0.25 * (p0.x + p1.x + p2.x + p3.x), 0.25 * (p0.y + p1.y + p2.y + p3.y),
           0.25 * (p0.z + p1.z + p2.z + p3.z)};
    double volume = 0.0;
    volume += tet_volume(p0, p1, pmB, p4);
    volume += tet_volume(p1, p2, pmB, p4);
    volume += tet_volume(p2, p3, pmB, p4);
    volume += tet_volume(p3, p0, pmB, p4);
    return volume;
}
__device__ Vd mid4(const Vd& a, const Vd& b, const Vd& c, const Vd& d) {
    return {0.25 * (a.x + b.x + c.x + d.x), 0.25 * (a.y + b.y + c.y + d.y),
            0.25 * (a.z + b.z + c.z + d.z)};
}

__global__ void k_geom_cells(BlockView b, const double* vtx) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        size_t c = pidx(b, i, j, k);
        double vol, iL, jL, kL;
        if (b.dim == 2) {
            // xyplane_quad_cell_properties, properties.d:177-236
            Vd p0 = vload(vtx, b, i, j, 0), p1 = vload(vtx, b, i + 1, j, 0);
            Vd p2 = vload(vtx, b, i + 1, j + 1, 0), p3 = vload(vtx, b, i, j + 1, 0);
            double xA = p1.x, yA = p1.y, xB = p2.x, yB = p2.y;
            double xC = p3.x, yC = p3.y, xD = p0.x, yD = p0.y;
            vol = 0.5 * ((xB + xA) * (yB - yA) + (xC + xB) * (yC - yB) + (xD + xC) * (yD - yC) +
                         (xA + xD) * (yA - yD));
            double xN = 0.5 * (xC + xB), yN = 0.5 * (yC + yB);
            double xS = 0.5 * (xD + xA), yS = 0.5 * (yD + yA);
            double xE = 0.5 * (xA + xB), yE = 0.5 * (yA + yB);
            double xW = 0.5 * (xD + xC), yW = 0.5 * (yD + yC);
            double dx = xN - xS, dy = yN - yS;
            jL = sqrt(dx * dx + dy * dy);
            dx = xE - xW; dy = yE - yW;
            iL = sqrt(dx * dx + dy * dy);
            kL = 0.0;
        } else {
            // hex_cell_properties, properties.d:568-648
            Vd p[8] = {vload(vtx, b, i, j, k),         vload(vtx, b, i + 1, j, k),
                       vload(vtx, b, i + 1, j + 1, k), vload(vtx, b, i, j + 1, k),
                       vload(vtx, b, i, j, k + 1),     vload(vtx, b, i + 1, j, k + 1),
                       vload(vtx, b, i + 1, j + 1, k + 1), vload(vtx, b, i, j + 1, k + 1)};
            Vd cc{0.125 * (p[0].x + p[1].x + p[2].x + p[3].x + p[4].x + p[5].x + p[6].x + p[7].x),
                  0.125 * (p[0].y + p[1].y + p[2].y + p[3].y + p[4].y + p[5].y + p[6].y + p[7].y),
                  0.125 * (p[0].z + p[1].z + p[2].z + p[3].z + p[4].z + p[5].z + p[6].z + p[7].z)};
            Vd pmN = mid4(p[3], p[2], p[6], p[7]), pmE = mid4(p[1], p[2], p[6], p[5]);
            Vd pmS = mid4(p[0], p[1], p[5], p[4]), pmW = mid4(p[0], p[3], p[7], p[4]);
            Vd pmT = mid4(p[4], p[5], p[6], p[7]), pmB = mid4(p[0], p[1], p[2], p[3]);
            double dx, dy, dz;
            dx = pmE.x - pmW.x; dy = pmE.y - pmW.y; dz = pmE.z - pmW.z;
            iL = sqrt(dx * dx + dy * dy + dz * dz);
            dx = pmN.x - pmS.x; dy = pmN.y - pmS.y; dz = pmN.z - pmS.z;
            jL = sqrt(dx * dx + dy * dy + dz * dz);
            dx = pmT.x - pmB.x; dy = pmT.y - pmB.y; dz = pmT.z - pmB.z;
            kL = sqrt(dx * dx + dy * dy + dz * dz);
            vol = 0.0;
            vol += pyr_volume(p[6], p[7], p[3], p[2], cc);
            vol += pyr_volume(p[5], p[6], p[2], p[1], cc);
            vol += pyr_volume(p[4], p[5], p[1], p[0], cc);
            vol += pyr_volume(p[7], p[4], p[0], p[3], cc);
            vol += pyr_volume(p[7], p[6], p[5], p[4], cc);
            vol += pyr_volume(p[0], p[1], p[2], p[3], cc);
            if ((vol < 0.0 && fabs(vol) < 1.0e-12) || (vol >= 0.0 && vol < 1.0e-20)) vol = 0.0;
        }
        b.cgeom[0 * b.npad + c] = vol;
        b.cgeom[1 * b.npad + c] = iL;
        b.cgeom[2 * b.npad + c] = jL;
        b.cgeom[3 * b.npad + c] = kL;
    }
}

__global__ void k_geom_faces(BlockView b, const double* vtx, int dir) {
    const int ni = b.ni + (dir == 0), nj = b.nj + (dir == 1), nk = b.nk + (dir == 2 && b.dim == 3);
    const long long n = (long long)ni * nj * nk;
    double* fg = dir == 0 ? b.fgi : (dir == 1 ? b.fgj : b.fgk);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % ni);
        int j = b.jmin + int((t / ni) % nj);
        int k = b.kmin + int(t / ((long long)ni * nj));
        double out[10];
        if (b.dim == 2) {
            if (dir == 0) face2d_props(vload(vtx, b, i, j, 0), vload(vtx, b, i, j + 1, 0), out);
            else face2d_props(vload(vtx, b, i + 1, j, 0), vload(vtx, b, i, j, 0), out);
        } else if (dir == 0) {
            quad_props(vload(vtx, b, i, j, k), vload(vtx, b, i, j + 1, k),
                       vload(vtx, b, i, j + 1, k + 1), vload(vtx, b, i, j, k + 1), out);
        } else if (dir == 1) {
            quad_props(vload(vtx, b, i, j, k), vload(vtx, b, i, j, k + 1),
                       vload(vtx, b, i + 1, j, k + 1), vload(vtx, b, i + 1, j, k), out);
        } else {
            quad_props(vload(vtx, b, i, j, k), vload(vtx, b, i + 1, j, k),
                       vload(vtx, b, i + 1, j + 1, k), vload(vtx, b, i, j + 1, k), out);
        }
        size_t f = pidx(b, i, j, k);
#pragma unroll
        for (int q = 0; q < 10; ++q) fg[q * b.npad + f] = out[q];
    }
}

// Ghost-cell lengths copied from the mirror interior cells (sfluidblock.d:675-712).
__global__ void k_geom_ghost_lengths(BlockView b) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    auto copy = [&](size_t dst, size_t src) {
        for (int q = 1; q < 4; ++q) b.cgeom[q * b.npad + dst] = b.cgeom[q * b.npad + src];
    };
    // i boundaries: over (j,k)
    if (t < b.nj * b.nk) {
        int j = b.jmin + t % b.nj, k = b.kmin + t / b.nj;
        copy(pidx(b, b.imin - 1, j, k), pidx(b, b.imin, j, k));
        copy(pidx(b, b.imin - 2, j, k), pidx(b, b.imin + 1, j, k));
        copy(pidx(b, b.imax + 1, j, k), pidx(b, b.imax, j, k));
        copy(pidx(b, b.imax + 2, j, k), pidx(b, b.imax - 1, j, k));
    }
    if (t < b.ni * b.nk) {
        int i = b.imin + t % b.ni, k = b.kmin + t / b.ni;
        copy(pidx(b, i, b.jmin - 1, k), pidx(b, i, b.jmin, k));
        copy(pidx(b, i, b.jmin - 2, k), pidx(b, i, b.jmin + 1, k));
        copy(pidx(b, i, b.jmax + 1, k), pidx(b, i, b.jmax, k));
        copy(pidx(b, i, b.jmax + 2, k), pidx(b, i, b.jmax - 1, k));
    }
    if (b.dim == 3 && t < b.ni * b.nj) {
        int i = b.imin + t % b.ni, j = b.jmin + t / b.ni;
        copy(pidx(b, i, j, b.kmin - 1), pidx(b, i, j, b.kmin));
        copy(pidx(b, i, j, b.kmin - 2), pidx(b, i, j, b.kmin + 1));
        copy(pidx(b, i, j, b.kmax + 1), pidx(b, i, j, b.kmax));
        copy(pidx(b, i, j, b.kmax + 2), pidx(b, i, j, b.kmax - 1));
    }
}

// ---------------------------------------------------------------------------
// Upload: primitive SoA over interior cells -> padded W and encoded U0
// (encode_conserved, src/eilmer/fvcell.d:494-560)
// ---------------------------------------------------------------------------
__global__ void k_upload(BlockView b, const double* prim) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    const int nw = W_NBASE + (b.nsp > 1 ? b.nsp : 0);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        size_t c = pidx(b, i, j, k);
        for (int q = 0; q < nw; ++q) b.W[q * b.npad + c] = prim[q * n + t];
        double rho = prim[W_RHO * n + t];
        double vx = prim[W_VX * n + t], vy = prim[W_VY * n + t], vz = prim[W_VZ * n + t];
        double u = prim[W_U * n + t];
        b.U0[0 * b.npad + c] = rho;
        b.U0[1 * b.npad + c] = rho * vx;
        b.U0[2 * b.npad + c] = rho * vy;
        b.U0[3 * b.npad + c] = rho * vz;
        double ke = 0.5 * (vx * vx + vy * vy + vz * vz);
        b.U0[4 * b.npad + c] = rho * (u + ke);
        for (int s = 0; s < b.nv - 5; ++s) b.U0[(5 + s) * b.npad + c] = rho * prim[(W_NBASE + s) * n + t];
    }
}

// Conserved state (dense, v * n + t) -> U0 and the decoded primitive state of
// the interior cells, ideal gas (decode_ideal).
__global__ void k_upload_cons(BlockView b, const double* cons, SimDev* sim, GasConsts gas) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        size_t c = pidx(b, i, j, k);
        double Un[5];
        for (int v = 0; v < 5; ++v) Un[v] = cons[v * n + t];
        double rho, vx, vy, vz, u, p, T, a;
        if (!decode_ideal(gas, Un, rho, vx, vy, vz, u, p, T, a)) set_status(sim, -5);
        double* W = b.W;
        W[W_RHO * b.npad + c] = rho;
        W[W_VX * b.npad + c] = vx; W[W_VY * b.npad + c] = vy; W[W_VZ * b.npad + c] = vz;
        W[W_P * b.npad + c] = p; W[W_T * b.npad + c] = T;
        W[W_U * b.npad + c] = u; W[W_A * b.npad + c] = a;
        for (int v = 0; v < 5; ++v) b.U0[v * b.npad + c] = Un[v];
    }
}

__global__ void k_download(BlockView b, double* prim, double* cons) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    const int nw = W_NBASE + (b.nsp > 1 ? b.nsp : 0);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        size_t c = pidx(b, i, j, k);
        if (prim)
            for (int q = 0; q < nw; ++q) prim[q * n + t] = b.W[q * b.npad + c];
        if (cons)
            for (int q = 0; q < b.nv; ++q) cons[q * n + t] = b.U0[q * b.npad + c];
    }
}

// ---------------------------------------------------------------------------
// Ghost cells: slip wall, supersonic inflow, zero-order extrapolate outflow
// (src/eilmer/bc/ghost_cell_effect/internal_copy_then_reflect.d:94+,
//  flow_state_copy.d:66+, extrapolate_copy.d:82+, ghost_cell.d:34-44)
// ---------------------------------------------------------------------------
template <int NSP>
__global__ void k_bc(BlockView b, const SimDev* sim) {
    if (sim->status != 0 || sim->finished) return;
    const int which = blockIdx.y;
    if (b.dim == 2 && which >= 4) return;
    int n1, n2;  // extent of the boundary layer of cells
    if (which == NORTH || which == SOUTH) { n1 = b.ni; n2 = b.nk; }
    else if (which == EAST || which == WEST) { n1 = b.nj; n2 = b.nk; }
    else { n1 = b.ni; n2 = b.nj; }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n1 * n2) return;
    const int a1 = t % n1, a2 = t / n1;
    int i, j, k, di = 0, dj = 0, dk = 0;
    switch (which) {
        case NORTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmax; dj = 1; break;
        case SOUTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmin; dj = -1; break;
        case EAST: j = b.jmin + a1; k = b.kmin + a2; i = b.imax; di = 1; break;
        case WEST: j = b.jmin + a1; k = b.kmin + a2; i = b.imin; di = -1; break;
        case TOP: i = b.imin + a1; j = b.jmin + a2; k = b.kmax; dk = 1; break;
        default: i = b.imin + a1; j = b.jmin + a2; k = b.kmin; dk = -1; break;
    }
    const size_t c0 = pidx(b, i, j, k);
    const size_t c1 = pidx(b, i - di, j - dj, k - dk);
    const size_t g1 = pidx(b, i + di, j + dj, k + dk);
    const size_t g2 = pidx(b, i + 2 * di, j + 2 * dj, k + 2 * dk);
    const int nw = W_NBASE + (NSP > 1 ? NSP : 0);
    const int type = b.bc[which];
    if (type == E4C_BC_OUTFLOW_EXTRAPOLATE_LINEAR) return;   // k_bc_linear
    if (type == 3) {  // full-face copy: the partner's first two cells
        const ExchangeSrc& o = b.ex[which];
        const size_t dst[2] = {g1, g2};
        for (int g = 0; g < 2; ++g) {
            int si, sj, sk;
            ffc_partner(which, o.face, o.orient, a1, a2, g, o.ni, o.nj, o.nk, si, sj, sk);
            const size_t sc = (size_t(sk + o.kmin) * o.njdim + sj + 2) * o.nidim + si + 2;
            for (int q = 0; q < nw; ++q) b.W[q * b.npad + dst[g]] = o.W[q * o.npad + sc];
            b.S[dst[g]] = o.S[sc];
        }
    } else if (type == 1) {  // InFlowBC_Supersonic: both ghosts <- inflow FlowState
        for (int q = 0; q < nw; ++q) {
            b.W[q * b.npad + g1] = b.inflow[q];
            b.W[q * b.npad + g2] = b.inflow[q];
        }
        b.S[g1] = 0;
        b.S[g2] = 0;
    } else if (type == 2 || type == 4) {
        // OutFlowBC_SimpleExtrapolate, x_order 0; also the ghost cells of
        // OutFlowBC_SimpleFlux (bc.lua:1124-1146)
        for (int q = 0; q < nw; ++q) {
            double v = b.W[q * b.npad + c0];
            b.W[q * b.npad + g1] = v;
            b.W[q * b.npad + g2] = v;
        }
        b.S[g1] = b.S[c0];
        b.S[g2] = b.S[c0];
    } else {  // WallBC_WithSlip: copy then reflect the normal velocity
        b.S[g1] = b.S[c0];
        b.S[g2] = b.S[c1];
        size_t f;
        const double* fg;
        switch (which) {
            case NORTH: f = pidx(b, i, j + 1, k); fg = b.fgj; break;
            case EAST: f = pidx(b, i + 1, j, k); fg = b.fgi; break;
            case SOUTH: f = pidx(b, i, j, k); fg = b.fgj; break;
            case WEST: f = pidx(b, i, j, k); fg = b.fgi; break;
            case TOP: f = pidx(b, i, j, k + 1); fg = b.fgk; break;
            default: f = pidx(b, i, j, k); fg = b.fgk; break;
        }
        Frame<double> fr;
        fr.n = {fg[0 * b.npad + f], fg[1 * b.npad + f], fg[2 * b.npad + f]};
        fr.t1 = {fg[3 * b.npad + f], fg[4 * b.npad + f], fg[5 * b.npad + f]};
        fr.t2 = {fg[6 * b.npad + f], fg[7 * b.npad + f], fg[8 * b.npad + f]};
        const size_t src[2] = {c0, c1}, dst[2] = {g1, g2};
        for (int g = 0; g < 2; ++g) {
            for (int q = 0; q < nw; ++q) b.W[q * b.npad + dst[g]] = b.W[q * b.npad + src[g]];
            V3<double> v{b.W[W_VX * b.npad + src[g]], b.W[W_VY * b.npad + src[g]],
                         b.W[W_VZ * b.npad + src[g]]};
            to_local(v, fr.n, fr.t1, fr.t2);
            v.x = -(v.x);
            to_global(v, fr.n, fr.t1, fr.t2);
            b.W[W_VX * b.npad + dst[g]] = v.x;
            b.W[W_VY * b.npad + dst[g]] = v.y;
            b.W[W_VZ * b.npad + dst[g]] = v.z;
        }
    }
}

// BFE_SimpleOutflowFlux (bc/boundary_flux_effect.d:367-546), the flux action
// of OutFlowBC_SimpleFlux, after the convective fluxes of every block
// (simcore.d:2373-2377): each face of the boundary takes the flux of its
// interior cell's flow state (fixed grid), or that of a closed face if the
// state would flow in.  The face fluxes the flux kernels computed there are
// overwritten, as the reference's flux loops skip those faces (sfluidblock.d:
// 2227-2228 and alike) after reconstructing them.
template <int NSP>
__global__ void k_bc_flux(BlockView b, const SimDev* sim, FluxOpts o) {
    if (sim->status != 0 || sim->finished) return;
    const int which = blockIdx.y;
    if (b.dim == 2 && which >= 4) return;
    if (b.bc[which] != E4C_BC_OUTFLOW_SIMPLE_FLUX) return;
    int n1, n2;
    if (which == NORTH || which == SOUTH) { n1 = b.ni; n2 = b.nk; }
    else if (which == EAST || which == WEST) { n1 = b.nj; n2 = b.nk; }
    else { n1 = b.ni; n2 = b.nj; }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n1 * n2) return;
    const int a1 = t % n1, a2 = t / n1;
    int i, j, k, fi, fj, fk, outsign;
    const double* fg;
    double* Fo;
    switch (which) {
        case NORTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmax; fi = i; fj = j + 1; fk = k;
                    fg = b.fgj; Fo = b.Fj; outsign = 1; break;
        case SOUTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmin; fi = i; fj = j; fk = k;
                    fg = b.fgj; Fo = b.Fj; outsign = -1; break;
        case EAST: j = b.jmin + a1; k = b.kmin + a2; i = b.imax; fi = i + 1; fj = j; fk = k;
                   fg = b.fgi; Fo = b.Fi; outsign = 1; break;
        case WEST: j = b.jmin + a1; k = b.kmin + a2; i = b.imin; fi = i; fj = j; fk = k;
                   fg = b.fgi; Fo = b.Fi; outsign = -1; break;
        case TOP: i = b.imin + a1; j = b.jmin + a2; k = b.kmax; fi = i; fj = j; fk = k + 1;
                  fg = b.fgk; Fo = b.Fk; outsign = 1; break;
        default: i = b.imin + a1; j = b.jmin + a2; k = b.kmin; fi = i; fj = j; fk = k;
                 fg = b.fgk; Fo = b.Fk; outsign = -1; break;
    }
    const size_t c = pidx(b, i, j, k), f = pidx(b, fi, fj, fk);
    const double rho = b.W[W_RHO * b.npad + c], p = b.W[W_P * b.npad + c];
    const double u = b.W[W_U * b.npad + c];
    V3<double> v{b.W[W_VX * b.npad + c], b.W[W_VY * b.npad + c], b.W[W_VZ * b.npad + c]};
    if (o.order2 && o.local_frame && !b.axis_frames) replay_all_roundtrips(b, i, j, k, v);
    const double nx = fg[0 * b.npad + f], ny = fg[1 * b.npad + f], nz = fg[2 * b.npad + f];
    const double vrx = v.x - 0.0, vry = v.y - 0.0, vrz = v.z - 0.0;
    const double mass_flux = rho * (vrx * nx + vry * ny + vrz * nz);
    constexpr int NSPC = NSP > 1 ? NSP : 0;
    double F[5 + NSPC];
    if ((outsign * mass_flux) > 0.0) {
        F[0] = mass_flux;
        F[1] = p * nx + v.x * mass_flux;
        F[2] = p * ny + v.y * mass_flux;
        F[3] = p * nz + v.z * mass_flux;
        const double utot = u + 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z);
        F[4] = mass_flux * utot + p * (v.x * nx + v.y * ny + v.z * nz);
#pragma unroll
        for (int q = 0; q < NSPC; ++q) F[5 + q] = mass_flux * b.W[(W_NBASE + q) * b.npad + c];
    } else {
        F[0] = 0.0;
        F[1] = nx * p;
        F[2] = ny * p;
        F[3] = nz * p;
        F[4] = p * (0.0 * nx + 0.0 * ny + 0.0 * nz);
#pragma unroll
        for (int q = 0; q < NSPC; ++q) F[5 + q] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < 5 + NSPC; ++q) Fo[q * b.npad + f] = F[q];
}

// detect_shock_points (fluidblock.d:415-431) with PJ_ShockDetector
// (shockdetectors.d:20-59): a face flags compression between its two cells,
// (uR - uL) / min(aL, aR) < tol with u the velocity along the face normal; a
// cell is a shock point if any of its faces is.  The flags of ghost cells are
// those copied by the boundary conditions (the previous detection's).
__device__ __forceinline__ int face_shock(const BlockView& b, const double* fg, size_t f,
                                          size_t cl, size_t cr, double tol) {
    const double nx = fg[0 * b.npad + f], ny = fg[1 * b.npad + f], nz = fg[2 * b.npad + f];
    const double uL = b.W[W_VX * b.npad + cl] * nx + b.W[W_VY * b.npad + cl] * ny +
                      b.W[W_VZ * b.npad + cl] * nz;
    const double uR = b.W[W_VX * b.npad + cr] * nx + b.W[W_VY * b.npad + cr] * ny +
                      b.W[W_VZ * b.npad + cr] * nz;
    const double aL = b.W[W_A * b.npad + cl], aR = b.W[W_A * b.npad + cr];
    const double a_min = (aL < aR) ? aL : aR;
    return quotient_below(uR - uL, a_min, tol) ? 1 : 0;
}

__global__ void k_shock(BlockView b, const SimDev* sim, double tol) {
    if (sim->status != 0 || sim->finished) return;
    const long long n = (long long)b.ni * b.nj * b.nk;
    const size_t si = 1, sj = size_t(b.nidim), sk = size_t(b.nidim) * b.njdim;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = b.imin + int(t % b.ni);
        const int j = b.jmin + int((t / b.ni) % b.nj);
        const int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        const size_t c = pidx(b, i, j, k);
        int S = 0;
        S |= face_shock(b, b.fgi, c, c - si, c, tol);
        S |= face_shock(b, b.fgi, c + si, c, c + si, tol);
        S |= face_shock(b, b.fgj, c, c - sj, c, tol);
        S |= face_shock(b, b.fgj, c + sj, c, c + sj, tol);
        if (b.dim == 3) {
            S |= face_shock(b, b.fgk, c, c - sk, c, tol);
            S |= face_shock(b, b.fgk, c + sk, c, c + sk, tol);
        }
        b.S[c] = S;
    }
}

// Ghost cells of an exchange boundary take the partner cells' volume and
// lengths (exchange_geometry, full_face_copy.d:963-1083, CopyDataOption.grid).
__global__ void k_exchange_geometry(BlockView b, int which) {
    int n1, n2;
    if (which == NORTH || which == SOUTH) { n1 = b.ni; n2 = b.nk; }
    else if (which == EAST || which == WEST) { n1 = b.nj; n2 = b.nk; }
    else { n1 = b.ni; n2 = b.nj; }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n1 * n2) return;
    const int a1 = t % n1, a2 = t / n1;
    int i, j, k, di = 0, dj = 0, dk = 0;
    switch (which) {
        case NORTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmax; dj = 1; break;
        case SOUTH: i = b.imin + a1; k = b.kmin + a2; j = b.jmin; dj = -1; break;
        case EAST: j = b.jmin + a1; k = b.kmin + a2; i = b.imax; di = 1; break;
        case WEST: j = b.jmin + a1; k = b.kmin + a2; i = b.imin; di = -1; break;
        case TOP: i = b.imin + a1; j = b.jmin + a2; k = b.kmax; dk = 1; break;
        default: i = b.imin + a1; j = b.jmin + a2; k = b.kmin; dk = -1; break;
    }
    const ExchangeSrc& o = b.ex[which];
    for (int g = 0; g < 2; ++g) {
        int si, sj, sk;
        ffc_partner(which, o.face, o.orient, a1, a2, g, o.ni, o.nj, o.nk, si, sj, sk);
        const size_t sc = (size_t(sk + o.kmin) * o.njdim + sj + 2) * o.nidim + si + 2;
        const size_t gc = pidx(b, i + (g + 1) * di, j + (g + 1) * dj, k + (g + 1) * dk);
        for (int q = 0; q < 4; ++q) b.cgeom[q * b.npad + gc] = o.cgeom[q * o.npad + sc];
    }
}

void launch_exchange_geometry(const BlockView& b, int which, cudaStream_t s) {
    int n;
    if (which == NORTH || which == SOUTH) n = b.ni * b.nk;
    else if (which == EAST || which == WEST) n = b.nj * b.nk;
    else n = b.ni * b.nj;
    k_exchange_geometry<<<(n + 127) / 128, 128, 0, s>>>(b, which);
}

// ---------------------------------------------------------------------------
// Time step: signal_frequency + block min/max (fvcell.d:1624-1705,
// fluidblock.d:776-862)
// ---------------------------------------------------------------------------
__global__ void k_dt(BlockView b, const SimDev* sim, double cfl_value, const double* dt_current_p,
                     unsigned long long* acc) {
    // acc[0] = min dt_local, acc[1] = max cfl_local (as ordered bits), acc[2] = last signal
    if (sim && (sim->status != 0 || sim->finished)) return;
    const long long n = (long long)b.ni * b.nj * b.nk;
    const double dt_current = *dt_current_p;
    double dmin = DBL_MAX, cmax = 0.0;
    bool any = false;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        const size_t c = pidx(b, i, j, k);
        V3<double> v{b.W[W_VX * b.npad + c], b.W[W_VY * b.npad + c], b.W[W_VZ * b.npad + c]};
        const double a = b.W[W_A * b.npad + c];
        const size_t sj = b.nidim, sk = size_t(b.nidim) * b.njdim;
        const size_t fN = c + sj, fE = c + 1, fT = c + sk;
        V3<double> nN{b.fgj[fN], b.fgj[b.npad + fN], b.fgj[2 * b.npad + fN]};
        V3<double> nE{b.fgi[fE], b.fgi[b.npad + fE], b.fgi[2 * b.npad + fE]};
        double un_N = fabs(dot3(v, nN));
        double un_E = fabs(dot3(v, nE));
        double un_T = 0.0;
        if (b.dim == 3) {
            V3<double> nT{b.fgk[fT], b.fgk[b.npad + fT], b.fgk[2 * b.npad + fT]};
            un_T = fabs(dot3(v, nT));
        }
        double signal = 0.0;
        signal = fmax(signal, (un_N + a) / b.cgeom[2 * b.npad + c]);
        signal = fmax(signal, (un_E + a) / b.cgeom[1 * b.npad + c]);
        if (b.dim == 3) signal = fmax(signal, (un_T + a) / b.cgeom[3 * b.npad + c]);
        double cfl_local = dt_current * signal;
        double dt_local = cfl_value / signal;
        dmin = fmin(dmin, dt_local);
        cmax = any ? fmax(cmax, cfl_local) : cfl_local;
        any = true;
        if (i == b.imax && j == b.jmax && k == b.kmax)
            acc[2] = static_cast<unsigned long long>(__double_as_longlong(signal));
    }
    // warp reduction then one atomic per warp
    for (int off = 16; off > 0; off >>= 1) {
        dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, off));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
    }
    if ((threadIdx.x & 31) == 0) {
        if (dmin >= 0.0) atomicMin(&acc[0], dbits(dmin));
        if (cmax >= 0.0) atomicMax(&acc[1], dbits(cmax));
    }
}

__global__ void k_dt_reset(unsigned long long* acc, int nb) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nb) {
        acc[3 * t + 0] = dbits(DBL_MAX);
        acc[3 * t + 1] = 0ull;
        acc[3 * t + 2] = 0ull;
    }
}

// The simcore.d:1347-1452 logic over all blocks (one thread).
__global__ void k_dt_finalize(SimDev* sim, const unsigned long long* acc, const int* hlist, int nb,
                              double cfl_allow, double dt_init, double dt_max, int check_cfl,
                              int step0, double* out_dt_allow, double* out_cfl_max) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (sim && (sim->status != 0 || sim->finished)) return;
    if (check_cfl < 0) {  // take SimState.step from the device-side loop
        check_cfl = sim->step > 0;
        step0 = sim->step == 0;
    }
    double dt_allow = DBL_MAX, cfl_max = 0.0;
    for (int q = 0; q < nb; ++q) {
        const int h = hlist[q];
        double d = __longlong_as_double(static_cast<long long>(acc[3 * h + 0]));
        double c = __longlong_as_double(static_cast<long long>(acc[3 * h + 1]));
        double last_signal = __longlong_as_double(static_cast<long long>(acc[3 * h + 2]));
        if (check_cfl && (c < 0.0 || c > cfl_allow)) {
            c = 0.5 * cfl_allow;
            d = c / last_signal;
        }
        dt_allow = (d < dt_allow) ? d : dt_allow;
        cfl_max = (c > cfl_max) ? c : cfl_max;
    }
    if (out_dt_allow) { *out_dt_allow = dt_allow; *out_cfl_max = cfl_max; }
    if (!sim) return;
    if (step0) dt_allow = fmin(dt_init, dt_allow);  // SimState.step == 0
    if (dt_allow <= sim->dt_global) {
        sim->dt_global = dt_allow;
    } else {
        double g = sim->dt_global * 1.5;
        g = (dt_allow < g) ? dt_allow : g;
        g = (dt_max < g) ? dt_max : g;
        sim->dt_global = g;
    }
}

__global__ void k_stage_check(SimDev* sim, int max_invalid_cells) {
    if (sim->status == 0 && sim->bad_cells > max_invalid_cells) {
        sim->status = -4;
        sim->status_step = sim->step;
    }
}

__global__ void k_reset_bad(SimDev* sim) { sim->bad_cells = 0; }

__global__ void k_end_step(SimDev* sim) {
    if (sim->status != 0 || sim->finished) return;
    sim->time = sim->time + sim->dt_global;  // simcore.d:2951
    sim->step = sim->step + 1;
    if (sim->time >= sim->max_time) sim->finished = 1;  // simcore.d:1099
}

__global__ void k_begin_run(SimDev* sim, double max_time) {
    sim->max_time = max_time;
    sim->finished = (sim->time >= max_time) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
static int grid_for(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 64) g = 148LL * 64;
    if (g < 1) g = 1;
    return int(g);
}

void launch_geometry(const BlockView& b, const double* vtx, cudaStream_t s) {
    const int T = 256;
    long long n = (long long)b.ni * b.nj * b.nk;
    k_geom_cells<<<grid_for(n, T), T, 0, s>>>(b, vtx);
    for (int d = 0; d < b.dim; ++d) {
        long long nf = (long long)(b.ni + (d == 0)) * (b.nj + (d == 1)) * (b.nk + (d == 2));
        k_geom_faces<<<grid_for(nf, T), T, 0, s>>>(b, vtx, d);
    }
    int m = b.ni * b.nj;
    m = m > b.nj * b.nk ? m : b.nj * b.nk;
    m = m > b.ni * b.nk ? m : b.ni * b.nk;
    k_geom_ghost_lengths<<<(m + T - 1) / T, T, 0, s>>>(b);
}

void launch_upload(const BlockView& b, const double* prim, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_upload<<<grid_for(n, 256), 256, 0, s>>>(b, prim);
}

void launch_upload_cons(const BlockView& b, const double* cons, SimDev* sim, const GasConsts& gas,
                        cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_upload_cons<<<grid_for(n, 256), 256, 0, s>>>(b, cons, sim, gas);
}

void launch_download(const BlockView& b, double* prim, double* cons, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_download<<<grid_for(n, 256), 256, 0, s>>>(b, prim, cons);
}

// Cells of the largest boundary face layer of the block (a 2-D block has no
// top or bottom face: its grid would otherwise be sized by the whole plane).
static int boundary_extent(const BlockView& b) {
    int m = b.ni * b.nk;
    m = m > b.nj * b.nk ? m : b.nj * b.nk;
    if (b.dim == 3) m = m > b.ni * b.nj ? m : b.ni * b.nj;
    return m;
}

void launch_bc(const BlockView& b, const SimDev* sim, cudaStream_t s) {
    const int m = boundary_extent(b);
    dim3 grid((m + 127) / 128, b.dim == 3 ? 6 : 4);
    if (b.nsp == 5) k_bc<5><<<grid, 128, 0, s>>>(b, sim);
    else k_bc<1><<<grid, 128, 0, s>>>(b, sim);
}

void launch_bc_linear(const BlockView& b, SimDev* sim, const GasConsts& gas, cudaStream_t s) {
    if (b.nsp == 5) {
        launch_bc_linear_tp(b, sim, gas, s);
        return;
    }
    const int m = boundary_extent(b);
    dim3 grid((m + 127) / 128, b.dim == 3 ? 6 : 4);
    k_bc_linear<1, 0><<<grid, 128, 0, s>>>(b, sim, gas);
}

void launch_ghost_defaults(const BlockView& b, const GasConsts& gas, cudaStream_t s) {
    if (b.nsp == 5) {
        launch_ghost_defaults_tp(b, gas, s);
        return;
    }
    const int m = boundary_extent(b);
    dim3 grid((m + 127) / 128, b.dim == 3 ? 6 : 4);
    k_ghost_defaults<1, 0><<<grid, 128, 0, s>>>(b, gas);
}

void launch_bc_flux(const BlockView& b, const SimDev* sim, const FluxOpts& o, cudaStream_t s) {
    const int m = boundary_extent(b);
    dim3 grid((m + 127) / 128, b.dim == 3 ? 6 : 4);
    if (b.nsp == 5) k_bc_flux<5><<<grid, 128, 0, s>>>(b, sim, o);
    else k_bc_flux<1><<<grid, 128, 0, s>>>(b, sim, o);
}

void launch_shock(const BlockView& b, const SimDev* sim, double tol, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_shock<<<grid_for(n, 256), 256, 0, s>>>(b, sim, tol);
}

// The velocity each interior cell of a block with general face frames holds
// when its j faces (V1) and its k faces (V2) begin: interp_l2r2 turns the
// velocities of its four stencil cells into the face frame and back in place
// (onedinterp.d:445-454, 576-584), so after the i-face loop of
// sfluidblock.d:2190-2344 a cell carries the round-off of the (up to) four i
// faces it took part in, in loop order, and after the j-face loop that of its
// j faces too.  Each cell depends only on its own velocity and the frames of
// its faces, so one thread per cell replays them once per stage for every
// face that reads the cell.
__global__ void k_replay_base(BlockView b, const SimDev* sim) {
    if (sim->status != 0 || sim->finished) return;
    const long long n = (long long)b.ni * b.nj * b.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = b.imin + int(t % b.ni);
        const int j = b.jmin + int((t / b.ni) % b.nj);
        const int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        const size_t c = pidx(b, i, j, k);
        V3<double> v{b.W[W_VX * b.npad + c], b.W[W_VY * b.npad + c], b.W[W_VZ * b.npad + c]};
        for (int g = i - 1; g <= i + 2; ++g) {
            if (g < b.imin || g > b.imax + 1) continue;
            roundtrip(v, b.fgi, b.npad, pidx(b, g, j, k));
        }
        b.Vrt[c] = v.x; b.Vrt[b.npad + c] = v.y; b.Vrt[2 * b.npad + c] = v.z;
        if (b.dim == 3) {
            for (int g = j - 1; g <= j + 2; ++g) {
                if (g < b.jmin || g > b.jmax + 1) continue;
                roundtrip(v, b.fgj, b.npad, pidx(b, i, g, k));
            }
            b.Vrt[3 * b.npad + c] = v.x; b.Vrt[4 * b.npad + c] = v.y;
            b.Vrt[5 * b.npad + c] = v.z;
        }
    }
}

void launch_replay_base(const BlockView& b, const SimDev* sim, cudaStream_t s) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    const int T = 128;
    k_replay_base<<<grid_for(n, T), T, 0, s>>>(b, sim);
}

// Faces per run of the row-walking flux kernel: i faces (runs of neighbouring
// threads interleave along the row) and j, k faces (threads along i).  Long
// runs share the stencil replay of a run's first face over more faces; small
// blocks halve them until the launch has about half an SM-full of threads on
// every SM.  e4c_set_flux_runs fixes both lengths.
#ifndef E4C_ROW_RUN_I
#define E4C_ROW_RUN_I 8
#endif
#ifndef E4C_ROW_RUN_JK
#define E4C_ROW_RUN_JK 32
#endif

static long long row_threads(const BlockView& b, const int r[3]) {
    long long n = (long long)b.nj * b.nk * r[0] + (long long)b.ni * b.nk * r[1];
    if (b.dim == 3) n += (long long)b.ni * b.nj * r[2];
    return n;
}

int3 flux_row_runs(const BlockView& b, const FluxOpts& o) {
    const int nf[3] = {b.ni + 1, b.nj + 1, b.nk + 1};
    const bool fixed = o.row_run_i > 0 && o.row_run_jk > 0;
    const long long want = fixed ? 0 : 148LL * 1024;
    const int base_i = fixed ? o.row_run_i : E4C_ROW_RUN_I;
    const int base_jk = fixed ? o.row_run_jk : E4C_ROW_RUN_JK;
    int r[3];
    for (int shift = 0;; ++shift) {
        bool all_single = true;
        for (int d = 0; d < 3; ++d) {
            int len = (d == 0 ? base_i : base_jk) >> shift;
            if (len < 1) len = 1;
            all_single = all_single && len == 1;
            r[d] = (nf[d] + len - 1) / len;
        }
        if (all_single || row_threads(b, r) >= want) break;
    }
    return make_int3(r[0], r[1], r[2]);
}

void launch_flux(const BlockView& b, const SimDev* sim, const FluxOpts& o, int dir,
                 cudaStream_t s) {
    if (dir < 0 && o.order2 && o.local_frame && b.dim == 3 && b.nsp == 1) {
        // a 3-D ideal-gas block: every direction's rows in one launch, each
        // stencil cell loaded once per run.  (The 5-species form of the row
        // kernel would spill under its register cap, and 2-D rows are too few
        // to run long: those blocks keep one thread per face, starting from
        // k_replay_base where their frames are general.)
        const int3 runs = flux_row_runs(b, o);
        const int r[3] = {runs.x, runs.y, runs.z};
        const long long n = row_threads(b, r);
        const int T = kRowThreads;
        const int g = grid_for(n, T);
        if (b.Vrt) {
            if (o.flux == 1) k_flux_rows<1, 1, 0, true><<<g, T, 0, s>>>(b, sim, o, runs);
            else if (o.flux == 2) k_flux_rows<1, 2, 0, true><<<g, T, 0, s>>>(b, sim, o, runs);
            else if (o.flux == 3) k_flux_rows<1, 3, 0, true><<<g, T, 0, s>>>(b, sim, o, runs);
            else k_flux_rows<1, 0, 0, true><<<g, T, 0, s>>>(b, sim, o, runs);
        } else {
            if (o.flux == 1) k_flux_rows<1, 1, 0, false><<<g, T, 0, s>>>(b, sim, o, runs);
            else if (o.flux == 2) k_flux_rows<1, 2, 0, false><<<g, T, 0, s>>>(b, sim, o, runs);
            else if (o.flux == 3) k_flux_rows<1, 3, 0, false><<<g, T, 0, s>>>(b, sim, o, runs);
            else k_flux_rows<1, 0, 0, false><<<g, T, 0, s>>>(b, sim, o, runs);
        }
        return;
    }
    long long n = 0;
    for (int d = 0; d < b.dim; ++d)
        if (dir < 0 || d == dir)
            n += (long long)(b.ni + (d == 0)) * (b.nj + (d == 1)) * (b.nk + (d == 2));
    const int T = 128;
    const int g = grid_for(n, T);
    if (b.nsp == 5) {
        launch_flux_tp(b, sim, o, dir, g, T, s);
    } else {
        if (o.flux == 1) k_flux<1, 1, 0><<<g, T, 0, s>>>(b, sim, o, dir);
        else if (o.flux == 2) k_flux<1, 2, 0><<<g, T, 0, s>>>(b, sim, o, dir);
        else if (o.flux == 3) k_flux<1, 3, 0><<<g, T, 0, s>>>(b, sim, o, dir);
        else k_flux<1, 0, 0><<<g, T, 0, s>>>(b, sim, o, dir);
    }
}

void launch_update(const BlockView& b, SimDev* sim, const GasConsts& gas, int stage,
                   int final_stage, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    const int T = 128;
    if (b.nsp == 5) launch_update_tp(b, sim, gas, stage, final_stage, grid_for(n, T), T, s);
    else k_update<1, 0><<<grid_for(n, T), T, 0, s>>>(b, sim, gas, stage, final_stage);
}

// Per-cell chemistry step suggestion of the interior cells (i fastest) to or
// from a dense array.
__global__ void k_dt_chem_copy(BlockView b, double* dense, int to_dense) {
    const long long n = (long long)b.ni * b.nj * b.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = b.imin + int(t % b.ni);
        const int j = b.jmin + int((t / b.ni) % b.nj);
        const int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        const size_t c = pidx(b, i, j, k);
        if (to_dense) dense[t] = b.dt_chem[c];
        else b.dt_chem[c] = dense[t];
    }
}

void launch_dt_chem_copy(const BlockView& b, double* dense, int to_dense, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_dt_chem_copy<<<grid_for(n, 256), 256, 0, s>>>(b, dense, to_dense);
}

void launch_dt_reset(unsigned long long* acc, int nb, cudaStream_t s) {
    k_dt_reset<<<(nb + 127) / 128, 128, 0, s>>>(acc, nb);
}

void launch_dt(const BlockView& b, const SimDev* sim, double cfl_value, const double* dt_current,
               unsigned long long* acc, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_dt<<<grid_for(n, 256), 256, 0, s>>>(b, sim, cfl_value, dt_current, acc);
}

void launch_dt_finalize(SimDev* sim, const unsigned long long* acc, const int* hlist, int nb,
                        double cfl_allow, double dt_init, double dt_max, int check_cfl, int step0,
                        double* out_dt_allow, double* out_cfl_max, cudaStream_t s) {
    k_dt_finalize<<<1, 32, 0, s>>>(sim, acc, hlist, nb, cfl_allow, dt_init, dt_max, check_cfl,
                                   step0, out_dt_allow, out_cfl_max);
}

// Is the geometry uniform: every interior cell's (vol, iLen, jLen, kLen) and
// every face's (n, t1, t2, area) of a direction identical to the first one?
__global__ void k_check_uniform(BlockView b, int* flag) {
    const size_t c0 = pidx(b, b.imin, b.jmin, b.kmin);
    const long long nc = (long long)b.ni * b.nj * b.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nc;
         t += (long long)gridDim.x * blockDim.x) {
        int i = b.imin + int(t % b.ni);
        int j = b.jmin + int((t / b.ni) % b.nj);
        int k = b.kmin + int(t / ((long long)b.ni * b.nj));
        const size_t c = pidx(b, i, j, k);
        for (int q = 0; q < 4; ++q)
            if (b.cgeom[q * b.npad + c] != b.cgeom[q * b.npad + c0]) atomicOr(flag, 1);
        // the west, south and bottom faces of the cell, plus the far boundary faces
        const double* fgs[3] = {b.fgi, b.fgj, b.fgk};
        const size_t far[3] = {pidx(b, i + 1, j, k), pidx(b, i, j + 1, k), pidx(b, i, j, k + 1)};
        const bool at_far[3] = {i == b.imax, j == b.jmax, k == b.kmax};
        for (int d = 0; d < b.dim; ++d) {
            for (int q = 0; q < 10; ++q) {
                const double ref = fgs[d][q * b.npad + c0];
                if (fgs[d][q * b.npad + c] != ref) atomicOr(flag, 1);
                if (at_far[d] && fgs[d][q * b.npad + far[d]] != ref) atomicOr(flag, 1);
            }
            if (!frame_is_axis(fgs[d], b.npad, c)) atomicOr(flag + 1, 1);
            if (at_far[d] && !frame_is_axis(fgs[d], b.npad, far[d])) atomicOr(flag + 1, 1);
        }
    }
}

void launch_check_uniform(const BlockView& b, int* flag, cudaStream_t s) {
    long long n = (long long)b.ni * b.nj * b.nk;
    k_check_uniform<<<grid_for(n, 256), 256, 0, s>>>(b, flag);
}

void launch_reset_bad(SimDev* sim, cudaStream_t s) { k_reset_bad<<<1, 1, 0, s>>>(sim); }
void launch_stage_check(SimDev* sim, int max_invalid, cudaStream_t s) {
    k_stage_check<<<1, 1, 0, s>>>(sim, max_invalid);
}
void launch_end_step(SimDev* sim, cudaStream_t s) { k_end_step<<<1, 1, 0, s>>>(sim); }
void launch_begin_run(SimDev* sim, double max_time, cudaStream_t s) {
    k_begin_run<<<1, 1, 0, s>>>(sim, max_time);
}

}  // namespace e4c
