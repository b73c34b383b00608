/*
 * e4_oracle.cpp -- CPU FP64 oracle for the explicit structured-block update.
 *
 * TEST INFRASTRUCTURE ONLY: a plain restatement of the reference algorithm
 * used to check the CUDA library (tests, smoke) and to time the CPU baseline.
 * It is never linked into, loaded by or called from the product library.
 *
 * What each piece restates (paths inside the reference project):
 *   geometry       src/eilmer/sfluidblock.d:506-642 (vertex binding),
 *                  :650-712 (ghost lengths); src/geom/elements/properties.d
 *                  :97-141 quad_properties, :177-236 xyplane_quad_cell_properties,
 *                  :293-304 tetrahedron_volume, :390-419 pyramid_properties,
 *                  :568-648 hex_cell_properties; src/eilmer/fvinterface.d:265-317
 *   frames         src/geom/elements/vector3.d:386-451 (normalize, dot,
 *                  transform_to_local_frame / transform_to_global_frame), :604 cross
 *   ghost cells    src/eilmer/bc/ghost_cell_effect/ghost_cell.d:34-44,
 *                  internal_copy_then_reflect.d:94+, flow_state_copy.d:66+,
 *                  extrapolate_copy.d:82+ (x_order 0)
 *   reconstruction src/eilmer/onedinterp.d:22, :118-162 (l2r2), :435-585,
 *                  :1039-1068; src/eilmer/limiters.d:31-38
 *   face loops     src/eilmer/sfluidblock.d:2190-2344
 *   flux           src/eilmer/fluxcalc.d:26-128 compute_interface_flux,
 *                  :376-529 ausmdv; HLLC has no reference counterpart (Toro)
 *   cell update    src/eilmer/fvcell.d:494-560 encode, :563-732 decode,
 *                  :735-875 time_derivatives, :1153-1311 stage updates
 *   validity       src/eilmer/fluidblock.d:433-499, src/eilmer/flowstate.d:345-388,
 *                  src/gas/gas_state.d:199-241, src/eilmer/fvcore.d:20-27
 *   time step      src/eilmer/fvcell.d:1624-1705 signal_frequency,
 *                  src/eilmer/fluidblock.d:776-862, src/eilmer/simcore.d:1347-1452
 *   stage loop     src/eilmer/simcore.d:2303-2952, main loop :856-1110
 *   ideal gas      src/gas/ideal_gas.d:66-144
 *
 * Floating-point discipline: built with -ffp-contract=off so that every
 * multiply and add rounds separately, as the reference's D code does, and
 * every expression keeps the reference's left-to-right evaluation order.
 */
#include "e4_oracle.h"
#include "e4_oracle_internal.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace e4o {

// ---------------------------------------------------------------------------
// Vector helpers (src/geom/elements/vector3.d)
// ---------------------------------------------------------------------------
static inline double dot(const Vec3& a, const Vec3& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;  // vector3.d:409-414
}
static inline void to_local(Vec3& v, const Vec3& n, const Vec3& t1, const Vec3& t2) {
    double vx = dot(v, n), vy = dot(v, t1), vz = dot(v, t2);  // vector3.d:425-434
    v.x = vx; v.y = vy; v.z = vz;
}
static inline void to_global(Vec3& v, const Vec3& n, const Vec3& t1, const Vec3& t2) {
    double gx = v.x * n.x + v.y * t1.x + v.z * t2.x;  // vector3.d:439-451
    double gy = v.x * n.y + v.y * t1.y + v.z * t2.y;
    double gz = v.x * n.z + v.y * t1.z + v.z * t2.z;
    v.x = gx; v.y = gy; v.z = gz;
}
static inline void cross(Vec3& v3, const Vec3& v1, const Vec3& v2) {
    v3.x = v1.y * v2.z - v2.y * v1.z;  // vector3.d:604-609
    v3.y = v2.x * v1.z - v1.x * v2.z;
    v3.z = v1.x * v2.y - v2.x * v1.y;
}
static inline void normalize(Vec3& v) {
    double mag = std::sqrt(dot(v, v));  // vector3.d:386-404
    if (mag > 0.0) { v.x /= mag; v.y /= mag; v.z /= mag; }
    else { v.x = v.y = v.z = 0.0; }
    const double small = 1.0e-30;
    if (std::fabs(v.x) < small) v.x = 0.0;
    if (std::fabs(v.y) < small) v.y = 0.0;
    if (std::fabs(v.z) < small) v.z = 0.0;
}

// ---------------------------------------------------------------------------
// Geometry (src/geom/elements/properties.d)
// ---------------------------------------------------------------------------
static void quad_properties(const Vec3& p0, const Vec3& p1, const Vec3& p2, const Vec3& p3,
                            Vec3& n, Vec3& t1, Vec3& t2, double& area) {
    // properties.d:97-141 (centroid not needed on the hot path)
    double p01x = p1.x - p0.x + p2.x - p3.x;
    double p01y = p1.y - p0.y + p2.y - p3.y;
    double p01z = p1.z - p0.z + p2.z - p3.z;
    double p03x = p3.x - p0.x + p2.x - p1.x;
    double p03y = p3.y - p0.y + p2.y - p1.y;
    double p03z = p3.z - p0.z + p2.z - p1.z;
    double vax = p01y * p03z - p01z * p03y;  // cross_product, vector3.d:634-641
    double vay = p01z * p03x - p01x * p03z;
    double vaz = p01x * p03y - p01y * p03x;
    vax *= 0.25; vay *= 0.25; vaz *= 0.25;
    area = std::sqrt(vax * vax + vay * vay + vaz * vaz);
    if (area > 1.0e-20) {
        n.x = vax / area; n.y = vay / area; n.z = vaz / area;
        t1.x = p01x; t1.y = p01y; t1.z = p01z;
        normalize(t1);
        cross(t2, n, t1);
        normalize(t2);
    } else {
        n = {1.0, 0.0, 0.0}; t1 = {0.0, 1.0, 0.0}; t2 = {0.0, 0.0, 1.0};
    }
}

static double tetrahedron_volume(const Vec3& p0, const Vec3& p1, const Vec3& p2, const Vec3& p3) {
    // properties.d:293-304
    double dx01 = p1.x - p0.x, dy01 = p1.y - p0.y, dz01 = p1.z - p0.z;
    double dx02 = p2.x - p0.x, dy02 = p2.y - p0.y, dz02 = p2.z - p0.z;
    double cx = dy01 * dz02 - dz01 * dy02;
    double cy = dz01 * dx02 - dx01 * dz02;
    double cz = dx01 * dy02 - dy01 * dx02;
    double dx03 = p3.x - p0.x, dy03 = p3.y - p0.y, dz03 = p3.z - p0.z;
    return (dx03 * cx + dy03 * cy + dz03 * cz) / 6.0;
}

static double pyramid_volume(const Vec3& p0, const Vec3& p1, const Vec3& p2, const Vec3& p3,
                             const Vec3& p4) {
    // properties.d:390-419 (volume part; the moment is not needed)
    Vec3 pmB{0.25 * (p0.x + p1.x + p2.x + p3.x), 0.25 * (p0.y + p1.y + p2.y + p3.y),
             0.25 * (p0.z + p1.z + p2.z + p3.z)};
    double volume = 0.0;
    volume += tetrahedron_volume(p0, p1, pmB, p4);
    volume += tetrahedron_volume(p1, p2, pmB, p4);
    volume += tetrahedron_volume(p2, p3, pmB, p4);
    volume += tetrahedron_volume(p3, p0, pmB, p4);
    return volume;
}

static void hex_cell_properties(const Vec3 p[8], double& volume, double& iLen, double& jLen,
                                double& kLen) {
    // properties.d:568-648
    Vec3 c{0.125 * (p[0].x + p[1].x + p[2].x + p[3].x + p[4].x + p[5].x + p[6].x + p[7].x),
           0.125 * (p[0].y + p[1].y + p[2].y + p[3].y + p[4].y + p[5].y + p[6].y + p[7].y),
           0.125 * (p[0].z + p[1].z + p[2].z + p[3].z + p[4].z + p[5].z + p[6].z + p[7].z)};
    auto mid4 = [](const Vec3& a, const Vec3& b, const Vec3& cc, const Vec3& d) {
        return Vec3{0.25 * (a.x + b.x + cc.x + d.x), 0.25 * (a.y + b.y + cc.y + d.y),
                    0.25 * (a.z + b.z + cc.z + d.z)};
    };
    Vec3 pmN = mid4(p[3], p[2], p[6], p[7]);
    Vec3 pmE = mid4(p[1], p[2], p[6], p[5]);
    Vec3 pmS = mid4(p[0], p[1], p[5], p[4]);
    Vec3 pmW = mid4(p[0], p[3], p[7], p[4]);
    Vec3 pmT = mid4(p[4], p[5], p[6], p[7]);
    Vec3 pmB = mid4(p[0], p[1], p[2], p[3]);
    double dx, dy, dz;
    dx = pmE.x - pmW.x; dy = pmE.y - pmW.y; dz = pmE.z - pmW.z;
    iLen = std::sqrt(dx * dx + dy * dy + dz * dz);
    dx = pmN.x - pmS.x; dy = pmN.y - pmS.y; dz = pmN.z - pmS.z;
    jLen = std::sqrt(dx * dx + dy * dy + dz * dz);
    dx = pmT.x - pmB.x; dy = pmT.y - pmB.y; dz = pmT.z - pmB.z;
    kLen = std::sqrt(dx * dx + dy * dy + dz * dz);
    volume = 0.0;
    volume += pyramid_volume(p[6], p[7], p[3], p[2], c);
    volume += pyramid_volume(p[5], p[6], p[2], p[1], c);
    volume += pyramid_volume(p[4], p[5], p[1], p[0], c);
    volume += pyramid_volume(p[7], p[4], p[0], p[3], c);
    volume += pyramid_volume(p[7], p[6], p[5], p[4], c);
    volume += pyramid_volume(p[0], p[1], p[2], p[3], c);
    if ((volume < 0.0 && std::fabs(volume) < 1.0e-12) || (volume >= 0.0 && volume < 1.0e-20))
        volume = 0.0;
}

static void xyplane_quad_cell_properties(const Vec3& p0, const Vec3& p1, const Vec3& p2,
                                         const Vec3& p3, double& area, double& iLen,
                                         double& jLen) {
    // properties.d:177-236 (centroid and minLen not needed on the hot path)
    double xA = p1.x, yA = p1.y, xB = p2.x, yB = p2.y;
    double xC = p3.x, yC = p3.y, xD = p0.x, yD = p0.y;
    area = 0.5 * ((xB + xA) * (yB - yA) + (xC + xB) * (yC - yB) + (xD + xC) * (yD - yC) +
                  (xA + xD) * (yA - yD));
    double xN = 0.5 * (xC + xB), yN = 0.5 * (yC + yB);
    double xS = 0.5 * (xD + xA), yS = 0.5 * (yD + yA);
    double xE = 0.5 * (xA + xB), yE = 0.5 * (yA + yB);
    double xW = 0.5 * (xD + xC), yW = 0.5 * (yD + yC);
    double dx = xN - xS, dy = yN - yS;
    jLen = std::sqrt(dx * dx + dy * dy);
    dx = xE - xW; dy = yE - yW;
    iLen = std::sqrt(dx * dx + dy * dy);
}

static void face_2d_properties(const Vec3& A, const Vec3& B, Vec3& n, Vec3& t1, Vec3& t2,
                               double& area) {
    // fvinterface.d:265-297 (planar, not axisymmetric)
    double xA = A.x, yA = A.y, xB = B.x, yB = B.y;
    double LAB = std::sqrt((xB - xA) * (xB - xA) + (yB - yA) * (yB - yA));
    if (LAB > 1.0e-12) {
        n = {(yB - yA) / LAB, -(xB - xA) / LAB, 0.0};
        t2 = {0.0, 0.0, 1.0};
        cross(t1, n, t2);
        area = LAB;
    } else {
        n = {1.0, 0.0, 0.0}; t2 = {0.0, 0.0, 1.0}; t1 = {0.0, 1.0, 0.0};
        area = 0.0;
    }
}

void Block::compute_geometry() {
    auto V = [&](int i, int j, int k) -> const Vec3& { return vtx[idx(i, j, k)]; };
    // Cells (interior only; sfluidblock.d:656-661 iterates over `cells`).
    for (int k = kmin; k <= kmax; ++k)
        for (int j = jmin; j <= jmax; ++j)
            for (int i = imin; i <= imax; ++i) {
                Cell& c = cell(i, j, k);
                if (dim == 2) {
                    double area;
                    xyplane_quad_cell_properties(V(i, j, 0), V(i + 1, j, 0), V(i + 1, j + 1, 0),
                                                 V(i, j + 1, 0), area, c.iLen, c.jLen);
                    c.vol = area;
                    c.kLen = 0.0;
                } else {
                    Vec3 p[8] = {V(i, j, k),         V(i + 1, j, k),         V(i + 1, j + 1, k),
                                 V(i, j + 1, k),     V(i, j, k + 1),         V(i + 1, j, k + 1),
                                 V(i + 1, j + 1, k + 1), V(i, j + 1, k + 1)};
                    hex_cell_properties(p, c.vol, c.iLen, c.jLen, c.kLen);
                }
            }
    // Faces (sfluidblock.d:535-642 vertex order).
    for (int k = kmin; k <= kmax; ++k)
        for (int j = jmin; j <= jmax; ++j)
            for (int i = imin; i <= imax + 1; ++i) {
                Face& f = ifi[idx(i, j, k)];
                if (dim == 2) face_2d_properties(V(i, j, 0), V(i, j + 1, 0), f.n, f.t1, f.t2, f.area);
                else quad_properties(V(i, j, k), V(i, j + 1, k), V(i, j + 1, k + 1), V(i, j, k + 1),
                                     f.n, f.t1, f.t2, f.area);
            }
    for (int k = kmin; k <= kmax; ++k)
        for (int j = jmin; j <= jmax + 1; ++j)
            for (int i = imin; i <= imax; ++i) {
                Face& f = ifj[idx(i, j, k)];
                if (dim == 2) face_2d_properties(V(i + 1, j, 0), V(i, j, 0), f.n, f.t1, f.t2, f.area);
                else quad_properties(V(i, j, k), V(i, j, k + 1), V(i + 1, j, k + 1), V(i + 1, j, k),
                                     f.n, f.t1, f.t2, f.area);
            }
    if (dim == 3) {
        for (int k = kmin; k <= kmax + 1; ++k)
            for (int j = jmin; j <= jmax; ++j)
                for (int i = imin; i <= imax; ++i) {
                    Face& f = ifk[idx(i, j, k)];
                    quad_properties(V(i, j, k), V(i + 1, j, k), V(i + 1, j + 1, k), V(i, j + 1, k),
                                    f.n, f.t1, f.t2, f.area);
                }
    }
    // Ghost-cell lengths copied from the mirror interior cells (sfluidblock.d:675-712).
    auto copy_len = [&](Cell& dst, const Cell& src) {
        dst.iLen = src.iLen; dst.jLen = src.jLen; dst.kLen = src.kLen;
    };
    for (int j = jmin; j <= jmax; ++j)
        for (int k = kmin; k <= kmax; ++k) {
            copy_len(cell(imin - 1, j, k), cell(imin, j, k));
            copy_len(cell(imin - 2, j, k), cell(imin + 1, j, k));
            copy_len(cell(imax + 1, j, k), cell(imax, j, k));
            copy_len(cell(imax + 2, j, k), cell(imax - 1, j, k));
        }
    for (int i = imin; i <= imax; ++i)
        for (int k = kmin; k <= kmax; ++k) {
            copy_len(cell(i, jmin - 1, k), cell(i, jmin, k));
            copy_len(cell(i, jmin - 2, k), cell(i, jmin + 1, k));
            copy_len(cell(i, jmax + 1, k), cell(i, jmax, k));
            copy_len(cell(i, jmax + 2, k), cell(i, jmax - 1, k));
        }
    if (dim == 3) {
        for (int i = imin; i <= imax; ++i)
            for (int j = jmin; j <= jmax; ++j) {
                copy_len(cell(i, j, kmin - 1), cell(i, j, kmin));
                copy_len(cell(i, j, kmin - 2), cell(i, j, kmin + 1));
                copy_len(cell(i, j, kmax + 1), cell(i, j, kmax));
                copy_len(cell(i, j, kmax + 2), cell(i, j, kmax - 1));
            }
    }
    // Are all face frames exact unit axes?  Then the in-place frame round
    // trips of interp_l2r2 leave the cell velocities numerically unchanged and
    // the face loops may run in parallel on copies.
    auto is_unit_axis = [](const Vec3& v) {
        int nz = 0, nu = 0;
        for (double c : {v.x, v.y, v.z}) {
            if (c == 0.0) ++nz;
            else if (c == 1.0 || c == -1.0) ++nu;
        }
        return nz == 2 && nu == 1;
    };
    axis_frames = true;
    auto check_faces = [&](std::vector<Face>& F, int i0, int i1, int j0, int j1, int k0, int k1) {
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i) {
                    const Face& f = F[idx(i, j, k)];
                    if (!is_unit_axis(f.n) || !is_unit_axis(f.t1) || !is_unit_axis(f.t2))
                        axis_frames = false;
                }
    };
    check_faces(ifi, imin, imax + 1, jmin, jmax, kmin, kmax);
    check_faces(ifj, imin, imax, jmin, jmax + 1, kmin, kmax);
    if (dim == 3) check_faces(ifk, imin, imax, jmin, jmax, kmin, kmax + 1);
}

// ---------------------------------------------------------------------------
// Ideal gas (src/gas/ideal_gas.d)
// ---------------------------------------------------------------------------
void GasModel::init_ideal(double mol_mass, double gamma_) {
    kind = E4O_GAS_IDEAL;
    nsp = 1;
    Rgas = R_universal / mol_mass;  // ideal_gas.d:66-69
    gamma = gamma_;
    Cv = Rgas / (gamma - 1.0);
    Cvinv = 1.0 / Cv;
    Cp = Rgas * gamma / (gamma - 1.0);
}

bool GasModel::update_thermo_from_pT(GasState& Q) const {
    if (kind != E4O_GAS_IDEAL) return tp_update_thermo_from_pT(Q);
    if (Q.T <= 0.0 || Q.p <= 0.0) return false;  // ideal_gas.d:89-96
    Q.rho = Q.p / (Q.T * Rgas);
    Q.u = Cv * Q.T;
    return true;
}
bool GasModel::update_thermo_from_rhou(GasState& Q) const {
    if (kind != E4O_GAS_IDEAL) return tp_update_thermo_from_rhou(Q);
    if (Q.u <= 0.0 || Q.rho <= 0.0) return false;  // ideal_gas.d:98-106
    Q.T = Q.u * Cvinv;
    Q.p = Q.rho * Rgas * Q.T;
    return true;
}
bool GasModel::update_thermo_from_rhoT(GasState& Q) const {
    if (kind != E4O_GAS_IDEAL) return tp_update_thermo_from_rhoT(Q);
    if (Q.T <= 0.0 || Q.rho <= 0.0) return false;  // ideal_gas.d:107-115
    Q.p = Q.rho * Rgas * Q.T;
    Q.u = Cv * Q.T;
    return true;
}
bool GasModel::update_sound_speed(GasState& Q) const {
    if (kind != E4O_GAS_IDEAL) return tp_update_sound_speed(Q);
    if (Q.T <= 0.0) return false;  // ideal_gas.d:137-144
    Q.a = std::sqrt(gamma * Rgas * Q.T);
    return true;
}

// ---------------------------------------------------------------------------
// Reconstruction (src/eilmer/onedinterp.d, src/eilmer/limiters.d)
// ---------------------------------------------------------------------------
static inline double clip_to_limits(double q, double A, double B) {
    double lower = (A <= B) ? A : B;  // limiters.d:31-38
    double upper = (A > B) ? A : B;
    double qc = (q > lower) ? q : lower;
    return (qc <= upper) ? qc : upper;
}

struct L2R2 {
    // l2r2_prepare, onedinterp.d:118-133
    double aL0, aR0, lenL0_, lenR0_, two_over_lenL0_plus_lenL1, two_over_lenR0_plus_lenL0,
        two_over_lenR1_plus_lenR0, two_lenL0_plus_lenL1, two_lenR0_plus_lenR1;
    bool apply_limiter, extrema_clipping;
    void prepare(double lenL1, double lenL0, double lenR0, double lenR1) {
        lenL0_ = lenL0;
        lenR0_ = lenR0;
        aL0 = 0.5 * lenL0 / (lenL1 + 2.0 * lenL0 + lenR0);
        aR0 = 0.5 * lenR0 / (lenL0 + 2.0 * lenR0 + lenR1);
        two_over_lenL0_plus_lenL1 = 2.0 / (lenL0 + lenL1);
        two_over_lenR0_plus_lenL0 = 2.0 / (lenR0 + lenL0);
        two_over_lenR1_plus_lenR0 = 2.0 / (lenR1 + lenR0);
        two_lenL0_plus_lenL1 = (2.0 * lenL0 + lenL1);
        two_lenR0_plus_lenR1 = (2.0 * lenR0 + lenR1);
    }
    // interp_l2r2_scalar, onedinterp.d:136-162
    void scalar(double qL1, double qL0, double qR0, double qR1, double& qL, double& qR) const {
        const double eps = 1.0e-12;  // epsilon_van_albada, onedinterp.d:22
        double delLminus = (qL0 - qL1) * two_over_lenL0_plus_lenL1;
        double del = (qR0 - qL0) * two_over_lenR0_plus_lenL0;
        double delRplus = (qR1 - qR0) * two_over_lenR1_plus_lenR0;
        double sL = 1.0, sR = 1.0;
        if (apply_limiter) {
            sL = (delLminus * del + std::fabs(delLminus * del) + eps) /
                 (delLminus * delLminus + del * del + eps);
            sR = (del * delRplus + std::fabs(del * delRplus) + eps) /
                 (del * del + delRplus * delRplus + eps);
        }
        qL = qL0 + sL * aL0 * (del * two_lenL0_plus_lenL1 + delLminus * lenR0_);
        qR = qR0 - sR * aR0 * (delRplus * lenL0_ + del * two_lenR0_plus_lenR1);
        if (extrema_clipping) {
            qL = clip_to_limits(qL, qL0, qR0);
            qR = clip_to_limits(qR, qL0, qR0);
        }
    }
};

// ---------------------------------------------------------------------------
// Flux calculators (src/eilmer/fluxcalc.d)
// ---------------------------------------------------------------------------
void Sim::ausmdv(const FlowState& Lft, const FlowState& Rght, double* F) const {
    // fluxcalc.d:376-529
    double rL = Lft.gas.rho, pL = Lft.gas.p;
    double pLrL = pL / rL;
    double uL = Lft.vel.x, vL = Lft.vel.y, wL = Lft.vel.z;
    double eL = Lft.gas.u;  // internal_energy()
    double aL = Lft.gas.a;
    double keL = 0.5 * (uL * uL + vL * vL + wL * wL);
    double HL = eL + pLrL + keL;
    double rR = Rght.gas.rho, pR = Rght.gas.p;
    double pRrR = pR / rR;
    double uR = Rght.vel.x, vR = Rght.vel.y, wR = Rght.vel.z;
    double eR = Rght.gas.u;
    double aR = Rght.gas.a;
    double keR = 0.5 * (uR * uR + vR * vR + wR * wR);
    double HR = eR + pRrR + keR;
    double alphaL = 2.0 * pLrL / (pLrL + pRrR);
    double alphaR = 2.0 * pRrR / (pLrL + pRrR);
    double am = std::fmax(aL, aR);
    double ML = uL / am;
    double MR = uR / am;
    double pLplus, uLplus;
    double duL = 0.5 * (uL + std::fabs(uL));
    if (std::fabs(ML) <= 1.0) {
        pLplus = pL * (ML + 1.0) * (ML + 1.0) * (2.0 - ML) * 0.25;
        uLplus = alphaL * ((uL + am) * (uL + am) / (4.0 * am) - duL) + duL;
    } else {
        pLplus = pL * duL / uL;
        uLplus = duL;
    }
    double pRminus, uRminus;
    double duR = 0.5 * (uR - std::fabs(uR));
    if (std::fabs(MR) <= 1.0) {
        pRminus = pR * (MR - 1.0) * (MR - 1.0) * (2.0 + MR) * 0.25;
        uRminus = alphaR * (-(uR - am) * (uR - am) / (4.0 * am) - duR) + duR;
    } else {
        pRminus = pR * duR / uR;
        uRminus = duR;
    }
    double ru_half = uLplus * rL + uRminus * rR;
    double p_half = pLplus + pRminus;
    double dp = pL - pR;
    const double K_SWITCH = 10.0;
    dp = K_SWITCH * std::fabs(dp) / std::fmin(pL, pR);
    double s = 0.5 * std::fmin(1.0, dp);
    double ru2_AUSMV = uLplus * rL * uL + uRminus * rR * uR;
    double ru2_AUSMD = 0.5 * (ru_half * (uL + uR) - std::fabs(ru_half) * (uR - uL));
    double ru2_half = (0.5 + s) * ru2_AUSMV + (0.5 - s) * ru2_AUSMD;
    F[0] = ru_half;
    if (ru_half >= 0.0) {
        F[1] = ru2_half + p_half; F[2] = ru_half * vL; F[3] = ru_half * wL;
        F[4] = ru_half * HL;
        for (int i = 0; i < nsp_cons; ++i) F[5 + i] = ru_half * Lft.gas.massf[i];
    } else {
        F[1] = ru2_half + p_half; F[2] = ru_half * vR; F[3] = ru_half * wR;
        F[4] = ru_half * HR;
        for (int i = 0; i < nsp_cons; ++i) F[5 + i] = ru_half * Rght.gas.massf[i];
    }
    const double C_EFIX = 0.125;
    bool caseA = ((uL - aL) < 0.0) && ((uR - aR) > 0.0);
    bool caseB = ((uL + aL) < 0.0) && ((uR + aR) > 0.0);
    double d_ua = 0.0;
    if (caseA && !caseB) d_ua = C_EFIX * ((uR - aR) - (uL - aL));
    if (caseB && !caseA) d_ua = C_EFIX * ((uR + aR) - (uL + aL));
    if (d_ua != 0.0) {
        F[0] -= d_ua * (rR - rL);
        F[1] -= d_ua * (rR * uR - rL * uL);
        F[2] -= d_ua * (rR * vR - rL * vL);
        F[3] -= d_ua * (rR * wR - rL * wL);
        F[4] -= d_ua * (rR * HR - rL * HL);
        for (int i = 0; i < nsp_cons; ++i)
            F[5 + i] -= d_ua * (rR * Rght.gas.massf[i] - rL * Lft.gas.massf[i]);
    }
}

void Sim::hanel(const FlowState& Lft, const FlowState& Rght, double* F) const {
    // fluxcalc.d:532-629 (Hanel, Schwane & Seider 1987, as in Wada & Liou 1997)
    double rL = Lft.gas.rho, pL = Lft.gas.p;
    double pLrL = pL / rL;
    double uL = Lft.vel.x, vL = Lft.vel.y, wL = Lft.vel.z;
    double eL = Lft.gas.u;
    double aL = Lft.gas.a;
    double keL = 0.5 * (uL * uL + vL * vL + wL * wL);
    double HL = eL + pLrL + keL;
    double rR = Rght.gas.rho, pR = Rght.gas.p;
    double pRrR = pR / rR;
    double uR = Rght.vel.x, vR = Rght.vel.y, wR = Rght.vel.z;
    double eR = Rght.gas.u;
    double aR = Rght.gas.a;
    double keR = 0.5 * (uR * uR + vR * vR + wR * wR);
    double HR = eR + pRrR + keR;
    double pLplus, uLplus;
    if (std::fabs(uL) <= aL) {
        uLplus = 1.0 / (4.0 * aL) * (uL + aL) * (uL + aL);
        pLplus = pL * uLplus * (1.0 / aL * (2.0 - uL / aL));
    } else {
        uLplus = 0.5 * (uL + std::fabs(uL));
        pLplus = pL * uLplus * (1.0 / uL);
    }
    double pRminus, uRminus;
    if (std::fabs(uR) <= aR) {
        uRminus = -1.0 / (4.0 * aR) * (uR - aR) * (uR - aR);
        pRminus = pR * uRminus * (1.0 / aR * (-2.0 - uR / aR));
    } else {
        uRminus = 0.5 * (uR - std::fabs(uR));
        pRminus = pR * uRminus * (1.0 / uR);
    }
    double p_half = pLplus + pRminus;
    F[0] = uLplus * rL + uRminus * rR;
    F[1] = uLplus * rL * uL + uRminus * rR * uR + p_half;
    F[2] = uLplus * rL * vL + uRminus * rR * vR;
    F[3] = uLplus * rL * wL + uRminus * rR * wR;
    F[4] = uLplus * rL * HL + uRminus * rR * HR;
    for (int i = 0; i < nsp_cons; ++i)
        F[5 + i] = uLplus * rL * Lft.gas.massf[i] + uRminus * rR * Rght.gas.massf[i];
}

void Sim::detect_shock_points(Block& b) {
    // fluidblock.d:415-431 with PJ_ShockDetector (shockdetectors.d:20-59):
    // every face flags compression between its two cells, every interior
    // cell is a shock point if any of its faces is.  All boundaries in scope
    // carry ghost cells, so both cells of a face always exist.
    const double tol = cfg.compression_tolerance;
    auto face_S = [&](const Face& f, const Cell& L, const Cell& R) {
        double uL = L.fs.vel.x * f.n.x + L.fs.vel.y * f.n.y + L.fs.vel.z * f.n.z;
        double uR = R.fs.vel.x * f.n.x + R.fs.vel.y * f.n.y + R.fs.vel.z * f.n.z;
        double aL = L.fs.gas.a, aR = R.fs.gas.a;
        double a_min = (aL < aR) ? aL : aR;
        return ((uR - uL) / a_min) < tol ? 1 : 0;
    };
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i) {
                int S = 0;
                S |= face_S(b.ifi[b.idx(i, j, k)], b.cell(i - 1, j, k), b.cell(i, j, k));
                S |= face_S(b.ifi[b.idx(i + 1, j, k)], b.cell(i, j, k), b.cell(i + 1, j, k));
                S |= face_S(b.ifj[b.idx(i, j, k)], b.cell(i, j - 1, k), b.cell(i, j, k));
                S |= face_S(b.ifj[b.idx(i, j + 1, k)], b.cell(i, j, k), b.cell(i, j + 1, k));
                if (b.dim == 3) {
                    S |= face_S(b.ifk[b.idx(i, j, k)], b.cell(i, j, k - 1), b.cell(i, j, k));
                    S |= face_S(b.ifk[b.idx(i, j, k + 1)], b.cell(i, j, k), b.cell(i, j, k + 1));
                }
                b.cell(i, j, k).fs.S = S;
            }
}

void Sim::hllc(const FlowState& Lft, const FlowState& Rght, double* F) const {
    // No reference counterpart: Toro's HLLC (Riemann Solvers and Numerical
    // Methods for Fluid Dynamics, 3rd ed., sec. 10.4-10.6) in the face frame,
    // with Davis wave-speed bounds SL = min(uL-aL, uR-aR), SR = max(uL+aL, uR+aR)
    // and the star-state flux F*K = FK + SK (U*K - UK).  Species ride on the
    // mass flux of the upwind star state.
    double rL = Lft.gas.rho, pL = Lft.gas.p, uL = Lft.vel.x, vL = Lft.vel.y, wL = Lft.vel.z;
    double aL = Lft.gas.a;
    double eL = Lft.gas.u + 0.5 * (uL * uL + vL * vL + wL * wL);  // total energy per mass
    double EL = rL * eL;
    double rR = Rght.gas.rho, pR = Rght.gas.p, uR = Rght.vel.x, vR = Rght.vel.y, wR = Rght.vel.z;
    double aR = Rght.gas.a;
    double eR = Rght.gas.u + 0.5 * (uR * uR + vR * vR + wR * wR);
    double ER = rR * eR;
    double SL = std::fmin(uL - aL, uR - aR);
    double SR = std::fmax(uL + aL, uR + aR);
    double mL = rL * (SL - uL);
    double mR = rR * (SR - uR);
    double Sstar = (pR - pL + mL * uL - mR * uR) / (mL - mR);
    if (SL >= 0.0) {
        double m = rL * uL;
        F[0] = m; F[1] = m * uL + pL; F[2] = m * vL; F[3] = m * wL; F[4] = uL * (EL + pL);
        for (int i = 0; i < nsp_cons; ++i) F[5 + i] = m * Lft.gas.massf[i];
    } else if (SR <= 0.0) {
        double m = rR * uR;
        F[0] = m; F[1] = m * uR + pR; F[2] = m * vR; F[3] = m * wR; F[4] = uR * (ER + pR);
        for (int i = 0; i < nsp_cons; ++i) F[5 + i] = m * Rght.gas.massf[i];
    } else if (Sstar >= 0.0) {
        double m = rL * uL;
        double coef = mL / (SL - Sstar);  // rho*L
        double Estar = coef * (eL + (Sstar - uL) * (Sstar + pL / mL));
        F[0] = m + SL * (coef - rL);
        F[1] = (m * uL + pL) + SL * (coef * Sstar - m);
        F[2] = m * vL + SL * (coef * vL - rL * vL);
        F[3] = m * wL + SL * (coef * wL - rL * wL);
        F[4] = uL * (EL + pL) + SL * (Estar - EL);
        for (int i = 0; i < nsp_cons; ++i) F[5 + i] = F[0] * Lft.gas.massf[i];
    } else {
        double m = rR * uR;
        double coef = mR / (SR - Sstar);
        double Estar = coef * (eR + (Sstar - uR) * (Sstar + pR / mR));
        F[0] = m + SR * (coef - rR);
        F[1] = (m * uR + pR) + SR * (coef * Sstar - m);
        F[2] = m * vR + SR * (coef * vR - rR * vR);
        F[3] = m * wR + SR * (coef * wR - rR * wR);
        F[4] = uR * (ER + pR) + SR * (Estar - ER);
        for (int i = 0; i < nsp_cons; ++i) F[5 + i] = F[0] * Rght.gas.massf[i];
    }
}

void Sim::interface_flux(FlowState& Lft, FlowState& Rght, Face& f) const {
    // compute_interface_flux, fluxcalc.d:26-128, for a fixed grid (gvel = 0):
    // the grid-velocity terms add signed zeros only and are left out.
    to_local(Lft.vel, f.n, f.t1, f.t2);
    to_local(Rght.vel, f.n, f.t1, f.t2);
    if (cfg.flux_calculator == E4O_FLUX_HLLC) {
        hllc(Lft, Rght, f.F);
    } else if (cfg.flux_calculator == E4O_FLUX_HANEL) {
        hanel(Lft, Rght, f.F);
    } else if (cfg.flux_calculator == E4O_FLUX_ADAPTIVE_HANEL_AUSMDV) {
        // adaptive_hanel_ausmdv, fluxcalc.d:824-838: Hanel next to shocks
        // unless the shear across the face is large, AUSMDV elsewhere
        double sound_speed = 0.5 * (Lft.gas.a + Rght.gas.a);
        double shear_y = std::fabs(Lft.vel.y - Rght.vel.y) / sound_speed;
        double shear_z = std::fabs(Lft.vel.z - Rght.vel.z) / sound_speed;
        bool shear_is_small = std::fmax(shear_y, shear_z) <= cfg.shear_tolerance;
        if ((Lft.S == 1 || Rght.S == 1) && shear_is_small) hanel(Lft, Rght, f.F);
        else ausmdv(Lft, Rght, f.F);
    } else {
        ausmdv(Lft, Rght, f.F);
    }
    Vec3 m{f.F[1], f.F[2], f.F[3]};
    to_global(m, f.n, f.t1, f.t2);
    f.F[1] = m.x; f.F[2] = m.y; f.F[3] = m.z;
}

bool Sim::scale_mass_fractions(double* massf) const {
    // gas_model.d:295-327 with the default tolerances (0.0, 0.1)
    double sum = 0.0;
    for (int i = 0; i < gm.nsp; ++i) {
        massf[i] = massf[i] >= 0.0 ? massf[i] : 0.0;
        sum += massf[i];
    }
    if (std::fabs(sum - 1.0) > 0.1) return false;
    if (std::fabs(sum - 1.0) > 0.0) {
        for (int i = 0; i < gm.nsp; ++i) massf[i] /= sum;
    }
    return true;
}

void Sim::interp_l2r2(Face& f, Cell& cL1, Cell& cL0, Cell& cR0, Cell& cR1, double lenL1,
                      double lenL0, double lenR0, double lenR1, FlowState& Lft,
                      FlowState& Rght) const {
    // onedinterp.d:435-585 with thermo_interpolator = rhou.  The cell
    // velocities are rotated in place and back again, as in the reference.
    Vec3 *vL1 = &cL1.fs.vel, *vL0 = &cL0.fs.vel, *vR0 = &cR0.fs.vel, *vR1 = &cR1.fs.vel;
    Vec3 cpL1, cpL0, cpR0, cpR1;
    if (!mutate_in_place) {
        cpL1 = *vL1; cpL0 = *vL0; cpR0 = *vR0; cpR1 = *vR1;
        vL1 = &cpL1; vL0 = &cpL0; vR0 = &cpR0; vR1 = &cpR1;
    }
    if (cfg.interpolate_in_local_frame) {
        to_local(*vL1, f.n, f.t1, f.t2);
        to_local(*vL0, f.n, f.t1, f.t2);
        to_local(*vR0, f.n, f.t1, f.t2);
        to_local(*vR1, f.n, f.t1, f.t2);
    }
    L2R2 r;
    r.apply_limiter = cfg.apply_limiter != 0;
    r.extrema_clipping = cfg.extrema_clipping != 0;
    r.prepare(lenL1, lenL0, lenR0, lenR1);
    r.scalar(vL1->x, vL0->x, vR0->x, vR1->x, Lft.vel.x, Rght.vel.x);
    r.scalar(vL1->y, vL0->y, vR0->y, vR1->y, Lft.vel.y, Rght.vel.y);
    r.scalar(vL1->z, vL0->z, vR0->z, vR1->z, Lft.vel.z, Rght.vel.z);
    const GasState &gL1 = cL1.fs.gas, &gL0 = cL0.fs.gas, &gR0 = cR0.fs.gas, &gR1 = cR1.fs.gas;
    if (gm.nsp > 1) {
        for (int isp = 0; isp < gm.nsp; ++isp)
            r.scalar(gL1.massf[isp], gL0.massf[isp], gR0.massf[isp], gR1.massf[isp],
                     Lft.gas.massf[isp], Rght.gas.massf[isp]);
        if (!scale_mass_fractions(Lft.gas.massf))
            for (int isp = 0; isp < gm.nsp; ++isp) Lft.gas.massf[isp] = gL0.massf[isp];
        if (!scale_mass_fractions(Rght.gas.massf))
            for (int isp = 0; isp < gm.nsp; ++isp) Rght.gas.massf[isp] = gR0.massf[isp];
    } else {
        Lft.gas.massf[0] = 1.0;
        Rght.gas.massf[0] = 1.0;
    }
    r.scalar(gL1.rho, gL0.rho, gR0.rho, gR1.rho, Lft.gas.rho, Rght.gas.rho);
    r.scalar(gL1.u, gL0.u, gR0.u, gR1.u, Lft.gas.u, Rght.gas.u);
    // codeForThermoUpdateBoth("rhou"), onedinterp.d:1039-1068: on failure the
    // whole cell-centre FlowState is copied (its velocity is in the local frame).
    if (!gm.update_thermo_from_rhou(Lft.gas)) { Lft = cL0.fs; Lft.vel = *vL0; }
    if (!gm.update_thermo_from_rhou(Rght.gas)) { Rght = cR0.fs; Rght.vel = *vR0; }
    if (cfg.interpolate_in_local_frame) {
        to_global(Lft.vel, f.n, f.t1, f.t2);
        to_global(Rght.vel, f.n, f.t1, f.t2);
        to_global(*vL1, f.n, f.t1, f.t2);
        to_global(*vL0, f.n, f.t1, f.t2);
        to_global(*vR0, f.n, f.t1, f.t2);
        to_global(*vR1, f.n, f.t1, f.t2);
    }
}

void Sim::face_flux(Block& b, Face& f, Cell& cL1, Cell& cL0, Cell& cR0, Cell& cR1, int dir) const {
    // One face of the loops at sfluidblock.d:2190-2344; all boundaries in scope
    // have ghost_cell_data_available = true.
    FlowState Lft = cL0.fs, Rght = cR0.fs;
    if (cfg.interpolation_order > 1) {
        double l1, l0, r0, r1;
        if (dir == 0) { l1 = cL1.iLen; l0 = cL0.iLen; r0 = cR0.iLen; r1 = cR1.iLen; }
        else if (dir == 1) { l1 = cL1.jLen; l0 = cL0.jLen; r0 = cR0.jLen; r1 = cR1.jLen; }
        else { l1 = cL1.kLen; l0 = cL0.kLen; r0 = cR0.kLen; r1 = cR1.kLen; }
        interp_l2r2(f, cL1, cL0, cR0, cR1, l1, l0, r0, r1, Lft, Rght);
    }
    (void)b;
    interface_flux(Lft, Rght, f);
}

// BFE_SimpleOutflowFlux (bc/boundary_flux_effect.d:367-546), the flux action
// of OutFlowBC_SimpleFlux: every face of the boundary takes the flux of the
// interior cell's flow state (fixed grid: v_rel = v), or that of a closed
// face if that state would flow in.  The convective-flux loops skip these
// faces (sfluidblock.d:2227-2228 and alike), after reconstructing them; the
// face flux computed there is overwritten here, which is the same.
void Sim::simple_outflow_flux(Block& b) {
    const int nb = (b.dim == 3) ? 6 : 4;
    const int nsp = gm.nsp;
    for (int which = 0; which < nb; ++which) {
        if (b.bc[which] != E4O_BC_OUTFLOW_SIMPLE_FLUX) continue;
        int i0 = b.imin, i1 = b.imax, j0 = b.jmin, j1 = b.jmax, k0 = b.kmin, k1 = b.kmax;
        if (which == 0) j0 = j1 = b.jmax;
        if (which == 2) j0 = j1 = b.jmin;
        if (which == 1) i0 = i1 = b.imax;
        if (which == 3) i0 = i1 = b.imin;
        if (which == 4) k0 = k1 = b.kmax;
        if (which == 5) k0 = k1 = b.kmin;
        const int outsign = (which == 0 || which == 1 || which == 4) ? 1 : -1;
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i) {
                    Face* f;
                    switch (which) {
                        case 0: f = &b.ifj[b.idx(i, j + 1, k)]; break;
                        case 1: f = &b.ifi[b.idx(i + 1, j, k)]; break;
                        case 2: f = &b.ifj[b.idx(i, j, k)]; break;
                        case 3: f = &b.ifi[b.idx(i, j, k)]; break;
                        case 4: f = &b.ifk[b.idx(i, j, k + 1)]; break;
                        default: f = &b.ifk[b.idx(i, j, k)]; break;
                    }
                    const FlowState& fs = b.cell(i, j, k).fs;
                    const Vec3 v_rel{fs.vel.x - 0.0, fs.vel.y - 0.0, fs.vel.z - 0.0};
                    const double mass_flux =
                        fs.gas.rho * (v_rel.x * f->n.x + v_rel.y * f->n.y + v_rel.z * f->n.z);
                    if ((outsign * mass_flux) > 0.0) {
                        f->F[0] = mass_flux;
                        f->F[1] = fs.gas.p * f->n.x + fs.vel.x * mass_flux;
                        f->F[2] = fs.gas.p * f->n.y + fs.vel.y * mass_flux;
                        f->F[3] = fs.gas.p * f->n.z + fs.vel.z * mass_flux;
                        const double utot =
                            fs.gas.u + 0.5 * (fs.vel.x * fs.vel.x + fs.vel.y * fs.vel.y +
                                              fs.vel.z * fs.vel.z);
                        f->F[4] = mass_flux * utot +
                                  fs.gas.p * (fs.vel.x * f->n.x + fs.vel.y * f->n.y + fs.vel.z * f->n.z);
                        if (nsp > 1)
                            for (int s = 0; s < nsp; ++s) f->F[5 + s] = mass_flux * fs.gas.massf[s];
                    } else {
                        f->F[0] = 0.0;
                        f->F[1] = f->n.x * fs.gas.p;
                        f->F[2] = f->n.y * fs.gas.p;
                        f->F[3] = f->n.z * fs.gas.p;
                        f->F[4] = fs.gas.p * (0.0 * f->n.x + 0.0 * f->n.y + 0.0 * f->n.z);
                        if (nsp > 1)
                            for (int s = 0; s < nsp; ++s) f->F[5 + s] = 0.0;
                    }
                }
    }
}

void Sim::convective_flux(Block& b) {
    const bool par = !mutate_in_place;
    // i-faces (east-facing), loops k, j, i.
#pragma omp parallel for collapse(2) schedule(static) if (par)
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax + 1; ++i)
                face_flux(b, b.ifi[b.idx(i, j, k)], b.cell(i - 2, j, k), b.cell(i - 1, j, k),
                          b.cell(i, j, k), b.cell(i + 1, j, k), 0);
    // j-faces (north-facing), loops k, j, i.
#pragma omp parallel for collapse(2) schedule(static) if (par)
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax + 1; ++j)
            for (int i = b.imin; i <= b.imax; ++i)
                face_flux(b, b.ifj[b.idx(i, j, k)], b.cell(i, j - 2, k), b.cell(i, j - 1, k),
                          b.cell(i, j, k), b.cell(i, j + 1, k), 1);
    if (b.dim == 2) return;
    // k-faces (top-facing), loops k, j, i.
#pragma omp parallel for collapse(2) schedule(static) if (par)
    for (int k = b.kmin; k <= b.kmax + 1; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i)
                face_flux(b, b.ifk[b.idx(i, j, k)], b.cell(i, j, k - 2), b.cell(i, j, k - 1),
                          b.cell(i, j, k), b.cell(i, j, k + 1), 2);
}

// ---------------------------------------------------------------------------
// Ghost cells (src/eilmer/bc/ghost_cell_effect/*)
// ---------------------------------------------------------------------------
// Cells of face f of block B along its two face indices: north/south (i, k),
// east/west (j, k), top/bottom (i, j).
static void face_extents(const Block& B, int f, int& P, int& Q) {
    P = (f == 1 || f == 3) ? B.nj : B.ni;
    Q = (f == 4 || f == 5) ? B.nj : B.nk;
}

// GhostCellFullFaceCopy.set_up_cell_mapping (src/eilmer/bc/ghost_cell_effect/
// full_face_copy.d:142-1083): the cell of partner block O (face fb, joint
// orientation r) that fills ghost layer g (0: next to the face) of boundary
// cell (i, j, k) on face `which` of block B, as padded indices of O.  The
// reference's 144 cases (and the 16 of 2-D) follow one rule: faces north,
// west, bottom form one class and east, south, top the other; seen from the
// second class the orientation turns the other way (r -> 4 - r); a joint
// within a class and a joint across the classes then each map the face
// indices (p, q) to the partner's (p', q') with P', Q' its extents:
//   within: r0 (P'-1-p, q)  r1 (q, p)      r2 (p, Q'-1-q)      r3 (P'-1-q, Q'-1-p)
//   across: r0 (p, q)       r1 (P'-1-q, p) r2 (P'-1-p, Q'-1-q) r3 (q, Q'-1-p)
static void map_face_cell(int which, int p, int q, int g, int fb, int r, int ni, int nj, int nk,
                          int& ai, int& aj, int& ak) {
    auto first_class = [](int f) { return f == 0 || f == 3 || f == 5; };
    const bool ca = first_class(which), cb = first_class(fb);
    if (!ca) r = (4 - r) % 4;
    const int P = (fb == 1 || fb == 3) ? nj : ni;
    const int Q = (fb == 4 || fb == 5) ? nj : nk;
    // rows: r; columns: (coefficient of p, of q, constant) for p' and for q',
    // where a constant of -1 stands for "extent - 1 -" (a reversed index)
    static const int within[4][2][3] = {{{1, 0, -1}, {0, 1, 0}},  {{0, 1, 0}, {1, 0, 0}},
                                        {{1, 0, 0}, {0, 1, -1}},  {{0, 1, -1}, {1, 0, -1}}};
    static const int across[4][2][3] = {{{1, 0, 0}, {0, 1, 0}},   {{0, 1, -1}, {1, 0, 0}},
                                        {{1, 0, -1}, {0, 1, -1}}, {{0, 1, 0}, {1, 0, -1}}};
    const int(*m)[3] = (ca == cb) ? within[r] : across[r];
    int out[2];
    for (int a = 0; a < 2; ++a) {
        const int v = m[a][0] * p + m[a][1] * q;
        const int ext = (a == 0) ? P : Q;
        out[a] = (m[a][2] < 0) ? ext - 1 - v : v;
    }
    switch (fb) {
        case 0: ai = out[0]; ak = out[1]; aj = nj - 1 - g; break;
        case 2: ai = out[0]; ak = out[1]; aj = g; break;
        case 1: aj = out[0]; ak = out[1]; ai = ni - 1 - g; break;
        case 3: aj = out[0]; ak = out[1]; ai = g; break;
        case 4: ai = out[0]; aj = out[1]; ak = nk - 1 - g; break;
        default: ai = out[0]; aj = out[1]; ak = g; break;
    }
}

static void mapped_cell(const Block& B, int which, int i, int j, int k, int g, const Block& O,
                        int fb, int r, int& si, int& sj, int& sk) {
    // face indices of the boundary cell
    const int p = (which == 1 || which == 3) ? j - B.jmin : i - B.imin;
    const int q = (which == 4 || which == 5) ? j - B.jmin : k - B.kmin;
    int ai, aj, ak;
    map_face_cell(which, p, q, g, fb, r, O.ni, O.nj, O.nk, ai, aj, ak);
    si = O.imin + ai;
    sj = O.jmin + aj;
    sk = O.kmin + ak;
}

static inline void reflect_normal_velocity(FlowState& fs, const Face& f) {
    to_local(fs.vel, f.n, f.t1, f.t2);  // ghost_cell.d:34-44
    fs.vel.x = -(fs.vel.x);
    to_global(fs.vel, f.n, f.t1, f.t2);
}

int Sim::apply_bcs(Block& b) {
    // Boundaries in the order north, east, south, west, top, bottom.
    const int nb = (b.dim == 3) ? 6 : 4;
    for (int which = 0; which < nb; ++which) {
        const int type = b.bc[which];
        // (di,dj,dk) steps outward; the boundary cell layer is at the edge.
        int di = 0, dj = 0, dk = 0;
        switch (which) {
            case 0: dj = 1; break;
            case 1: di = 1; break;
            case 2: dj = -1; break;
            case 3: di = -1; break;
            case 4: dk = 1; break;
            case 5: dk = -1; break;
        }
        int i0 = b.imin, i1 = b.imax, j0 = b.jmin, j1 = b.jmax, k0 = b.kmin, k1 = b.kmax;
        if (which == 0) j0 = j1 = b.jmax;
        if (which == 2) j0 = j1 = b.jmin;
        if (which == 1) i0 = i1 = b.imax;
        if (which == 3) i0 = i1 = b.imin;
        if (which == 4) k0 = k1 = b.kmax;
        if (which == 5) k0 = k1 = b.kmin;
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i) {
                    Cell& g1 = b.cell(i + di, j + dj, k + dk);
                    Cell& g2 = b.cell(i + 2 * di, j + 2 * dj, k + 2 * dk);
                    if (type == E4O_BC_EXCHANGE && b.ex_block[which] < 0) {
                        // a partner on another rank: the ghost cells hold
                        // what e4o_unpack_face wrote before this stage
                        // (full_face_copy.d exchange over MPI, :1134, :1255)
                        continue;
                    } else if (type == E4O_BC_EXCHANGE) {
                        // full_face_copy.d: the ghost layers take the cells of
                        // the partner mapped to them (set_up_cell_mapping)
                        Block& o = *blocks[b.ex_block[which]];
                        for (int g = 0; g < 2; ++g) {
                            int si, sj, sk;
                            mapped_cell(b, which, i, j, k, g, o, b.ex_face[which],
                                        b.ex_orient[which], si, sj, sk);
                            (g == 0 ? g1 : g2).fs = o.cell(si, sj, sk).fs;
                        }
                    } else if (type == E4O_BC_OUTFLOW_EXTRAPOLATE_LINEAR) {
                        // extrapolate_copy.d:206-258 (east; alike for every
                        // face), x_order 1: each ghost layer from the two
                        // cells before it, rho, u and mass fractions, then
                        // update_thermo_from_rhou, then the velocity; the
                        // sound speed and shock flag are not touched
                        const Cell* c1 = &b.cell(i, j, k);
                        const Cell* c2 = &b.cell(i - di, j - dj, k - dk);
                        Cell* dst[2] = {&g1, &g2};
                        for (int g = 0; g < 2; ++g) {
                            GasState& d = dst[g]->fs.gas;
                            const GasState &q1 = c1->fs.gas, &q2 = c2->fs.gas;
                            d.rho = 2.0 * q1.rho - q2.rho;
                            d.u = 2.0 * q1.u - q2.u;
                            if (gm.nsp > 1) {
                                for (int sp = 0; sp < gm.nsp; ++sp)
                                    d.massf[sp] = 2.0 * q1.massf[sp] - q2.massf[sp];
                                if (!scale_mass_fractions(d.massf)) return E4O_ERR_THERMO;
                            } else {
                                d.massf[0] = 1.0;
                            }
                            if (!gm.update_thermo_from_rhou(d)) return E4O_ERR_THERMO;
                            Vec3& v = dst[g]->fs.vel;
                            v.x = 2.0 * c1->fs.vel.x - c2->fs.vel.x;
                            v.y = 2.0 * c1->fs.vel.y - c2->fs.vel.y;
                            v.z = 2.0 * c1->fs.vel.z - c2->fs.vel.z;
                            c2 = c1;
                            c1 = dst[g];
                        }
                    } else if (type == E4O_BC_INFLOW_SUPERSONIC) {
                        g1.fs = b.inflow;  // flow_state_copy.d:66+
                        g2.fs = b.inflow;
                    } else if (type == E4O_BC_OUTFLOW_EXTRAPOLATE ||
                               type == E4O_BC_OUTFLOW_SIMPLE_FLUX) {
                        // extrapolate_copy.d:82+, x_order 0 (also the ghost
                        // cells of OutFlowBC_SimpleFlux, bc.lua:1124-1146)
                        const Cell& src = b.cell(i, j, k);
                        g1.fs = src.fs;
                        g2.fs = src.fs;
                    } else {
                        // internal_copy_then_reflect.d:94+ ; the face is that of the
                        // boundary cell on this boundary.
                        const Face* f;
                        switch (which) {
                            case 0: f = &b.ifj[b.idx(i, j + 1, k)]; break;
                            case 1: f = &b.ifi[b.idx(i + 1, j, k)]; break;
                            case 2: f = &b.ifj[b.idx(i, j, k)]; break;
                            case 3: f = &b.ifi[b.idx(i, j, k)]; break;
                            case 4: f = &b.ifk[b.idx(i, j, k + 1)]; break;
                            default: f = &b.ifk[b.idx(i, j, k)]; break;
                        }
                        g1.fs = b.cell(i, j, k).fs;
                        reflect_normal_velocity(g1.fs, *f);
                        g2.fs = b.cell(i - di, j - dj, k - dk).fs;
                        reflect_normal_velocity(g2.fs, *f);
                    }
                }
    }
    return 0;
}

// The ghost cells of a block's x_order 1 boundaries as a cell's initial
// FlowState (fvcell.d:168-170, flowstate.d:115-131): 100 kPa, 300 K, at rest,
// mass fractions (1, 0, ...), from update_thermo_from_pT and update_sound_speed.
void Sim::reset_linear_ghosts(Block& b) {
    FlowState fs;
    fs.gas.p = 100.0e3;
    fs.gas.T = 300.0;
    for (int sp = 0; sp < NSPMAX; ++sp) fs.gas.massf[sp] = (sp == 0) ? 1.0 : 0.0;
    gm.update_thermo_from_pT(fs.gas);
    gm.update_sound_speed(fs.gas);
    fs.vel = {0.0, 0.0, 0.0};
    fs.S = 0;
    const int nb = (b.dim == 3) ? 6 : 4;
    for (int which = 0; which < nb; ++which) {
        if (b.bc[which] != E4O_BC_OUTFLOW_EXTRAPOLATE_LINEAR) continue;
        int di = 0, dj = 0, dk = 0;
        switch (which) {
            case 0: dj = 1; break;
            case 1: di = 1; break;
            case 2: dj = -1; break;
            case 3: di = -1; break;
            case 4: dk = 1; break;
            default: dk = -1; break;
        }
        int i0 = b.imin, i1 = b.imax, j0 = b.jmin, j1 = b.jmax, k0 = b.kmin, k1 = b.kmax;
        if (which == 0) j0 = j1 = b.jmax;
        if (which == 2) j0 = j1 = b.jmin;
        if (which == 1) i0 = i1 = b.imax;
        if (which == 3) i0 = i1 = b.imin;
        if (which == 4) k0 = k1 = b.kmax;
        if (which == 5) k0 = k1 = b.kmin;
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i)
                    for (int g = 1; g <= 2; ++g) b.cell(i + g * di, j + g * dj, k + g * dk).fs = fs;
    }
}

// ---------------------------------------------------------------------------
// Cell update (src/eilmer/fvcell.d)
// ---------------------------------------------------------------------------
void Sim::encode_conserved(Cell& c, int ftl) const {
    // fvcell.d:494-560
    double* U = c.U[ftl];
    const FlowState& fs = c.fs;
    U[0] = fs.gas.rho;
    U[1] = fs.gas.rho * fs.vel.x;
    U[2] = fs.gas.rho * fs.vel.y;
    U[3] = fs.gas.rho * fs.vel.z;
    double u = fs.gas.u;
    double ke = 0.5 * (fs.vel.x * fs.vel.x + fs.vel.y * fs.vel.y + fs.vel.z * fs.vel.z);
    U[4] = fs.gas.rho * (u + ke);
    for (int isp = 0; isp < nsp_cons; ++isp) U[5 + isp] = fs.gas.rho * fs.gas.massf[isp];
}

int Sim::decode_conserved(Cell& c, int ftl) const {
    // fvcell.d:563-732 with adjust_invalid_cell_data = false,
    // ignore_low_T_thermo_update_failure = true, suggested_low_T_value = 200 K.
    const double* U = c.U[ftl];
    FlowState& fs = c.fs;
    if (!(U[0] > 0.0)) return -1;  // "Bad cell with negative mass."
    double rho = U[0];
    fs.gas.rho = rho;
    double dinv = 1.0 / rho;
    fs.vel.x = U[1] * dinv; fs.vel.y = U[2] * dinv; fs.vel.z = U[3] * dinv;
    double rE = U[4];
    double u = rE * dinv;
    double ke = 0.5 * (fs.vel.x * fs.vel.x + fs.vel.y * fs.vel.y + fs.vel.z * fs.vel.z);
    u -= ke;
    fs.gas.u = u;
    if (nsp_cons > 0) {
        for (int isp = 0; isp < nsp_cons; ++isp) fs.gas.massf[isp] = U[5 + isp] * dinv;
        if (!scale_mass_fractions(fs.gas.massf)) return -2;
    }
    if (!gm.update_thermo_from_rhou(fs.gas)) {
        if (rho > 0.0) {
            fs.gas.T = 200.0;
            if (!gm.update_thermo_from_rhoT(fs.gas)) return -2;
            encode_conserved(c, ftl);
        } else {
            return -2;
        }
    }
    if (!gm.update_sound_speed(fs.gas)) return -2;
    return 0;
}

static bool check_data(const FlowState& fs, int nsp) {
    // flowstate.d:345-388, gas_state.d:199-241, limits fvcore.d:20-27
    bool ok = true;
    const GasState& g = fs.gas;
    if (!std::isfinite(g.rho) || g.rho < 1.01 * 0.0) ok = false;
    if (!std::isfinite(g.T) || g.T < 1.01 * 1.0) ok = false;
    if (!std::isfinite(g.p)) ok = false;
    if (!std::isfinite(g.a)) ok = false;
    double f_sum = 0.0;
    for (int i = 0; i < nsp; ++i) f_sum += g.massf[i];
    if (f_sum < 0.99 || f_sum > 1.01 || !std::isfinite(f_sum)) ok = false;
    if (std::fabs(fs.vel.x) > 30000.0 || std::fabs(fs.vel.y) > 30000.0 ||
        std::fabs(fs.vel.z) > 30000.0) ok = false;
    if (g.T < 0.0) ok = false;
    if (g.T > 50000.0) ok = false;
    return ok;
}

void Sim::time_derivatives(Block& b, Cell& c, int i, int j, int k, int ftl) const {
    // fvcell.d:735-875; faces in the order north, east, south, west, top, bottom
    // with outsign +1, +1, -1, -1, +1, -1 (sfluidblock.d:506-517).
    const Face* faces[6] = {&b.ifj[b.idx(i, j + 1, k)], &b.ifi[b.idx(i + 1, j, k)],
                            &b.ifj[b.idx(i, j, k)],     &b.ifi[b.idx(i, j, k)],
                            nullptr, nullptr};
    const double outsign[6] = {1.0, 1.0, -1.0, -1.0, 1.0, -1.0};
    int nf = 4;
    if (b.dim == 3) {
        faces[4] = &b.ifk[b.idx(i, j, k + 1)];
        faces[5] = &b.ifk[b.idx(i, j, k)];
        nf = 6;
    }
    const int nv = 5 + nsp_cons;
    double integral[5 + NSPMAX];
    for (int v = 0; v < nv; ++v) integral[v] = 0.0;
    for (int q = 0; q < nf; ++q) {
        const double* F = faces[q]->F;
        double area = outsign[q] * faces[q]->area;
        integral[0] -= F[0] * area;
        integral[1] -= F[1] * area;
        integral[2] -= F[2] * area;
        if (b.dim == 3) integral[3] -= F[3] * area;
        integral[4] -= F[4] * area;
        for (int isp = 0; isp < nsp_cons; ++isp) integral[5 + isp] -= F[5 + isp] * area;
    }
    double vol_inv = 1.0 / c.vol;
    double* dUdt = c.dUdt[ftl];
    for (int v = 0; v < nv; ++v) dUdt[v] = vol_inv * integral[v];  // + Q (zero source)
}

void Sim::stage_update(Cell& c, int stage, double dt) const {
    const int nv = 5 + nsp_cons;
    if (stage == 1) {
        // fvcell.d:1153-1238, gamma_1 = 1 for euler and predictor-corrector
        const double gamma_1 = 1.0;
        for (int v = 0; v < nv; ++v) c.U[1][v] = c.U[0][v] + dt * gamma_1 * c.dUdt[0][v];
    } else {
        // fvcell.d:1241-1311, predictor-corrector gamma_1 = gamma_2 = 0.5
        const double gamma_1 = 0.5, gamma_2 = 0.5;
        for (int v = 0; v < nv; ++v)
            c.U[2][v] = c.U[0][v] + dt * (gamma_1 * c.dUdt[0][v] + gamma_2 * c.dUdt[1][v]);
    }
}

int Sim::stage_cells(Block& b, int stage, double dt) {
    // simcore.d:2439-2478 (stage 1) and the stage-2 twin.
    const int ftl = stage - 1;
    int bad = 0, err = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : bad) reduction(min : err)
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i) {
                Cell& c = b.cell(i, j, k);
                time_derivatives(b, c, i, j, k, ftl);
                stage_update(c, stage, dt);
                int rc = decode_conserved(c, ftl + 1);
                if (rc != 0) { err = std::min(err, rc); c.data_is_bad = true; }
                if (c.data_is_bad || !check_data(c.fs, gm.nsp)) ++bad;
            }
    last_bad_cells = std::max(last_bad_cells, bad);
    if (err == -1) return E4O_ERR_BAD_MASS;
    if (err == -2) return E4O_ERR_THERMO;
    if (bad > cfg.max_invalid_cells) return E4O_ERR_BAD_CELLS;
    return 0;
}

// ---------------------------------------------------------------------------
// Time step (fvcell.d:1624-1705, fluidblock.d:776-862, simcore.d:1347-1452)
// ---------------------------------------------------------------------------
double Sim::signal_frequency(Block& b, Cell& c, int i, int j, int k) const {
    const Vec3& v = c.fs.vel;
    double un_N = std::fabs(dot(v, b.ifj[b.idx(i, j + 1, k)].n));
    double un_E = std::fabs(dot(v, b.ifi[b.idx(i + 1, j, k)].n));
    double un_T = (b.dim == 3) ? std::fabs(dot(v, b.ifk[b.idx(i, j, k + 1)].n)) : 0.0;
    double signal = 0.0;
    double signalN = (un_N + c.fs.gas.a) / c.jLen;
    signal = std::fmax(signal, signalN);
    double signalE = (un_E + c.fs.gas.a) / c.iLen;
    signal = std::fmax(signal, signalE);
    if (b.dim == 3) {
        double signalT = (un_T + c.fs.gas.a) / c.kLen;
        signal = std::fmax(signal, signalT);
    }
    return signal;
}

void Sim::block_dt(Block& b, double dt_current, bool check_cfl, double& dt_allow,
                   double& cfl_max) {
    const double cfl_value = cfg.cfl_value;
    const double cfl_allow = (cfg.update_scheme == E4O_UPDATE_PC) ? 1.2 : 0.9;
    double dta = DBL_MAX, cmax = -DBL_MAX;
    double last_signal = 0.0;
    const int li = b.imax, lj = b.jmax, lk = b.kmax;
#pragma omp parallel for collapse(2) schedule(static) reduction(min : dta) reduction(max : cmax)
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i) {
                double signal = signal_frequency(b, b.cell(i, j, k), i, j, k);
                double cfl_local = dt_current * signal;
                double dt_local = cfl_value / signal;
                dta = std::fmin(dta, dt_local);
                cmax = std::fmax(cmax, cfl_local);
            }
    // The rescale below uses the signal of the last cell of the loop.
    last_signal = signal_frequency(b, b.cell(li, lj, lk), li, lj, lk);
    if (check_cfl && (cmax < 0.0 || cmax > cfl_allow)) {
        cmax = 0.5 * cfl_allow;
        dta = cmax / last_signal;
    }
    dt_allow = dta;
    cfl_max = cmax;
}

void Sim::determine_time_step_size() {
    bool do_dt_check_now = (step % cfg.cfl_count) == 0;
    if (!do_dt_check_now) return;
    double dt_allow = DBL_MAX, cfl_max = 0.0;
    for (Block* b : blocks) {
        double d, c;
        block_dt(*b, dt_global, step > 0, d, c);
        dt_allow = std::min(dt_allow, d);
        cfl_max = std::max(cfl_max, c);
    }
    if (step == 0) dt_allow = std::fmin(cfg.dt_init, dt_allow);
    if (dt_allow <= dt_global) {
        dt_global = dt_allow;
    } else {
        dt_global = std::min(dt_global * 1.5, dt_allow);
        dt_global = std::min(dt_global, cfg.dt_max);
    }
    last_cfl_max = cfl_max;
}

int Sim::gasdynamic_stage(int stage) {
    // one stage of simcore.d:2303-2952 (euler / predictor-corrector, fixed
    // grid): every block's ghost cells first (exchange copies see no
    // flux-loop state), then every block's fluxes, then the cell updates
    if (stage == 1) last_bad_cells = 0;
    for (Block* b : blocks) {
        int rc = apply_bcs(*b);
        if (rc != 0) return rc;
    }
    // simcore.d:2354-2358, turned on by the adaptive flux calculator
    // (globalconfig.d:1942-1950)
    if (cfg.flux_calculator == E4O_FLUX_ADAPTIVE_HANEL_AUSMDV)
        for (Block* b : blocks) detect_shock_points(*b);
    for (Block* b : blocks) convective_flux(*b);
    // applyPostConvFluxAction of every block (simcore.d:2373-2377)
    for (Block* b : blocks) simple_outflow_flux(*b);
    for (Block* b : blocks) {
        int rc = stage_cells(*b, stage, dt_global);
        if (rc != 0) return rc;
    }
    return 0;
}

void Sim::finish_gasdynamic_step() {
    const int nstages = (cfg.update_scheme == E4O_UPDATE_PC) ? 2 : 1;
    const int end_indx = (nstages == 2) ? 2 : 1;
    for (Block* b : blocks)
        for (Cell& c : b->cells) std::swap(c.U[0], c.U[end_indx]);
    time = time + dt_global;
}

int Sim::gasdynamic_increment() {
    const int nstages = (cfg.update_scheme == E4O_UPDATE_PC) ? 2 : 1;
    for (int stage = 1; stage <= nstages; ++stage) {
        int rc = gasdynamic_stage(stage);
        if (rc != 0) return rc;
    }
    finish_gasdynamic_step();
    return 0;
}

// After the gas-dynamic increment: chemistry, then the step count.
int Sim::end_step() {
    if (cfg.reacting) {
        int rc = chemistry_step(dt_global);
        if (rc != 0) { error = "chemistry step failed"; return rc; }
    }
    step = step + 1;
    return 0;
}

int Sim::run(int nsteps, double max_time) {
#ifdef _OPENMP
    if (cfg.n_threads > 0) omp_set_num_threads(cfg.n_threads);
#endif
    int target = step + nsteps;
    bool finished = (time >= max_time) || (step >= target);
    while (!finished) {
        determine_time_step_size();
        int rc = gasdynamic_increment();
        if (rc != 0) { error = "gasdynamic step failed"; return rc; }
        rc = end_step();
        if (rc != 0) return rc;
        if (time >= max_time) finished = true;
        if (step >= target) finished = true;
    }
    return 0;
}

}  // namespace e4o

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
using namespace e4o;

extern "C" {

void e4o_default_config(e4o_config* c) {
    // Defaults of src/eilmer/globalconfig.d:440-734 for the keys in scope.
    std::memset(c, 0, sizeof(*c));
    c->dimensions = 2;
    c->flux_calculator = E4O_FLUX_AUSMDV;
    c->interpolation_order = 2;
    c->apply_limiter = 1;
    c->extrema_clipping = 1;
    c->interpolate_in_local_frame = 1;
    c->update_scheme = E4O_UPDATE_PC;
    c->cfl_value = 0.5;
    c->dt_init = 1.0e-3;
    c->dt_max = 1.0e-3;
    c->cfl_count = 10;
    c->max_invalid_cells = 0;
    c->gas_model = E4O_GAS_IDEAL;
    c->ideal_mol_mass = 0.02896;
    c->ideal_gamma = 1.4;
    c->reacting = 0;
    c->T_frozen = 300.0;
    c->n_threads = 1;
    c->shear_tolerance = 0.20;
    c->compression_tolerance = -0.30;
    c->chem_newton_iterations = 12;
    c->chem_method = 0;
}

void* e4o_sim_new(const e4o_config* cfg) {
    Sim* s = new Sim();
    s->cfg = *cfg;
    if (cfg->gas_model == E4O_GAS_IDEAL) s->gm.init_ideal(cfg->ideal_mol_mass, cfg->ideal_gamma);
    else s->gm.init_therm_perf_air5();
    s->nsp_cons = (s->gm.nsp > 1) ? s->gm.nsp : 0;
    s->dt_global = cfg->dt_init;  // simcore.d:562
    return s;
}

void e4o_sim_free(void* sim) { delete static_cast<Sim*>(sim); }

int e4o_add_block(void* sim, int ni, int nj, int nk, const double* vtx, const int* bc,
                  const double* inflow) {
    Sim* s = static_cast<Sim*>(sim);
    Block* b = new Block();
    b->init(s->cfg.dimensions, ni, nj, nk);
    const int nvi = ni + 1, nvj = nj + 1, nvk = (b->dim == 3) ? nk + 1 : 1;
    for (int k = 0; k < nvk; ++k)
        for (int j = 0; j < nvj; ++j)
            for (int i = 0; i < nvi; ++i) {
                const double* p = vtx + 3 * ((size_t(k) * nvj + j) * nvi + i);
                b->vtx[b->idx(i + b->imin, j + b->jmin, k + b->kmin)] = {p[0], p[1], p[2]};
            }
    for (int q = 0; q < 6; ++q) b->bc[q] = bc[q];
    s->unpack_prim(inflow, 1, 0, b->inflow);
    b->compute_geometry();
    s->mutate_in_place = s->mutate_in_place || !b->axis_frames;
    s->blocks.push_back(b);
    return int(s->blocks.size()) - 1;
}

void e4o_ffc_map(int fa, int fb, int r, int p, int q, int depth, int ni, int nj, int nk,
                 int* out3) {
    e4o::map_face_cell(fa, p, q, depth, fb, r, ni, nj, nk, out3[0], out3[1], out3[2]);
}

int e4o_connect_blocks(void* sim, int a, int fa, int b, int fb, int orientation) {
    Sim* s = static_cast<Sim*>(sim);
    const int nb = int(s->blocks.size());
    if (a < 0 || a >= nb || b < 0 || b >= nb || a == b) return E4O_ERR_ARG;
    if (fa < 0 || fa > 5 || fb < 0 || fb > 5 || orientation < 0 || orientation > 3)
        return E4O_ERR_ARG;
    Block& A = *s->blocks[a];
    Block& B = *s->blocks[b];
    if (A.dim == 2 && (fa >= 4 || fb >= 4 || orientation != 0)) return E4O_ERR_ARG;
    int Pa, Qa, Pb, Qb;
    face_extents(A, fa, Pa, Qa);
    face_extents(B, fb, Pb, Qb);
    if (orientation % 2 == 0 ? (Pa != Pb || Qa != Qb) : (Pa != Qb || Qa != Pb)) return E4O_ERR_ARG;
    A.bc[fa] = E4O_BC_EXCHANGE; A.ex_block[fa] = b; A.ex_face[fa] = fb; A.ex_orient[fa] = orientation;
    B.bc[fb] = E4O_BC_EXCHANGE; B.ex_block[fb] = a; B.ex_face[fb] = fa; B.ex_orient[fb] = orientation;
    // exchange_geometry (full_face_copy.d:963-1083, CopyDataOption.grid):
    // ghost cells take the partner cells' volume and lengths
    auto copy_geom = [](Block& D, int which, Block& O) {
        int di = 0, dj = 0, dk = 0;
        switch (which) {
            case 0: dj = 1; break;
            case 1: di = 1; break;
            case 2: dj = -1; break;
            case 3: di = -1; break;
            case 4: dk = 1; break;
            default: dk = -1; break;
        }
        int i0 = D.imin, i1 = D.imax, j0 = D.jmin, j1 = D.jmax, k0 = D.kmin, k1 = D.kmax;
        if (which == 0) j0 = j1 = D.jmax;
        if (which == 2) j0 = j1 = D.jmin;
        if (which == 1) i0 = i1 = D.imax;
        if (which == 3) i0 = i1 = D.imin;
        if (which == 4) k0 = k1 = D.kmax;
        if (which == 5) k0 = k1 = D.kmin;
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i)
                    for (int g = 0; g < 2; ++g) {
                        int si, sj, sk;
                        mapped_cell(D, which, i, j, k, g, O, D.ex_face[which], D.ex_orient[which],
                                    si, sj, sk);
                        Cell& gc = D.cell(i + (g + 1) * di, j + (g + 1) * dj, k + (g + 1) * dk);
                        const Cell& sc = O.cell(si, sj, sk);
                        gc.vol = sc.vol;
                        gc.iLen = sc.iLen;
                        gc.jLen = sc.jLen;
                        gc.kLen = sc.kLen;
                    }
    };
    copy_geom(A, fa, B);
    copy_geom(B, fb, A);
    return 0;
}

// ---------------------------------------------------------------------------
// Blocks whose partner lives on another rank (the reference's MPI exchange,
// full_face_copy.d:1134-1255, with the dt and bad-cell reductions of
// simcore.d:1399-1401, 2489 left to the caller)
// ---------------------------------------------------------------------------
static int face_cells(const Block& B, int which, int& i0, int& i1, int& j0, int& j1, int& k0,
                      int& k1, int& di, int& dj, int& dk) {
    di = dj = dk = 0;
    switch (which) {
        case 0: dj = 1; break;
        case 1: di = 1; break;
        case 2: dj = -1; break;
        case 3: di = -1; break;
        case 4: dk = 1; break;
        default: dk = -1; break;
    }
    i0 = B.imin; i1 = B.imax; j0 = B.jmin; j1 = B.jmax; k0 = B.kmin; k1 = B.kmax;
    if (which == 0) j0 = j1 = B.jmax;
    if (which == 2) j0 = j1 = B.jmin;
    if (which == 1) i0 = i1 = B.imax;
    if (which == 3) i0 = i1 = B.imin;
    if (which == 4) k0 = k1 = B.kmax;
    if (which == 5) k0 = k1 = B.kmin;
    return (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1);
}

static int fs_fields(const Sim& s) { return 8 + s.gm.nsp + 1; }

int e4o_set_remote(void* sim, int blk, int face) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size()) || face < 0 || face > 5) return E4O_ERR_ARG;
    Block& B = *s->blocks[blk];
    if (B.dim == 2 && face >= 4) return E4O_ERR_ARG;
    B.bc[face] = E4O_BC_EXCHANGE;
    B.ex_block[face] = -2;
    return 0;
}

int e4o_face_values(void* sim, int blk, int face) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size()) || face < 0 || face > 5) return E4O_ERR_ARG;
    int i0, i1, j0, j1, k0, k1, di, dj, dk;
    const int n = face_cells(*s->blocks[blk], face, i0, i1, j0, j1, k0, k1, di, dj, dk);
    return 2 * n * fs_fields(*s);
}

// The flow states of the two cell layers next to a face, nearest first, as
// the partner's ghost layers take them: [layer][face cell][field], fields
// rho, vx, vy, vz, p, T, u, a, massf[nsp], shock flag.
int e4o_pack_face(void* sim, int blk, int face, double* out) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size()) || face < 0 || face > 5 || !out)
        return E4O_ERR_ARG;
    Block& B = *s->blocks[blk];
    int i0, i1, j0, j1, k0, k1, di, dj, dk;
    const int n = face_cells(B, face, i0, i1, j0, j1, k0, k1, di, dj, dk);
    const int nf = fs_fields(*s), nsp = s->gm.nsp;
    for (int g = 0; g < 2; ++g) {
        int q = 0;
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i, ++q) {
                    const FlowState& fs = B.cell(i - g * di, j - g * dj, k - g * dk).fs;
                    double* o = out + (size_t(g) * n + q) * nf;
                    o[0] = fs.gas.rho; o[1] = fs.vel.x; o[2] = fs.vel.y; o[3] = fs.vel.z;
                    o[4] = fs.gas.p; o[5] = fs.gas.T; o[6] = fs.gas.u; o[7] = fs.gas.a;
                    for (int sp = 0; sp < nsp; ++sp) o[8 + sp] = fs.gas.massf[sp];
                    o[8 + nsp] = double(fs.S);
                }
    }
    return 0;
}

// The ghost layers of a remote face from the partner's packed layers.
int e4o_unpack_face(void* sim, int blk, int face, const double* in) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size()) || face < 0 || face > 5 || !in)
        return E4O_ERR_ARG;
    Block& B = *s->blocks[blk];
    int i0, i1, j0, j1, k0, k1, di, dj, dk;
    const int n = face_cells(B, face, i0, i1, j0, j1, k0, k1, di, dj, dk);
    const int nf = fs_fields(*s), nsp = s->gm.nsp;
    for (int g = 0; g < 2; ++g) {
        int q = 0;
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i, ++q) {
                    FlowState& fs =
                        B.cell(i + (g + 1) * di, j + (g + 1) * dj, k + (g + 1) * dk).fs;
                    const double* v = in + (size_t(g) * n + q) * nf;
                    fs.gas.rho = v[0]; fs.vel.x = v[1]; fs.vel.y = v[2]; fs.vel.z = v[3];
                    fs.gas.p = v[4]; fs.gas.T = v[5]; fs.gas.u = v[6]; fs.gas.a = v[7];
                    for (int sp = 0; sp < nsp; ++sp) fs.gas.massf[sp] = v[8 + sp];
                    fs.S = int(v[8 + nsp]);
                }
    }
    return 0;
}

// This rank's share of determine_time_step_size (simcore.d:1362-1386): the
// minimum dt_allow and maximum CFL over its blocks, each block's rescale
// applied; the caller reduces over ranks and takes the global decision.
int e4o_dt_allow(void* sim, double dt_current, int check_cfl, double* dt_allow, double* cfl_max) {
    Sim* s = static_cast<Sim*>(sim);
    double d_all = DBL_MAX, c_all = 0.0;
    for (Block* b : s->blocks) {
        double d, c;
        s->block_dt(*b, dt_current, check_cfl != 0, d, c);
        d_all = std::min(d_all, d);
        c_all = std::max(c_all, c);
    }
    *dt_allow = d_all;
    *cfl_max = c_all;
    return 0;
}

void e4o_set_dt_global(void* sim, double dt) { static_cast<Sim*>(sim)->dt_global = dt; }

// One stage of the gas-dynamic increment over every block with dt_global;
// the last stage also ends the step (time, chemistry, step count).
int e4o_stage(void* sim, int stage) {
    Sim* s = static_cast<Sim*>(sim);
    const int nstages = (s->cfg.update_scheme == E4O_UPDATE_PC) ? 2 : 1;
    if (stage < 1 || stage > nstages) return E4O_ERR_ARG;
    int rc = s->gasdynamic_stage(stage);
    if (rc != 0) { s->error = "gasdynamic step failed"; return rc; }
    if (stage == nstages) {
        s->finish_gasdynamic_step();
        rc = s->end_step();
        if (rc != 0) return rc;
    }
    return 0;
}

int e4o_set_flow(void* sim, int blk, const double* prim) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size())) return E4O_ERR_ARG;
    Block& b = *s->blocks[blk];
    const size_t n = b.ncell();
    size_t q = 0;
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i, ++q) {
                Cell& c = b.cell(i, j, k);
                s->unpack_prim(prim, n, q, c.fs);
                s->encode_conserved(c, 0);
                c.dt_chem = -1.0;
            }
    s->reset_linear_ghosts(b);
    return 0;
}

int e4o_get_flow(void* sim, int blk, double* prim, double* cons) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size())) return E4O_ERR_ARG;
    Block& b = *s->blocks[blk];
    const size_t n = b.ncell();
    const int nv = 5 + s->nsp_cons;
    size_t q = 0;
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i, ++q) {
                const Cell& c = b.cell(i, j, k);
                if (prim) s->pack_prim(c.fs, prim, n, q);
                if (cons)
                    for (int v = 0; v < nv; ++v) cons[v * n + q] = c.U[0][v];
            }
    return 0;
}

int e4o_get_cell_geometry(void* sim, int blk, double* out) {
    Sim* s = static_cast<Sim*>(sim);
    if (blk < 0 || blk >= int(s->blocks.size())) return E4O_ERR_ARG;
    Block& b = *s->blocks[blk];
    const size_t n = b.ncell();
    size_t q = 0;
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax; ++i, ++q) {
                const Cell& c = b.cell(i, j, k);
                out[q] = c.vol; out[n + q] = c.iLen; out[2 * n + q] = c.jLen; out[3 * n + q] = c.kLen;
            }
    double* fo = out + 4 * n;
    auto put = [&](const Face& f) {
        const double vals[10] = {f.n.x, f.n.y, f.n.z, f.t1.x, f.t1.y, f.t1.z,
                                 f.t2.x, f.t2.y, f.t2.z, f.area};
        for (double v : vals) *fo++ = v;
    };
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax; ++j)
            for (int i = b.imin; i <= b.imax + 1; ++i) put(b.ifi[b.idx(i, j, k)]);
    for (int k = b.kmin; k <= b.kmax; ++k)
        for (int j = b.jmin; j <= b.jmax + 1; ++j)
            for (int i = b.imin; i <= b.imax; ++i) put(b.ifj[b.idx(i, j, k)]);
    if (b.dim == 3)
        for (int k = b.kmin; k <= b.kmax + 1; ++k)
            for (int j = b.jmin; j <= b.jmax; ++j)
                for (int i = b.imin; i <= b.imax; ++i) put(b.ifk[b.idx(i, j, k)]);
    return 0;
}

int e4o_run(void* sim, int nsteps, double max_time) {
    return static_cast<Sim*>(sim)->run(nsteps, max_time);
}
double e4o_time(void* sim) { return static_cast<Sim*>(sim)->time; }
double e4o_dt_global(void* sim) { return static_cast<Sim*>(sim)->dt_global; }
int e4o_step_count(void* sim) { return static_cast<Sim*>(sim)->step; }
int e4o_last_bad_cells(void* sim) { return static_cast<Sim*>(sim)->last_bad_cells; }
const char* e4o_last_error(void* sim) { return static_cast<Sim*>(sim)->error.c_str(); }

int e4o_ideal_gas_pT(double mol_mass, double gamma, double p, double T, double* rho, double* u,
                     double* a) {
    GasModel gm;
    gm.init_ideal(mol_mass, gamma);
    GasState Q;
    Q.p = p; Q.T = T;
    if (!gm.update_thermo_from_pT(Q) || !gm.update_sound_speed(Q)) return E4O_ERR_THERMO;
    *rho = Q.rho; *u = Q.u; *a = Q.a;
    return 0;
}

}  // extern "C"
