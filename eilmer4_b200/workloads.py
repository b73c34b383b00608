"""Grids and initial flow states for the structured-block workloads.

These play the part of the reference's preparation step (``e4shared --prep``:
``prep.lua`` builds the grid, evaluates the initial ``FlowState`` at each cell
centroid and writes the flow file).  Flow states are built from (p, T) exactly
as ``IdealGas.update_thermo_from_pT`` + ``update_sound_speed`` do
(src/gas/ideal_gas.d:89-96, 137-144), in IEEE double arithmetic with the same
operation order, so the library and any checker start from identical bits.

Workloads (sizes as stated; all data synthetic, generated from a fixed seed):
  * ``sod_2d``        2-D Sod shock tube, 256 x 64 cells on the unit square,
                      slip walls all round (ausmdv, 1000 steps).
  * ``sod_3d_tube``   the reference's own 3-D Sod regression deck
                      (examples/eilmer/3D/sod-shock-tube/sg/sod.lua):
                      100 x 2 x 2 cells on 1.0 x 0.1 x 0.1.
  * ``inflow_3d``     256^3 ideal-air block on the unit cube, Mach 3 inflow at
                      i-min, extrapolate outflow at i-max, slip walls elsewhere,
                      density perturbed by 8 seeded random-phase sines.
  * ``batched_blocks`` 64 independent 3-D blocks with edges drawn
                      log-uniformly in [16, 96], each initialised like
                      ``inflow_3d`` with its own seed offset.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

R_UNIVERSAL = 8.31451  # J/(mol.K), src/gas/physical_constants.d:13

# Boundary order north, east, south, west, top, bottom (src/eilmer/fvcore.d Face).
NORTH, EAST, SOUTH, WEST, TOP, BOTTOM = range(6)
BC_SLIP_WALL = 0
BC_INFLOW_SUPERSONIC = 1
BC_OUTFLOW_EXTRAPOLATE = 2
BC_OUTFLOW_SIMPLE_FLUX = 4   # OutFlowBC_SimpleFlux (bc.lua:1124-1146)
BC_OUTFLOW_EXTRAPOLATE_LINEAR = 5   # OutFlowBC_SimpleExtrapolate{xOrder=1}

DEFAULT_SEED = 20261203

# Primitive variable order used at the library boundary.
PRIM_VARS = ("rho", "velx", "vely", "velz", "p", "T", "u", "a")


def splitmix64(seed: int):
    """The project RNG: SplitMix64 (Steele, Lea & Flood 2014), yields floats in [0,1)."""
    state = seed & 0xFFFFFFFFFFFFFFFF
    mask = 0xFFFFFFFFFFFFFFFF
    while True:
        state = (state + 0x9E3779B97F4A7C15) & mask
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z = z ^ (z >> 31)
        yield (z >> 11) * (1.0 / (1 << 53))


@dataclass
class IdealGas:
    """Ideal air as in src/gas/sample-data/ideal-air-gas-model.lua."""
    mol_mass: float = 0.02896
    gamma: float = 1.4

    @property
    def R(self):
        return R_UNIVERSAL / self.mol_mass  # ideal_gas.d:66

    @property
    def Cv(self):
        return self.R / (self.gamma - 1.0)

    def from_pT(self, p, T):
        """rho, u, a from p and T (ideal_gas.d:89-96 and :137-144)."""
        p = np.asarray(p, dtype=np.float64)
        T = np.asarray(T, dtype=np.float64)
        rho = p / (T * self.R)
        u = self.Cv * T
        a = np.sqrt(self.gamma * self.R * T)
        return rho, u, a

    def from_rhop(self, rho, p):
        """T, u, a from rho and p (ideal_gas.d:116-123 and :137-144)."""
        rho = np.asarray(rho, dtype=np.float64)
        p = np.asarray(p, dtype=np.float64)
        T = p / (rho * self.R)
        u = self.Cv * T
        a = np.sqrt(self.gamma * self.R * T)
        return T, u, a


@dataclass
class BlockSpec:
    """One structured block: grid, boundary conditions and initial state."""
    ni: int
    nj: int
    nk: int
    vtx: np.ndarray            # ((nk+1)*(nj+1)*(ni+1), 3), i fastest; nk+1 -> 1 in 2-D
    bc: tuple                  # 6 ints, order N, E, S, W, T, B
    inflow: np.ndarray         # primitive FlowState used by inflow boundaries
    prim: np.ndarray           # (8 [+nsp], ncell) primitive SoA over interior cells

    @property
    def ncell(self):
        return self.ni * self.nj * self.nk


@dataclass
class Workload:
    name: str
    dimensions: int
    blocks: list = field(default_factory=list)
    flux_calculator: str = "ausmdv"
    nsteps: int = 1
    gas: IdealGas = field(default_factory=IdealGas)

    @property
    def ncell(self):
        return sum(b.ncell for b in self.blocks)


def box_vertices(ni, nj, nk, lx, ly, lz, dimensions, origin=(0.0, 0.0, 0.0), spacing=None):
    """Vertices of a Cartesian box; x = origin + lx*(i/ni) like a parametric map,
    or x = origin + i*spacing when a cell spacing is given."""
    def axis(n, L, o):
        r = np.arange(n + 1, dtype=np.float64)
        return o + (r * spacing if spacing is not None else L * (r / n))
    xs = axis(ni, lx, origin[0])
    ys = axis(nj, ly, origin[1])
    if dimensions == 3:
        zs = axis(nk, lz, origin[2])
    else:
        zs = np.zeros(1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).copy()


def cell_centres(vtx, ni, nj, nk, dimensions):
    """Average of the cell's corner vertices (exact for dyadic Cartesian grids)."""
    nvk = nk + 1 if dimensions == 3 else 1
    V = vtx.reshape(nvk, nj + 1, ni + 1, 3)
    if dimensions == 3:
        c = (V[:-1, :-1, :-1] + V[:-1, :-1, 1:] + V[:-1, 1:, 1:] + V[:-1, 1:, :-1]
             + V[1:, :-1, :-1] + V[1:, :-1, 1:] + V[1:, 1:, 1:] + V[1:, 1:, :-1]) * 0.125
    else:
        c = (V[:, :-1, :-1] + V[:, :-1, 1:] + V[:, 1:, 1:] + V[:, 1:, :-1]) * 0.25
    return c.reshape(-1, 3)


def prim_from(rho, vx, vy, vz, p, T, u, a):
    n = np.broadcast(rho, vx, vy, vz, p, T, u, a).shape
    out = np.empty((8,) + n, dtype=np.float64)
    for q, v in enumerate((rho, vx, vy, vz, p, T, u, a)):
        out[q] = v
    return out.reshape(8, -1)


def flowstate_pT(gas: IdealGas, p, T, vel=(0.0, 0.0, 0.0)):
    rho, u, a = gas.from_pT(p, T)
    return np.array([float(rho), vel[0], vel[1], vel[2], p, T, float(u), float(a)])


def sod_2d(ni=256, nj=64, T_right=278.7, nsteps=1000) -> Workload:
    gas = IdealGas()
    vtx = box_vertices(ni, nj, 1, 1.0, 1.0, 0.0, 2)
    xc = cell_centres(vtx, ni, nj, 1, 2)[:, 0]
    left = xc < 0.5
    p = np.where(left, 1.0e5, 1.0e4)
    T = np.where(left, 348.4, 278.7 if T_right is None else T_right)
    rho, u, a = gas.from_pT(p, T)
    z = np.zeros_like(p)
    prim = prim_from(rho, z, z, z, p, T, u, a)
    bc = (BC_SLIP_WALL,) * 6
    inflow = flowstate_pT(gas, 1.0e5, 300.0)
    wl = Workload("sod_2d_%dx%d" % (ni, nj), 2, flux_calculator="ausmdv", nsteps=nsteps, gas=gas)
    wl.blocks.append(BlockSpec(ni, nj, 1, vtx, bc, inflow, prim))
    return wl


def sod_3d_tube(ni=100, nj=2, nk=2, T_right=278.8) -> Workload:
    """examples/eilmer/3D/sod-shock-tube/sg/sod.lua: 1.0 x 0.1 x 0.1, ausmdv."""
    gas = IdealGas()
    vtx = box_vertices(ni, nj, nk, 1.0, 0.1, 0.1, 3)
    xc = cell_centres(vtx, ni, nj, nk, 3)[:, 0]
    left = xc < 0.5
    p = np.where(left, 1.0e5, 1.0e4)
    T = np.where(left, 348.4, T_right)
    rho, u, a = gas.from_pT(p, T)
    z = np.zeros_like(p)
    prim = prim_from(rho, z, z, z, p, T, u, a)
    wl = Workload("sod_3d_tube", 3, flux_calculator="ausmdv", nsteps=600, gas=gas)
    wl.blocks.append(BlockSpec(ni, nj, nk, vtx, (BC_SLIP_WALL,) * 6,
                               flowstate_pT(gas, 1.0e5, 300.0), prim))
    return wl


def _perturbation(centres, seed):
    rng = splitmix64(seed)
    s = np.zeros(centres.shape[0])
    for m in range(1, 9):
        # random direction (uniform on the sphere) and phase for term m
        cz = 2.0 * next(rng) - 1.0
        phi = 2.0 * math.pi * next(rng)
        sz = math.sqrt(max(0.0, 1.0 - cz * cz))
        d = np.array([sz * math.cos(phi), sz * math.sin(phi), cz])
        phase = 2.0 * math.pi * next(rng)
        s += np.sin(2.0 * math.pi * m * (centres @ d) + phase)
    return s


def inflow_3d_block(ni, nj, nk, seed, spacing=None, mach=3.0, p_in=1.0e5, T_in=300.0,
                    gas=None) -> BlockSpec:
    """Mach-3 inflow block: inflow at i-min (west), outflow at i-max (east)."""
    gas = gas or IdealGas()
    if spacing is None:
        lx, ly, lz = 1.0, 1.0, 1.0
    else:
        lx, ly, lz = ni * spacing, nj * spacing, nk * spacing
    vtx = box_vertices(ni, nj, nk, lx, ly, lz, 3, spacing=spacing)
    centres = cell_centres(vtx, ni, nj, nk, 3)
    rho_in, u_in, a_in = gas.from_pT(p_in, T_in)
    vx_in = mach * float(a_in)
    inflow = np.array([float(rho_in), vx_in, 0.0, 0.0, p_in, T_in, float(u_in), float(a_in)])
    rho = float(rho_in) * (1.0 + 0.05 * _perturbation(centres, seed))
    p = np.full_like(rho, p_in)
    T, u, a = gas.from_rhop(rho, p)
    z = np.zeros_like(rho)
    prim = prim_from(rho, np.full_like(rho, vx_in), z, z, p, T, u, a)
    bc = [BC_SLIP_WALL] * 6
    bc[WEST] = BC_INFLOW_SUPERSONIC
    bc[EAST] = BC_OUTFLOW_EXTRAPOLATE
    return BlockSpec(ni, nj, nk, vtx, tuple(bc), inflow, prim)


def skewed_box_3d(ni=12, nj=10, nk=8, flux="ausmdv", amp=0.04, seed=DEFAULT_SEED,
                  reacting=False) -> Workload:
    """A curvilinear 3-D block: the unit box with every vertex displaced by
    smooth sines (amplitude amp in each direction), so no face frame is an
    axis permutation and cell volumes and lengths vary.  Mach-3 inflow at
    i-min, extrapolate outflow at i-max, slip walls elsewhere; the density
    perturbed as in inflow_3d.  reacting: 5-species air at the reacting
    channel's inflow state (Mach 10, 2000 K, 20 kPa) instead of ideal air,
    the density perturbed at constant pressure."""
    vtx = box_vertices(ni, nj, nk, 1.0, 1.0, 1.0, 3)
    x, y, z = vtx[:, 0].copy(), vtx[:, 1].copy(), vtx[:, 2].copy()
    tp = 2.0 * math.pi
    vtx[:, 0] = x + amp * np.sin(tp * y) * np.sin(tp * z)
    vtx[:, 1] = y + amp * np.sin(tp * z) * np.sin(tp * x)
    vtx[:, 2] = z + amp * np.sin(tp * x) * np.sin(tp * y)
    centres = cell_centres(vtx, ni, nj, nk, 3)
    bc = [BC_SLIP_WALL] * 6
    bc[WEST] = BC_INFLOW_SUPERSONIC
    bc[EAST] = BC_OUTFLOW_EXTRAPOLATE
    wl = Workload("skewed_box_3d_%dx%dx%d" % (ni, nj, nk), 3, flux_calculator=flux, nsteps=50)
    if not reacting:
        gas = IdealGas()
        rho_in, u_in, a_in = gas.from_pT(1.0e5, 300.0)
        vx = 3.0 * float(a_in)
        inflow = np.array([float(rho_in), vx, 0.0, 0.0, 1.0e5, 300.0, float(u_in), float(a_in)])
        rho = float(rho_in) * (1.0 + 0.05 * _perturbation(centres, seed))
        p = np.full_like(rho, 1.0e5)
        T, u, a = gas.from_rhop(rho, p)
        z0 = np.zeros_like(rho)
        prim = prim_from(rho, np.full_like(rho, vx), z0, z0, p, T, u, a)
        wl.gas = gas
    else:
        from .thermochem import load_air5
        tc = load_air5()
        massf = (0.767, 0.233, 0.0, 0.0, 0.0)
        rho_in, u_in, a_in = tc.state_pT(2.0e4, 2000.0, massf)
        inflow = np.array([rho_in, 10.0 * a_in, 0.0, 0.0, 2.0e4, 2000.0, u_in, a_in] + list(massf))
        # the stream with the density perturbed at constant pressure (an
        # entropy wave it carries through the block)
        n = ni * nj * nk
        prim = np.repeat(inflow[:, None], n, axis=1).copy()
        pert = 1.0 + 0.05 * _perturbation(centres, seed)
        for q in range(n):
            T = 2000.0 / pert[q]
            rho, u, a = tc.state_pT(2.0e4, T, massf)
            prim[0, q], prim[5, q], prim[6, q], prim[7, q] = rho, T, u, a
        wl.thermochem = tc
    wl.blocks.append(BlockSpec(ni, nj, nk, vtx, tuple(bc), inflow, prim))
    return wl


def inflow_3d(n=256, seed=DEFAULT_SEED, flux="hllc", nsteps=500) -> Workload:
    wl = Workload("inflow_3d_%d^3" % n, 3, flux_calculator=flux, nsteps=nsteps)
    wl.blocks.append(inflow_3d_block(n, n, n, seed))
    return wl


def batched_blocks(nblocks=64, lo=16, hi=96, seed=DEFAULT_SEED, spacing=1.0 / 64.0,
                   nsteps=200, flux="ausmdv") -> Workload:
    """Independent blocks with log-uniform edges; cell spacing 1/64 keeps each
    block's geometry exactly uniform."""
    rng = splitmix64(seed ^ 0xB10C)
    wl = Workload("batched_%d_blocks" % nblocks, 3, flux_calculator=flux, nsteps=nsteps)
    for b in range(nblocks):
        dims = [int(round(math.exp(math.log(lo) + (math.log(hi) - math.log(lo)) * next(rng))))
                for _ in range(3)]
        wl.blocks.append(inflow_3d_block(dims[0], dims[1], dims[2], seed + 1 + b,
                                         spacing=spacing))
    return wl


def reacting_channel(ni=512, nj=256, nsteps=300, length=1.0, height=0.5, ramp_x=0.25,
                     ramp_deg=15.0, mach=10.0, p_in=2000.0, T_in=300.0,
                     massf=(0.767, 0.233, 0.0, 0.0, 0.0)):
    """2-D hypersonic channel with a compression ramp on the lower wall:
    5-species air (N2, O2, NO, N, O), Mach-10 inflow at i-min, extrapolate
    outflow at i-max, slip walls below (ramp) and above.  Grid lines of
    constant i are vertical; the lower wall rises at ramp_deg from ramp_x."""
    from .thermochem import load_air5
    tc = load_air5()
    x = length * (np.arange(ni + 1, dtype=np.float64) / ni)
    yw = np.where(x > ramp_x, (x - ramp_x) * math.tan(math.radians(ramp_deg)), 0.0)
    eta = np.arange(nj + 1, dtype=np.float64) / nj
    Y = yw[None, :] + (height - yw[None, :]) * eta[:, None]
    X = np.broadcast_to(x[None, :], Y.shape)
    vtx = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1).copy()
    rho, u, a = tc.state_pT(p_in, T_in, massf)
    vx = mach * a
    inflow = np.array([rho, vx, 0.0, 0.0, p_in, T_in, u, a] + list(massf))
    n = ni * nj
    prim = np.repeat(inflow[:, None], n, axis=1).copy()
    bc = [BC_SLIP_WALL] * 6
    bc[WEST] = BC_INFLOW_SUPERSONIC
    bc[EAST] = BC_OUTFLOW_EXTRAPOLATE
    wl = Workload("reacting_channel_%dx%d" % (ni, nj), 2, flux_calculator="ausmdv",
                  nsteps=nsteps)
    wl.blocks.append(BlockSpec(ni, nj, 1, vtx, tuple(bc), inflow, prim))
    wl.thermochem = tc
    return wl


def reacting_channel_hot(ni=512, nj=256, nsteps=300):
    """The reacting channel with a high-enthalpy free stream: Mach 10 at
    2000 K and 20 kPa.  Behind the ramp shock the air reaches about 6000 K and
    dissociates within a few flow steps; the 300 K, 2 kPa free stream of
    reacting_channel stays below 1000 K behind the shock, where the chemistry
    is frozen over a flow step."""
    wl = reacting_channel(ni, nj, nsteps, T_in=2000.0, p_in=2.0e4)
    wl.name = "reacting_channel_hot_%dx%d" % (ni, nj)
    return wl


def split_block(b: BlockSpec, dimensions, parts=(2, 1, 1)):
    """Cut a block into parts[0] x parts[1] x parts[2] blocks joined by
    exchange boundaries (the FluidBlockArray split of the reference's prep,
    src/eilmer/prep.lua).  Returns (blocks, connections), connections as
    (block a, face a, block b, face b) with orientation 0, blocks numbered
    i fastest."""
    pi, pj, pk = parts
    if dimensions == 2:
        pk = 1
    nk1 = b.nk + 1 if dimensions == 3 else 1
    v = np.asarray(b.vtx).reshape(nk1, b.nj + 1, b.ni + 1, 3)
    nv = b.prim.shape[0]
    pr = b.prim.reshape(nv, b.nk, b.nj, b.ni)

    def cuts(n, p):
        e = [round(n * q / p) for q in range(p + 1)]
        if any(e[q + 1] - e[q] < 2 for q in range(p)):
            raise ValueError("a part would have fewer than 2 cells")
        return e

    ei, ej = cuts(b.ni, pi), cuts(b.nj, pj)
    ek = cuts(b.nk, pk) if dimensions == 3 else [0, 1]
    blocks, index = [], {}
    for ck in range(pk):
        for cj in range(pj):
            for ci in range(pi):
                i0, i1, j0, j1, k0, k1 = ei[ci], ei[ci + 1], ej[cj], ej[cj + 1], ek[ck], ek[ck + 1]
                kv = slice(k0, k1 + 1) if dimensions == 3 else slice(0, 1)
                vtx = v[kv, j0:j1 + 1, i0:i1 + 1].reshape(-1, 3).copy()
                prim = pr[:, k0:k1, j0:j1, i0:i1].reshape(nv, -1).copy()
                bc = list(b.bc)
                # faces inside the original block become exchange boundaries
                if ci > 0: bc[WEST] = BC_SLIP_WALL
                if ci < pi - 1: bc[EAST] = BC_SLIP_WALL
                if cj > 0: bc[SOUTH] = BC_SLIP_WALL
                if cj < pj - 1: bc[NORTH] = BC_SLIP_WALL
                if ck > 0: bc[BOTTOM] = BC_SLIP_WALL
                if ck < pk - 1: bc[TOP] = BC_SLIP_WALL
                index[(ci, cj, ck)] = len(blocks)
                blocks.append(BlockSpec(i1 - i0, j1 - j0, (k1 - k0) if dimensions == 3 else 1,
                                        vtx, tuple(bc), b.inflow, prim))
    conns = []
    for (ci, cj, ck), a in index.items():
        if ci + 1 < pi:
            conns.append((a, EAST, index[(ci + 1, cj, ck)], WEST))
        if cj + 1 < pj:
            conns.append((a, NORTH, index[(ci, cj + 1, ck)], SOUTH))
        if ck + 1 < pk:
            conns.append((a, TOP, index[(ci, cj, ck + 1)], BOTTOM))
    return blocks, conns


# faces as (index axis, side): axis 0 = i, 1 = j, 2 = k; side 0 = low, 1 = high
FACE_AXIS = {WEST: (0, 0), EAST: (0, 1), SOUTH: (1, 0), NORTH: (1, 1), BOTTOM: (2, 0), TOP: (2, 1)}
AXIS_FACE = {v: f for f, v in FACE_AXIS.items()}


def reindex_block(b: BlockSpec, axes, dimensions):
    """The same block with its index axes turned: new axis a (i', j', k')
    runs along old axis axes[a][0], forwards (axes[a][1] = +1) or backwards
    (-1).  The turn must be proper (determinant +1) so cells stay
    right-handed.  Returns (block, face_map, cell_map): face_map[old face] =
    new face, cell_map(i, j, k) = the new indices of an old cell."""
    nd = 3 if dimensions == 3 else 2
    axes = [tuple(a) for a in axes][:nd]
    if dimensions == 2:
        axes.append((2, 1))
    M = np.zeros((3, 3))
    for a, (o, sgn) in enumerate(axes):
        M[a, o] = sgn
    if sorted(o for o, _ in axes) != [0, 1, 2] or round(np.linalg.det(M)) != 1:
        raise ValueError("not a proper turn of the index axes")
    n_old = (b.ni, b.nj, b.nk)
    n_new = tuple(n_old[o] for o, _ in axes)

    def turn(G, lead):
        # G has axes (lead..., k, j, i, trailing...); numpy axis of index axis a is lead + 2 - a
        order = list(range(lead)) + [lead + 2 - axes[a][0] for a in (2, 1, 0)]
        order += list(range(lead + 3, G.ndim))
        T = np.transpose(G, order)
        for a in range(3):
            if axes[a][1] < 0:
                T = np.flip(T, axis=lead + 2 - a)
        return np.ascontiguousarray(T)

    nk1 = b.nk + 1 if dimensions == 3 else 1
    V = turn(np.asarray(b.vtx).reshape(nk1, b.nj + 1, b.ni + 1, 3), 0)
    nv = b.prim.shape[0]
    P = turn(b.prim.reshape(nv, b.nk, b.nj, b.ni), 1)
    face_map = {}
    for f, (o, side) in FACE_AXIS.items():
        a = next(q for q in range(3) if axes[q][0] == o)
        face_map[f] = AXIS_FACE[(a, side if axes[a][1] > 0 else 1 - side)]
    bc = [0] * 6
    for f in range(6):
        bc[face_map[f]] = b.bc[f]

    def cell_map(i, j, k):
        x = (i, j, k)
        return tuple(x[o] if sgn > 0 else n_old[o] - 1 - x[o] for o, sgn in axes)

    nb = BlockSpec(n_new[0], n_new[1], n_new[2], V.reshape(-1, 3).copy(), tuple(bc), b.inflow,
                   P.reshape(nv, -1).copy())
    return nb, face_map, cell_map


def unturn_prim(prim, b_new: BlockSpec, axes, dimensions):
    """The primitive array of a block made by reindex_block(…, axes, …),
    back in the original block's cell order."""
    nv = prim.shape[0]
    P = prim.reshape(nv, b_new.nk, b_new.nj, b_new.ni)
    nd = 3 if dimensions == 3 else 2
    axes = [tuple(a) for a in axes][:nd]
    if dimensions == 2:
        axes.append((2, 1))
    for a in range(3):
        if axes[a][1] < 0:
            P = np.flip(P, axis=1 + 2 - a)
    # numpy axis 1 + 2 - a of P holds old axis axes[a][0]
    inv = [0, 0, 0]
    for a in range(3):
        inv[2 - axes[a][0]] = 1 + 2 - a
    return np.ascontiguousarray(np.transpose(P, [0] + inv)).reshape(nv, -1)


def join_prims(blocks, b_shape, dimensions, parts=(2, 1, 1)):
    """Reassemble the primitive arrays of split_block's blocks (list of
    (nv, n) arrays) into the original block's (nv, ni*nj*nk) layout."""
    ni, nj, nk = b_shape
    pi, pj, pk = parts
    if dimensions == 2:
        pk = 1
    nv = blocks[0].shape[0]
    out = np.zeros((nv, nk, nj, ni))

    def cuts(n, p):
        return [round(n * q / p) for q in range(p + 1)]

    ei, ej = cuts(ni, pi), cuts(nj, pj)
    ek = cuts(nk, pk) if dimensions == 3 else [0, 1]
    q = 0
    for ck in range(pk):
        for cj in range(pj):
            for ci in range(pi):
                i0, i1, j0, j1, k0, k1 = ei[ci], ei[ci + 1], ej[cj], ej[cj + 1], ek[ck], ek[ck + 1]
                out[:, k0:k1, j0:j1, i0:i1] = blocks[q].reshape(nv, k1 - k0, j1 - j0, i1 - i0)
                q += 1
    return out.reshape(nv, -1)
