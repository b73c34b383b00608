"""ctypes wrapper of the CPU FP64 oracle (oracle/_build/libe4oracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's explicit
structured-block update in plain C++ (see e4_oracle.cpp for the file:line map
into the reference).  Only tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import this module; the product package never
does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libe4oracle.so")

BC_SLIP_WALL = 0
BC_INFLOW_SUPERSONIC = 1
BC_OUTFLOW_EXTRAPOLATE = 2
BC_EXCHANGE = 3
BC_OUTFLOW_SIMPLE_FLUX = 4
FLUX_AUSMDV = 0
FLUX_HLLC = 1
FLUX_HANEL = 2
FLUX_ADAPTIVE_HANEL_AUSMDV = 3
UPDATE_EULER = 0
UPDATE_PC = 1
GAS_IDEAL = 0
GAS_THERM_PERF_5SP_AIR = 1


class Config(ctypes.Structure):
    _fields_ = [
        ("dimensions", ctypes.c_int),
        ("flux_calculator", ctypes.c_int),
        ("interpolation_order", ctypes.c_int),
        ("apply_limiter", ctypes.c_int),
        ("extrema_clipping", ctypes.c_int),
        ("interpolate_in_local_frame", ctypes.c_int),
        ("update_scheme", ctypes.c_int),
        ("cfl_value", ctypes.c_double),
        ("dt_init", ctypes.c_double),
        ("dt_max", ctypes.c_double),
        ("cfl_count", ctypes.c_int),
        ("max_invalid_cells", ctypes.c_int),
        ("gas_model", ctypes.c_int),
        ("ideal_mol_mass", ctypes.c_double),
        ("ideal_gamma", ctypes.c_double),
        ("reacting", ctypes.c_int),
        ("T_frozen", ctypes.c_double),
        ("n_threads", ctypes.c_int),
        ("shear_tolerance", ctypes.c_double),
        ("compression_tolerance", ctypes.c_double),
        ("chem_newton_iterations", ctypes.c_int),
        ("chem_method", ctypes.c_int),
    ]


MAXSP, MAXSEG, MAXR = 8, 4, 8


class ThermoChem(ctypes.Structure):
    _fields_ = [
        ("nsp", ctypes.c_int),
        ("M", ctypes.c_double * MAXSP),
        ("nseg", ctypes.c_int * MAXSP),
        ("T_break", (ctypes.c_double * (MAXSEG + 1)) * MAXSP),
        ("T_blend", (ctypes.c_double * MAXSEG) * MAXSP),
        ("coeffs", ((ctypes.c_double * 9) * MAXSEG) * MAXSP),
        ("nreac", ctypes.c_int),
        ("A_f", ctypes.c_double * MAXR), ("n_f", ctypes.c_double * MAXR),
        ("C_f", ctypes.c_double * MAXR),
        ("A_b", ctypes.c_double * MAXR), ("n_b", ctypes.c_double * MAXR),
        ("C_b", ctypes.c_double * MAXR),
        ("nu_r", (ctypes.c_int * MAXSP) * MAXR),
        ("nu_p", (ctypes.c_int * MAXSP) * MAXR),
        ("third_body", ctypes.c_int * MAXR),
        ("eff", (ctypes.c_double * MAXSP) * MAXR),
        ("T_lower", ctypes.c_double),
        ("T_upper", ctypes.c_double),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, no GPU needed; make rebuilds
    only when a source is newer than the library)."""
    if force and os.path.exists(_LIB_PATH):
        os.remove(_LIB_PATH)
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None
_lib_libm = None


def lib(libm: bool = False):
    """The oracle library; libm=True: its build with the C library's exp, log
    and pow in place of the portable restatements the GPU shares."""
    global _lib, _lib_libm
    if libm:
        if _lib_libm is None:
            build()
            _lib_libm = _declare(ctypes.CDLL(os.path.join(_HERE, "_build", "libe4oracle_libm.so")))
        return _lib_libm
    if _lib is None:
        _lib = _declare(ctypes.CDLL(build()))
    return _lib


def _declare(L):
    """Argument and result types of the oracle's C functions."""
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    P = ctypes.POINTER
    L.e4o_default_config.argtypes = [P(Config)]
    L.e4o_sim_new.argtypes = [P(Config)]
    L.e4o_sim_new.restype = vp
    L.e4o_sim_free.argtypes = [vp]
    L.e4o_add_block.argtypes = [vp, ip, ip, ip, P(dp), P(ip), P(dp)]
    L.e4o_add_block.restype = ip
    L.e4o_set_flow.argtypes = [vp, ip, P(dp)]
    L.e4o_connect_blocks.argtypes = [vp, ip, ip, ip, ip, ip]
    L.e4o_ffc_map.argtypes = [ip, ip, ip, ip, ip, ip, ip, ip, ip, P(ip)]
    L.e4o_ffc_map.restype = None
    L.e4o_get_flow.argtypes = [vp, ip, P(dp), P(dp)]
    L.e4o_get_cell_geometry.argtypes = [vp, ip, P(dp)]
    L.e4o_run.argtypes = [vp, ip, dp]
    L.e4o_time.argtypes = [vp]
    L.e4o_time.restype = dp
    L.e4o_dt_global.argtypes = [vp]
    L.e4o_dt_global.restype = dp
    L.e4o_step_count.argtypes = [vp]
    L.e4o_last_bad_cells.argtypes = [vp]
    L.e4o_last_error.argtypes = [vp]
    L.e4o_last_error.restype = ctypes.c_char_p
    L.e4o_ideal_gas_pT.argtypes = [dp, dp, dp, dp, P(dp), P(dp), P(dp)]
    L.e4o_set_thermochem.argtypes = [vp, P(ThermoChem)]
    L.e4o_tp_update.argtypes = [P(ThermoChem), ip, P(dp), P(dp), P(dp), P(dp), P(dp), P(dp)]
    L.e4o_chem_cell.argtypes = [P(ThermoChem), dp, dp, dp, P(dp), P(dp), P(dp), P(dp), P(dp)]
    L.e4o_chem_update.argtypes = [P(ThermoChem), dp, dp, dp, P(dp), P(dp)]
    L.e4o_rates.argtypes = [P(ThermoChem), dp, P(dp), P(dp), P(dp)]
    L.e4o_set_chem_newton_iterations.argtypes = [ip]
    L.e4o_newton_test.argtypes = [ip, P(dp)]
    L.e4o_gpuchem_prepare.argtypes = [P(ThermoChem), ip] + [P(dp)] * 8
    L.e4o_gpuchem_finish.argtypes = [P(ThermoChem), ip] + [P(dp)] * 8
    L.e4o_set_chem_method.argtypes = [ip]
    L.e4o_rkf_step.argtypes = [P(ThermoChem), dp, P(dp), dp, P(dp), P(dp)]
    L.e4o_set_remote.argtypes = [vp, ip, ip]
    L.e4o_face_values.argtypes = [vp, ip, ip]
    L.e4o_pack_face.argtypes = [vp, ip, ip, P(dp)]
    L.e4o_unpack_face.argtypes = [vp, ip, ip, P(dp)]
    L.e4o_dt_allow.argtypes = [vp, dp, ip, P(dp), P(dp)]
    L.e4o_set_dt_global.argtypes = [vp, dp]
    L.e4o_set_dt_global.restype = None
    L.e4o_stage.argtypes = [vp, ip]
    return L


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def default_config(**kw) -> Config:
    c = Config()
    lib().e4o_default_config(ctypes.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def ffc_map(fa, fb, r, p, q, depth, ni, nj, nk):
    """The partner cell (active indices) filling ghost layer `depth` behind
    cell (p, q) of face fa, for a joint with face fb at orientation r."""
    out = (ctypes.c_int * 3)()
    lib().e4o_ffc_map(fa, fb, r, p, q, depth, ni, nj, nk, out)
    return tuple(out)


class OracleSim:
    """One simulation (a set of blocks sharing dt_global), as simcore.d runs it."""

    def __init__(self, cfg: Config, thermochem=None, libm: bool = False):
        self.cfg = cfg
        self._L = lib(libm)
        self._h = self._L.e4o_sim_new(ctypes.byref(cfg))
        self.blocks = []
        self.nsp = 5 if cfg.gas_model == GAS_THERM_PERF_5SP_AIR else 1
        if thermochem is not None:
            self._tc = thermochem.fill(ThermoChem())
            self._L.e4o_set_thermochem(self._h, ctypes.byref(self._tc))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.e4o_sim_free(h)
            self._h = None

    def add_block(self, ni, nj, nk, vtx, bc, inflow):
        vtx = np.ascontiguousarray(vtx, dtype=np.float64)
        inflow = np.ascontiguousarray(inflow, dtype=np.float64)
        bca = (ctypes.c_int * 6)(*bc)
        b = self._L.e4o_add_block(self._h, ni, nj, nk, _dptr(vtx), bca, _dptr(inflow))
        if b < 0:
            raise RuntimeError(f"e4o_add_block failed: {b}")
        self.blocks.append((ni, nj, nk if self.cfg.dimensions == 3 else 1))
        return b

    def connect(self, a, fa, b, fb, orientation=0):
        rc = self._L.e4o_connect_blocks(self._h, a, fa, b, fb, orientation)
        if rc != 0:
            raise RuntimeError(f"e4o_connect_blocks failed: {rc}")

    def nvar_prim(self):
        return 8 + (self.nsp if self.nsp > 1 else 0)

    def nvar_cons(self):
        return 5 + (self.nsp if self.nsp > 1 else 0)

    def set_flow(self, b, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        rc = self._L.e4o_set_flow(self._h, b, _dptr(prim))
        if rc != 0:
            raise RuntimeError(f"e4o_set_flow failed: {rc}")

    def get_flow(self, b):
        ni, nj, nk = self.blocks[b]
        n = ni * nj * nk
        prim = np.zeros((self.nvar_prim(), n))
        cons = np.zeros((self.nvar_cons(), n))
        self._L.e4o_get_flow(self._h, b, _dptr(prim), _dptr(cons))
        return prim, cons

    def geometry(self, b):
        ni, nj, nk = self.blocks[b]
        n = ni * nj * nk
        nf = (ni + 1) * nj * nk + ni * (nj + 1) * nk
        if self.cfg.dimensions == 3:
            nf += ni * nj * (nk + 1)
        out = np.zeros(4 * n + 10 * nf)
        self._L.e4o_get_cell_geometry(self._h, b, _dptr(out))
        return out[: 4 * n].reshape(4, n), out[4 * n:].reshape(nf, 10)

    def run(self, nsteps, max_time=1.0e300):
        rc = self._L.e4o_run(self._h, nsteps, max_time)
        return rc

    # -- faces joined to blocks of another rank --------------------------------
    def set_remote(self, b, face):
        rc = self._L.e4o_set_remote(self._h, b, face)
        if rc != 0:
            raise RuntimeError(f"e4o_set_remote failed: {rc}")

    def pack_face(self, b, face):
        out = np.zeros(self._L.e4o_face_values(self._h, b, face))
        rc = self._L.e4o_pack_face(self._h, b, face, _dptr(out))
        if rc != 0:
            raise RuntimeError(f"e4o_pack_face failed: {rc}")
        return out

    def unpack_face(self, b, face, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        rc = self._L.e4o_unpack_face(self._h, b, face, _dptr(v))
        if rc != 0:
            raise RuntimeError(f"e4o_unpack_face failed: {rc}")

    def dt_allow(self, dt_current, check_cfl):
        d, c = ctypes.c_double(), ctypes.c_double()
        self._L.e4o_dt_allow(self._h, dt_current, int(check_cfl), ctypes.byref(d),
                             ctypes.byref(c))
        return d.value, c.value

    def set_dt_global(self, dt):
        self._L.e4o_set_dt_global(self._h, dt)

    def stage(self, stage):
        return self._L.e4o_stage(self._h, stage)

    @property
    def time(self):
        return self._L.e4o_time(self._h)

    @property
    def dt_global(self):
        return self._L.e4o_dt_global(self._h)

    @property
    def step(self):
        return self._L.e4o_step_count(self._h)

    @property
    def last_bad_cells(self):
        return self._L.e4o_last_bad_cells(self._h)


def ideal_gas_pT(mol_mass, gamma, p, T):
    rho, u, a = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    rc = lib().e4o_ideal_gas_pT(mol_mass, gamma, p, T, ctypes.byref(rho), ctypes.byref(u),
                                ctypes.byref(a))
    if rc != 0:
        raise ValueError("bad state")
    return rho.value, u.value, a.value


def tp_update(thermochem, mode, massf, rho=0.0, p=0.0, T=0.0, u=0.0):
    """Thermally perfect state update: mode 0 (p,T), 1 (rho,u; T = guess), 2 (rho,T)."""
    tc = thermochem.fill(ThermoChem())
    mf = np.ascontiguousarray(massf, dtype=np.float64)
    r, pp, TT, uu, a = (ctypes.c_double(rho), ctypes.c_double(p), ctypes.c_double(T),
                        ctypes.c_double(u), ctypes.c_double())
    rc = lib().e4o_tp_update(ctypes.byref(tc), mode, _dptr(mf), ctypes.byref(r), ctypes.byref(pp),
                             ctypes.byref(TT), ctypes.byref(uu), ctypes.byref(a))
    if rc != 0:
        raise ValueError(f"tp_update failed: {rc}")
    return {"rho": r.value, "p": pp.value, "T": TT.value, "u": uu.value, "a": a.value}


def chem_cell(thermochem, T_frozen, dt, rho, T, u, p, massf, dt_chem=-1.0):
    """One chemistry update of one cell (thermochemical_increment)."""
    tc = thermochem.fill(ThermoChem())
    mf = np.array(massf, dtype=np.float64)
    TT, uu, pp, dc = (ctypes.c_double(T), ctypes.c_double(u), ctypes.c_double(p),
                      ctypes.c_double(dt_chem))
    rc = lib().e4o_chem_cell(ctypes.byref(tc), T_frozen, dt, rho, ctypes.byref(TT),
                             ctypes.byref(uu), ctypes.byref(pp), _dptr(mf), ctypes.byref(dc))
    return rc, {"T": TT.value, "u": uu.value, "p": pp.value, "massf": mf, "dt_chem": dc.value}


def chem_update(thermochem, dt, rho, T, massf, dt_chem=-1.0):
    """The chemistry update alone at constant rho and T (no temperature update)."""
    tc = thermochem.fill(ThermoChem())
    mf = np.array(massf, dtype=np.float64)
    dc = ctypes.c_double(dt_chem)
    rc = lib().e4o_chem_update(ctypes.byref(tc), dt, rho, T, _dptr(mf), ctypes.byref(dc))
    return rc, mf


def gpuchem_prepare(thermochem, rho, T, massf, dt_chem):
    """Inputs of the reference's GPU chemistry kernel for n cells
    (GPUChem.prepareDataForGPU): conc (nsp, n), kf, kb (nreac, n), h (n,)."""
    tc = thermochem.fill(ThermoChem())
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    n = rho.size
    T = np.ascontiguousarray(T, dtype=np.float64)
    mf = np.ascontiguousarray(massf, dtype=np.float64).reshape(thermochem.nsp, n)
    dc = np.ascontiguousarray(dt_chem, dtype=np.float64)
    conc = np.zeros((thermochem.nsp, n))
    kf = np.zeros((thermochem.nreac, n))
    kb = np.zeros((thermochem.nreac, n))
    h = np.zeros(n)
    rc = lib().e4o_gpuchem_prepare(ctypes.byref(tc), n, _dptr(rho), _dptr(T), _dptr(mf),
                                   _dptr(dc), _dptr(conc), _dptr(kf), _dptr(kb), _dptr(h))
    if rc != 0:
        raise ValueError(f"gpuchem_prepare failed: {rc}")
    return conc, kf, kb, h


def gpuchem_finish(thermochem, conc, h, rho, T, u, p):
    """The cell loop after the reference's GPU chemistry kernel: massf (nsp, n),
    T, u, p and dt_chem (n,) as GPUChem.thermochemical_increment leaves them,
    and the return code (0, or the thermo error if a temperature solve failed)."""
    tc = thermochem.fill(ThermoChem())
    conc = np.ascontiguousarray(conc, dtype=np.float64)
    n = conc.shape[1]
    h = np.ascontiguousarray(h, dtype=np.float64)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    T = np.array(T, dtype=np.float64)
    u = np.array(u, dtype=np.float64)
    p = np.array(p, dtype=np.float64)
    mf = np.zeros((thermochem.nsp, n))
    dc = np.zeros(n)
    rc = lib().e4o_gpuchem_finish(ctypes.byref(tc), n, _dptr(conc), _dptr(h), _dptr(rho),
                                  _dptr(T), _dptr(u), _dptr(p), _dptr(mf), _dptr(dc))
    return rc, {"massf": mf, "T": T, "u": u, "p": p, "dt_chem": dc}


def rates(thermochem, T, conc):
    """Production and loss rates (q, L) of every species at T and conc."""
    tc = thermochem.fill(ThermoChem())
    c = np.ascontiguousarray(conc, dtype=np.float64)
    q = np.zeros(thermochem.nsp)
    L = np.zeros(thermochem.nsp)
    lib().e4o_rates(ctypes.byref(tc), float(T), _dptr(c), _dptr(q), _dptr(L))
    return q, L


def newton_test(which):
    """Root of the reference's Newton unit-test problem `which` (0 or 1)."""
    r = ctypes.c_double()
    rc = lib().e4o_newton_test(int(which), ctypes.byref(r))
    return rc, r.value


def set_chem_newton_iterations(n):
    """Newton iterations of the whole-interval step for chem_cell / chem_update."""
    lib().e4o_set_chem_newton_iterations(int(n))


def set_chem_method(m):
    """Chemistry method of the single-cell entry points: 0 point-implicit
    (with opCall's sub-cycled recovery), 1 the reference's RKF (opCall with
    RKF sub-steps)."""
    rc = lib().e4o_set_chem_method(int(m))
    if rc != 0:
        raise ValueError("unknown chemistry method")


def rkf_step(thermochem, T, conc0, h):
    """One RKF step of the rate equations at T from conc0 over h:
    (succeeded, concOut, suggested next step)."""
    tc = thermochem.fill(ThermoChem())
    c0 = np.ascontiguousarray(conc0, dtype=np.float64)
    out = np.zeros_like(c0)
    hs = ctypes.c_double()
    rc = lib().e4o_rkf_step(ctypes.byref(tc), float(T), _dptr(c0), float(h), _dptr(out),
                            ctypes.byref(hs))
    return rc == 0, out, hs.value
