"""ctypes binding of libe4cuda.so (the C ABI declared in include/e4cuda.h).

The shared library is built in-tree (``python -m eilmer4_b200.build``).  There
is no fallback: if the library is missing, loading fails with an error.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libe4cuda.so")

E4C_OK = 0
E4C_ERR_ARG = -1
E4C_ERR_CUDA = -2
E4C_ERR_UNSUPPORTED = -3
E4C_ERR_BAD_CELLS = -4
E4C_ERR_BAD_MASS = -5
E4C_ERR_THERMO = -6
E4C_ERR_CHEM = -7
E4C_ERR_TIMEOUT = -8
E4C_ERR_STATE = -9

KCLASS = ("dt", "bc", "flux", "update", "stage", "other", "chem", "seed", "chem_work")

ERROR_NAMES = {
    E4C_ERR_ARG: "E4C_ERR_ARG", E4C_ERR_CUDA: "E4C_ERR_CUDA",
    E4C_ERR_UNSUPPORTED: "E4C_ERR_UNSUPPORTED", E4C_ERR_BAD_CELLS: "E4C_ERR_BAD_CELLS",
    E4C_ERR_BAD_MASS: "E4C_ERR_BAD_MASS", E4C_ERR_THERMO: "E4C_ERR_THERMO",
    E4C_ERR_CHEM: "E4C_ERR_CHEM", E4C_ERR_TIMEOUT: "E4C_ERR_TIMEOUT",
    E4C_ERR_STATE: "E4C_ERR_STATE",
}

FLUX = {"ausmdv": 0, "hllc": 1, "hanel": 2, "adaptive_hanel_ausmdv": 3, "adaptive": 3}
UPDATE = {"euler": 0, "pc": 1, "predictor-corrector": 1, "predictor_corrector": 1}
PRECISION = {"fp64": 0, "fp32_flux": 1}
GAS = {"ideal": 0, "therm_perf_5sp_air": 1}


class E4CConfig(ctypes.Structure):
    _fields_ = [
        ("dimensions", ctypes.c_int),
        ("flux_calculator", ctypes.c_int),
        ("interpolation_order", ctypes.c_int),
        ("apply_limiter", ctypes.c_int),
        ("extrema_clipping", ctypes.c_int),
        ("interpolate_in_local_frame", ctypes.c_int),
        ("gasdynamic_update_scheme", ctypes.c_int),
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
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
        ("shear_tolerance", ctypes.c_double),
        ("compression_tolerance", ctypes.c_double),
        ("chem_newton_iterations", ctypes.c_int),
        ("chem_method", ctypes.c_int),
    ]


MAXSP, MAXSEG, MAXR = 8, 4, 8


class E4CThermoChem(ctypes.Structure):
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


class E4CRunInfo(ctypes.Structure):
    _fields_ = [
        ("steps_taken", ctypes.c_int),
        ("time", ctypes.c_double),
        ("dt_global", ctypes.c_double),
        ("status", ctypes.c_int),
        ("status_step", ctypes.c_int),
        ("bad_cells", ctypes.c_int),
    ]


class E4CError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


_lib = None


def load():
    """Load libe4cuda.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m eilmer4_b200.build` "
            "(the CUDA library is required, there is no CPU path)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    i, d, dp, ip = ctypes.c_int, ctypes.c_double, P(ctypes.c_double), P(ctypes.c_int)
    sigs = {
        "e4c_config_default": ([P(E4CConfig)], i),
        "e4c_init": ([P(E4CConfig)], i),
        "e4c_finalize": ([], i),
        "e4c_block_create": ([i, i, i, dp, ip, dp], i),
        "e4c_block_upload": ([i, dp], i),
        "e4c_block_download": ([i, dp, dp], i),
        "e4c_block_upload_async": ([i, dp], i),
        "e4c_block_upload_cons": ([i, dp], i),
        "e4c_block_upload_cons_async": ([i, dp], i),
        "e4c_block_download_async": ([i, dp, dp], i),
        "e4c_transfers_wait": ([], i),
        "e4c_integrate_async": ([i, d], i),
        "e4c_block_get_dt_chem": ([i, dp], i),
        "e4c_connect_blocks": ([i, i, i, i, i], i),
        "e4c_block_set_dt_chem": ([i, dp], i),
        "e4c_dt_allow": ([ip, i, d, i, dp, dp], i),
        "e4c_gasdynamic_step": ([ip, i, d, ip], i),
        "e4c_integrate": ([i, d, P(E4CRunInfo)], i),
        "e4c_sim_state": ([dp, dp, ip], i),
        "e4c_synchronize": ([], i),
        "e4c_last_error": ([ctypes.c_char_p, i], i),
        "e4c_stream": ([], ctypes.c_void_p),
        "e4c_kernel_launches": ([], ctypes.c_longlong),
        "e4c_profile_steps": ([i, dp, ip], i),
        "e4c_set_tile": ([i, i, i], i),
        "e4c_get_tile": ([ip, ip, ip], i),
        "e4c_set_flux_runs": ([i, i], i),
        "e4c_autotune": ([i, ip, ip, ip, dp], i),
        "e4c_dt_allow_noalloc": ([ip, i, d, i, dp, dp], i),
        "e4c_seed_set_wait_limit": ([i], i),
        "e4c_stage": ([ip, i, i, d, ip], i),
        "e4c_connect_remote": ([i, i], i),
        "e4c_face_slab_bytes": ([i, i, P(ctypes.c_longlong)], i),
        "e4c_pack_face": ([i, i, i, ctypes.c_void_p], i),
        "e4c_unpack_face": ([i, i, ctypes.c_void_p], i),
        "e4c_set_thermochem": ([P(E4CThermoChem)], i),
        "e4c_chemistry_step": ([ip, i, d], i),
        "e4c_chemistry_counters": ([P(ctypes.c_longlong), i], i),
        "e4c_seed_collect": ([ip, i, d, ctypes.c_longlong, ctypes.c_ulonglong], i),
        "e4c_seed_dataset": ([P(ctypes.c_longlong)], i),
        "e4c_seed_clear": ([], i),
        "e4c_seed_train": ([i, i, d, ctypes.c_ulonglong, dp], i),
        "e4c_seed_get": ([P(ctypes.c_float), dp], i),
        "e4c_seed_set": ([P(ctypes.c_float), dp], i),
        "e4c_seed_enable": ([i], i),
        "e4c_seed_predict": ([dp, ctypes.c_longlong, dp], i),
        "e4c_seed_loss_grad": ([P(ctypes.c_float), P(ctypes.c_float), i, dp, P(ctypes.c_float)], i),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    load().e4c_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int) -> int:
    if rc < 0:
        raise E4CError(rc, last_error())
    return rc


SEED_NPARAM = 9286
SEED_NNORM = 30


def fptr(a):
    """ctypes float* of a C-contiguous float32 numpy array."""
    assert a.dtype.name == "float32" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), ctypes.POINTER(ctypes.c_double))
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
