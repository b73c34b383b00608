"""The C-ABI library: it loads, exports every entry point include/e4cuda.h
declares, maps the reference config keys, and fails cleanly without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^\s*(?:int|void|double|const char\*)\s+(e4c_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("e4c_init", "e4c_block_create", "e4c_gasdynamic_step", "e4c_integrate",
                 "e4c_dt_allow", "e4c_block_download", "e4c_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(e4lib):
    from eilmer4_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(e4c_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(e4lib, n)


def test_config_default_matches_reference_defaults(e4lib):
    from eilmer4_b200 import _lib
    c = _lib.E4CConfig()
    assert e4lib.e4c_config_default(c) == 0
    assert c.cfl_value == 0.5 and c.dt_init == 1.0e-3 and c.dt_max == 1.0e-3
    assert c.cfl_count == 10 and c.interpolation_order == 2 and c.apply_limiter == 1
    assert c.extrema_clipping == 1 and c.interpolate_in_local_frame == 1
    assert c.gasdynamic_update_scheme == 1 and c.max_invalid_cells == 0
    assert c.flux_calculator == 3 and c.shear_tolerance == 0.2 and c.compression_tolerance == -0.3


def test_config_keys_select_path(e4lib):
    from eilmer4_b200.config import UnsupportedConfig, make_config
    cfg = make_config({"dimensions": 3, "flux_calculator": "hllc"}, {"cfl_value": 0.4})
    assert cfg.flux_calculator == 1 and cfg.cfl_value == 0.4 and cfg.dimensions == 3
    # the reference's default flux calculator is on the path
    cfg = make_config({})
    assert cfg.flux_calculator == 3 and cfg.shear_tolerance == 0.2
    assert cfg.compression_tolerance == -0.3
    with pytest.raises(UnsupportedConfig):
        make_config({"flux_calculator": "efm"})
    with pytest.raises(UnsupportedConfig):
        make_config({"flux_calculator": "ausmdv", "viscous": True})
    with pytest.raises(UnsupportedConfig):
        make_config({"flux_calculator": "ausmdv", "thermo_interpolator": "pT"})


def test_calls_before_init_are_rejected(e4lib):
    from eilmer4_b200 import _lib
    e4lib.e4c_finalize()
    assert e4lib.e4c_integrate(1, 1.0, None) == _lib.E4C_ERR_STATE
    assert "not initialised" in _lib.last_error()
    vtx = np.zeros(12)
    bc = (ctypes.c_int * 6)(0, 0, 0, 0, 0, 0)
    assert e4lib.e4c_block_create(2, 2, 1, _lib.dptr(vtx), bc, _lib.dptr(vtx)) == _lib.E4C_ERR_STATE
    # chemistry and the learned seed refuse as well, without touching a GPU
    h = (ctypes.c_int * 1)(0)
    assert e4lib.e4c_chemistry_step(h, 1, 1e-7) == _lib.E4C_ERR_STATE
    out = (ctypes.c_longlong * 4)()
    assert e4lib.e4c_chemistry_counters(out, 0) == _lib.E4C_ERR_STATE
    assert e4lib.e4c_seed_enable(1) == _lib.E4C_ERR_STATE
    assert e4lib.e4c_seed_train(1, 1024, 1e-3, 1, None) == _lib.E4C_ERR_STATE
    assert e4lib.e4c_seed_collect(h, 1, 1e-7, 10, 1) == _lib.E4C_ERR_STATE
    params = np.zeros(_lib.SEED_NPARAM, dtype=np.float32)
    norm = np.ones(_lib.SEED_NNORM)
    assert e4lib.e4c_seed_set(_lib.fptr(params), _lib.dptr(norm)) == _lib.E4C_ERR_STATE


def test_init_rejects_unsupported_config(e4lib):
    from eilmer4_b200 import _lib
    c = _lib.E4CConfig()
    e4lib.e4c_config_default(c)
    c.flux_calculator = 7
    assert e4lib.e4c_init(c) == _lib.E4C_ERR_UNSUPPORTED
    c.flux_calculator = 0
    c.interpolation_order = 3
    assert e4lib.e4c_init(c) == _lib.E4C_ERR_UNSUPPORTED


def test_init_without_gpu_fails_cleanly(e4lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from eilmer4_b200 import _lib
    c = _lib.E4CConfig()
    e4lib.e4c_config_default(c)
    assert e4lib.e4c_init(c) == _lib.E4C_ERR_CUDA
    assert "CUDA" in _lib.last_error() or "device" in _lib.last_error()


def test_noalloc_source_allocates_nothing():
    """The allocation-free dt control's translation unit calls no allocating
    routine: its only device memory is the file-scope scratch array."""
    src = open(os.path.join(ROOT, "eilmer4_b200", "csrc", "e4c_noalloc.cu")).read()
    code = "\n".join(line.split("//")[0] for line in src.splitlines())
    for banned in ("cudaMalloc", "cudaFree", "dalloc", "dfree", "malloc(", "new ",
                   "cudaMallocAsync", "ensure_"):
        assert banned not in code, banned
    assert "static __device__ __align__(256)" in code
    assert "cudaGetSymbolAddress" in code
