"""Configuration keys of the explicit structured-block path.

Mirrors what ``read_config_file`` and ``read_control_file``
(src/eilmer/globalconfig.d:1189, :1741) take from the JSON files that
``prep.lua`` writes (``write_config_file`` prep.lua:1752,
``write_control_file`` prep.lua:1685), for the keys that select this path.
Defaults are those of GlobalConfig (globalconfig.d:440-734).  A value
outside the implemented path raises ``UnsupportedConfig`` (the library
itself answers E4C_ERR_UNSUPPORTED); there is no CPU fallback.
"""
from __future__ import annotations

import json

from . import _lib


class UnsupportedConfig(ValueError):
    pass


CONFIG_DEFAULTS = {
    "dimensions": 2,
    "flux_calculator": "adaptive_hanel_ausmdv",   # globalconfig.d:533
    "interpolation_order": 2,                     # :544
    "apply_limiter": True,                        # :567
    "extrema_clipping": True,                     # :568
    "interpolate_in_local_frame": True,           # :569
    "thermo_interpolator": "rhou",                # :565
    "gasdynamic_update_scheme": "predictor-corrector",
    "max_invalid_cells": 0,                       # :519
    "reacting": False,
    "T_frozen": 300.0,                            # :692
    "n_ghost_cell_layers": 2,
    "axisymmetric": False,
    "viscous": False,
    "grid_motion": "none",
    "with_local_time_stepping": False,
    "with_super_time_stepping": False,
    "high_order_flux_calculator": False,
    "strang_splitting": "full_T_full_R",          # :456
    "shear_tolerance": 0.20,                      # :585
    "compression_tolerance": -0.30,               # :600
    "chem_newton_iterations": 12,                 # whole-interval point-implicit step
    # chemistry method: "point-implicit" (this library's update, opCall's
    # sub-cycling as its recovery) or "rkf" (the reference's default
    # odeStep.method, chemistry_update.d:75-80 with prep_chem.lua:51)
    "chem_method": "point-implicit",
}

CHEM_METHOD = {"point-implicit": 0, "rkf": 1}

CONTROL_DEFAULTS = {
    "dt_init": 1.0e-3,    # globalconfig.d:726
    "dt_max": 1.0e-3,     # :727
    "cfl_value": 0.5,     # :728
    "cfl_count": 10,      # :733
    "max_step": 100,
    "max_time": 1.0e-3,
    "fixed_time_step": False,
    "stringent_cfl": False,
}


def make_config(config: dict | None = None, control: dict | None = None, *,
                precision: str = "fp64", device: int = 0, use_graphs: bool = True,
                gas: dict | None = None) -> _lib.E4CConfig:
    """Build an e4c_config from reference-style config/control dictionaries."""
    c = dict(CONFIG_DEFAULTS)
    c.update(config or {})
    k = dict(CONTROL_DEFAULTS)
    k.update(control or {})
    g = {"model": "ideal", "mMass": 0.02896, "gamma": 1.4}
    g.update(gas or {})

    def need(cond, msg):
        if not cond:
            raise UnsupportedConfig(msg)

    need(c["dimensions"] in (2, 3), "dimensions must be 2 or 3")
    need(c["flux_calculator"] in _lib.FLUX,
         f"flux_calculator {c['flux_calculator']!r} is not on this path "
         "(ausmdv, hllc, hanel, adaptive_hanel_ausmdv)")
    need(c["interpolation_order"] in (1, 2), "interpolation_order must be 1 or 2")
    need(c["thermo_interpolator"] == "rhou", "thermo_interpolator must be rhou")
    need(c["gasdynamic_update_scheme"] in _lib.UPDATE,
         "gasdynamic_update_scheme must be euler or predictor-corrector")
    need(c["n_ghost_cell_layers"] == 2, "n_ghost_cell_layers must be 2")
    for flag in ("axisymmetric", "viscous", "with_local_time_stepping",
                 "with_super_time_stepping", "high_order_flux_calculator"):
        need(not c[flag], f"{flag} is not on this path")
    need(c["grid_motion"] == "none", "moving grids are not on this path")
    need(not k["stringent_cfl"], "stringent_cfl is not on this path")
    need(not k["fixed_time_step"], "fixed_time_step is not on this path")
    need(precision in _lib.PRECISION, "precision must be fp64 or fp32_flux")
    need(g["model"] in _lib.GAS, f"gas model {g['model']!r} is not on this path")

    L = _lib.load()
    cfg = _lib.E4CConfig()
    L.e4c_config_default(cfg)
    cfg.dimensions = int(c["dimensions"])
    cfg.flux_calculator = _lib.FLUX[c["flux_calculator"]]
    cfg.interpolation_order = int(c["interpolation_order"])
    cfg.apply_limiter = int(bool(c["apply_limiter"]))
    cfg.extrema_clipping = int(bool(c["extrema_clipping"]))
    cfg.interpolate_in_local_frame = int(bool(c["interpolate_in_local_frame"]))
    cfg.gasdynamic_update_scheme = _lib.UPDATE[c["gasdynamic_update_scheme"]]
    cfg.cfl_value = float(k["cfl_value"])
    cfg.dt_init = float(k["dt_init"])
    cfg.dt_max = float(k["dt_max"])
    cfg.cfl_count = int(k["cfl_count"])
    cfg.max_invalid_cells = int(c["max_invalid_cells"])
    cfg.gas_model = _lib.GAS[g["model"]]
    cfg.ideal_mol_mass = float(g["mMass"])
    cfg.ideal_gamma = float(g["gamma"])
    cfg.reacting = int(bool(c["reacting"]))
    cfg.T_frozen = float(c["T_frozen"])
    cfg.precision = _lib.PRECISION[precision]
    cfg.device = int(device)
    cfg.use_graphs = int(bool(use_graphs))
    cfg.shear_tolerance = float(c["shear_tolerance"])
    cfg.compression_tolerance = float(c["compression_tolerance"])
    cfg.chem_newton_iterations = int(c["chem_newton_iterations"])
    if c["chem_method"] not in CHEM_METHOD:
        raise UnsupportedConfig(f"chem_method {c['chem_method']!r} is not on this path")
    cfg.chem_method = CHEM_METHOD[c["chem_method"]]
    return cfg


def load_job_files(config_path: str, control_path: str):
    """Read the config/<job>.config and .control JSON files prep.lua writes."""
    with open(config_path) as f:
        config = json.load(f)
    with open(control_path) as f:
        control = json.load(f)
    return config, control
