"""e4c_dt_allow_noalloc: the time-step control without device allocation.

Some hosts cannot let a library call cudaMalloc inside their time loop (the
GPU's memory belongs to the host's own pool, or a fixed budget); this entry
point keeps its scratch in a fixed device array inside the library.  It must
give exactly what e4c_dt_allow gives, call after call, in both arithmetic
forms, and a warmed-up call must leave the device's free memory unchanged.
This file is collected last so that, should it fail, every other test has
already run.
"""
import ctypes

import numpy as np
import pytest

from eilmer4_b200 import workloads as W

pytestmark = pytest.mark.gpu


def noalloc(L, hs, dt_current, check_cfl):
    from eilmer4_b200 import _lib
    arr = (ctypes.c_int * len(hs))(*hs)
    d, c = ctypes.c_double(), ctypes.c_double()
    rc = L.e4c_dt_allow_noalloc(arr, len(hs), float(dt_current), int(check_cfl),
                                ctypes.byref(d), ctypes.byref(c))
    _lib.check(rc)
    return d.value, c.value


def mixed_workload(precision="fp64"):
    wl = W.Workload("mixed", 3, flux_calculator="hllc")
    # FP64: one block on the fused uniform path, one on the general path; the
    # FP32-flux form takes uniform blocks only, so there both are fused
    wl.blocks.append(W.inflow_3d_block(40, 24, 20, 5, spacing=1.0 / 64.0))
    if precision == "fp64":
        wl.blocks.append(W.inflow_3d_block(20, 12, 10, 7))
    else:
        wl.blocks.append(W.inflow_3d_block(20, 12, 10, 7, spacing=1.0 / 32.0))
    return wl


@pytest.mark.parametrize("precision", ["fp64", "fp32_flux"])
def test_noalloc_dt_matches_dt_allow(e4lib, precision):
    from eilmer4_b200.simcore import Simulation
    with Simulation.from_workload(mixed_workload(precision), precision=precision) as sim:
        hs = [0, 1]
        # two calls in a row, on the uploaded state
        for dt_current, check in ((1.0e-3, 0), (2.0e-7, 1)):
            ref = sim.dt_allow(hs, dt_current, check)
            got = noalloc(sim.L, hs, dt_current, check)
            assert got == ref, (got, ref)
        # and again after some steps (decoded state), single blocks and both
        # (fused blocks are reduced all together)
        sim.run(7)
        subsets = ([0], [1], [1, 0]) if precision == "fp64" else ([0, 1], [1, 0])
        for sub in subsets:
            for call in range(2):
                ref = sim.dt_allow(sub, 3.0e-7, 1)
                got = noalloc(sim.L, sub, 3.0e-7, 1)
                assert got == ref, (sub, call, got, ref)
        assert np.isfinite(got[0]) and got[0] > 0.0


def test_noalloc_calls_leave_free_memory_unchanged(e4lib):
    import torch

    from eilmer4_b200.simcore import Simulation
    with Simulation.from_workload(mixed_workload()) as sim:
        sim.run(3)
        first = noalloc(sim.L, [0, 1], 2.0e-7, 1)
        torch.cuda.mem_get_info(0)       # the runtime's own set-up, outside the window
        sim.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        outs = [noalloc(sim.L, [0, 1], 2.0e-7, 1) for _ in range(5)]
        free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert all(o == first for o in outs)


def test_noalloc_rejects_too_many_blocks(e4lib):
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    wl = W.sod_2d(16, 4)
    with Simulation.from_workload(wl) as sim:
        hs = [0] * 1025
        with pytest.raises(_lib.E4CError) as ei:
            noalloc(sim.L, hs, 1.0e-3, 0)
        assert ei.value.code == _lib.E4C_ERR_ARG
        assert "1024" in str(ei.value)
