"""OutFlowBC_SimpleExtrapolate with xOrder=1 (ExtrapolateCopy x_order 1,
src/eilmer/bc/ghost_cell_effect/extrapolate_copy.d:206-258 and alike for each
face): linear extrapolation of rho, u, mass fractions and velocity into both
ghost layers, T and p from the rhou update, the ghost's sound speed left at
its initial FlowState's (100 kPa, 300 K).  The oracle keeps a uniform stream
at those conditions exactly uniform; the GPU gives the oracle's bits on an
ideal-gas 2-D case, a curvilinear 3-D block and the thermally perfect ramp
channel."""
import dataclasses

import numpy as np
import pytest

from eilmer4_b200 import workloads as W
from parity import assert_same, compare, run_oracle


def with_bc(wl, **faces):
    b = wl.blocks[0]
    bc = list(b.bc)
    for name, code in faces.items():
        bc[getattr(W, name.upper())] = code
    wl.blocks[0] = dataclasses.replace(b, bc=tuple(bc))
    return wl


LIN = W.BC_OUTFLOW_EXTRAPOLATE_LINEAR


@pytest.mark.parametrize("dimensions", [2, 3])
def test_oracle_uniform_stream_at_300K_as_with_zero_order(oracle, dimensions):
    # 2 q1 - q2 = q1 for equal cells, and the ghosts' stale sound speed is
    # the stream's own at 300 K: the first-order boundary gives the state the
    # zero-order copy gives, to the rounding of the cells' decoded T
    gas = W.IdealGas()
    rho, u, a = gas.from_pT(1.0e5, 300.0)
    n = 12
    if dimensions == 2:
        vtx = W.box_vertices(n, 6, 1, 1.0, 0.5, 0.0, 2)
        nk = 1
    else:
        vtx = W.box_vertices(n, 6, 4, 1.0, 0.5, 0.25, 3)
        nk = 4
    ncell = n * 6 * nk
    state = np.array([float(rho), 2.0 * float(a), 0.0, 0.0, 1.0e5, 300.0, float(u), float(a)])
    prim = np.repeat(state[:, None], ncell, axis=1).copy()
    outs = []
    for east in (W.BC_OUTFLOW_EXTRAPOLATE, LIN):
        bc = [W.BC_SLIP_WALL] * 6
        bc[W.WEST] = W.BC_INFLOW_SUPERSONIC
        bc[W.EAST] = east
        wl = W.Workload("uniform", dimensions, flux_calculator="ausmdv")
        wl.blocks.append(W.BlockSpec(n, 6, nk, vtx, tuple(bc), state, prim))
        rc, st, t, dt, out = run_oracle(oracle, wl, 20)
        assert rc == 0 and st == 20
        outs.append(out[0][0])
    for q in range(8):
        scale = max(np.abs(state[1:4]).max() if q in (1, 2, 3) else abs(state[q]), 1.0)
        assert np.abs(outs[1][q] - outs[0][q]).max() <= 1e-12 * scale, q


def test_oracle_linear_outflow_changes_only_the_cells_near_it(oracle):
    wl0 = W.skewed_box_3d(ni=16, nj=6, nk=6)
    wl1 = with_bc(W.skewed_box_3d(ni=16, nj=6, nk=6), east=LIN)
    _, _, _, _, out0 = run_oracle(oracle, wl0, 2)
    _, _, _, _, out1 = run_oracle(oracle, wl1, 2)
    p0 = out0[0][0].reshape(-1, 6, 6, 16)
    p1 = out1[0][0].reshape(-1, 6, 6, 16)
    diff = np.abs(p1 - p0).max(axis=(0, 1, 2))
    assert diff[-1] > 0.0                     # the boundary cells see the new ghosts
    assert np.all(diff[:16 - 6] == 0.0)       # two steps reach no further than six cells


@pytest.mark.gpu
def test_gpu_linear_outflow_2d_matches_oracle(oracle, e4lib):
    # both ends open: the waves reach them by step 40; near step 100 the
    # extrapolated rarefaction drives a ghost state out of range (the
    # reference's rhou update throws there), so the comparison stops at 60
    wl = with_bc(W.sod_2d(40, 12), east=LIN, west=LIN)
    compare(oracle, wl, 60)


@pytest.mark.gpu
def test_gpu_linear_outflow_curvilinear_3d_matches_oracle(oracle, e4lib):
    wl = with_bc(W.skewed_box_3d(ni=16, nj=8, nk=6), east=LIN, north=LIN)
    compare(oracle, wl, 40)


@pytest.mark.gpu
def test_gpu_linear_outflow_thermally_perfect_matches_oracle(oracle, e4lib):
    from test_gpu_reacting import run_pair
    wl = W.reacting_channel(ni=48, nj=24)
    wl = with_bc(wl, east=LIN)
    (gp, gc), (op, oc) = run_pair(oracle, wl, 30, reacting=True)
    assert_same(gc, oc, "conserved")
    assert_same(gp, op, "primitive")


@pytest.mark.gpu
def test_gpu_linear_outflow_keeps_a_block_off_the_fused_path(e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = with_bc(W.inflow_3d(n=16), east=LIN)
    with Simulation.from_workload(wl) as sim:
        sim.run(2)
        prof = sim.profile(1)
        assert prof["stage"][1] == 0 and prof["flux"][1] > 0
