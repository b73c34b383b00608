"""The reference's default flux, adaptive_hanel_ausmdv (fluxcalc.d:824-838,
globalconfig.d:533), and plain Hanel on the fused FP64 path: the stage kernel
runs the shock detector (shockdetectors.d:20-59) on each plane of its ring,
the ghost cells taking the previous stage's flags as the boundary copies
leave them (flowstate.d:177-193), and chooses the flux per face.  A blast in
a box of cubic cells (waves along every axis) matches the oracle bit for
bit, for several tile shapes and across joints, and stays on the fused
path."""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W
from parity import FLUX, assert_same

pytestmark = pytest.mark.gpu


def blast_box(ni=40, nj=24, nk=16):
    gas = W.IdealGas()
    h = 1.0 / 32.0
    vtx = W.box_vertices(ni, nj, nk, 0.0, 0.0, 0.0, 3, spacing=h)
    c = W.cell_centres(vtx, ni, nj, nk, 3)
    r2 = ((c[:, 0] - 0.4 * ni * h) ** 2 + (c[:, 1] - 0.45 * nj * h) ** 2 +
          (c[:, 2] - 0.5 * nk * h) ** 2)
    hot = r2 < (0.2 * nj * h) ** 2
    p = np.where(hot, 5.0e5, 1.0e5)
    T = np.where(hot, 600.0, 300.0)
    rho, u, a = gas.from_pT(p, T)
    z = np.zeros_like(p)
    prim = W.prim_from(rho, z, z, z, p, T, u, a)
    bc = [W.BC_SLIP_WALL] * 6
    bc[W.EAST] = W.BC_OUTFLOW_EXTRAPOLATE
    wl = W.Workload("blast", 3, flux_calculator="adaptive_hanel_ausmdv", gas=gas)
    wl.blocks.append(W.BlockSpec(ni, nj, nk, vtx, tuple(bc), W.flowstate_pT(gas, 1.0e5, 300.0),
                                 prim))
    return wl


def run_both(oracle, wl, blocks, conns, nsteps, tile=None):
    from eilmer4_b200.simcore import Simulation
    cfg = oracle.default_config(dimensions=3, flux_calculator=FLUX[wl.flux_calculator],
                                n_threads=0)
    osim = oracle.OracleSim(cfg)
    for q in blocks:
        hh = osim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
        osim.set_flow(hh, q.prim)
    for cn in conns:
        osim.connect(*cn)
    assert osim.run(nsteps) == 0
    with Simulation({"dimensions": 3, "flux_calculator": wl.flux_calculator}) as sim:
        for q in blocks:
            hh = sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
            sim.upload(hh, q.prim)
        for cn in conns:
            sim.connect(*cn)
        if tile:
            sim.set_tile(*tile)
        sim.run(nsteps)
        prof = sim.profile(1)
        assert prof["stage"][1] > 0 and prof["flux"][1] == 0   # the fused path
        out = [sim.download(hh, want_cons=False)[0] for hh in range(len(blocks))]
        t, dt, st = sim.state()
    assert st == osim.step + 1 and t > osim.time
    return out, [osim.get_flow(hh)[0] for hh in range(len(blocks))]


@pytest.mark.parametrize("tile", [(32, 16, 32), (16, 8, 8), (64, 4, 16)])
def test_fused_adaptive_flux_matches_oracle(oracle, e4lib, tile):
    wl = blast_box()
    b = wl.blocks[0]
    g, o = run_both(oracle, wl, [b], [], 30, tile)
    # the profile step ran one more step on the GPU: compare a fresh run
    from eilmer4_b200.simcore import Simulation
    with Simulation({"dimensions": 3, "flux_calculator": wl.flux_calculator}) as sim:
        sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
        sim.upload(0, b.prim)
        sim.set_tile(*tile)
        sim.run(30)
        gp = sim.download(0, want_cons=False)[0]
    assert_same(gp, o[0], f"adaptive, tile {tile}")


def test_fused_hanel_flux_matches_oracle(oracle, e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = blast_box()
    wl.flux_calculator = "hanel"
    b = wl.blocks[0]
    cfg = oracle.default_config(dimensions=3, flux_calculator=FLUX["hanel"], n_threads=0)
    osim = oracle.OracleSim(cfg)
    osim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    osim.set_flow(0, b.prim)
    assert osim.run(25) == 0
    with Simulation({"dimensions": 3, "flux_calculator": "hanel"}) as sim:
        sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
        sim.upload(0, b.prim)
        sim.run(25)
        gp = sim.download(0, want_cons=False)[0]
        prof = sim.profile(1)
        assert prof["stage"][1] > 0 and prof["flux"][1] == 0
    assert_same(gp, osim.get_flow(0)[0], "hanel")


def test_fused_adaptive_flux_across_joints_matches_oracle(oracle, e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = blast_box()
    b = wl.blocks[0]
    parts = (2, 1, 2)
    blocks, conns = W.split_block(b, 3, parts)
    nsteps = 30
    cfg = oracle.default_config(dimensions=3, flux_calculator=FLUX[wl.flux_calculator],
                                n_threads=0)
    osim = oracle.OracleSim(cfg)
    for q in blocks:
        hh = osim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
        osim.set_flow(hh, q.prim)
    for cn in conns:
        osim.connect(*cn)
    assert osim.run(nsteps) == 0
    with Simulation({"dimensions": 3, "flux_calculator": wl.flux_calculator}) as sim:
        for q in blocks:
            hh = sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
            sim.upload(hh, q.prim)
        for cn in conns:
            sim.connect(*cn)
        sim.run(nsteps)
        out = [sim.download(hh, want_cons=False)[0] for hh in range(len(blocks))]
    for hh, gp in enumerate(out):
        assert_same(gp, osim.get_flow(hh)[0], f"block {hh}")
