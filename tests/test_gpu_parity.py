"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle.

The plain FP64 path keeps the reference's operation order with no fused
multiply-adds, so the comparison is exact (==) on every primitive and
conserved quantity, on the step count, simulation time and dt_global.
"""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W
from parity import FLUX, assert_same, compare, run_gpu, run_oracle  # noqa: F401

pytestmark = pytest.mark.gpu


def test_sod_2d_small_bitexact(oracle, e4lib):
    compare(oracle, W.sod_2d(64, 16), 120)


def test_sod_tube_3d_reference_deck(oracle, e4lib):
    # examples/eilmer/3D/sod-shock-tube/sg: run to t = 0.6 ms like the deck
    info = compare(oracle, W.sod_3d_tube(), 600, max_time=0.6e-3)
    assert abs(info.steps_taken - 75) < 3


@pytest.mark.parametrize("flux", ["hanel", "adaptive_hanel_ausmdv"])
def test_sod_2d_hanel_and_adaptive_bitexact(oracle, e4lib, flux):
    """Hanel's flux and the reference's default adaptive Hanel/AUSMDV
    switch, with the shock detector run after every stage's ghost cells."""
    wl = W.sod_2d(64, 16)
    wl.flux_calculator = flux
    compare(oracle, wl, 120)


def test_adaptive_3d_inflow_and_reference_deck(oracle, e4lib):
    wl = W.Workload("inflow3d", 3, flux_calculator="adaptive_hanel_ausmdv")
    wl.blocks.append(W.inflow_3d_block(16, 10, 8, seed=3))
    compare(oracle, wl, 30)
    wl = W.sod_3d_tube()
    wl.flux_calculator = "adaptive_hanel_ausmdv"
    info = compare(oracle, wl, 600, max_time=0.6e-3)
    assert abs(info.steps_taken - 75) < 4


def test_inflow_3d_ausmdv_bitexact(oracle, e4lib):
    wl = W.Workload("inflow3d", 3, flux_calculator="ausmdv")
    wl.blocks.append(W.inflow_3d_block(20, 12, 10, seed=7))
    compare(oracle, wl, 40)


def test_inflow_3d_hllc_bitexact(oracle, e4lib):
    wl = W.Workload("inflow3d", 3, flux_calculator="hllc")
    wl.blocks.append(W.inflow_3d_block(16, 14, 12, seed=11))
    compare(oracle, wl, 40)


def test_multiblock_shared_dt(oracle, e4lib):
    wl = W.batched_blocks(nblocks=3, lo=6, hi=12, nsteps=25)
    compare(oracle, wl, 25)


def test_euler_and_first_order(oracle, e4lib):
    # the one-stage Euler update with second-order fluxes is unstable at CFL
    # 0.5 and fails within a few dozen steps (the reference would throw);
    # run it over a few steps, and first order over more
    compare(oracle, W.sod_2d(40, 8), 6, update_scheme=0)
    compare(oracle, W.sod_2d(40, 8), 30, interpolation_order=1)
    compare(oracle, W.sod_2d(40, 8), 30, update_scheme=0, interpolation_order=1)


def test_unstable_euler_fails_like_the_oracle(oracle, e4lib):
    """Both stop with the same error at the same step."""
    from eilmer4_b200 import _lib
    wl = W.sod_2d(40, 8)
    rc, ost, *_ = run_oracle(oracle, wl, 60, update_scheme=0)
    assert rc != 0
    with pytest.raises(_lib.E4CError) as ei:
        run_gpu(wl, 60, gasdynamic_update_scheme="euler")
    assert ei.value.code in (_lib.E4C_ERR_BAD_MASS, _lib.E4C_ERR_BAD_CELLS)
    assert f"at step {ost}" in str(ei.value), (str(ei.value), ost)


def test_without_graphs_matches(oracle, e4lib):
    compare(oracle, W.sod_2d(32, 8), 25, use_graphs=False)


def test_dt_allow_and_single_step_calls(oracle, e4lib):
    """The per-call entry points a D host would use inside its own loop."""
    from eilmer4_b200.simcore import Simulation
    wl = W.sod_2d(32, 8)
    with Simulation.from_workload(wl) as sim:
        dt_allow, cfl_max = sim.dt_allow([0], 1.0e-3, False)
        dt = min(1.0e-3, dt_allow)  # step 0: fmin(dt_init, dt_allow)
        bad = sim.gasdynamic_step([0], dt)
        assert bad == 0
        gp, gc = sim.download(0)
    _, ost, _, odt, oout = run_oracle(oracle, wl, 1)
    assert dt == odt
    assert_same(gc, oout[0][1], "conserved after one step")


def test_bad_cells_reported(oracle, e4lib):
    """A state past the velocity limit (flowstate.d:345-388) makes the stage
    report E4C_ERR_BAD_CELLS, as the reference throws 'Too many bad cells'."""
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    wl = W.sod_2d(16, 4)
    b = wl.blocks[0]
    b.prim[1, 5] = 40000.0
    with Simulation.from_workload(wl) as sim:
        with pytest.raises(_lib.E4CError) as ei:
            sim.run(3)
        assert ei.value.code == _lib.E4C_ERR_BAD_CELLS
    rc, *_ = run_oracle(oracle, wl, 3)
    assert rc == -4


# --- fused uniform path (dyadic Cartesian blocks) ---------------------------

def uniform_block(ni, nj, nk, seed, spacing=1.0 / 64.0, all_walls=False, swirl=False):
    b = W.inflow_3d_block(ni, nj, nk, seed, spacing=spacing)
    if all_walls:
        b.bc = (W.BC_SLIP_WALL,) * 6
    if swirl:
        c = W.cell_centres(b.vtx, ni, nj, nk, 3)
        b.prim[2] = 120.0 * np.sin(9.0 * c[:, 0] + 2.0 * c[:, 2])
        b.prim[3] = -80.0 * np.cos(7.0 * c[:, 1] + 3.0 * c[:, 0])
    return b


def test_fused_path_selected_for_uniform_blocks(e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(40, 24, 20, 3))
    with Simulation.from_workload(wl) as sim:
        sim.run(2)
        prof = sim.profile(2)
    assert prof["stage"][1] == 4 and prof["flux"][1] == 0, prof


def test_fused_fp64_ausmdv_bitexact(oracle, e4lib):
    wl = W.Workload("u", 3, flux_calculator="ausmdv")
    wl.blocks.append(uniform_block(40, 24, 20, 5))
    compare(oracle, wl, 30)


def test_fused_fp64_hllc_partial_tiles(oracle, e4lib):
    # odd extents exercise partial tiles in i, j and k chunks
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(37, 19, 41, 9, spacing=1.0 / 32.0))
    compare(oracle, wl, 25)


def test_fused_slip_walls_every_face(oracle, e4lib):
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(24, 20, 18, 13, all_walls=True, swirl=True))
    compare(oracle, wl, 40)


def test_fused_multiblock(oracle, e4lib):
    wl = W.batched_blocks(nblocks=4, lo=10, hi=28, nsteps=20)
    compare(oracle, wl, 20)


@pytest.mark.parametrize("kc", [3, 5, 64])
def test_fused_one_cta_tile_bitexact(oracle, e4lib, kc):
    """The 32x16 tile (one 16-warp CTA per SM): with partial tiles in i and j,
    k chunks with remainders, slip walls on every face and blocks joined by
    exchange boundaries, the state stays bit for bit the oracle's."""
    from eilmer4_b200.simcore import Simulation
    b = uniform_block(70, 37, 23, 41, all_walls=True, swirl=True)
    nsteps = 12
    blocks, conns = W.split_block(b, 3, (2, 1, 1))
    cfg = oracle.default_config(dimensions=3, n_threads=0, flux_calculator=oracle.FLUX_HLLC)
    osim = oracle.OracleSim(cfg)
    for q in blocks:
        h = osim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
        osim.set_flow(h, q.prim)
    for (a, fa, bb, fb) in conns:
        osim.connect(a, fa, bb, fb)
    assert osim.run(nsteps) == 0
    with Simulation({"dimensions": 3, "flux_calculator": "hllc"}) as sim:
        for q in blocks:
            h = sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
            sim.upload(h, q.prim)
        for (a, fa, bb, fb) in conns:
            sim.connect(a, fa, bb, fb)
        sim.set_tile(32, 16, kc)
        sim.run(nsteps)
        for h in range(len(blocks)):
            gp, gc = sim.download(h)
            op, oc = osim.get_flow(h)
            assert_same(gc, oc, f"conserved, block {h}")
            assert_same(gp, op, f"primitive, block {h}")
        assert sim.state()[2] == osim.step


def test_fused_dt_allow_and_step_calls(oracle, e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(32, 16, 16, 21))
    with Simulation.from_workload(wl) as sim:
        dt_allow, _ = sim.dt_allow([0], 1.0e-3, False)
        dt = min(1.0e-3, dt_allow)
        assert sim.gasdynamic_step([0], dt) == 0
        gp, gc = sim.download(0)
    _, _, _, odt, oout = run_oracle(oracle, wl, 1)
    assert dt == odt
    assert_same(gc, oout[0][1], "conserved after one step")


def test_fp32_flux_form_error_vs_fp64(oracle, e4lib):
    """FP32 reconstruction/flux with FP64 accumulation and decode: relative
    density error against the FP64 oracle stays below 1e-5."""
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(48, 32, 32, 17))
    nsteps = 40
    _, ost, otime, _, oout = run_oracle(oracle, wl, nsteps)
    info, gst, gtime, _, gout = run_gpu(wl, nsteps, precision="fp32_flux")
    assert gst == ost
    assert abs(gtime - otime) / otime < 1e-5
    rho_g, rho_o = gout[0][1][0], oout[0][1][0]
    err = np.max(np.abs(rho_g - rho_o) / np.abs(rho_o))
    assert err < 1.0e-5, err
    E_g, E_o = gout[0][1][4], oout[0][1][4]
    assert np.max(np.abs(E_g - E_o) / np.abs(E_o)) < 1.0e-5


def test_autotune_keeps_state_and_parity(oracle, e4lib):
    """The autotuner's trial steps leave the flow state and clock untouched,
    and every tile shape it may pick gives the same bits."""
    from eilmer4_b200.simcore import Simulation
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(36, 20, 28, 31))
    nsteps = 12
    _, ost, otime, odt, oout = run_oracle(oracle, wl, nsteps)
    with Simulation.from_workload(wl) as sim:
        (ti, tj, kc), ms = sim.autotune(2)
        assert ms > 0.0 and (ti, tj) in ((32, 8), (32, 4), (16, 8), (64, 4), (16, 16), (32, 16))
        t, dt, st = sim.state()
        assert st == 0 and t == 0.0
        sim.run(nsteps)
        gp, gc = sim.download(0)
        assert sim.state()[2] == ost
    assert_same(gc, oout[0][1], "conserved after autotune + run")
    for shape in ((16, 16, 16), (64, 4, 128), (32, 4, 7), (32, 16, 5), (32, 16, 64)):
        with Simulation.from_workload(wl) as sim:
            sim.set_tile(*shape)
            sim.run(nsteps)
            gp, gc = sim.download(0)
        assert_same(gc, oout[0][1], f"conserved with tile {shape}")


def test_async_transfers_match_sync(e4lib):
    """Upload, steps and download through the asynchronous entry points (two
    copy streams, event ordering, steps queued without waiting) give the same
    bits and the same clock as the synchronous ones, call after call."""
    import torch

    from eilmer4_b200.simcore import Simulation
    wl = W.inflow_3d(n=32)
    b = wl.blocks[0]
    n = b.ncell
    host_in = torch.from_numpy(b.prim.copy()).pin_memory()
    outs = []
    for use_async in (False, True):
        with Simulation.from_workload(wl) as sim:
            res = []
            for _ in range(3):
                if use_async:
                    out = torch.empty((8, n), dtype=torch.float64).pin_memory()
                    sim.upload_async(0, host_in)
                    sim.run_async(2)
                    sim.download_async(0, prim=out)
                    sim.wait_transfers()
                    res.append(out.numpy().copy())
                else:
                    sim.upload(0, b.prim)
                    sim.run(2)
                    res.append(sim.download(0, want_cons=False)[0])
            sim.run(0)
            res.append(np.array(sim.state()))
            outs.append(res)
    for a, c in zip(outs[0], outs[1]):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("case", ["fused3d", "fused3d_fp32", "general2d"])
def test_conserved_handoff_continues_bit_for_bit(e4lib, case):
    """A host that takes the conserved state off the device between steps and
    hands it back (e4c_block_upload_cons, decoded on the device as a stage's
    end decodes it) continues exactly as the uninterrupted run: the decoded
    primitive state and U are the run's own, and the next steps give the
    same bits (fused 3-D FP64 and FP32-flux, general 2-D)."""
    from eilmer4_b200.simcore import Simulation
    if case.startswith("fused3d"):
        wl = W.Workload("u", 3, flux_calculator="hllc")
        wl.blocks.append(uniform_block(40, 24, 20, 7))
    else:
        wl = W.sod_2d(48, 16)
    prec = "fp32_flux" if case.endswith("fp32") else "fp64"
    with Simulation.from_workload(wl, precision=prec) as a:
        dt = 1.0e-3
        for q in range(6):
            dta, _ = a.dt_allow([0], dt, q > 0)
            dt = min(dta, 1.0e-3)
            assert a.gasdynamic_step([0], dt) == 0
        pA, cA = a.download(0)
        dt_more = 0.5 * a.dt_allow([0], dt, True)[0]
        for q in range(4):
            assert a.gasdynamic_step([0], dt_more) == 0
        pA2, cA2 = a.download(0)
    with Simulation.from_workload(wl, precision=prec) as b:
        b.upload_cons(0, cA)
        pB, cB = b.download(0)
        assert_same(cB, cA, "conserved after the upload")
        assert_same(pB, pA, "decoded primitive state")
        for q in range(4):
            assert b.gasdynamic_step([0], dt_more) == 0
        pB2, cB2 = b.download(0)
    assert_same(cB2, cA2, "conserved after four more steps")
    assert_same(pB2, pA2, "primitive after four more steps")


def test_conserved_upload_rejects_bad_mass_and_the_mixture(e4lib):
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    wl = W.sod_2d(16, 8)
    with Simulation.from_workload(wl) as sim:
        _, c = sim.download(0)
        c = c.copy()
        c[0, 5] = -1.0
        with pytest.raises(_lib.E4CError) as err:
            sim.upload_cons(0, c)
        assert err.value.code == _lib.E4C_ERR_BAD_MASS
    with Simulation.from_workload(W.reacting_channel(ni=16, nj=8), reacting=True) as sim:
        _, c = sim.download(0)
        with pytest.raises(_lib.E4CError) as err:
            sim.upload_cons(0, c[:5].copy())
        assert err.value.code == _lib.E4C_ERR_UNSUPPORTED


@pytest.mark.parametrize("tile", [(32, 4, 7), (32, 8, 16), (32, 16, 64), (16, 16, 16)])
@pytest.mark.parametrize("case", ["inflow", "walls"])
def test_fp32_flux_tile_shapes_error_vs_fp64(oracle, e4lib, tile, case):
    """The FP32-flux form with each kernel and tile shape it runs: 32-wide
    tiles (edge warps, per-cell reconstruction, ghost cells copied with
    cp.async and fixed up) and the 16x16 tile of the per-face kernel, on a
    block with partial tiles in i, j and k: Mach-3 inflow and outflow with
    slip walls, or slip walls on every face around a swirling state.  The
    relative density and energy differences from the FP64 oracle stay below
    1e-5, and the steps and clock agree."""
    from eilmer4_b200.simcore import Simulation
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(uniform_block(45, 27, 21, 23, all_walls=(case == "walls"),
                                   swirl=(case == "walls")))
    nsteps = 30
    _, ost, otime, _, oout = run_oracle(oracle, wl, nsteps)
    with Simulation.from_workload(wl, precision="fp32_flux") as sim:
        sim.set_tile(*tile)
        sim.run(nsteps)
        gp, gc = sim.download(0)
        t, _, st = sim.state()
    assert st == ost and abs(t - otime) / otime < 1e-5
    for v in (0, 4):
        err = np.max(np.abs(gc[v] - oout[0][1][v]) / np.abs(oout[0][1][v]))
        assert err < 1.0e-5, (v, err)
