"""OutFlowBC_SimpleFlux (bc.lua:1124-1146): extrapolated ghost cells plus
the boundary-face flux of BFE_SimpleOutflowFlux
(bc/boundary_flux_effect.d:367-546), computed from the interior cell after the
convective fluxes.  The oracle against the physics of the boundary; the GPU
against the oracle bit for bit (ideal gas on a Cartesian grid, thermally
perfect air on the curvilinear ramp grid, where the boundary cells' velocities
carry the round-off of the reference's in-place frame round trips)."""
import dataclasses

import numpy as np
import pytest

from eilmer4_b200 import workloads as W


def with_bc(wl, **faces):
    b = wl.blocks[0]
    bc = list(b.bc)
    for name, t in faces.items():
        bc[getattr(W, name.upper())] = t
    wl.blocks[0] = dataclasses.replace(b, bc=tuple(bc))
    return wl


def oracle_run(oracle, wl, nsteps, reacting=False, **kw):
    cfg = oracle.default_config(dimensions=wl.dimensions, n_threads=0, reacting=int(reacting), **kw)
    tc = getattr(wl, "thermochem", None)
    sim = oracle.OracleSim(cfg, tc) if tc is not None else oracle.OracleSim(cfg)
    b = wl.blocks[0]
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    sim.set_flow(0, b.prim)
    assert sim.run(nsteps) == 0
    p, c = sim.get_flow(0)
    return p, c, (sim.time, sim.dt_global, sim.step)


def test_uniform_supersonic_outflow_stays_uniform(oracle):
    """Mach-3 uniform flow leaving through a simple-flux boundary: the
    boundary flux is the flux of the cell state, so nothing changes."""
    wl = with_bc(W.inflow_3d(n=8), east=W.BC_OUTFLOW_SIMPLE_FLUX)
    b = wl.blocks[0]
    prim = np.repeat(np.asarray(b.inflow)[:, None], b.ncell, axis=1).copy()
    wl.blocks[0] = dataclasses.replace(b, prim=prim)
    p, _, _ = oracle_run(oracle, wl, 20, flux_calculator=oracle.FLUX_AUSMDV)
    assert np.allclose(p[:5], prim[:5], rtol=1e-12, atol=1e-9)


def test_inflowing_state_closes_the_face(oracle):
    """Gas drifting west, away from a simple-flux east boundary: the state
    would flow in there, so the face closes (the wall branch of
    BFE_SimpleOutflowFlux) and a rarefaction lowers the density at the east
    end; with extrapolated ghost cells gas flows in and the state stays."""
    out = {}
    for name, east in (("simple", W.BC_OUTFLOW_SIMPLE_FLUX), ("extrap", W.BC_OUTFLOW_EXTRAPOLATE)):
        wl = with_bc(W.sod_2d(40, 4), east=east, west=W.BC_OUTFLOW_EXTRAPOLATE)
        b = wl.blocks[0]
        prim = np.repeat(b.prim[:, -1:], b.ncell, axis=1).copy()
        prim[1] = -50.0
        wl.blocks[0] = dataclasses.replace(b, prim=prim)
        p, _, _ = oracle_run(oracle, wl, 20, flux_calculator=oracle.FLUX_AUSMDV)
        out[name] = p[0].reshape(4, 40)
    rho0 = prim[0, 0]
    assert out["simple"][:, -1].max() < rho0 * (1.0 - 1e-3)
    assert np.abs(out["extrap"] - rho0).max() <= 1e-12 * rho0


def test_supersonic_outflow_equals_the_extrapolated_one(oracle):
    """Through a supersonic outflow the upwind face flux is the cell's own:
    the simple-flux boundary and the extrapolated ghost cells (whose face
    state reconstructs to the cell's) agree to round-off on the perturbed
    Mach-3 block."""
    wl_a = with_bc(W.inflow_3d(n=10), east=W.BC_OUTFLOW_SIMPLE_FLUX)
    wl_b = W.inflow_3d(n=10)
    pa, _, _ = oracle_run(oracle, wl_a, 12, flux_calculator=oracle.FLUX_HLLC)
    pb, _, _ = oracle_run(oracle, wl_b, 12, flux_calculator=oracle.FLUX_HLLC)
    assert not np.array_equal(pa, pb)
    assert np.abs(pa[:5] - pb[:5]).max() <= 1e-12 * np.abs(pb[:5]).max()


# ---------------------------------------------------------------------------
# GPU parity
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sod2d", "inflow3d_hllc", "ramp_tp"])
def test_simple_flux_bitexact(oracle, e4lib, case):
    from eilmer4_b200.simcore import Simulation
    if case == "sod2d":
        wl = with_bc(W.sod_2d(48, 16), east=W.BC_OUTFLOW_SIMPLE_FLUX, north=W.BC_OUTFLOW_SIMPLE_FLUX)
        b = wl.blocks[0]
        prim = b.prim.copy()
        prim[1] = 30.0
        prim[2] = -10.0
        wl.blocks[0] = dataclasses.replace(b, prim=prim)
        kw, n, reacting = {"flux_calculator": oracle.FLUX_AUSMDV}, 40, False
    elif case == "inflow3d_hllc":
        wl = with_bc(W.inflow_3d(n=16), east=W.BC_OUTFLOW_SIMPLE_FLUX,
                     top=W.BC_OUTFLOW_SIMPLE_FLUX)
        kw, n, reacting = {"flux_calculator": oracle.FLUX_HLLC}, 25, False
    else:
        wl = with_bc(W.reacting_channel_hot(ni=48, nj=24), east=W.BC_OUTFLOW_SIMPLE_FLUX)
        kw = {"flux_calculator": oracle.FLUX_AUSMDV,
              "gas_model": oracle.GAS_THERM_PERF_5SP_AIR}
        n, reacting = 30, True
    op, oc, ost = oracle_run(oracle, wl, n, reacting=reacting, **kw)
    with Simulation.from_workload(wl, reacting=reacting) as sim:
        sim.run(n)
        gp, gc = sim.download(0)
        st = sim.state()
    assert (st[0], st[1], st[2]) == ost
    assert np.array_equal(gc, oc)
    assert np.array_equal(gp, op)
