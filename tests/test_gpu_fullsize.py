"""Size-independent properties at the full benchmark size (256^3 cells),
where the CPU oracle would take too long to run alongside: a closed box of
slip walls keeps its total mass and energy to round-off, a uniform
supersonic stream through inflow and outflow boundaries stays uniform, and
the FP32-flux form conserves mass and energy as well (its state and
accumulation are FP64)."""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W

pytestmark = pytest.mark.gpu

N = 256


def box(all_walls):
    b = W.inflow_3d_block(N, N, N, 20261203, spacing=1.0 / 64.0)
    if all_walls:
        b.bc = (W.BC_SLIP_WALL,) * 6
    wl = W.Workload("box", 3, flux_calculator="hllc")
    wl.blocks.append(b)
    return wl


@pytest.mark.parametrize("precision", ["fp64", "fp32_flux"])
def test_closed_box_conserves_mass_and_energy(e4lib, precision):
    from eilmer4_b200.simcore import Simulation
    wl = box(all_walls=True)
    with Simulation.from_workload(wl, precision=precision) as sim:
        _, c0 = sim.download(0)
        sim.run(12)
        _, c1 = sim.download(0)
    # every cell has the same volume: the totals are sums over cells.  Each
    # interior face flux enters its two cells with opposite signs, so the
    # totals change only by the rounding of 16.8 M cell updates a step (FP64)
    # or, in the FP32-flux form, by the FP32 rounding of the wall fluxes,
    # whose mass and energy parts are zero in exact arithmetic.
    tol = 1e-10 if precision == "fp64" else 1e-6
    for v, name in ((0, "mass"), (4, "energy")):
        s0 = np.sum(c0[v], dtype=np.float64)
        s1 = np.sum(c1[v], dtype=np.float64)
        assert abs(s1 - s0) <= tol * abs(s0), (name, s0, s1)
    # and something moved: the density perturbation has evolved
    assert np.abs(c1[0] - c0[0]).max() > 1e-6 * np.abs(c0[0]).max()


def test_uniform_stream_stays_uniform(e4lib):
    from eilmer4_b200.simcore import Simulation
    wl = box(all_walls=False)
    b = wl.blocks[0]
    b.prim = np.repeat(np.asarray(b.inflow)[:, None], b.ncell, axis=1).copy()
    with Simulation.from_workload(wl) as sim:
        sim.run(8)
        p, _ = sim.download(0)
    for q in (0, 1, 4, 6):
        assert np.abs(p[q] - b.inflow[q]).max() <= 1e-12 * abs(b.inflow[q]), q
    assert np.abs(p[2]).max() <= 1e-9 and np.abs(p[3]).max() <= 1e-9
