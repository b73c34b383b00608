"""Turned joints on the GPU: a block cut in two, the second part's index
axes turned so the cut joins the first part's east face to each face of the
second part at each orientation (every face-pair and orientation case of
GhostCellFullFaceCopy.set_up_cell_mapping, src/eilmer/bc/ghost_cell_effect/
full_face_copy.d:142-1083, from an east face).  The library gives the
oracle's bits, and the uncut block's state to rounding."""
import numpy as np
import pytest

from eilmer4_b200 import workloads as W
import joints
from test_ffc_map import oracle_run


def gpu_run(dimensions, blocks, joint, nsteps):
    from eilmer4_b200.simcore import Simulation
    with Simulation({"dimensions": dimensions, "flux_calculator": "ausmdv"}) as sim:
        for q in blocks:
            h = sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
            sim.upload(h, q.prim)
        if joint is not None:
            sim.connect(*joint)
        sim.run(nsteps)
        prims = [sim.download(h, want_cons=False)[0] for h in range(len(blocks))]
        return prims, sim.state()


CASES = [(2, t) for t in range(4)] + [(3, t) for t in range(24)]


@pytest.mark.gpu
@pytest.mark.parametrize("dimensions,turn", CASES)
def test_gpu_turned_joint_matches_oracle_and_uncut_block(oracle, e4lib, dimensions, turn):
    b = joints.cubic_block(12, 8, 6, 5, dimensions)
    axes = joints.proper_turns(dimensions)[turn]
    blocks, joint, unturn = joints.turned_domain(oracle, b, axes, dimensions)
    nsteps = 10
    prims, st = gpu_run(dimensions, blocks, joint, nsteps)
    oprims, ost = oracle_run(oracle, dimensions, blocks, joint, nsteps)
    for gp, op in zip(prims, oprims):
        assert np.array_equal(gp, op), joint
    assert st[2] == ost[1] == nsteps and st[0] == ost[0]
    (uncut,), _ = gpu_run(dimensions, [b], None, nsteps)
    joined = unturn(prims)
    for q in range(uncut.shape[0]):
        scale = np.abs(uncut[1:4]).max() if q in (1, 2, 3) else np.abs(uncut[q]).max()
        assert np.abs(joined[q] - uncut[q]).max() <= 1e-11 * scale, (q, joint)


@pytest.mark.gpu
def test_gpu_connect_checks_the_joint(e4lib):
    from eilmer4_b200 import _lib
    from eilmer4_b200.simcore import Simulation
    b = W.inflow_3d_block(8, 6, 4, 1, spacing=1.0 / 16.0)
    blocks, _ = W.split_block(b, 3, (2, 1, 1))   # 4 x 6 x 4 each
    with Simulation({"dimensions": 3, "flux_calculator": "ausmdv"}) as sim:
        for q in blocks:
            sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
        with pytest.raises(_lib.E4CError) as e:
            sim.connect(0, W.EAST, 1, W.NORTH)     # 6 x 4 against 4 x 4
        assert e.value.code == _lib.E4C_ERR_ARG
        with pytest.raises(_lib.E4CError) as e:
            sim.connect(0, W.EAST, 1, W.WEST, 4)   # no such orientation
        assert e.value.code == _lib.E4C_ERR_ARG
        # the parts are uniform (fused): their joints are opposite faces at orientation 0
        with pytest.raises(_lib.E4CError) as e:
            sim.connect(0, W.EAST, 1, W.WEST, 2)
        assert e.value.code == _lib.E4C_ERR_UNSUPPORTED
        sim.connect(0, W.EAST, 1, W.WEST, 0)
