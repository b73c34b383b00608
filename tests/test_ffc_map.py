"""The full-face-copy cell mapping for any pair of faces and orientation
(GhostCellFullFaceCopy.set_up_cell_mapping, src/eilmer/bc/ghost_cell_effect/
full_face_copy.d:142-1083): the oracle's rule against the reference's own
table (tests/golden/ffc_map.json, made by tests/golden/make_ffc_map.py from
the reference source), the rule's inverse, its geometric meaning, and the
oracle's turned joints against the uncut block."""
import itertools
import json
import os

import numpy as np
import pytest

from eilmer4_b200 import workloads as W
import joints

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_mapping_matches_the_reference_table(oracle):
    with open(os.path.join(HERE, "golden", "ffc_map.json")) as f:
        d = json.load(f)
    ni, nj, nk = d["partner_extents"]
    cases = set()
    for dim, fa, fb, r, p, q, g, i, j, k in d["rows"]:
        got = oracle.ffc_map(fa, fb, r, p, q, g, ni, nj, nk if dim == 3 else 1)
        assert tuple(got) == (i, j, k), (dim, fa, fb, r, p, q, g)
        cases.add((dim, fa, fb, r))
    assert len(cases) == 6 * 6 * 4 + 4 * 4   # every 3-D and 2-D case of the reference


def test_mapping_maps_back_with_the_same_orientation(oracle):
    # connectBlocks gives both blocks the joint's orientation (src/eilmer/prep.lua)
    n = 4
    for fa, fb, r in itertools.product(range(6), range(6), range(4)):
        for p, q in itertools.product(range(n), range(n)):
            c = oracle.ffc_map(fa, fb, r, p, q, 0, n, n, n)
            # the partner cell's own face indices on fb
            pb = c[1] if fb in (W.EAST, W.WEST) else c[0]
            qb = c[1] if fb in (W.TOP, W.BOTTOM) else c[2]
            back = oracle.ffc_map(fb, fa, r, pb, qb, 0, n, n, n)
            pa = back[1] if fa in (W.EAST, W.WEST) else back[0]
            qa = back[1] if fa in (W.TOP, W.BOTTOM) else back[2]
            assert (pa, qa) == (p, q), (fa, fb, r, p, q)


@pytest.mark.parametrize("dimensions", [2, 3])
def test_every_turn_of_the_partner_is_one_face_and_orientation(oracle, dimensions):
    b = joints.cubic_block(8, 6, 4, 3, dimensions, bump=False)
    seen = set()
    for axes in joints.proper_turns(dimensions):
        _, (a, fa, hb, fb, r), _ = joints.turned_domain(oracle, b, axes, dimensions)
        seen.add((fb, r))
    assert len(seen) == (24 if dimensions == 3 else 4)


def oracle_run(oracle, dimensions, blocks, joint, nsteps):
    cfg = oracle.default_config(dimensions=dimensions, n_threads=0,
                                flux_calculator=oracle.FLUX_AUSMDV)
    sim = oracle.OracleSim(cfg)
    for q in blocks:
        h = sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
        sim.set_flow(h, q.prim)
    if joint is not None:
        a, fa, hb, fb, r = joint
        sim.connect(a, fa, hb, fb, r)
    assert sim.run(nsteps) == 0
    return [sim.get_flow(h)[0] for h in range(len(blocks))], (sim.time, sim.step)


@pytest.mark.parametrize("dimensions,turn", [(2, 1), (2, 2), (3, 5), (3, 11), (3, 18)])
def test_oracle_turned_joint_matches_the_uncut_block(oracle, dimensions, turn):
    b = joints.cubic_block(12, 8, 6, 5, dimensions)
    axes = joints.proper_turns(dimensions)[turn]
    nsteps = 10
    (uncut,), st = oracle_run(oracle, dimensions, [b], None, nsteps)
    blocks, joint, unturn = joints.turned_domain(oracle, b, axes, dimensions)
    prims, st2 = oracle_run(oracle, dimensions, blocks, joint, nsteps)
    assert st2[1] == st[1]
    joined = unturn(prims)
    for q in range(uncut.shape[0]):
        scale = np.abs(uncut[1:4]).max() if q in (1, 2, 3) else np.abs(uncut[q]).max()
        assert np.abs(joined[q] - uncut[q]).max() <= 1e-11 * scale, (q, axes, joint)
