"""Domains whose blocks meet at turned joints, for the full-face-copy tests:
a block cut in two along i, the second part re-indexed by a proper turn of
its index axes, so the cut becomes a joint of the first part's east face with
any face of the second part at any orientation."""
import itertools

import numpy as np

from eilmer4_b200 import workloads as W


def proper_turns(dimensions):
    """Every proper turn of the index axes, as ((old axis, sign), ...) per
    new axis; the 2-D turns keep k."""
    out = []
    nd = 3 if dimensions == 3 else 2
    for perm in itertools.permutations(range(nd)):
        for sg in itertools.product((1, -1), repeat=nd):
            M = np.zeros((nd, nd))
            for a in range(nd):
                M[a, perm[a]] = sg[a]
            if round(np.linalg.det(M)) == 1:
                out.append(tuple(zip(perm, sg)))
    return out


def orientation_of(oracle, A, Bt, fb, cell_map, dimensions):
    """The orientations r under which the reference's mapping sends the ghost
    layers behind A's east face to the cells of the turned partner Bt that
    lie there (the first cells of the uncut partner, turned)."""
    found = []
    for r in range(4 if dimensions == 3 else 1):
        ok = True
        for j in range(A.nj):
            for k in range(A.nk):
                for g in range(2):
                    want = cell_map(g, j, k)
                    got = oracle.ffc_map(W.EAST, fb, r, j, k, g, Bt.ni, Bt.nj, Bt.nk)
                    ok = ok and tuple(got) == tuple(want)
        if ok:
            found.append(r)
    return found


def turned_domain(oracle, b, axes, dimensions):
    """(blocks, joint, unturn): b cut in two along i, the second part turned
    by axes; joint = (0, EAST, 1, face, orientation); unturn(prims) gives the
    uncut block's primitive array from the two parts' arrays."""
    blocks, conns = W.split_block(b, dimensions, (2, 1, 1))
    A, B = blocks
    Bt, face_map, cell_map = W.reindex_block(B, axes, dimensions)
    fb = face_map[W.WEST]
    rs = orientation_of(oracle, A, Bt, fb, cell_map, dimensions)
    assert len(rs) == 1, (axes, fb, rs)

    def unturn(prims):
        pa, pbt = prims
        pb = W.unturn_prim(pbt, Bt, axes, dimensions)
        return W.join_prims([pa, pb], (b.ni, b.nj, b.nk), dimensions, (2, 1, 1))

    return [A, Bt], (0, W.EAST, 1, fb, rs[0]), unturn


def cubic_block(ni, nj, nk, seed, dimensions, bump=True):
    """A Mach-3 inflow block of cubic cells (so every ghost length the joint
    copies agrees with the uncut block) with an interior vertex of its first
    and of its last quarter moved a little (so neither it nor either half is
    uniform: they take the general path)."""
    if dimensions == 3:
        b = W.inflow_3d_block(ni, nj, nk, seed, spacing=1.0 / 16.0)
    else:
        wl = W.sod_2d(ni, ni)   # a unit square: square cells
        b = wl.blocks[0]
    if bump:
        nk1 = b.nk + 1 if dimensions == 3 else 1
        V = b.vtx.reshape(nk1, b.nj + 1, b.ni + 1, 3).copy()
        V[nk1 // 2, b.nj // 2, max(1, b.ni // 4), 0] += 1.0e-3 / 16.0
        V[nk1 // 2, b.nj // 2, b.ni - max(1, b.ni // 4), 0] -= 1.0e-3 / 16.0
        b = W.BlockSpec(b.ni, b.nj, b.nk, V.reshape(-1, 3), b.bc, b.inflow, b.prim)
    return b
