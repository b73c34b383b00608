"""Blocks shared out over ranks (eilmer4_b200/sharding.py): the partition
plan, two gloo ranks on the CPU advancing a split domain with the oracle as
each rank's engine (bit for bit the uncut block), and, on one GPU, the
library's remote faces (pack, transfer, unpack into a shadow) driven by the
same host loop with a loopback transport (bit for bit the uncut block in the
FP64 form)."""
import os
import socket
import tempfile

import numpy as np
import pytest

from eilmer4_b200 import sharding as S
from eilmer4_b200 import workloads as W


def domain(parts):
    b = W.inflow_3d_block(24, 12, 10, 5, spacing=1.0 / 64.0)
    blocks, conns = W.split_block(b, 3, parts)
    return b, blocks, conns


def test_plan_pairs_every_remote_face():
    _, blocks, conns = domain((2, 2, 1))
    owner = [0, 1, 1, 0]
    plans = [S.plan(len(blocks), conns, owner, r) for r in (0, 1)]
    assert plans[0].blocks == [0, 3] and plans[1].blocks == [1, 2]
    keys = {}
    for r, p in enumerate(plans):
        for rf in p.remote:
            keys.setdefault(rf.key, []).append((r, rf))
    assert len(keys) == len(conns)   # no joint stays inside a rank here
    for key, sides in keys.items():
        (ra, a), (rb, b) = sides
        assert ra != rb and a.peer == rb and b.peer == ra
        assert S.OPPOSITE[a.face] == b.face
    # the order of a pair's joints is the same on both ranks
    for r, p in enumerate(plans):
        other = plans[1 - r]
        assert [rf.key for rf in p.remote] == [rf.key for rf in other.remote]


def test_dt_control_follows_the_device_rule():
    c = S.DtControl(cfl_count=10, dt_init=1.0e-3, dt_max=2.0e-6)
    assert c.update(0, 5.0e-7, 0.4) == 5.0e-7           # fmin(dt_init, dt_allow)
    assert c.update(10, 1.0e-6, 0.3) == 7.5e-7           # x1.5 growth cap
    assert c.update(20, 1.0e-5, 0.2) == 1.125e-6
    assert c.update(30, 1.0e-5, 0.2) == 1.6875e-06
    assert c.update(40, 1.0e-5, 0.2) == 2.0e-6           # dt_max
    assert c.update(50, 1.0e-7, 0.9) == 1.0e-7           # shrink at once


class OracleEngine:
    """One rank's blocks in the CPU oracle (test infrastructure)."""

    def __init__(self, osim, nblocks):
        self.sim = osim
        self.nblocks = nblocks

    def dt_allow(self, dt_current, check_cfl):
        return self.sim.dt_allow(dt_current, check_cfl)

    def stage(self, stage, dt):
        if stage == 1:
            self.sim.set_dt_global(dt)
        rc = self.sim.stage(stage)
        if rc != 0:
            raise RuntimeError(f"oracle stage failed: {rc}")

    def pack_face(self, h, face, stage):
        import torch
        return torch.from_numpy(self.sim.pack_face(h, face))

    def recv_buffer(self, h, face):
        import torch
        return torch.zeros(self.sim.pack_face(h, face).size, dtype=torch.float64)

    def unpack_face(self, h, face, buf):
        self.sim.unpack_face(h, face, buf.numpy())


def oracle_for(oracle, blocks, nthreads=2):
    cfg = oracle.default_config(dimensions=3, flux_calculator=oracle.FLUX_HLLC,
                                n_threads=nthreads)
    osim = oracle.OracleSim(cfg)
    for q in blocks:
        h = osim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
        osim.set_flow(h, q.prim)
    return osim


def _rank_main(rank, world, port, parts, nsteps, outdir):
    import torch.distributed as dist

    from oracle import e4_oracle as O
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        _, blocks, conns = domain(parts)
        owner = [g % world for g in range(len(blocks))]
        p = S.plan(len(blocks), conns, owner, rank)
        osim = oracle_for(O, [blocks[g] for g in p.blocks])
        for (ha, fa, hb, fb) in p.local:
            osim.connect(ha, fa, hb, fb)
        for rf in p.remote:
            osim.set_remote(rf.handle, rf.face)
        cfg = osim.cfg
        run = S.ShardedRun(OracleEngine(osim, len(p.blocks)), p.remote, S.TorchComm(dist, "cpu"),
                           S.DtControl(cfg.cfl_count, cfg.dt_init, cfg.dt_max))
        run.run(nsteps)
        out = {f"prim{g}": osim.get_flow(h)[0] for h, g in enumerate(p.blocks)}
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), time=run.time, step=run.step_count,
                 dt=run.control.dt_global, ostep=osim.step, otime=osim.time, **out)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("parts", [(2, 1, 1), (1, 1, 2), (2, 2, 1)])
def test_two_gloo_ranks_match_the_uncut_block(oracle, parts):
    import torch.multiprocessing as mp
    nsteps = 14
    b, blocks, conns = domain(parts)
    with tempfile.TemporaryDirectory() as tmp:
        mp.spawn(_rank_main, args=(2, free_port(), parts, nsteps, tmp), nprocs=2, join=True)
        res = [dict(np.load(os.path.join(tmp, f"rank{r}.npz"))) for r in (0, 1)]
    uncut = oracle_for(oracle, [b], nthreads=0)
    assert uncut.run(nsteps) == 0
    prims = [None] * len(blocks)
    for r in res:
        for k, v in r.items():
            if k.startswith("prim"):
                prims[int(k[4:])] = v
    joined = W.join_prims(prims, (b.ni, b.nj, b.nk), 3, parts)
    assert np.array_equal(joined, uncut.get_flow(0)[0])
    for r in res:
        assert int(r["step"]) == nsteps == int(r["ostep"])
        assert float(r["time"]) == uncut.time == float(r["otime"])
        assert float(r["dt"]) == uncut.dt_global


class LoopbackComm:
    """Both sides of every joint in one process: each face receives what the
    other side of its joint packed; the reductions are over one rank."""

    def exchange(self, items):
        by_key = {}
        for rf, sbuf, _ in items:
            by_key.setdefault(rf.key, []).append((rf, sbuf))
        for rf, _, rbuf in items:
            (other,) = [s for (r, s) in by_key[rf.key] if (r.handle, r.face) != (rf.handle, rf.face)]
            rbuf.copy_(other)

    def min(self, x):
        return x

    def max(self, x):
        return x


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32_flux"])
@pytest.mark.parametrize("parts", [(2, 1, 1), (1, 2, 2)])
def test_gpu_remote_faces_match_the_uncut_block(e4lib, precision, parts):
    """The library's remote faces on one GPU: the blocks of a split domain in
    one context, every joint declared remote, the layers packed, moved and
    unpacked into the shadows before each stage by the sharded host loop."""
    import torch

    from eilmer4_b200.simcore import Simulation
    nsteps = 14
    b, blocks, conns = domain(parts)
    wl = W.Workload("u", 3, flux_calculator="hllc")
    wl.blocks.append(b)
    with Simulation.from_workload(wl, precision=precision) as sim:
        sim.run(nsteps)
        ref = sim.download(0, want_cons=False)[0]
        t_ref, dt_ref, st_ref = sim.state()
    owner = [0] * len(blocks)
    p = S.plan(len(blocks), conns, owner, 0)
    remote = []
    for (a, fa, bb, fb) in conns:   # every joint through the remote path
        key = (a, fa, bb, fb)
        remote += [S.RemoteFace(a, fa, 0, key), S.RemoteFace(bb, fb, 0, key)]
    with Simulation({"dimensions": 3, "flux_calculator": "hllc"}, precision=precision) as sim:
        for q in blocks:
            h = sim.add_block(q.ni, q.nj, q.nk, q.vtx, q.bc, q.inflow)
            sim.upload(h, q.prim)
        eng = S.LibraryEngine(sim, remote, torch.device("cuda", 0))
        c = sim.cfg
        run = S.ShardedRun(eng, remote, LoopbackComm(), S.DtControl(c.cfl_count, c.dt_init, c.dt_max))
        run.run(nsteps)
        prims = [sim.download(h, want_cons=False)[0] for h in range(len(blocks))]
        t, dt, st = sim.state()
        # a simulation with remote faces advances one stage at a time
        from eilmer4_b200 import _lib
        with pytest.raises(_lib.E4CError) as ei:
            sim.run(1)
        assert ei.value.code == _lib.E4C_ERR_STATE
    assert p.blocks == list(range(len(blocks)))
    joined = W.join_prims(prims, (b.ni, b.nj, b.nk), 3, parts)
    assert st == st_ref == nsteps and run.step_count == nsteps
    if precision == "fp64":
        assert np.array_equal(joined, ref)
        assert t == t_ref == run.time and dt == dt_ref
    else:
        speed = np.abs(ref[1:4]).max()
        for q in range(ref.shape[0]):
            scale = speed if q in (1, 2, 3) else np.abs(ref[q]).max()
            assert np.abs(joined[q] - ref[q]).max() <= 1e-6 * scale, q
