"""Structured blocks shared out over ranks, one rank per GPU.

This is the host side of the reference's MPI runs for the explicit update:
- the full-face exchange between blocks on different ranks: the two cell
  layers next to a joint are sent to the partner block's rank before every
  stage (src/eilmer/bc/ghost_cell_effect/full_face_copy.d:1134-1255; simcore.d
  calls exchange_ghost_cell_boundary_data before each stage's fluxes, :1599);
- the global time-step reductions, MIN of dt_allow and MAX of the CFL number
  over ranks (simcore.d:1399-1401), and the bad-cell MAX (simcore.d:2489),
  after which every rank takes the same dt decision (simcore.d:1347-1452).

The transport is torch.distributed: NCCL send/receive of device buffers
between GPUs (each buffer lands in the receiving GPU's own memory; nothing
reads another GPU's memory directly), gloo on the host for tests.  The
per-rank compute is an engine object:

    dt_allow(dt_current, check_cfl) -> (dt_allow, cfl_max)   this rank's blocks
    stage(stage, dt)                 one stage; the last one ends the step;
                                     raises on a failed stage
    pack_face(h, face, stage)        the two layers next to a remote face
    recv_buffer(h, face)             a buffer for the partner's layers
    unpack_face(h, face, buffer)     the partner's layers as ghost cells

LibraryEngine runs a Simulation (the CUDA library) on this rank's GPU.
"""
from __future__ import annotations

from dataclasses import dataclass

OPPOSITE = {0: 2, 1: 3, 2: 0, 3: 1, 4: 5, 5: 4}


@dataclass(frozen=True)
class RemoteFace:
    """A face of one of this rank's blocks joined to a block on rank `peer`.
    `key` names the joint the same way on both ranks (the global block and
    face numbers of both sides, lower block first)."""
    handle: int
    face: int
    peer: int
    key: tuple


@dataclass
class Plan:
    blocks: list          # global indices of this rank's blocks, in handle order
    local: list           # joints with both blocks here: (ha, fa, hb, fb)
    remote: list          # RemoteFace of this rank


def plan(nblocks, conns, owner, rank):
    """This rank's share of a domain cut into blocks: its blocks (handles in
    the order of their global indices), the joints inside the rank and the
    faces joined to other ranks.  conns: (a, fa, b, fb) joints of opposite
    faces by global block index; owner[g]: the rank of block g."""
    mine = [g for g in range(nblocks) if owner[g] == rank]
    handle = {g: h for h, g in enumerate(mine)}
    local, remote = [], []
    for (a, fa, b, fb) in conns:
        if OPPOSITE[fa] != fb:
            raise ValueError("only opposite faces join")
        key = (a, fa, b, fb) if a < b else (b, fb, a, fa)
        if owner[a] == rank and owner[b] == rank:
            local.append((handle[a], fa, handle[b], fb))
        elif owner[a] == rank:
            remote.append(RemoteFace(handle[a], fa, owner[b], key))
        elif owner[b] == rank:
            remote.append(RemoteFace(handle[b], fb, owner[a], key))
    remote.sort(key=lambda r: (r.peer, r.key))
    return Plan(mine, local, remote)


class DtControl:
    """The global time-step decision every rank takes from the reduced
    values (simcore.d:1347-1452, as the device loop takes it): dt_init at step
    0, at most x1.5 growth, dt_max; checked every cfl_count steps."""

    def __init__(self, cfl_count, dt_init, dt_max):
        self.cfl_count = int(cfl_count)
        self.dt_init = float(dt_init)
        self.dt_max = float(dt_max)
        self.dt_global = float(dt_init)

    def due(self, step):
        return step % self.cfl_count == 0

    def update(self, step, dt_allow, cfl_max):
        if step == 0 and not (self.dt_init >= dt_allow):   # fmin(dt_init, dt_allow)
            dt_allow = self.dt_init
        if dt_allow <= self.dt_global:
            self.dt_global = dt_allow
        else:
            g = self.dt_global * 1.5
            g = dt_allow if dt_allow < g else g
            g = self.dt_max if self.dt_max < g else g
            self.dt_global = g
        self.last_cfl_max = cfl_max
        return self.dt_global


class TorchComm:
    """Exchange and reductions over a torch.distributed process group."""

    def __init__(self, dist, device):
        self.dist = dist
        self.device = device

    def exchange(self, items):
        """items: (RemoteFace, send buffer, receive buffer).  All sends and
        receives are posted as one group (the order of a pair's joints is the
        same on both ranks)."""
        d = self.dist
        ops = []
        seen = {}
        for rf, sbuf, rbuf in items:
            tag = seen.get(rf.peer, 0)
            seen[rf.peer] = tag + 1
            ops.append(d.P2POp(d.isend, sbuf, rf.peer, tag=tag))
            ops.append(d.P2POp(d.irecv, rbuf, rf.peer, tag=tag))
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()

    def _reduce(self, x, op):
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def min(self, x):
        return self._reduce(x, self.dist.ReduceOp.MIN)

    def max(self, x):
        return self._reduce(x, self.dist.ReduceOp.MAX)


class ShardedRun:
    """Advance this rank's blocks in step with the other ranks'."""

    def __init__(self, engine, remote_faces, comm, control: DtControl, nstages=2):
        self.engine = engine
        self.remote = list(remote_faces)
        self.comm = comm
        self.control = control
        self.nstages = nstages
        self.step_count = 0
        self.time = 0.0
        self._recv = [engine.recv_buffer(rf.handle, rf.face) for rf in self.remote]

    def exchange(self, stage):
        items = [(rf, self.engine.pack_face(rf.handle, rf.face, stage), rb)
                 for rf, rb in zip(self.remote, self._recv)]
        self.comm.exchange(items)
        for rf, rb in zip(self.remote, self._recv):
            self.engine.unpack_face(rf.handle, rf.face, rb)

    def step(self):
        c = self.control
        if c.due(self.step_count):
            d, cfl = self.engine.dt_allow(c.dt_global, self.step_count > 0)
            d = self.comm.min(d)
            cfl = self.comm.max(cfl)
            c.update(self.step_count, d, cfl)
        dt = c.dt_global
        for stage in range(1, self.nstages + 1):
            self.exchange(stage)
            failed, err = 0.0, None
            try:
                self.engine.stage(stage, dt)
            except Exception as e:  # every rank learns of it before going on
                failed, err = 1.0, e
            if self.comm.max(failed) > 0.0:
                if err is not None:
                    raise err
                raise RuntimeError(f"a stage failed on another rank at step {self.step_count}")
        self.time = self.time + dt
        self.step_count += 1

    def run(self, nsteps):
        for _ in range(nsteps):
            self.step()


class LibraryEngine:
    """This rank's blocks in the CUDA library (a Simulation on its GPU)."""

    def __init__(self, sim, remote_faces, device):
        import torch
        self.sim = sim
        self.device = device
        self.handles = list(range(len(sim.blocks)))
        self._torch = torch
        for rf in remote_faces:
            sim.connect_remote(rf.handle, rf.face)

    def dt_allow(self, dt_current, check_cfl):
        return self.sim.dt_allow(self.handles, dt_current, check_cfl)

    def stage(self, stage, dt):
        self.sim.stage(self.handles, stage, dt)

    def _buffer(self, h, face):
        n = self.sim.face_slab_bytes(h, face)
        return self._torch.empty(n, dtype=self._torch.uint8, device=self.device)

    def pack_face(self, h, face, stage):
        buf = self._buffer(h, face)
        self.sim.pack_face(h, face, stage, buf.data_ptr())
        return buf

    def recv_buffer(self, h, face):
        return self._buffer(h, face)

    def unpack_face(self, h, face, buf):
        self.sim.unpack_face(h, face, buf.data_ptr())
