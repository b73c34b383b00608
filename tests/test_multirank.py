"""The N > 1 host logic of bench.py on CPU ranks (gloo, world size 2): the
timing reduction is the max over ranks, the whole-job value sums the
replicas, and the reference arm runs on rank 0 alone."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (r + 1) * 10 ms: every rank sees the slowest
        ms = bench.max_over_ranks(10.0 * (rank + 1), dist, device="cpu")
        value = bench.replica_rate(1000 * 5, world, ms * 1e-3)
        # the reference arm: rank 0 alone does work, the others return at once
        ref = bench.run_reference(None, rank, world) if rank != 0 else "rank0"
        out[rank] = (ms, value, ref)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    assert res[0][1] == res[1][1] == pytest.approx(2 * 5000 / 0.020)
    assert res[1][2] is None


def test_single_process_reduction_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replica_rate(100, 1, 0.5) == 200.0
