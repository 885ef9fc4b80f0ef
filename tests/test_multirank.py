"""CPU multi-rank checks of the sharding and timing logic (gloo, world size 2)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dendro_b200.parallel import shard_meshes


def test_shard_meshes_partitions_by_weight():
    w = np.random.default_rng(0).integers(1000, 500000, 32)
    for world in (1, 2, 3, 4, 8):
        ranges = [shard_meshes(w, r, world) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == len(w)
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        if world > 1:
            loads = [w[lo:hi].sum() for lo, hi in ranges]
            assert max(loads) <= w.sum() / world + w.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    from dendro_b200.parallel import max_over_ranks, shard_meshes, sum_over_ranks
    w = np.arange(1, 33) * 1000
    lo, hi = shard_meshes(w, rank, world)
    t = max_over_ranks(10.0 + rank)
    s = sum_over_ranks(float(hi - lo))
    out[rank] = (lo, hi, t, s)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][1] == res[1][0] and res[0][0] == 0 and res[1][1] == 32
    assert res[0][2] == res[1][2] == 11.0      # max over ranks
    assert res[0][3] == res[1][3] == 32.0      # every mesh counted once
