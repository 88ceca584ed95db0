"""Multi-process host logic on CPU (gloo, world size 2): replicas shard the
ensemble members with no data exchange, the ensemble-mean P(k) is the one
collective, and the bench's timing reduction takes the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from conan_b200.ensemble import allreduce_mean_pk, shard, standard_members
        import bench
        members = standard_members()
        mine = shard(members, rank, world)
        # per-member "spectra": P = member seed * ones, one member per bin
        P = np.array([np.full(4, float(m[3])) for m in mine])
        cnt = np.full(4, float(len(mine)))
        mean = allreduce_mean_pk(P, cnt, dist)
        t = bench.max_over_ranks(10.0 + rank, dist, device="cpu")
        q.put((rank, [m[3] for m in mine], mean.tolist(), t))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_sharding_and_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    out.sort()
    seeds = out[0][1] + out[1][1]
    assert sorted(seeds) == list(range(1000, 1096))  # every member exactly once
    assert not set(out[0][1]) & set(out[1][1])
    expect = np.mean(np.arange(1000, 1096, dtype=float))
    for r in out:
        assert np.allclose(r[2], expect)
        assert r[3] == 11.0  # max over ranks
