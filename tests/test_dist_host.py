"""The host side of a row-sharded fit on CPU: two gloo ranks (world size 2,
127.0.0.1) run the protocol bench.py and a multi-GPU fit use -- shard ranges,
the fit's initial score chained through the ranks in row order, and rank 0's
communicator id shared with the other -- and must agree with each other and
with a one-process computation bit for bit. No GPU is touched: the id is a
stand-in, the sums are host floats."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

N_ROWS = 10_007


def _labels():
    rng = np.random.Generator(np.random.PCG64(17))
    return (rng.random(N_ROWS) < 0.37).astype(np.float32) * rng.uniform(0.5, 1.5, N_ROWS).astype(
        np.float32)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bonsai_b200 import dist as bdist
        y = _labels()
        a, b = bdist.shard_range(N_ROWS, world, rank)
        s = bdist.chained_label_sum(y[a:b], world, rank)
        init = bdist.sharded_init_score(y[a:b], N_ROWS, "logloss", world, rank)
        uid = bdist.share_comm_id(world, rank, make=lambda: bytes(range(128)))
        out.put((rank, a, b, float(s), float(init), uid))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_with_one_process():
    import torch.multiprocessing as mp

    from bonsai_b200 import init_score, label_sum
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    y = _labels()
    # contiguous, covering, disjoint shards
    assert got[0][1] == 0 and got[-1][2] == N_ROWS
    assert all(got[i][2] == got[i + 1][1] for i in range(world - 1))
    # one serial float sum, on every rank
    want = label_sum(y)
    for r in got:
        assert np.float32(r[3]) == want
        assert np.float32(r[4]) == init_score(y, "logloss")
        assert r[5] == bytes(range(128))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_ranges_partition_rows(world):
    from bonsai_b200 import shard_range
    spans = [shard_range(N_ROWS, world, r) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == N_ROWS
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1
    assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
