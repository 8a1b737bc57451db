"""The row-sharded fit's exchange steps on CPU, over two gloo ranks.

A row-sharded quantised fit (bonsai_b200/csrc/shard.cu, the Reducer calls in
bonsai_b200/csrc/grow.cu) reduces, in stream order and in the same sequence
on every rank: the gradient maxima (max), the root's integer cells, each
frontier node's left count, the next frontier's smaller-child cells, and the
leaves' fixed-point sums (all int64 sums). This test runs that call sequence
with a CPU restatement of the depthwise step around it -- integer histograms
of each rank's rows, FP64 gain from the reduced cells, min_data_in_leaf on
global counts, the smaller child built and the larger subtracted, leaf values
from the reduced fixed-point sums -- on two gloo ranks (127.0.0.1), and checks
that both ranks take every decision a one-process fit takes: the same split
per node, the same node counts, the same leaf values, bit for bit. No GPU is
touched; the device kernels' own equality with a one-GPU fit is the GPU test
tests/test_gpu_sharded.py."""

from __future__ import annotations

import os
import socket

import numpy as np

N, F, NB, DEPTH = 6_007, 5, 16, 4
LAMBDA, MIN_DATA = 1.0, 20
UNIT = float(2 ** 38)


def _data():
    rng = np.random.Generator(np.random.PCG64(31))
    bins = rng.integers(0, NB, (N, F)).astype(np.int64)
    g = rng.normal(0, 1, N) + 0.8 * (bins[:, 0] > 7) - 0.5 * (bins[:, 2] < 4)
    h = rng.uniform(0.05, 0.25, N)
    return bins, g.astype(np.float32), h.astype(np.float32)


class Local:
    """One process: every reduction is the identity."""

    def max_u32(self, a):
        return a

    def sum_i64(self, a):
        return a


class Gloo:
    """The Reducer's two operations over torch.distributed (gloo)."""

    def max_u32(self, a):
        import torch
        import torch.distributed as dist
        t = torch.from_numpy(np.asarray(a, np.int64).copy())
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.numpy()

    def sum_i64(self, a):
        import torch
        import torch.distributed as dist
        t = torch.from_numpy(np.asarray(a, np.int64).copy())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.numpy()


def _cells(bins, qg, qh, rows):
    """Integer (g, h, count) cells [F, NB, 3] of the given rows."""
    c = np.zeros((F, NB, 3), np.int64)
    for f in range(F):
        np.add.at(c[f, :, 0], bins[rows, f], qg[rows])
        np.add.at(c[f, :, 1], bins[rows, f], qh[rows])
        np.add.at(c[f, :, 2], bins[rows, f], 1)
    return c


def _best(c, sg, sh):
    """The split with the largest FP64 gain (first maximum: feature, then bin)."""
    G, H, n = c[0, :, 0].sum(), c[0, :, 1].sum(), c[0, :, 2].sum()
    parent = (G * sg) ** 2 / (H * sh + LAMBDA)
    best = (0.0, -1, -1)
    for f in range(F):
        lg = np.cumsum(c[f, :-1, 0]) * sg
        lh = np.cumsum(c[f, :-1, 1]) * sh
        ln = np.cumsum(c[f, :-1, 2])
        for b in range(NB - 1):
            if ln[b] < MIN_DATA or n - ln[b] < MIN_DATA:
                continue
            rg, rh = G * sg - lg[b], H * sh - lh[b]
            gain = lg[b] ** 2 / (lh[b] + LAMBDA) + rg ** 2 / (rh + LAMBDA) - parent
            if gain > best[0]:
                best = (gain, f, b)
    return best


def grow(bins, g, h, row0, red):
    """One depthwise tree over this rank's rows (global ids row0 + local
    index), every cross-rank quantity through `red` in the device order."""
    n = len(g)
    # 1. the fit's maxima -> one quantisation scale on every rank
    mx = red.max_u32(np.array([np.abs(g).max().view(np.uint32), h.max().view(np.uint32)],
                              np.int64))
    mg = np.uint32(mx[0]).view(np.float32)
    mh = np.uint32(mx[1]).view(np.float32)
    sg, sh = float(mg) / 127.0, float(mh) / 127.0
    # deterministic rounding keyed by the global row id (the device uses Philox)
    rid = np.arange(n) + row0
    u = ((rid * 2654435761) % 1000003) / 1000003.0
    qg = np.floor(g / sg + u).astype(np.int64)
    qh = np.floor(h / sh + u).astype(np.int64)
    # 2. the root's cells
    nodes = {0: np.arange(n)}
    cells = {0: red.sum_i64(_cells(bins, qg, qh, nodes[0]))}
    tree, frontier = {}, [0]
    for _ in range(DEPTH):
        nxt = []
        splits = {}
        for nd in frontier:
            gain, f, b = _best(cells[nd], sg, sh)
            if f >= 0:
                splits[nd] = (f, b)
        if not splits:
            break
        # 3. every split node's rows routed left, summed over the ranks
        lefts = np.array([(bins[nodes[nd], splits[nd][0]] <= splits[nd][1]).sum()
                          for nd in splits], np.int64)
        glefts = red.sum_i64(lefts)
        smaller = {}
        for (nd, (f, b)), gl in zip(splits.items(), glefts):
            total = cells[nd][0, :, 2].sum()
            go = bins[nodes[nd], f] <= b
            nodes[2 * nd + 1] = nodes[nd][go]
            nodes[2 * nd + 2] = nodes[nd][~go]
            smaller[nd] = 2 * nd + 1 if gl <= total - gl else 2 * nd + 2
            tree[nd] = (f, b, int(total), int(gl))
        # 4. the smaller children's cells (partial per rank), larger by subtraction
        built = red.sum_i64(np.stack([_cells(bins, qg, qh, nodes[smaller[nd]])
                                      for nd in splits]))
        for k, nd in enumerate(splits):
            s = smaller[nd]
            other = 2 * nd + 1 if s == 2 * nd + 2 else 2 * nd + 2
            cells[s] = built[k]
            cells[other] = cells[nd] - built[k]
            nxt += [2 * nd + 1, 2 * nd + 2]
        frontier = nxt
    # 5. the leaves' fixed-point sums of full-precision gradients
    leaves = sorted(nd for nd in nodes if nd not in tree)
    fix = np.zeros((len(leaves), 2), np.int64)
    for i, nd in enumerate(leaves):
        fix[i, 0] = np.rint(g[nodes[nd]].astype(np.float64) * (UNIT / float(mg))).sum()
        fix[i, 1] = np.rint(h[nodes[nd]].astype(np.float64) * (UNIT / float(mh))).sum()
    fix = red.sum_i64(fix)
    values = {nd: float(-(fix[i, 0] * float(mg) / UNIT) / (fix[i, 1] * float(mh) / UNIT + LAMBDA))
              for i, nd in enumerate(leaves)}
    return tree, values


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
        from bonsai_b200 import shard_range
        bins, g, h = _data()
        a, b = shard_range(N, world, rank)
        out.put((rank, grow(bins[a:b], g[a:b], h[a:b], a, Gloo())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_one_process_decisions():
    import torch.multiprocessing as mp
    bins, g, h = _data()
    want_tree, want_values = grow(bins, g, h, 0, Local())
    assert len(want_tree) >= 7 and len(want_values) >= 8     # a real tree
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        tree, values = got[r]
        assert tree == want_tree, r
        assert values == want_values, r
