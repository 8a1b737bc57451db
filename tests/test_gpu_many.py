"""Many fits at once (the many-datasets batch: 64 datasets of 1k-200k rows x 28):
boosters run on private streams and a round is one CUDA graph, so launching every
booster's rounds before waiting on any lets the GPU run them concurrently. The
fits must equal the same fits run one at a time, tree for tree and score for
score."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

pytestmark = pytest.mark.gpu


def _datasets(k, seed=64):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(k):
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
        X = rng.standard_normal((n, 28)).astype(np.float32)
        w = rng.standard_normal(28)
        y = (X @ w + 0.1 * rng.standard_normal(n)).astype(np.float32)
        out.append((X, y))
    return out


@pytest.mark.parametrize("mode", ["exact", "int8"])
def test_concurrent_fits_equal_sequential(bb, mode):
    sets = _datasets(12)
    params = bb.TrainParams(max_depth=6, learning_rate=0.1, hist_mode=mode, use_graph=True)
    rounds = 10

    def make():
        out = []
        for X, y in sets:
            cuts, off = bb.fit_cuts(X)
            out.append(bb.Booster(bb.Plane(X, cuts, off), y, params, max_trees=rounds))
        return out

    seq = make()
    for b in seq:
        b.update(rounds)           # one fit at a time
    con = make()
    for b in con:
        b.update(rounds, sync=False)  # every fit in flight
    for b in con:
        b.sync()
    for i, (a, c) in enumerate(zip(seq, con)):
        assert np.array_equal(a.scores(), c.scores()), i
        for t in range(rounds):
            ta, tc = a.tree(t), c.tree(t)
            for f in TREE_FIELDS:
                assert np.array_equal(getattr(ta, f).view(np.uint8),
                                      getattr(tc, f).view(np.uint8)), (i, t, f)


@pytest.mark.parametrize("mode,grower", [("exact", "depthwise"), ("int8", "depthwise"),
                                         ("int8", "levelwise")])
def test_one_launch_batch_equals_sequential(bb, mode, grower):
    """bb_batch: every booster's round graph a child of one parent graph, one
    launch per round for the whole batch; the fits equal the same fits run one
    at a time, and a batch round can follow ordinary rounds of its boosters."""
    sets = _datasets(10, seed=65)
    params = bb.TrainParams(max_depth=5, learning_rate=0.1, hist_mode=mode, grower=grower,
                            use_graph=True)
    rounds = 8

    def make():
        out = []
        for X, y in sets:
            cuts, off = bb.fit_cuts(X)
            out.append(bb.Booster(bb.Plane(X, cuts, off), y, params, max_trees=rounds))
        return out

    seq = make()
    for b in seq:
        b.update(rounds)
    bat = make()
    bat[0].update(2)                 # ordinary rounds first, then the batch
    batch = bb.BoosterBatch(bat[1:])
    batch.update(rounds)
    bat[0].update(rounds - 2)
    assert batch.last_ms > 0
    batch.close()
    for i, (a, c) in enumerate(zip(seq, bat)):
        assert c.n_trees == rounds, i
        assert np.array_equal(a.scores(), c.scores()), i
        for t in range(rounds):
            ta, tc = a.tree(t), c.tree(t)
            for f in TREE_FIELDS:
                assert np.array_equal(getattr(ta, f).view(np.uint8),
                                      getattr(tc, f).view(np.uint8)), (i, t, f)


def test_batch_refuses_sampled_and_leafwise(bb):
    (X, y), = _datasets(1, seed=66)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    for kw in (dict(subsample=0.8), dict(grower="leafwise", max_leaves=15),
               dict(feature_fraction=0.5)):
        b = bb.Booster(plane, y, bb.TrainParams(use_graph=True, **kw), max_trees=2)
        with pytest.raises(bb.ConfigError):
            bb.BoosterBatch([b])
        b.close()
