"""Row-sharded fits (bb_comm, bb_booster_create_sharded) on one GPU: the shards
of an in-process group run from one host thread each and combine their
integer partial sums through CUDA events, so a fit split over 2 or 3 shards
must equal the unsharded fit bit for bit -- every tree (features, thresholds,
gains, covers, leaf values) and every row's score. A one-rank NCCL
communicator runs the same calls through ncclAllReduce inside the round's
CUDA graph."""

from __future__ import annotations

import threading

import numpy as np
import pytest
from conftest import TREE_FIELDS

pytestmark = pytest.mark.gpu


def _data(seed, n=120_000, F=9):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    y = ((np.nan_to_num(X[:, 0]) + np.nan_to_num(X[:, 1]) * np.nan_to_num(X[:, 2])
          + 0.5 * rng.standard_normal(n)) > 0).astype(np.float32)
    return X, y


def _same_tree(a, b, where):
    for k in TREE_FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), f"{where} {k}"


def _sharded(bb, X, y, cuts, off, params, k, rounds, init):
    n = len(X)
    comms = bb.Comm.group(k)
    boosters = []
    for s in range(k):
        a, b = bb.shard_range(n, k, s)
        plane = bb.Plane(X[a:b], cuts, off)
        boosters.append(bb.Booster(plane, y[a:b], params, max_trees=rounds, comm=comms[s],
                                   row_offset=a, total_rows=n, init_score=init))
    errors = []

    def run(bst):
        try:
            bst.update(rounds)
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=run, args=(bst,)) for bst in boosters]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    return boosters


@pytest.mark.parametrize("k,grower,ff", [(2, "depthwise", 1.0), (3, "levelwise", 1.0),
                                         (2, "depthwise", 0.5), (3, "levelwise", 0.6)])
def test_group_shards_equal_unsharded_fit(bb, k, grower, ff):
    # ff < 1: every shard draws each tree's features from the same seed
    X, y = _data(3 + k)
    cuts, off = bb.fit_cuts(X)
    params = bb.TrainParams(objective="logloss", grower=grower, max_depth=6,
                            hist_mode="int8", seed=9, learning_rate=0.2, feature_fraction=ff,
                            feature_seed=4)
    rounds = 6
    full = bb.Booster(bb.Plane(X, cuts, off), y, params, max_trees=rounds)
    full.update(rounds)
    shards = _sharded(bb, X, y, cuts, off, params, k, rounds, full.init_score)
    for i in range(rounds):
        want = full.tree(i)
        for s, bst in enumerate(shards):
            _same_tree(bst.tree(i), want, f"tree {i} shard {s}")
    scores = np.concatenate([bst.scores() for bst in shards])
    assert np.array_equal(scores, full.scores())


def test_nccl_single_rank_in_graph_equals_unsharded(bb):
    X, y = _data(11, n=60_000)
    cuts, off = bb.fit_cuts(X)
    params = bb.TrainParams(objective="logloss", max_depth=5, hist_mode="int8",
                            use_graph=True)
    full = bb.Booster(bb.Plane(X, cuts, off), y, params, max_trees=4)
    full.update(4)
    comm = bb.Comm.nccl(bb.Comm.unique_id(), 1, 0)
    one = bb.Booster(bb.Plane(X, cuts, off), y, params, max_trees=4, comm=comm,
                     row_offset=0, total_rows=len(X), init_score=full.init_score)
    one.update(4)
    for i in range(4):
        _same_tree(one.tree(i), full.tree(i), f"tree {i}")
    assert np.array_equal(one.scores(), full.scores())


def test_init_score_helper_matches_booster(bb):
    X, y = _data(2, n=10_000)
    cuts, off = bb.fit_cuts(X)
    for obj in ("mse", "logloss"):
        b = bb.Booster(bb.Plane(X, cuts, off), y, bb.TrainParams(objective=obj), max_trees=1)
        assert np.float32(b.init_score) == bb.init_score(y, obj)


def test_sharding_refuses_the_exact_form(bb):
    X, y = _data(1, n=5_000)
    cuts, off = bb.fit_cuts(X)
    comms = bb.Comm.group(2)
    with pytest.raises(bb.ConfigError):
        bb.Booster(bb.Plane(X[:2500], cuts, off), y[:2500], bb.TrainParams(), max_trees=1,
                   comm=comms[0], row_offset=0, total_rows=5_000, init_score=0.0)
