"""Parity at the shapes of the wide-sparse and multiclass configurations,
with fewer rows so the reference's CPU grower finishes in seconds.

Wide sparse: 2,000 lognormal features, 90% of cells missing (the missing bin
everywhere), max_bin 256, leafwise with 255 leaves, a Bernoulli 0.8 row
sample drawn by the harness and handed to both sides, squared-error
gradients: the whole node table and every sampled row's leaf must equal the
reference's LeafwiseGrower bit for bit (the plane spans 63 mirror tiles).

Multiclass: 54 features (10 continuous, one-hot blocks of 4 and 40), seven
classes, softmax over the levelwise grower at depth 8: the first round's
seven oblivious trees must equal the reference MulticlassBooster's level
tables bit for bit."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg

pytestmark = pytest.mark.gpu


def test_wide_sparse_leafwise_tree_matches_reference(bb, ref):
    from bonsai_b200 import synth
    X, y = synth.wide_sparse(n=20_000, F=2_000)
    cuts, off = ref.fit_cuts(X, max_bin=256)
    rng = np.random.Generator(np.random.PCG64(2_001))
    rows = np.flatnonzero(rng.random(len(y)) < 0.8).astype(np.uint32)
    init = np.float32(y.mean(dtype=np.float64))
    g = (init - y).astype(np.float32)
    h = np.ones_like(g)
    cfg = dict(max_leaves=255, max_depth=255, min_data_in_leaf=20)
    ds = ref.dataset(X, np.zeros(len(X), np.float32), cuts, off)
    rt, rvals, rids, _ = ref.grow_tree(ds, TreeCfg(grower="leafwise", **cfg), g, h, rows)
    plane = bb.Plane(X, cuts, off)
    assert plane.u8
    t, vals, ids = bb.grow_tree(plane, bb.TrainParams(grower="leafwise", **cfg), g, h, rows)
    n = len(rt.feature)
    assert n > 400  # the 255-leaf budget is (nearly) spent
    for k in TREE_FIELDS:
        a, b = np.asarray(getattr(t, k)), np.asarray(getattr(rt, k))
        assert len(a) == n, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    # sampled rows carry their leaf (bb_grow_tree leaves unsampled rows to the
    # caller, who routes them through the finished tree)
    assert np.array_equal(vals[rows].view(np.uint32), rvals[rows].view(np.uint32))
    assert np.array_equal(ids[rows], rids[rows])


def test_multiclass_levelwise_first_round_matches_reference(bb, ref):
    from bonsai_b200 import synth
    K = 7
    X, y = synth.multiclass_onehot(n=30_000, n_classes=K)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=K, grower="levelwise",
                              max_depth=8, n_iters=1, learning_rate=0.1))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K,
                                            grower="levelwise", max_depth=8,
                                            learning_rate=0.1, use_graph=True), max_trees=1)
    b.update(1)
    assert np.array_equal(b.init_scores, m.init_scores())
    for k in range(K):
        for x, z in zip(bb.oblivious_tables(b.tree(k)), m.oblivious(k)):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(z).view(np.uint8)), k
