"""Row subsampling in the resident booster: with subsample < 1 every tree
grows over the rows the reference's BernoulliSampler keeps (src/sampler.cpp:
36-55; the booster's std::mt19937 seeded by booster_config.random_seed,
include/bonsai/booster.hpp:496), and every row -- kept or not -- takes the
tree's leaf into its score (the unsampled ones routed through the finished
tree as route_unsampled does, src/grower_impl.hpp:438-461).

Against the reference's own booster with the same sampler and seed: every
tree of every round bit for bit (depthwise eager and graph-captured,
levelwise, leafwise, over two update batches so the draw stream carries
across calls) and the final predictions bit for bit; a softmax round's
class trees (one draw per class tree). The quantised form, which has no
reference counterpart, is checked against the restated draws (each tree's
root cover is its kept-row count) and against the plain sampled fit's AUC."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg, bernoulli_keep

pytestmark = pytest.mark.gpu


def _data(seed=3, n=20_000, F=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.04] = np.nan
    x = np.nan_to_num(X)
    y = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.3 * np.abs(x[:, 3])
         + 0.1 * rng.standard_normal(n)).astype(np.float32)
    return X, y


def _same(a, b, where):
    for k in TREE_FIELDS:
        x, z = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert len(x) == len(z), f"{where} {k}"
        assert np.array_equal(x.view(np.uint8), z.view(np.uint8)), f"{where} {k}"


@pytest.mark.parametrize("grower,graph", [("depthwise", True), ("depthwise", False),
                                          ("levelwise", True), ("leafwise", False)])
def test_sampled_fit_matches_reference(bb, ref, grower, graph):
    X, y = _data()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    tc = dict(grower=grower, max_depth=6, max_leaves=31)
    m = ref.train(ds, TreeCfg(n_iters=8, learning_rate=0.1, subsample=0.7, random_seed=11,
                              **tc))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(learning_rate=0.1, subsample=0.7, random_seed=11,
                                            use_graph=graph, **tc), max_trees=8)
    b.update(3)
    b.update(5)
    keep = bernoulli_keep(len(y), 0.7, 11, 8)
    for i in range(8):
        if grower == "levelwise":
            for x, z in zip(bb.oblivious_tables(b.tree(i)), m.oblivious(i)):
                assert np.array_equal(np.asarray(x).view(np.uint8),
                                      np.asarray(z).view(np.uint8)), i
        else:
            _same(b.tree(i), m.tree(i), f"tree {i}")
        assert int(b.tree(i).covers[0]) == int(keep[i].sum())
    assert np.array_equal(bb.predict(plane, b.trees(), b.init_score, 0.1), m.predict_binned(ds))


def test_sampled_scores_route_every_row(bb, ref):
    """The device scores equal init + lr x leaf summed tree by tree in round
    order over every row (kept or not): the oracle's bin-space predict of
    each prefix of the ensemble, differenced."""
    X, y = _data(seed=4, n=6_000)
    cuts, off = ref.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(learning_rate=0.1, subsample=0.5, random_seed=3,
                                            max_depth=5, use_graph=True), max_trees=4)
    b.update(4)
    trees = b.trees()
    s = np.full(len(y), np.float32(b.init_score), np.float32)
    for t in trees:
        leaf = bb.predict(plane, [t], np.float32(0.0), 1.0)  # the tree's leaf value per row
        s = (s + np.float32(0.1) * leaf).astype(np.float32)
    assert np.array_equal(b.scores().view(np.uint32), s.view(np.uint32))


def test_sampled_softmax_round_matches_reference(bb, ref):
    from bonsai_b200 import synth
    K = 4
    X, y = synth.multiclass_onehot(n=12_000, n_classes=K)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=K, max_depth=5, n_iters=1,
                              learning_rate=0.1, subsample=0.6, random_seed=9))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K, max_depth=5,
                                            learning_rate=0.1, subsample=0.6, random_seed=9,
                                            use_graph=True), max_trees=1)
    b.update(1)
    for k in range(K):
        _same(b.tree(k), m.tree(k), f"class {k}")


@pytest.mark.parametrize("grower", ["depthwise", "leafwise"])
def test_sampled_quantised_follows_the_draws(bb, grower):
    rng = np.random.Generator(np.random.PCG64(8))
    n, F = 60_000, 8
    X = rng.standard_normal((n, F)).astype(np.float32)
    y = ((X[:, 0] + X[:, 1] * X[:, 2] + 0.3 * rng.standard_normal(n)) > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    keep = bernoulli_keep(n, 0.8, 21, 12)
    auc = {}
    for mode in ("exact", "int16"):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", grower=grower, max_depth=6,
                                                max_leaves=31, hist_mode=mode, seed=2,
                                                subsample=0.8, random_seed=21,
                                                use_graph=grower == "depthwise"), max_trees=12)
        b.update(12)
        assert [int(b.tree(i).covers[0]) for i in range(12)] == [int(k.sum()) for k in keep]
        s = b.scores()
        order = np.argsort(s)
        ranks = np.empty(n)
        ranks[order] = np.arange(1, n + 1)
        pos = y == 1
        auc[mode] = (ranks[pos].sum() - pos.sum() * (pos.sum() + 1) / 2) / (pos.sum() * (~pos).sum())
    assert abs(auc["exact"] - auc["int16"]) < 2e-3, auc


def test_subsample_refusals(bb):
    X, y = _data(n=500)
    cuts, off = bb.fit_cuts(X)
    with pytest.raises(bb.BonsaiError):
        bb.Booster(bb.Plane(X, cuts, off), y, bb.TrainParams(subsample=-0.5))


@pytest.mark.parametrize("grower,graph", [("depthwise", True), ("levelwise", True),
                                          ("leafwise", False)])
@pytest.mark.parametrize("seed", [0, 5])
def test_empty_and_single_row_samples_match_reference(bb, ref, grower, graph, seed):
    """Samples of zero or one row (subsample 0.002 of 300 rows: seed 0 keeps 1, 0
    and 1 rows over three trees, seed 5 none): the reference grows a root leaf
    of value -0.0 and cover 0 from an empty sample, and every row still takes
    each tree's leaf."""
    rng = np.random.Generator(np.random.PCG64(1))
    X = rng.standard_normal((300, 4)).astype(np.float32)
    y = X[:, 0].astype(np.float32)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    tc = dict(grower=grower, max_depth=3, max_leaves=7)
    m = ref.train(ds, TreeCfg(n_iters=3, subsample=0.002, random_seed=seed, **tc))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(subsample=0.002, random_seed=seed, use_graph=graph,
                                            **tc), max_trees=3)
    b.update(3)
    keep = bernoulli_keep(300, 0.002, seed, 3)
    for i in range(3):
        assert int(b.tree(i).covers[0]) == int(keep[i].sum())
        if grower == "levelwise":
            for x, z in zip(bb.oblivious_tables(b.tree(i)), m.oblivious(i)):
                assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(z).view(np.uint8))
        else:
            _same(b.tree(i), m.tree(i), f"tree {i}")
    assert np.array_equal(bb.predict(plane, b.trees(), b.init_score, 0.1).view(np.uint32),
                          m.predict_binned(ds).view(np.uint32))
    s = np.full(300, np.float32(b.init_score), np.float32)
    for t in b.trees():
        s = (s + np.float32(0.1) * bb.predict(plane, [t], np.float32(0.0), 1.0)).astype(np.float32)
    assert np.array_equal(b.scores().view(np.uint32), s.view(np.uint32))
