"""Per-tree feature sampling in the resident booster (tree_config.feature_fraction
with feature_seed): every tree grows over the features sample_features draws
(src/grower_impl.hpp:163-180: a sorted std::sample of max(1, ceil(fraction x
F)) ids from the grower's std::mt19937), one draw per tree and per class tree.

Against the reference's own booster with the same fraction and seed: every
tree of eight rounds over two update batches bit for bit and the predictions
bit for bit (depthwise eager and graph-captured, levelwise, leafwise, u16
bins, with the Bernoulli sampler and sample weights), a softmax round's class
trees, and a one-feature sample. The quantised form, which has no reference
counterpart, is checked on a plane of several mirror tiles (samples that
leave tile slots unused): a one-feature sample splits every node of a tree on
one feature, two fits are identical, and the AUC is within 2e-3 of the plain
sampled fit's."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg

pytestmark = pytest.mark.gpu
LEAF = 0xFFFFFFFF


def _data(seed=4, n=12_000, F=9):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.04] = np.nan
    x = np.nan_to_num(X)
    w = rng.normal(0, 1, F)
    y = (x @ w + 0.5 * x[:, 0] * x[:, 1] + 0.1 * rng.standard_normal(n)).astype(np.float32)
    return X, y


def _same(a, b, where):
    for k in TREE_FIELDS:
        x, z = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert len(x) == len(z), f"{where} {k}"
        assert np.array_equal(x.view(np.uint8), z.view(np.uint8)), f"{where} {k}"


@pytest.mark.parametrize("grower,graph,extra", [
    ("depthwise", True, {}), ("depthwise", False, {}), ("levelwise", True, {}),
    ("leafwise", False, {}), ("depthwise", True, {"subsample": 0.7, "weights": True}),
    ("depthwise", True, {"max_bin": 700}), ("depthwise", True, {"fraction": 0.05}),
])
def test_feature_fraction_matches_reference(bb, ref, grower, graph, extra):
    X, y = _data()
    frac = extra.get("fraction", 0.5)
    sub = extra.get("subsample", 1.0)
    w = (np.random.Generator(np.random.PCG64(9)).uniform(0.2, 2.0, len(y)).astype(np.float32)
         if extra.get("weights") else None)
    cuts, off = ref.fit_cuts(X, max_bin=extra.get("max_bin", 255))
    ds = ref.dataset(X, y, cuts, off, weights=w)
    tc = dict(grower=grower, max_depth=6, max_leaves=31)
    m = ref.train(ds, TreeCfg(n_iters=8, learning_rate=0.1, feature_fraction=frac,
                              feature_seed=13, subsample=sub, random_seed=5, **tc))
    plane = bb.Plane(X, cuts, off)
    assert plane.u8 == ("max_bin" not in extra)
    b = bb.Booster(plane, y, bb.TrainParams(learning_rate=0.1, feature_fraction=frac,
                                            feature_seed=13, subsample=sub, random_seed=5,
                                            use_graph=graph, **tc), max_trees=8, weights=w)
    b.update(3)
    b.update(5)
    for i in range(8):
        if grower == "levelwise":
            for x, z in zip(bb.oblivious_tables(b.tree(i)), m.oblivious(i)):
                assert np.array_equal(np.asarray(x).view(np.uint8),
                                      np.asarray(z).view(np.uint8)), i
        else:
            _same(b.tree(i), m.tree(i), f"tree {i}")
        if frac < 0.1:  # one feature per tree
            f = b.tree(i).feature
            assert len(set(f[f != LEAF].tolist())) <= 1
    assert np.array_equal(bb.predict(plane, b.trees(), b.init_score, 0.1), m.predict_binned(ds))


def test_feature_fraction_softmax_round_matches_reference(bb, ref):
    from bonsai_b200 import synth
    K = 3
    X, y = synth.multiclass_onehot(n=10_000, n_classes=K)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=K, max_depth=5, n_iters=1,
                              learning_rate=0.1, feature_fraction=0.3, feature_seed=21))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K, max_depth=5,
                                            learning_rate=0.1, feature_fraction=0.3,
                                            feature_seed=21, use_graph=True), max_trees=1)
    b.update(1)
    for k in range(K):
        _same(b.tree(k), m.tree(k), f"class {k}")


@pytest.mark.parametrize("max_bin", [255, 700])
def test_feature_fraction_quantised(bb, max_bin):
    rng = np.random.Generator(np.random.PCG64(17))
    n, F = 60_000, 40  # two u8 mirror tiles, three u16 ones
    X = rng.standard_normal((n, F)).astype(np.float32)
    w = rng.normal(0, 1, F)
    y = ((X @ w + 0.3 * rng.standard_normal(n)) > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X, max_bin=max_bin)
    plane = bb.Plane(X, cuts, off)

    def fit(mode, frac, graph=True):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=6,
                                                hist_mode=mode, seed=3, feature_fraction=frac,
                                                feature_seed=8, use_graph=graph), max_trees=15)
        b.update(15)
        return b

    # one feature per tree: every split of a tree on the same feature
    one = fit("int8", 0.01)
    for t in one.trees():
        assert len(set(t.feature[t.feature != LEAF].tolist())) == 1
    a, c = fit("int8", 0.3), fit("int8", 0.3, graph=False)
    for i in range(15):
        _same(a.tree(i), c.tree(i), f"tree {i}")
    auc = {}
    for mode, b in (("int8", a), ("exact", fit("exact", 0.3))):
        s = b.scores()
        order = np.argsort(s)
        ranks = np.empty(n)
        ranks[order] = np.arange(1, n + 1)
        pos = y == 1
        auc[mode] = (ranks[pos].sum() - pos.sum() * (pos.sum() + 1) / 2) / (pos.sum() * (~pos).sum())
    assert abs(auc["exact"] - auc["int8"]) < 2e-3, auc


def test_feature_fraction_refusals(bb):
    X, y = _data(n=500)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    with pytest.raises(bb.BonsaiError):
        bb.Booster(plane, y, bb.TrainParams(feature_fraction=-0.5))
    with pytest.raises(bb.BonsaiError):
        bb.Booster(plane, y, bb.TrainParams(feature_fraction=0.5, selected=[0, 2]))
