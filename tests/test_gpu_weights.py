"""Per-row sample weights (Dataset::weights, include/bonsai/dataset.hpp:73,86)
on the resident booster: every round's gradient and hessian scaled by the
row's weight, one float multiply each (Booster::update_one_iter,
include/bonsai/booster.hpp:546-555; the softmax pass,
include/bonsai/multiclass_booster.hpp:121-135), the initial scores unweighted.

Against the reference's own booster over a weighted Dataset: every tree of
every round bit for bit and the predictions bit for bit (depthwise eager and
graph-captured, levelwise, leafwise, and with the Bernoulli sampler); a
weighted softmax round's class trees; the reference's booster over the
drop-in grower with weights equals its CPU grower. Unit weights reproduce the
unweighted fit bit for bit; weights after the first round are refused."""

from __future__ import annotations

import os

import numpy as np
import pytest
from conftest import TREE_FIELDS, assert_trees_equal

from oracle import REF_B200_SO, RefLib, TreeCfg

pytestmark = pytest.mark.gpu


def _data(seed=6, n=15_000, F=6):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    x = np.nan_to_num(X)
    y = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.1 * rng.standard_normal(n)).astype(np.float32)
    w = rng.uniform(0.1, 3.0, n).astype(np.float32)
    w[rng.random(n) < 0.05] = 0.0
    return X, y, w


def _same(a, b, where):
    for k in TREE_FIELDS:
        x, z = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert len(x) == len(z), f"{where} {k}"
        assert np.array_equal(x.view(np.uint8), z.view(np.uint8)), f"{where} {k}"


@pytest.mark.parametrize("grower,graph,subsample", [
    ("depthwise", True, 1.0), ("depthwise", False, 1.0), ("levelwise", True, 1.0),
    ("leafwise", False, 1.0), ("depthwise", True, 0.75), ("leafwise", False, 0.75)])
def test_weighted_fit_matches_reference(bb, ref, grower, graph, subsample):
    X, y, w = _data()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off, weights=w)
    tc = dict(grower=grower, max_depth=6, max_leaves=31)
    m = ref.train(ds, TreeCfg(n_iters=8, learning_rate=0.1, subsample=subsample,
                              random_seed=4, **tc))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(learning_rate=0.1, use_graph=graph,
                                            subsample=subsample, random_seed=4, **tc),
                   max_trees=8, weights=w)
    b.update(8)
    for i in range(8):
        if grower == "levelwise":
            for x, z in zip(bb.oblivious_tables(b.tree(i)), m.oblivious(i)):
                assert np.array_equal(np.asarray(x).view(np.uint8),
                                      np.asarray(z).view(np.uint8)), i
        else:
            _same(b.tree(i), m.tree(i), f"tree {i}")
    assert np.array_equal(bb.predict(plane, b.trees(), b.init_score, 0.1), m.predict_binned(ds))


def test_weighted_softmax_round_matches_reference(bb, ref):
    from bonsai_b200 import synth
    K = 3
    X, y = synth.multiclass_onehot(n=10_000, n_classes=K)
    w = np.random.Generator(np.random.PCG64(2)).uniform(0.2, 2.0, len(y)).astype(np.float32)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off, weights=w)
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=K, max_depth=5, n_iters=1,
                              learning_rate=0.1))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K, max_depth=5,
                                            learning_rate=0.1, use_graph=True),
                   max_trees=1, weights=w)
    b.update(1)
    assert np.array_equal(b.init_scores, m.init_scores())
    for k in range(K):
        _same(b.tree(k), m.tree(k), f"class {k}")


def test_weighted_reference_booster_over_dropin_grower(bb):
    if not os.path.exists(REF_B200_SO):
        pytest.skip("the drop-in harness is not built (make -C oracle dropin)")
    dref = RefLib(REF_B200_SO)
    X, y, w = _data(seed=7, n=8_000)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off, weights=w)
    tc = TreeCfg(max_depth=5, n_iters=10, learning_rate=0.1)
    cpu, gpu = dref.train(ds, tc), dref.train_b200(ds, tc)
    for i in range(10):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")


def test_unit_weights_are_the_unweighted_fit(bb):
    X, y, _ = _data(seed=8, n=5_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    p = bb.TrainParams(max_depth=5, use_graph=True, hist_mode="int8", seed=1)
    a = bb.Booster(plane, y, p, max_trees=5)
    c = bb.Booster(plane, y, p, max_trees=5, weights=np.ones(len(y), np.float32))
    a.update(5)
    c.update(5)
    for i in range(5):
        _same(a.tree(i), c.tree(i), f"tree {i}")
    assert np.array_equal(a.scores().view(np.uint32), c.scores().view(np.uint32))


def test_weights_after_the_first_round_are_refused(bb):
    X, y, w = _data(seed=9, n=2_000)
    cuts, off = bb.fit_cuts(X)
    b = bb.Booster(bb.Plane(X, cuts, off), y, bb.TrainParams(max_depth=3), max_trees=3)
    b.update(1)
    with pytest.raises(bb.BonsaiError):
        b.set_weights(w)
