"""GPU parity of the levelwise grower (ObliviousGrower, src/grower_impl.hpp:579-720)
against the reference's own CPU implementation: one split per level chosen over the
whole frontier (update_best_for_feature_for_level, src/split.cpp:164-235, infeasible
nodes contributing their parent score), broadcast to every node, empty children kept.
Trees are compared as the reference's ObliviousTree tables (level features,
thresholds, default directions, leaf values, level gains) and per-row leaf values, bit
for bit."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import level_gains

from oracle import TreeCfg

pytestmark = pytest.mark.gpu


def _case(seed, n=4000, F=6):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[:, 1] = np.round(X[:, 1] * 2)
    X[rng.random(n) < 0.2, 2] = np.nan
    X[:, 3] = np.where(rng.random(n) < 0.7, 0.0, X[:, 3])
    g = rng.normal(0, 1, n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    return X, g, h


def _ref_tables(m):
    f, thr, dl, leaves = m.oblivious(0)
    return f, thr, dl, leaves


@pytest.mark.parametrize("seed,cfg", [
    (1, dict(max_depth=6)),
    (2, dict(max_depth=8, min_child_hess=5.0)),          # infeasible nodes (issue #60)
    (3, dict(max_depth=8, min_child_hess=0.0, lambda_l2=0.0)),
    (4, dict(max_depth=3, lambda_l1=0.5, min_gain_to_split=0.5)),
    (5, dict(max_depth=1)),
    (6, dict(max_depth=7, min_data_in_leaf=400)),        # no effect on a level split
])
def test_levelwise_tree_matches_reference(bb, ref, seed, cfg):
    X, g, h = _case(seed)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, np.zeros(len(X), np.float32), cuts, off)
    _, rvals, _, m = ref.grow_tree(ds, TreeCfg(grower="levelwise", **cfg), g, h)
    plane = bb.Plane(X, cuts, off)
    params = bb.TrainParams(grower="levelwise", **cfg)
    t, vals, _ = bb.grow_tree(plane, params, g, h)
    mine = bb.oblivious_tables(t)
    theirs = _ref_tables(m)
    for a, b, what in zip(mine, theirs, ("features", "thresholds", "default_left", "leaves")):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8)), what
    assert np.array_equal(level_gains(t).view(np.uint32), level_gains(m.tree(0)).view(np.uint32))
    assert np.array_equal(vals.view(np.uint32), rvals.view(np.uint32))


def test_levelwise_u16_bins_matches_reference(bb, ref):
    X, g, h = _case(9, n=3000)
    cuts, off = ref.fit_cuts(X, max_bin=700)
    ds = ref.dataset(X, np.zeros(len(X), np.float32), cuts, off)
    _, rvals, _, m = ref.grow_tree(ds, TreeCfg(grower="levelwise", max_depth=5), g, h)
    plane = bb.Plane(X, cuts, off)
    assert not plane.u8
    t, vals, _ = bb.grow_tree(plane, bb.TrainParams(grower="levelwise", max_depth=5), g, h)
    for a, b in zip(bb.oblivious_tables(t), _ref_tables(m)):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert np.array_equal(vals.view(np.uint32), rvals.view(np.uint32))


@pytest.mark.parametrize("use_graph", [False, True])
def test_levelwise_booster_matches_reference(bb, ref, use_graph):
    from bonsai_b200 import synth
    X, y = synth.regression_small()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    tc = TreeCfg(grower="levelwise", max_depth=6, n_iters=30, learning_rate=0.1)
    m = ref.train(ds, tc)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(grower="levelwise", max_depth=6,
                                            learning_rate=0.1, use_graph=use_graph),
                   max_trees=30)
    b.update(30)
    for i in range(30):
        mine = bb.oblivious_tables(b.tree(i))
        theirs = m.oblivious(i)
        for a, c in zip(mine, theirs):
            assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(c).view(np.uint8)), i
        assert np.array_equal(level_gains(b.tree(i)).view(np.uint32),
                              level_gains(m.tree(i)).view(np.uint32)), i
    pred = bb.predict(plane, b.trees(), b.init_score, 0.1)
    assert np.array_equal(pred, m.predict_binned(ds))


def test_levelwise_rejects_monotone(bb):
    X, g, h = _case(1, n=500)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    with pytest.raises(bb.ConfigError):
        bb.grow_tree(plane, bb.TrainParams(grower="levelwise", monotone=[1]), g, h)


def test_levelwise_quantised_close_to_plain(bb):
    rng = np.random.Generator(np.random.PCG64(31))
    n, F = 200_000, 12
    X = rng.standard_normal((n, F)).astype(np.float32)
    y = ((X[:, 0] + X[:, 1] * X[:, 2] + 0.3 * rng.standard_normal(n)) > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    out = {}
    for mode in ("exact", "int8"):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", grower="levelwise",
                                                max_depth=6, hist_mode=mode, seed=5),
                       max_trees=30)
        b.update(30)
        out[mode] = b.scores()
    # same ranking quality: AUC within 2e-3
    def auc(p):
        order = np.argsort(p, kind="stable")
        r = np.empty(n); r[order] = np.arange(1, n + 1)
        pos = y > 0.5
        return (r[pos].sum() - pos.sum() * (pos.sum() + 1) / 2) / (pos.sum() * (~pos).sum())
    assert abs(auc(out["exact"]) - auc(out["int8"])) < 2e-3


def test_levelwise_tree_matches_golden(bb):
    from conftest import load_golden
    d = load_golden("missing_values.npz")
    lv = load_golden("levelwise.npz")
    plane = bb.Plane(d["X"], d["cuts"], d["cut_off"])
    t, vals, _ = bb.grow_tree(plane, bb.TrainParams(grower="levelwise", max_depth=7,
                                                    min_child_hess=5.0),
                              lv["grad"], lv["hess"])
    for a, b in zip(bb.oblivious_tables(t), (lv["one_features"], lv["one_thresholds"],
                                             lv["one_default_left"], lv["one_leaves"])):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert np.array_equal(vals.view(np.uint32), lv["one_values"].view(np.uint32))


def test_levelwise_booster_matches_golden(bb):
    from conftest import load_golden
    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    lv = load_golden("levelwise.npz")
    X, y = synth.regression_small()
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    b = bb.Booster(plane, y, bb.TrainParams(grower="levelwise", max_depth=6, use_graph=True),
                   max_trees=20)
    b.update(20)
    assert np.float32(b.init_score) == lv["boost_init"]
    for i in range(20):
        want = (lv[f"boost{i}_features"], lv[f"boost{i}_thresholds"],
                lv[f"boost{i}_default_left"], lv[f"boost{i}_leaves"])
        for a, c in zip(bb.oblivious_tables(b.tree(i)), want):
            assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(c).view(np.uint8)), i
    assert np.array_equal(bb.predict(plane, b.trees(), b.init_score, 0.1), lv["boost_pred"])
