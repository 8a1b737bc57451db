"""GPU parity of the plain (exact) form against the reference: bin codes,
trees (features, thresholds, default directions, gains, covers, leaf values),
per-row leaf assignments and predictions bit-exact against the golden
fixtures the reference produced and against the oracle restatement."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import assert_trees_equal, load_golden, unpack_trees

from oracle import TreeCfg

pytestmark = pytest.mark.gpu


def _params(bb, **kw):
    return bb.TrainParams(**kw)


def test_ingest_small_regression_bit_exact(bb):
    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    X, _ = synth.regression_small()
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    assert plane.u8
    assert np.array_equal(plane.bins(), d["bins"].astype(np.uint16))


def test_ingest_missing_values_bit_exact(bb):
    d = load_golden("missing_values.npz")
    plane = bb.Plane(d["X"], d["cuts"], d["cut_off"])
    assert np.array_equal(plane.bins(), d["bins"])


def test_ingest_u16_and_ragged_rows(bb, orc):
    rng = np.random.Generator(np.random.PCG64(17))
    for n, F in [(1, 3), (257, 5), (3001, 33), (70000, 7)]:
        X = rng.standard_normal((n, F)).astype(np.float32)
        X[rng.random((n, F)) < 0.1] = np.nan
        X[0, 0] = np.inf
        X[-1, -1] = -np.inf
        cuts, off = bb.fit_cuts(X, max_bin=1000)
        plane = bb.Plane(X, cuts, off)
        assert plane.u8 == (np.diff(off).max() <= 256)
        assert np.array_equal(plane.bins(), orc.transform(X, cuts, off)), (n, F)


def test_ingest_from_device_memory(bb, orc):
    import torch
    rng = np.random.Generator(np.random.PCG64(3))
    X = rng.standard_normal((5000, 12)).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    Xd = torch.from_numpy(X).cuda()
    plane = bb.Plane(Xd, cuts, off, x_on_device=True)
    assert np.array_equal(plane.bins(), orc.transform(X, cuts, off))


def test_one_tree_with_missing_values_bit_exact(bb):
    d = load_golden("missing_values.npz")
    plane = bb.Plane(d["X"], d["cuts"], d["cut_off"])
    t, vals, ids = bb.grow_tree(plane, _params(bb, max_depth=5, min_data_in_leaf=10),
                                d["grad"], d["hess"])
    assert_trees_equal(t, unpack_trees(d, "one_")[0])
    assert np.array_equal(vals, d["values"])
    assert np.array_equal(ids, d["leaf_ids"])


def _case(seed, n=3000, F=5):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[:, 1] = np.round(X[:, 1] * 2)
    X[rng.random(n) < 0.2, 2] = np.nan
    X[:, 3] = np.where(rng.random(n) < 0.7, 0.0, X[:, 3])
    g = rng.normal(0, 1, n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    return X, g, h


@pytest.mark.parametrize("seed,cfg", [
    (1, dict(max_depth=6, min_data_in_leaf=5)),
    (2, dict(max_depth=4, lambda_l1=0.5, lambda_l2=2.0)),
    (3, dict(max_depth=5, min_child_hess=3.0, min_gain_to_split=0.01)),
    (4, dict(max_depth=6, min_data_in_leaf=2, monotone=[1, 0, -1, 0, 1])),
    (5, dict(max_depth=3, lambda_l2=0.0, min_child_hess=0.0, min_data_in_leaf=1)),
    (6, dict(max_depth=8, min_data_in_leaf=1)),
    (7, dict(max_depth=0)),
    (8, dict(max_depth=1)),
])
def test_grow_tree_matches_oracle(bb, orc, seed, cfg):
    X, g, h = _case(seed)
    cuts, off = bb.fit_cuts(X, max_bin=64)
    plane = bb.Plane(X, cuts, off)
    tc = TreeCfg(**cfg)
    ot, ov, oids = orc.grow(plane.bins(), np.diff(off), cuts, off, g, h, tc)
    mono = cfg.get("monotone", [])
    p = _params(bb, **{k: v for k, v in cfg.items() if k != "monotone"}, monotone=mono)
    t, v, ids = bb.grow_tree(plane, p, g, h)
    assert_trees_equal(t, ot, f"seed {seed}")
    assert np.array_equal(v, ov)
    assert np.array_equal(ids, oids)


def test_grow_tree_sampled_rows_and_feature_subset(bb, orc):
    X, g, h = _case(9, n=6000, F=7)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    rng = np.random.Generator(np.random.PCG64(4))
    rows = np.flatnonzero(rng.random(len(g)) < 0.6).astype(np.uint32)
    sel = np.array([1, 2, 4, 6], np.uint32)
    tc = TreeCfg(max_depth=6)
    ot, ov, oids = orc.grow(plane.bins(), np.diff(off), cuts, off, g, h, tc, rows=rows,
                            selected=sel)
    t, v, ids = bb.grow_tree(plane, _params(bb, max_depth=6, selected=list(sel)), g, h,
                             rows=rows)
    assert_trees_equal(t, ot)
    assert np.array_equal(v[rows], ov[rows])
    assert np.array_equal(ids[rows], oids[rows])


def test_u16_bins_tree_matches_oracle(bb, orc):
    X, g, h = _case(12, n=8000, F=4)
    cuts, off = bb.fit_cuts(X, max_bin=700)
    plane = bb.Plane(X, cuts, off)
    assert not plane.u8
    tc = TreeCfg(max_depth=5)
    ot, ov, oids = orc.grow(plane.bins(), np.diff(off), cuts, off, g, h, tc)
    t, v, ids = bb.grow_tree(plane, _params(bb, max_depth=5), g, h)
    assert_trees_equal(t, ot)
    assert np.array_equal(v, ov)


@pytest.mark.parametrize("use_graph", [False, True])
def test_booster_100_trees_bit_exact_vs_reference(bb, orc, use_graph):
    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    X, y = synth.regression_small()
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    b = bb.Booster(plane, y, _params(bb, max_depth=6, learning_rate=0.1,
                                     use_graph=use_graph), max_trees=100)
    b.update(100)
    assert np.float32(b.init_score) == d["init"]
    gold = unpack_trees(d)
    for i in range(100):
        assert_trees_equal(b.tree(i), gold[i], f"tree {i}")
    trees = b.trees()                      # all 100 in one transfer per array
    for i in range(100):
        assert_trees_equal(trees[i], gold[i], f"bulk tree {i}")
    assert [len(t.feature) for t in b.trees()[40:]] == [len(b.tree(i).feature)
                                                        for i in range(40, 100)]
    pred = bb.predict(plane, trees, b.init_score, 0.1)
    assert np.array_equal(pred, d["pred"])
    # the fused training-score update: scores[r] += lr * leaf, round by round
    _, _, scores = orc.train(d["bins"].astype(np.uint16), np.diff(d["cut_off"]), d["cuts"],
                             d["cut_off"], y, TreeCfg(max_depth=6, n_iters=100,
                                                      learning_rate=0.1))
    assert np.array_equal(b.scores(), scores)


def test_booster_logloss_close_to_reference(bb):
    d = load_golden("missing_values.npz")
    plane = bb.Plane(d["X"], d["cuts"], d["cut_off"])
    b = bb.Booster(plane, d["yb"], _params(bb, objective="logloss", max_depth=4,
                                           learning_rate=0.1), max_trees=20)
    b.update(20)
    assert np.float32(b.init_score) == d["logloss_init"]
    pred = bb.predict(plane, b.trees(), b.init_score, 0.1)
    # device expf is not glibc's expf: gradients may differ in the last ulp
    np.testing.assert_allclose(pred, d["logloss_pred"], rtol=1e-4, atol=1e-4)
    gold = unpack_trees(d, "ll_")
    same = sum(np.array_equal(b.tree(i).feature, gold[i].feature) for i in range(20))
    assert same >= 18


def test_determinism_bit_identical_runs(bb):
    X, g, h = _case(21, n=50000, F=9)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    y = (g > 0).astype(np.float32)
    outs = []
    for _ in range(2):
        b = bb.Booster(plane, y, _params(bb, objective="logloss", max_depth=7), max_trees=5)
        b.update(5)
        outs.append((b.scores(), [b.tree(i) for i in range(5)]))
    assert np.array_equal(outs[0][0], outs[1][0])
    for a, c in zip(outs[0][1], outs[1][1]):
        assert_trees_equal(a, c)


def test_large_tree_structural_invariants(bb):
    """At a size the oracle is slow on: covers add up, leaf ids agree with the
    bin-space walk, and the fused scores equal predict."""
    rng = np.random.Generator(np.random.PCG64(99))
    n, F = 1_500_000, 16
    X = rng.standard_normal((n, F)).astype(np.float32)
    y = (X[:, 0] + X[:, 1] * X[:, 2] > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, _params(bb, objective="logloss", max_depth=8,
                                     record_leaf_ids=True), max_trees=3)
    b.update(3)
    trees = b.trees()
    for t in trees:
        internal = t.feature != bb.LEAF
        for i in np.flatnonzero(internal):
            assert t.covers[t.left[i]] + t.covers[t.right[i]] == t.covers[i]
    assert trees[0].covers[0] == n
    # the fused score update equals init + sum of lr * leaf(tree) round by round
    s = np.full(n, np.float32(b.init_score), np.float32)
    for t in trees:
        v = bb.predict(plane, [t], 0.0, 1.0)
        s = (s + np.float32(0.1) * v).astype(np.float32)
    np.testing.assert_array_equal(b.scores(), s)
    ids = b.leaf_ids()
    t = trees[-1]
    v = bb.predict(plane, [t], 0.0, 1.0)
    np.testing.assert_array_equal(t.value[ids], v)
