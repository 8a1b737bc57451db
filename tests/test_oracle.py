"""The oracle (oracle/bonsai_oracle.c) pinned against the reference: golden
fixtures produced by the reference's own CPU grower (tests/golden), and, where
the reference library is built, live comparisons on fresh seeded inputs."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import assert_trees_equal, level_gains, load_golden, unpack_trees

from oracle import Oracle, TreeCfg, orc_find_split


def test_transform_matches_golden(orc: Oracle):
    for name in ("missing_values.npz",):
        d = load_golden(name)
        bins = orc.transform(d["X"], d["cuts"], d["cut_off"])
        assert np.array_equal(bins, d["bins"])


def test_depthwise_100_trees_match_golden(orc: Oracle):
    d = load_golden("small_regression.npz")
    bins = d["bins"].astype(np.uint16)
    from bonsai_b200 import synth
    _, y = synth.regression_small()
    nb = np.diff(d["cut_off"])
    trees, init, _ = orc.train(bins, nb, d["cuts"], d["cut_off"], y,
                               TreeCfg(max_depth=6, n_iters=100, learning_rate=0.1))
    assert np.float32(init) == d["init"]
    for i, (a, b) in enumerate(zip(trees, unpack_trees(d))):
        assert_trees_equal(a, b, f"tree {i}")
    pred = orc.predict_binned(bins, nb, trees, init, 0.1)
    assert np.array_equal(pred, d["pred"])


def test_one_tree_with_missing_values_matches_golden(orc: Oracle):
    d = load_golden("missing_values.npz")
    nb = np.diff(d["cut_off"])
    t, vals, ids = orc.grow(d["bins"], nb, d["cuts"], d["cut_off"], d["grad"], d["hess"],
                            TreeCfg(max_depth=5, min_data_in_leaf=10))
    assert_trees_equal(t, unpack_trees(d, "one_")[0])
    assert np.array_equal(vals, d["values"])
    assert np.array_equal(ids, d["leaf_ids"])


def test_logloss_trees_match_golden(orc: Oracle):
    d = load_golden("missing_values.npz")
    nb = np.diff(d["cut_off"])
    tc = TreeCfg(objective="logloss", max_depth=4, n_iters=20)
    trees, init, _ = orc.train(d["bins"], nb, d["cuts"], d["cut_off"], d["yb"], tc)
    assert np.float32(init) == d["logloss_init"]
    for i, (a, b) in enumerate(zip(trees, unpack_trees(d, "ll_"))):
        assert_trees_equal(a, b, f"logloss tree {i}")


def test_split_finder_matches_golden_cases(orc: Oracle):
    d = load_golden("split_cases.npz")
    for i in range(int(d["n"])):
        n_rows, l2, mch, mdl = d[f"meta{i}"]
        tc = TreeCfg(lambda_l2=float(l2), min_child_hess=float(mch),
                     min_data_in_leaf=int(mdl))
        s = orc_find_split(orc, d[f"hist{i}"], int(n_rows), tc)
        gain, feat, b, dl, valid = d[f"split{i}"]
        assert s["valid"] == int(valid), f"case {i}"
        if valid:
            assert (s["feature"], s["bin"], s["default_left"]) == (int(feat), int(b), int(dl)), f"case {i}"
            assert s["gain"] == gain, f"case {i}"


def _random_case(seed, n=3000, F=5):
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
])
def test_live_grow_matches_reference(orc: Oracle, ref, seed, cfg):
    X, g, h = _random_case(seed)
    cuts, off = ref.fit_cuts(X, max_bin=64)
    ds = ref.dataset(X, g, cuts, off)
    tc = TreeCfg(**cfg)
    rt, rv, rids, _ = ref.grow_tree(ds, tc, g, h)
    ot, ov, oids = orc.grow(ds.bins(), np.diff(off), cuts, off, g, h, tc)
    assert_trees_equal(ot, rt, f"seed {seed}")
    assert np.array_equal(ov, rv)
    assert np.array_equal(oids, rids)


def test_live_sampled_rows_match_reference(orc: Oracle, ref):
    X, g, h = _random_case(9, n=4000)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, g, cuts, off)
    rows = np.flatnonzero(np.random.Generator(np.random.PCG64(3)).random(len(g)) < 0.7)
    tc = TreeCfg(max_depth=5)
    rt, rv, rids, _ = ref.grow_tree(ds, tc, g, h, rows)
    ot, ov, oids = orc.grow(ds.bins(), np.diff(off), cuts, off, g, h, tc, rows=rows)
    assert_trees_equal(ot, rt)
    assert np.array_equal(ov, rv)
    assert np.array_equal(oids, rids)


# ---- levelwise (ObliviousGrower) ------------------------------------------------

def _tables_equal(mine, theirs, where=""):
    for a, b, what in zip(mine, theirs, ("features", "thresholds", "default_left", "leaves")):
        a, b = np.asarray(a), np.asarray(b)
        assert a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8)), (
            f"{where} {what}")


def test_levelwise_tree_matches_golden(orc: Oracle):
    from bonsai_b200 import oblivious_tables
    d = load_golden("missing_values.npz")
    lv = load_golden("levelwise.npz")
    nb = np.diff(d["cut_off"])
    t, vals, _ = orc.grow(d["bins"], nb, d["cuts"], d["cut_off"], lv["grad"], lv["hess"],
                          TreeCfg(grower="levelwise", max_depth=7, min_child_hess=5.0))
    _tables_equal(oblivious_tables(t), (lv["one_features"], lv["one_thresholds"],
                                        lv["one_default_left"], lv["one_leaves"]))
    assert np.array_equal(vals.view(np.uint32), lv["one_values"].view(np.uint32))


def test_levelwise_boosting_matches_golden(orc: Oracle):
    from bonsai_b200 import oblivious_tables, synth
    d = load_golden("small_regression.npz")
    lv = load_golden("levelwise.npz")
    _, y = synth.regression_small()
    bins = d["bins"].astype(np.uint16)
    nb = np.diff(d["cut_off"])
    trees, init, _ = orc.train(bins, nb, d["cuts"], d["cut_off"], y,
                               TreeCfg(grower="levelwise", max_depth=6, n_iters=20))
    assert np.float32(init) == lv["boost_init"]
    for i, t in enumerate(trees):
        _tables_equal(oblivious_tables(t), (lv[f"boost{i}_features"], lv[f"boost{i}_thresholds"],
                                            lv[f"boost{i}_default_left"], lv[f"boost{i}_leaves"]),
                      f"tree {i}")
    assert np.array_equal(orc.predict_binned(bins, nb, trees, init, 0.1), lv["boost_pred"])


@pytest.mark.parametrize("seed,cfg", [
    (11, dict(max_depth=8)),
    (12, dict(max_depth=8, min_child_hess=4.0, lambda_l2=0.0)),
    (13, dict(max_depth=4, lambda_l1=0.7, min_gain_to_split=0.3)),
])
def test_levelwise_live_matches_reference(orc: Oracle, ref, seed, cfg):
    from bonsai_b200 import oblivious_tables
    rng = np.random.Generator(np.random.PCG64(seed))
    n, F = 3000, 5
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random(n) < 0.15, 1] = np.nan
    X[:, 2] = np.round(X[:, 2])
    g = rng.normal(0, 1, n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, np.zeros(n, np.float32), cuts, off)
    tc = TreeCfg(grower="levelwise", **cfg)
    _, rvals, _, m = ref.grow_tree(ds, tc, g, h)
    t, vals, _ = orc.grow(ds.bins(), np.diff(off), cuts, off, g, h, tc)
    _tables_equal(oblivious_tables(t), m.oblivious(0))
    assert np.array_equal(level_gains(t).view(np.uint32), level_gains(m.tree(0)).view(np.uint32))
    assert np.array_equal(vals.view(np.uint32), rvals.view(np.uint32))
