"""Regenerates the golden fixtures in this folder from the reference itself.

Runs the reference's own CPU implementation (oracle/_ref/libbonsai_ref.so,
compiled from the reference sources by oracle/Makefile) on seeded synthetic
inputs and stores inputs and outputs as .npz:

  small_regression.npz   20,640 x 8 regression: cuts, bin codes, 100 MSE
                         depthwise trees (depth 6, lr 0.1), training-set
                         predictions, tree 0's per-row leaf ids, the
                         reference's binned TreeSHAP contributions of the
                         first 1,024 rows
  missing_values.npz     4,096 x 6 with NaN columns and duplicate-heavy
                         values (the reference's test_cuda_grower scenario
                         shape): cuts, bins, one tree from fixed gradients
                         with its per-row values/leaf ids, 20 logloss trees
                         and their binned TreeSHAP contributions
  split_cases.npz        hand-built histograms and the reference finder's
                         chosen split for each (the test_split_node cases)
  levelwise.npz          the levelwise (oblivious) grower: one depth-7 tree
                         from fixed gradients over the missing-values data
                         (min_child_hess 5: infeasible nodes) with its per-row
                         values, and 20 MSE rounds at depth 6 on the small
                         regression data with their training predictions;
                         trees as level tables (features, thresholds,
                         default directions, leaf values)

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from bonsai_b200 import synth  # noqa: E402
from oracle import RefLib, TreeCfg  # noqa: E402

TREE_KEYS = ("feature", "value", "left", "right", "default_left", "gains", "covers")


def pack_trees(trees):
    out = {}
    sizes = np.array([len(t.feature) for t in trees], np.uint32)
    out["tree_sizes"] = sizes
    for k in TREE_KEYS:
        out["tree_" + k] = np.concatenate([getattr(t, k) for t in trees])
    return out


def missing_values_data(n=4096, seed=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = np.empty((n, 6), np.float32)
    X[:, 0] = rng.standard_normal(n)
    X[:, 1] = rng.integers(0, 5, n)               # duplicate-heavy
    X[:, 2] = rng.lognormal(0, 1, n)
    X[rng.random(n) < 0.3, 2] = np.nan            # 30% missing
    X[:, 3] = np.round(rng.standard_normal(n), 1)
    X[:, 4] = rng.random(n)
    X[rng.random(n) < 0.05, 4] = np.nan
    X[:, 5] = np.where(rng.random(n) < 0.9, 0.0, rng.standard_normal(n))  # heavy zero
    y = (X[:, 0] + np.nan_to_num(X[:, 2]) * (X[:, 1] > 2) + 0.3 * X[:, 5]
         + rng.normal(0, 0.1, n)).astype(np.float32)
    return X, y


def split_cases():
    """(hist [F, n_bins, 2], n_rows, lambda_l2, min_child_hess, min_data) cases."""
    cases = []
    # an obvious cut: left bins negative gradient, right positive
    h = np.zeros((1, 6, 2), np.float32)
    h[0, :, 1] = 10.0
    h[0, :2, 0] = -5.0
    h[0, 2:4, 0] = 5.0
    cases.append((h, 40, 1.0, 1.0, 1))
    # missing mass that must route right (default_left = false)
    h = np.zeros((1, 6, 2), np.float32)
    h[0, :4, 1] = 5.0
    h[0, :2, 0] = -4.0
    h[0, 2:4, 0] = 4.0
    h[0, 5] = (6.0, 5.0)
    cases.append((h, 60, 1.0, 1.0, 1))
    # two features, a tie in gain: the lower feature id must win
    h = np.zeros((2, 5, 2), np.float32)
    h[:, :, 1] = 3.0
    h[:, :2, 0] = -2.0
    h[:, 2:, 0] = 2.0
    cases.append((h, 40, 1.0, 1.0, 1))
    # min_child_hess gates every cut
    h = np.zeros((1, 5, 2), np.float32)
    h[0, :, 1] = 0.5
    h[0, :2, 0] = -1.0
    cases.append((h, 40, 1.0, 3.0, 1))
    # too few rows for two children of min_data_in_leaf
    h = np.zeros((1, 5, 2), np.float32)
    h[0, :, 1] = 5.0
    h[0, :2, 0] = -3.0
    cases.append((h, 30, 1.0, 1.0, 20))
    # lambda_l2 = 0 with an empty side
    h = np.zeros((1, 6, 2), np.float32)
    h[0, 1:4, 1] = 2.0
    h[0, 1, 0] = -3.0
    h[0, 3, 0] = 3.0
    cases.append((h, 40, 0.0, 0.0, 1))
    # random dense histograms
    rng = np.random.Generator(np.random.PCG64(11))
    for _ in range(6):
        F, nb = 4, int(rng.integers(3, 40))
        h = np.zeros((F, nb, 2), np.float32)
        h[:, :, 0] = rng.normal(0, 3, (F, nb)).astype(np.float32)
        h[:, :, 1] = rng.uniform(0.1, 4, (F, nb)).astype(np.float32)
        # every feature sums the same rows: share the totals through the last bin
        tg, th = h[0, :, 0].sum(dtype=np.float64), h[0, :, 1].sum(dtype=np.float64)
        for f in range(1, F):
            h[f, -1, 0] += np.float32(tg - h[f, :, 0].sum(dtype=np.float64))
            h[f, -1, 1] = max(np.float32(0.0), np.float32(h[f, -1, 1] + th - h[f, :, 1].sum(dtype=np.float64)))
        cases.append((h, 500, 1.0, 1.0, 20))
    return cases


def main():
    ref = RefLib()
    # --- small regression
    X, y = synth.regression_small()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    bins = ds.bins()
    tc = TreeCfg(max_depth=6, n_iters=100, learning_rate=0.1)
    m = ref.train(ds, tc)
    trees = m.trees()
    pred = m.predict_binned(ds)
    contribs = m.contribs_binned(ds)[:1024]
    g = np.zeros(len(y), np.float32)
    h = np.ones(len(y), np.float32)
    init = m.init_score()
    g[:] = np.float32(init) - y
    _, v0, ids0 = ref.grow_tree(ds, TreeCfg(max_depth=6), g, h)[:3]
    np.savez_compressed(os.path.join(HERE, "small_regression.npz"), cuts=cuts, cut_off=off,
                        bins=bins.astype(np.uint8), init=np.float32(init), pred=pred,
                        tree0_values=v0, tree0_leaf_ids=ids0, contribs=contribs,
                        **pack_trees(trees))
    # --- missing values
    X, y = missing_values_data()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    rng = np.random.Generator(np.random.PCG64(5))
    g = rng.normal(0, 1, len(y)).astype(np.float32)
    hh = rng.uniform(0.2, 1.0, len(y)).astype(np.float32)
    t, vals, ids, _ = ref.grow_tree(ds, TreeCfg(max_depth=5, min_data_in_leaf=10), g, hh)
    yb = (y > np.median(y)).astype(np.float32)
    dsb = ref.dataset(X, yb, cuts, off)
    mb = ref.train(dsb, TreeCfg(objective="logloss", max_depth=4, n_iters=20))
    np.savez_compressed(os.path.join(HERE, "missing_values.npz"), X=X, y=y, yb=yb,
                        cuts=cuts, cut_off=off, bins=ds.bins(), grad=g, hess=hh,
                        values=vals, leaf_ids=ids, logloss_init=np.float32(mb.init_score()),
                        logloss_pred=mb.predict_binned(dsb),
                        ll_contribs=mb.contribs_binned(dsb),
                        **{"one_" + k: v for k, v in pack_trees([t]).items()},
                        **{"ll_" + k: v for k, v in pack_trees(mb.trees()).items()})
    # --- split finder cases
    out = {}
    for i, (hist, n_rows, l2, mch, mdl) in enumerate(split_cases()):
        s = ref.find_split(hist, n_rows, TreeCfg(lambda_l2=l2, min_child_hess=mch,
                                                 min_data_in_leaf=mdl))
        out[f"hist{i}"] = hist
        out[f"meta{i}"] = np.array([n_rows, l2, mch, mdl], np.float64)
        out[f"split{i}"] = np.array([s["gain"], s["feature"], s["bin"], s["default_left"],
                                     s["valid"]], np.float64)
    np.savez_compressed(os.path.join(HERE, "split_cases.npz"), n=len(split_cases()), **out)
    # --- levelwise
    X, y = missing_values_data()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    rng = np.random.Generator(np.random.PCG64(5))
    g = rng.normal(0, 1, len(y)).astype(np.float32)
    hh = rng.uniform(0.2, 1.0, len(y)).astype(np.float32)
    _, lv_vals, _, m1 = ref.grow_tree(ds, TreeCfg(grower="levelwise", max_depth=7,
                                                  min_child_hess=5.0), g, hh)
    f1, t1, d1, l1 = m1.oblivious(0)
    Xs, ys = synth.regression_small()
    cs, os_ = ref.fit_cuts(Xs)
    dss = ref.dataset(Xs, ys, cs, os_)
    mb = ref.train(dss, TreeCfg(grower="levelwise", max_depth=6, n_iters=20))
    lv = {}
    for i in range(20):
        f, t, d, lf = mb.oblivious(i)
        lv[f"boost{i}_features"] = f
        lv[f"boost{i}_thresholds"] = t
        lv[f"boost{i}_default_left"] = d
        lv[f"boost{i}_leaves"] = lf
    np.savez_compressed(os.path.join(HERE, "levelwise.npz"), grad=g, hess=hh,
                        one_values=lv_vals, one_features=f1, one_thresholds=t1,
                        one_default_left=d1, one_leaves=l1, boost_init=np.float32(mb.init_score()),
                        boost_pred=mb.predict_binned(dss), **lv)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
