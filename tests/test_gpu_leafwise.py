"""GPU parity of the leafwise grower (LeafwiseGrower, src/grower_impl.hpp:744-850,
over the leaf plane) against the reference's own CPU implementation: best-first
growth from a gain heap (the lower node id on a tie), child ids allocated at each
pop, demotion of a split whose partition empties a side, no children's split at
the depth cap, the max_leaves budget. The whole node table -- DenseTree fields,
gains and covers, demotion placeholders included -- and every row's leaf value
must match bit for bit."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg

pytestmark = pytest.mark.gpu


def _case(seed, n=6000, F=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[:, 1] = np.round(X[:, 1] * 2)
    X[rng.random(n) < 0.2, 2] = np.nan
    X[:, 3] = np.where(rng.random(n) < 0.7, 0.0, X[:, 3])
    g = rng.normal(0, 1, n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    return X, g, h


def _same(a, b, where=""):
    n = int(b.feature.shape[0])
    for k in TREE_FIELDS:
        x = np.asarray(getattr(a, k))[:n]
        y = np.asarray(getattr(b, k))
        assert len(np.asarray(getattr(a, k))) == n, f"{where} node count"
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (
            f"{where} {k} differs at {np.flatnonzero(x != y)[:8]}")


@pytest.mark.parametrize("seed,cfg", [
    (1, dict(max_leaves=31, max_depth=6)),
    (2, dict(max_leaves=255, max_depth=255, min_data_in_leaf=5)),
    (3, dict(max_leaves=64, max_depth=4)),                       # depth cap binds
    (4, dict(max_leaves=40, max_depth=12, lambda_l1=0.5, min_gain_to_split=0.2)),
    (5, dict(max_leaves=50, max_depth=10, min_child_hess=4.0, lambda_l2=0.0)),
    (6, dict(max_leaves=30, max_depth=8, monotone=[1, 0, -1])),
    (7, dict(max_leaves=1, max_depth=6)),                        # the root alone
])
def test_leafwise_tree_matches_reference(bb, ref, seed, cfg):
    X, g, h = _case(seed)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, np.zeros(len(X), np.float32), cuts, off)
    rt, rvals, rids, _ = ref.grow_tree(ds, TreeCfg(grower="leafwise", **cfg), g, h)
    plane = bb.Plane(X, cuts, off)
    t, vals, ids = bb.grow_tree(plane, bb.TrainParams(grower="leafwise", **cfg), g, h)
    _same(t, rt, f"seed {seed}")
    assert np.array_equal(vals.view(np.uint32), rvals.view(np.uint32))
    assert np.array_equal(ids, rids)


def test_leafwise_sampled_rows_and_u16_bins(bb, ref):
    X, g, h = _case(9, n=4000)
    cuts, off = ref.fit_cuts(X, max_bin=700)
    ds = ref.dataset(X, np.zeros(len(X), np.float32), cuts, off)
    rows = np.flatnonzero(np.random.Generator(np.random.PCG64(1)).random(len(X)) < 0.7)
    rows = rows.astype(np.uint32)
    tc = dict(max_leaves=48, max_depth=9)
    rt, rvals, _, _ = ref.grow_tree(ds, TreeCfg(grower="leafwise", **tc), g, h, rows=rows)
    plane = bb.Plane(X, cuts, off)
    assert not plane.u8
    t, vals, _ = bb.grow_tree(plane, bb.TrainParams(grower="leafwise", **tc), g, h, rows=rows)
    _same(t, rt)
    assert np.array_equal(vals[rows].view(np.uint32), rvals[rows].view(np.uint32))


def test_leafwise_booster_matches_reference(bb, ref):
    from bonsai_b200 import synth
    X, y = synth.regression_small()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    tc = TreeCfg(grower="leafwise", max_leaves=31, max_depth=10, n_iters=15,
                 learning_rate=0.1)
    m = ref.train(ds, tc)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(grower="leafwise", max_leaves=31, max_depth=10,
                                            learning_rate=0.1, use_graph=True), max_trees=15)
    b.update(15)
    for i, rt in enumerate(m.trees()):
        _same(b.tree(i), rt, f"tree {i}")
    assert np.array_equal(bb.predict(plane, b.trees(), b.init_score, 0.1), m.predict_binned(ds))


def test_leafwise_quantised_close_to_plain(bb):
    rng = np.random.Generator(np.random.PCG64(12))
    n, F = 150_000, 10
    X = rng.standard_normal((n, F)).astype(np.float32)
    y = ((X[:, 0] + X[:, 1] * X[:, 2] + 0.3 * rng.standard_normal(n)) > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    out = {}
    for mode in ("exact", "int8"):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", grower="leafwise",
                                                max_leaves=63, max_depth=20, hist_mode=mode,
                                                seed=3), max_trees=20)
        b.update(20)
        out[mode] = b.scores()

    def auc(p):
        order = np.argsort(p, kind="stable")
        r = np.empty(n); r[order] = np.arange(1, n + 1)
        pos = y > 0.5
        return (r[pos].sum() - pos.sum() * (pos.sum() + 1) / 2) / (pos.sum() * (~pos).sum())
    assert abs(auc(out["exact"]) - auc(out["int8"])) < 2e-3
