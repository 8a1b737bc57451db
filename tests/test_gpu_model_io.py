"""Model files on the device path: boosters trained here (depthwise, levelwise,
leafwise, softmax) saved in the reference's format v7 and loaded back give
the same trees field for field (split bins recovered from the thresholds) and
the same predictions; a levelwise fit's ObliviousTree records equal the
reference's own (its level splits and leaf table, and the level gains and
leaf covers its dense_equivalent carries, src/tree.cpp:64-117); the
reference's committed models (tests/golden/model_v7_*.bonsai) predict through
this package's plan exactly as the oracle's bin-space walk and a float-space
walk of DenseTree::leaf_for (src/tree.cpp:18-38: x <= threshold, NaN by
default_left) predict them."""

from __future__ import annotations

import os

import numpy as np
import pytest
from conftest import TREE_FIELDS

from bonsai_b200 import model as M
from oracle import TreeCfg

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _data(seed=12, n=8_000, F=6):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    x = np.nan_to_num(X)
    y = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.1 * rng.standard_normal(n)).astype(np.float32)
    return X, y


def _same(a, b, where):
    for k in TREE_FIELDS + ("split_bin",):
        x, z = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert np.array_equal(x.view(np.uint8), z.view(np.uint8)), f"{where} {k}"
    assert (a.depth, a.n_leaves) == (b.depth, b.n_leaves), where


@pytest.mark.parametrize("params", [
    dict(grower="depthwise", max_depth=6),
    dict(grower="levelwise", max_depth=5),
    dict(grower="leafwise", max_leaves=31, max_depth=12),
    dict(objective="softmax", n_classes=3, max_depth=4),
])
def test_booster_saves_and_loads(bb, tmp_path, params):
    X, y = _data()
    if params.get("objective") == "softmax":
        y = np.floor(np.clip(y + 1.5, 0, 2.99)).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    p = bb.TrainParams(learning_rate=0.1, use_graph=params.get("grower") != "leafwise",
                       **params)
    b = bb.Booster(plane, y, p, max_trees=6 * max(1, params.get("n_classes", 1)))
    b.update(6)
    m = M.from_booster(b, cuts, off)
    path = str(tmp_path / "fit.bonsai")
    m.save(path)
    back = M.load(path)
    assert back.objective == m.objective and back.grower == m.grower
    assert np.array_equal(back.init_scores, b.init_scores)
    assert len(back.trees) == b.n_trees
    for i, (t, u) in enumerate(zip(b.trees(), back.trees)):
        _same(u, t, f"tree {i}")
    for k in range(back.n_classes):
        got = bb.PredictPlan(plane, back.class_trees(k), float(back.init_scores[k]),
                             back.learning_rate).run(plane)
        want = bb.predict(plane, b.trees()[k::back.n_classes], float(b.init_scores[k]), 0.1)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), k
    # the file is what the encoder makes of the document, byte for byte
    with open(path, "rb") as f:
        assert f.read() == M.packb(back.document())


def test_levelwise_records_are_the_references(bb, ref):
    X, y = _data(seed=13)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    r = ref.train(ds, TreeCfg(grower="levelwise", max_depth=5, n_iters=4, learning_rate=0.1))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(grower="levelwise", max_depth=5, learning_rate=0.1,
                                            use_graph=True), max_trees=4)
    b.update(4)
    for i in range(4):
        j = M.oblivious_to_json(b.tree(i))
        f, thr, dl, leaves = r.oblivious(i)
        assert [s["feature_id"] for s in j["splits"]] == f.tolist()
        assert np.array_equal(np.float32([s["threshold"] for s in j["splits"]]), thr)
        assert [int(s["default_left"]) for s in j["splits"]] == dl.tolist()
        assert np.array_equal(np.float32(j["leaves"]), leaves)
        # the reference's dense_equivalent: preorder, level gains on the left spine,
        # leaf covers in path order
        rt = r.tree(i)
        spine, n = [], 0
        while rt.feature[n] != M.LEAF:
            spine.append(rt.gains[n])
            n = int(rt.left[n])
        assert np.array_equal(np.float32(j["gains"]), np.float32(spine))
        assert np.array_equal(np.float32(j["covers"]), rt.covers[rt.feature == M.LEAF])


def _float_walk(t, X):
    out = np.zeros(len(X), np.float32)
    for r in range(len(X)):
        i = 0
        while t.feature[i] != M.LEAF:
            v = X[r, t.feature[i]]
            left = (not np.isnan(v) and v <= t.value[i]) or (np.isnan(v) and t.default_left[i])
            i = int(t.left[i] if left else t.right[i])
        out[r] = t.value[i]
    return out


@pytest.mark.parametrize("kind", ["regressor", "softmax"])
def test_reference_models_predict(bb, orc, kind):
    m = M.load(os.path.join(GOLDEN, f"model_v7_{kind}.bonsai"))
    F = len(m.cut_off) - 1
    rng = np.random.Generator(np.random.PCG64(31))
    X = (rng.standard_normal((3_000, F)) * 1.5 + 0.5).astype(np.float32)
    X[rng.random(X.shape) < 0.05] = np.nan
    plane = bb.Plane(X, m.cuts, m.cut_off)
    codes = plane.bins()
    nb = np.diff(m.cut_off).astype(np.uint32)
    for k in range(m.n_classes):
        trees = m.class_trees(k)
        init = float(m.init_scores[k])
        got = bb.PredictPlan(plane, trees, init, m.learning_rate).run(plane)
        want = orc.predict_binned(codes, nb, trees, init, m.learning_rate)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), k
        raw = np.zeros(len(X), np.float32)
        for t in trees:
            raw = (raw + _float_walk(t, X)).astype(np.float32)
        fw = (np.float32(init) + np.float32(m.learning_rate) * raw).astype(np.float32)
        np.testing.assert_allclose(got, fw, rtol=1e-6, atol=1e-6)
