"""Softmax multiclass boosting on the device (objective 2) against the
reference's MulticlassBooster (include/bonsai/multiclass_booster.hpp): per-class
log-prior init scores, one tree per class per round (round-major), the round's
softmax gradients g = p - 1[y == k], h = max(p (1 - p), 1e-6). The first round's
trees grow from identical gradients (init scores are per-class constants) and
must match bit for bit; later rounds differ only where the device's double exp
rounds differently from the host's, so the fit is compared by its raw scores."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg

pytestmark = pytest.mark.gpu


def _data(n=8000, F=6, K=4, seed=21):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    logits = np.nan_to_num(X[:, :K]) + 0.5 * rng.standard_normal((n, K))
    y = np.argmax(logits, axis=1).astype(np.float32)
    return X, y


def _with_bins(bb, t, cuts, off):
    """A reference tree with each split's bin recovered from its threshold."""
    sb = np.zeros(len(t.feature), np.uint32)
    for i, f in enumerate(t.feature):
        if f != bb.LEAF:
            sb[i] = np.flatnonzero(cuts[off[f]:off[f + 1]] == t.value[i])[0]
    return bb.Tree(feature=t.feature.astype(np.uint32), value=t.value.astype(np.float32),
                   left=t.left.astype(np.uint32), right=t.right.astype(np.uint32),
                   default_left=t.default_left.astype(np.uint8), gains=t.gains, covers=t.covers,
                   split_bin=sb)


def _oblivious_tree(bb, feats, thr, dl, leaves, cuts, off):
    """An ObliviousTree's tables as the perfect tree they expand to (BFS)."""
    d = len(feats)
    n = (2 << d) - 1
    t = dict(feature=np.full(n, bb.LEAF, np.uint32), value=np.zeros(n, np.float32),
             left=np.zeros(n, np.uint32), right=np.zeros(n, np.uint32),
             default_left=np.zeros(n, np.uint8), gains=np.zeros(n, np.float32),
             covers=np.zeros(n, np.float32), split_bin=np.zeros(n, np.uint32))
    for lvl in range(d):
        f = int(feats[lvl])
        b = np.flatnonzero(cuts[off[f]:off[f + 1]] == thr[lvl])[0]
        for i in range((1 << lvl) - 1, (2 << lvl) - 1):
            t["feature"][i], t["value"][i], t["split_bin"][i] = f, thr[lvl], b
            t["default_left"][i] = dl[lvl]
            t["left"][i], t["right"][i] = 2 * i + 1, 2 * i + 2
    t["value"][(1 << d) - 1:] = leaves
    return bb.Tree(**t)


@pytest.mark.parametrize("grower", ["depthwise", "levelwise"])
def test_softmax_matches_reference(bb, ref, grower):
    K = 4
    X, y = _data(K=K)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    rounds = 8
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=K, grower=grower, max_depth=5,
                              n_iters=rounds, learning_rate=0.2))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K, grower=grower,
                                            max_depth=5, learning_rate=0.2, use_graph=True),
                   max_trees=rounds)
    b.update(rounds)
    assert b.n_trees == rounds * K
    assert np.array_equal(b.init_scores, m.init_scores())
    theirs = m.trees()
    for k in range(K):  # round 0, every class
        mine = b.tree(k)
        if grower == "levelwise":
            # the reference keeps ObliviousTrees: compare their level tables
            for x, z in zip(bb.oblivious_tables(mine), m.oblivious(k)):
                assert np.array_equal(np.asarray(x).view(np.uint8),
                                      np.asarray(z).view(np.uint8)), k
            continue
        for f in TREE_FIELDS:
            x, z = getattr(mine, f), getattr(theirs[k], f)
            assert np.array_equal(x[:len(z)].view(np.uint8), z.view(np.uint8)), (k, f)
    raw = bb.predict_classes(plane, b.trees(), b.init_scores, 0.2)
    # training scores add lr * leaf round by round; predict forms init + lr * sum
    np.testing.assert_allclose(b.scores(), raw, rtol=1e-5, atol=1e-5)
    if grower == "levelwise":
        ref_trees = [_oblivious_tree(bb, *m.oblivious(t), cuts, off) for t in range(len(theirs))]
    else:
        ref_trees = [_with_bins(bb, t, cuts, off) for t in theirs]
    ref_raw = np.stack([bb.predict(plane, ref_trees[k::K], float(m.init_scores()[k]), 0.2)
                        for k in range(K)], axis=1)
    np.testing.assert_allclose(raw, ref_raw, rtol=1e-4, atol=1e-4)
    assert (np.argmax(raw, 1) == np.argmax(ref_raw, 1)).mean() > 0.999


def test_softmax_quantised_accuracy(bb):
    K = 5
    X, y = _data(n=60_000, F=8, K=K, seed=4)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    acc = {}
    for mode in ("exact", "int8"):
        b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K,
                                                grower="levelwise", max_depth=6,
                                                hist_mode=mode, learning_rate=0.3),
                       max_trees=15)
        b.update(15)
        acc[mode] = (np.argmax(b.scores(), 1) == y).mean()
    assert acc["exact"] > 0.6
    assert abs(acc["exact"] - acc["int8"]) < 5e-3
