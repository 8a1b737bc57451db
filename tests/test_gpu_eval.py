"""The device validation plane (bb_booster_eval_*): the reference's eval plane
(CudaDeviceContext::eval_begin / eval_accumulate, src/cuda/detail/
device_context.cu:1666-1760) behind Booster::begin_resident_validation /
accumulate_last_round_resident (include/bonsai/booster.hpp:1008-1021) and
the early-stopping loop of src/cli/pipeline.cpp:413-462.

Every round adds lr x leaf of its new tree(s) to the validation scores
(scores[i] += lr * value, accumulate_last_round): checked bit for bit
against a float32 host accumulation over the trees the booster returns. The
recorded loss is the reference's device form (FP64 sum of per-row terms,
/ n) and is checked against a numpy FP64 restatement over those scores to
1e-6 relative; softmax cross-entropy follows logloss_from_scores
(include/bonsai/multiclass_booster.hpp:545-559)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LEAF = 0xFFFFFFFF


def leaf_values(codes, n_bins, tree):
    """Each row's leaf value under `tree` (routes_left in bin space)."""
    F, n = codes.shape
    last = np.asarray(n_bins, np.int64) - 1
    rows = np.arange(n)
    idx = np.zeros(n, np.int64)
    feat = tree.feature.astype(np.int64)
    while True:
        f = feat[idx]
        live = f != LEAF
        if not live.any():
            break
        fl = np.where(live, f, 0)
        b = codes[fl, rows].astype(np.int64)
        left = np.where(b == last[fl], tree.default_left[idx] != 0, b <= tree.split_bin[idx])
        idx = np.where(live, np.where(left, tree.left[idx], tree.right[idx]), idx).astype(np.int64)
    return tree.value[idx].astype(np.float32)


def host_scores(codes, n_bins, trees, init, lr, K=1):
    """scores[i] += lr * leaf, round by round, in float32 (K columns)."""
    n = codes.shape[1]
    s = np.tile(np.asarray(init, np.float32).reshape(1, -1), (n, 1)) if K > 1 else \
        np.full(n, np.float32(init), np.float32)
    lr = np.float32(lr)
    out = []
    for r in range(len(trees) // K):
        for k in range(K):
            v = leaf_values(codes, n_bins, trees[r * K + k])
            if K > 1:
                s[:, k] = (s[:, k] + lr * v).astype(np.float32)
            else:
                s = (s + lr * v).astype(np.float32)
        out.append(s.copy())
    return out


def loss64(s, y, objective):
    if objective == "mse":
        d = s.astype(np.float64) - y.astype(np.float64)
        return float(np.sum(d * d) / len(y))
    if objective == "logloss":
        s = s.astype(np.float32)
        t = np.maximum(np.float32(0), s) + np.log1p(np.exp(-np.abs(s))) - y * s
        return float(np.sum(t.astype(np.float64)) / len(y))
    sd = s.astype(np.float64)
    m = sd.max(axis=1)
    lse = np.log(np.exp(sd - m[:, None]).sum(axis=1))
    c = y.astype(np.int64)
    return float(-np.sum(sd[np.arange(len(y)), c] - m - lse) / len(y))


def _data(seed, n, F=10, classes=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    z = np.nan_to_num(X[:, 0]) * 1.5 + np.sin(2 * np.nan_to_num(X[:, 1])) + \
        np.nan_to_num(X[:, 2]) * np.nan_to_num(X[:, 3])
    if classes:
        y = np.digitize(z + rng.normal(0, 0.5, n), np.quantile(z, np.linspace(0, 1, classes + 1)[1:-1]))
        return X, y.astype(np.float32)
    return X, (z + rng.normal(0, 0.3, n)).astype(np.float32)


@pytest.mark.parametrize("objective,grower,graph", [
    ("logloss", "depthwise", True), ("logloss", "depthwise", False),
    ("mse", "levelwise", True), ("mse", "leafwise", False),
])
def test_eval_plane_scores_and_losses(bb, objective, grower, graph):
    X, y = _data(3, 30_000)
    Xv, yv = _data(4, 7_001)
    if objective == "logloss":
        y, yv = (y > 0).astype(np.float32), (yv > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane, valid = bb.Plane(X, cuts, off), bb.Plane(Xv, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective=objective, grower=grower, max_depth=6,
                                            max_leaves=40, learning_rate=0.2,
                                            use_graph=graph), max_trees=40)
    b.update(3)  # rounds before arming start from the booster's initial score
    b.eval_arm(valid, yv)
    b.update(25)
    trees = b.trees()
    losses = b.eval_losses()
    assert len(losses) == 25
    codes = valid.bins()
    want = host_scores(codes, valid.n_bins, trees[3:], b.init_score, 0.2)
    assert np.array_equal(b.eval_scores().view(np.uint32), want[-1].view(np.uint32))
    ref = np.array([loss64(s, yv, objective) for s in want])
    np.testing.assert_allclose(losses, ref.astype(np.float32), rtol=1e-6)
    assert losses[-1] < losses[0]


def test_eval_plane_softmax(bb):
    K = 3
    X, y = _data(5, 20_000, classes=K)
    Xv, yv = _data(6, 5_000, classes=K)
    cuts, off = bb.fit_cuts(X)
    plane, valid = bb.Plane(X, cuts, off), bb.Plane(Xv, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="softmax", n_classes=K, max_depth=5,
                                            learning_rate=0.3, use_graph=True), max_trees=20)
    b.eval_arm(valid, yv)
    b.update(12)
    trees = b.trees()
    want = host_scores(valid.bins(), valid.n_bins, trees, b.init_scores, 0.3, K=K)
    assert np.array_equal(b.eval_scores().view(np.uint32), want[-1].view(np.uint32))
    ref = np.array([loss64(s, yv, "softmax") for s in want])
    np.testing.assert_allclose(b.eval_losses(), ref.astype(np.float32), rtol=1e-6)


def test_early_stopping_keeps_the_rule_s_rounds(bb):
    """Strong learning rate on noise: the validation loss turns up, the fit
    stops, and the booster keeps exactly the rounds the per-round rule keeps
    over the recorded losses."""
    rng = np.random.Generator(np.random.PCG64(8))
    X = rng.standard_normal((4_000, 6)).astype(np.float32)
    y = (X[:, 0] + rng.normal(0, 2.0, 4_000)).astype(np.float32)
    Xv = rng.standard_normal((4_000, 6)).astype(np.float32)
    yv = (Xv[:, 0] + rng.normal(0, 2.0, 4_000)).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane, valid = bb.Plane(X, cuts, off), bb.Plane(Xv, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(max_depth=6, learning_rate=0.5, min_data_in_leaf=2,
                                            use_graph=True), max_trees=200)
    kept = bb.fit_early_stopping(b, valid, yv, n_iters=200, patience=5, check_every=8)
    losses = b.eval_losses()
    want, stopped = bb.early_stop_round(losses, 5)
    assert stopped and kept == want < 200
    assert b.n_trees == kept
    # the kept round has the lowest loss up to the stop (rounds past the stop
    # ran inside the last check_every batch and do not count)
    assert losses[kept - 1] == losses[:kept + 5].min()
    with pytest.raises(bb.BonsaiError):
        b.update(1)


def test_eval_plane_refusals(bb):
    X, y = _data(9, 5_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(max_depth=4), max_trees=4)
    other_cuts, other_off = bb.fit_cuts(X[:, :9])
    with pytest.raises(bb.BonsaiError):
        b.eval_arm(bb.Plane(X[:, :9], other_cuts, other_off), y)
    with pytest.raises(bb.BonsaiError):
        b.eval_losses()  # nothing armed
    shard = bb.Comm.group(1)[0]
    bs = bb.Booster(plane, y, bb.TrainParams(max_depth=4, hist_mode="int8"), max_trees=4,
                    comm=shard, row_offset=0, total_rows=len(y),
                    init_score=bb.init_score(y, "mse"))
    with pytest.raises(bb.ConfigError):
        bs.eval_arm(plane, y)
