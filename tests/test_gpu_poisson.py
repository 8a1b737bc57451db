"""The Poisson objective (PoissonObjective, src/objective.cpp:253-308; a
resident device kind of the reference, include/bonsai/objective_traits.hpp)
on the device booster: log link, g = exp(s) - y and h = exp(s) with the raw
score clamped to +-30, the initial score the log of the mean label (FP64
sum, floored at 1e-9), exp rounded by CUDA's expf as the reference's own
device gradient kernel does (src/cuda/detail/kernels.cuh:994-999). Against
the reference: the same initial score as its CPU booster; the first round's
tree bit for bit the reference grower's for the rate the device rounded;
predictions after ten rounds within float tolerance of the CPU booster's
except at rows that rounding-decided defaults move; the device validation
loss is the reference's device form; negative labels are refused."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg

pytestmark = pytest.mark.gpu


def _data(seed, n=10_000, F=6):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    rate = np.exp(0.4 * np.nan_to_num(X[:, 0]) - 0.3 * np.abs(np.nan_to_num(X[:, 1])) + 0.5)
    y = rng.poisson(rate).astype(np.float32)
    return X, y


def _ulps(r, k):
    for _ in range(abs(k)):
        r = np.nextafter(r, np.float32(np.inf if k > 0 else -np.inf))
    return r


@pytest.mark.parametrize("grower", ["depthwise", "leafwise"])
def test_poisson_matches_reference(bb, ref, grower):
    X, y = _data(3)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    tc = dict(grower=grower, max_depth=6, max_leaves=31)
    m = ref.train(ds, TreeCfg(objective="poisson", n_iters=10, learning_rate=0.1, **tc))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="poisson", learning_rate=0.1,
                                            use_graph=True, **tc), max_trees=10)
    b.update(10)
    init = np.float32(m.init_score())
    assert np.float32(b.init_score) == init
    assert np.float32(bb.init_score(y, "poisson")) == init
    # Round 0: every row's rate is exp(init). The device rounds it with CUDA's
    # expf (within 2 ulp), the reference's CPU booster with the host's, and
    # this tree has defaults decided by near-ties that flip with one ulp of
    # the rate. So the device tree must be, bit for bit, the reference
    # grower's tree for g = r - y, h = r with r one of the floats within
    # 2 ulp of exp(init).
    rows = np.arange(len(y), dtype=np.uint32)
    mine, hits = b.tree(0), []
    for k in range(-2, 3):
        r = _ulps(np.exp(init), k)
        g = (r - y).astype(np.float32)
        want, *_ = ref.grow_tree(ds, TreeCfg(**tc), g, np.full_like(g, r), rows)
        if all(np.array_equal(np.asarray(getattr(mine, f)).view(np.uint8),
                              np.asarray(getattr(want, f)).view(np.uint8))
               for f in TREE_FIELDS):
            hits.append(k)
    assert hits, "no rate within 2 ulp of exp(init) reproduces the device tree"
    # Ten rounds: the same model up to those rounding-decided defaults, which
    # move only the missing rows of a few small nodes.
    p = bb.predict(plane, b.trees(), b.init_score, 0.1)
    q = m.predict_binned(ds)
    off_rows = np.abs(p - q) > 1e-5 * (1 + np.abs(q))
    assert off_rows.mean() < 0.02, off_rows.mean()
    np.testing.assert_allclose(np.median(p), np.median(q), rtol=1e-5)


def test_poisson_validation_loss(bb):
    X, y = _data(4)
    Xv, yv = _data(5, n=3_000)
    cuts, off = bb.fit_cuts(X)
    plane, valid = bb.Plane(X, cuts, off), bb.Plane(Xv, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="poisson", max_depth=5, learning_rate=0.2,
                                            use_graph=True), max_trees=15)
    b.eval_arm(valid, yv)
    b.update(15)
    s = b.eval_scores()
    f = np.clip(s, -30, 30).astype(np.float32)
    want = float(np.sum(np.exp(f).astype(np.float32).astype(np.float64)
                        - yv.astype(np.float64) * f.astype(np.float64)) / len(yv))
    losses = b.eval_losses()
    np.testing.assert_allclose(losses[-1], want, rtol=1e-6)
    assert losses[-1] < losses[0]


def test_poisson_refuses_negative_labels(bb):
    X, y = _data(6, n=500)
    y[3] = -1.0
    cuts, off = bb.fit_cuts(X)
    with pytest.raises(bb.BonsaiError):
        bb.Booster(bb.Plane(X, cuts, off), y, bb.TrainParams(objective="poisson"))
