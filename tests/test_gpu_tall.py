"""The int8 form past 16,909,320 rows (127 x rows >= 2^31): histogram cells
widen to two words (an int64 gradient and a uint64 hessian sum) and the
fixed-point leaf sums take a smaller unit, so a fit of 20,000,000 rows --
the reference's own tall GPU benches run 16.7M and more rows on one card --
keeps exact integer histograms: a 20M-row bin sums exactly, the fit equals
its own two-shard fit tree for tree, and its validation AUC stays within
the quantised form's bound of the plain form's."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_TALL = 20_000_000


@pytest.mark.parametrize("hist_ctas", [0, 1])
def test_int8_cells_past_the_packed_range(bb, hist_ctas):
    """One bin holding all 20M rows with the largest code: 20M x 127 would
    wrap a packed 32-bit half; the two-word cell sums it exactly. With one
    CTA asked for, the build still spreads the rows over enough CTAs that no
    CTA's 32-bit shared words sum more than 16,908,288 codes."""
    rng = np.random.Generator(np.random.PCG64(5))
    X = np.empty((N_TALL, 2), np.float32)
    X[:, 0] = 1.0                                  # every row in one bin
    X[:, 1] = rng.standard_normal(N_TALL, dtype=np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    g = np.ones(N_TALL, np.float32)
    h = np.full(N_TALL, 0.25, np.float32)
    q = bb.populate(plane, bb.TrainParams(hist_mode="int8", seed=1, hist_ctas=hist_ctas),
                    g, h)
    nb0 = int(off[1] - off[0])
    cells = q[:nb0]
    assert cells[:, 0].max() == N_TALL            # 20M codes of 127 x scale 1/127
    assert cells[:, 1].max() == 0.25 * N_TALL
    assert cells[:, 0].sum() == N_TALL and cells[:, 1].sum() == 0.25 * N_TALL
    other = q[nb0:]                               # every row counted once per feature
    np.testing.assert_allclose(other[:, 0].sum(), N_TALL, rtol=1e-12)


def _auc(y, p):
    order = np.argsort(p, kind="stable")
    ranks = np.empty(len(p)); ranks[order] = np.arange(1, len(p) + 1)
    pos = y > 0.5
    n1, n0 = pos.sum(), (~pos).sum()
    return (ranks[pos].sum() - n1 * (n1 + 1) / 2) / (n1 * n0)


def test_int8_tall_fit_equals_its_sharded_fit_and_tracks_plain(bb):
    from test_gpu_sharded import _same_tree, _sharded

    from bonsai_b200 import synth
    X, y = synth.tall_binary(n=N_TALL)
    cuts, off = bb.fit_cuts(X)
    rounds = 12
    params = bb.TrainParams(objective="logloss", max_depth=6, hist_mode="int8", seed=3,
                            learning_rate=0.2, use_graph=True)
    plane = bb.Plane(X, cuts, off)
    full = bb.Booster(plane, y, params, max_trees=rounds)
    full.update(rounds)
    trees = full.trees()
    shards = _sharded(bb, X, y, cuts, off, bb.TrainParams(
        objective="logloss", max_depth=6, hist_mode="int8", seed=3, learning_rate=0.2),
        2, rounds, full.init_score)
    for i in range(rounds):
        for s, bst in enumerate(shards):
            _same_tree(bst.tree(i), trees[i], f"tree {i} shard {s}")
    assert np.array_equal(np.concatenate([b.scores() for b in shards]), full.scores())
    for b in shards:
        b.close()
    plain = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=6,
                                                learning_rate=0.2, use_graph=True),
                       max_trees=rounds)
    plain.update(rounds)
    Xv, yv = synth.tall_binary(n=500_000, seed=10_000_001)
    pv = bb.Plane(Xv, cuts, off)
    a_q = _auc(yv, bb.predict(pv, trees, full.init_score, 0.2))
    a_p = _auc(yv, bb.predict(pv, plain.trees(), plain.init_score, 0.2))
    assert abs(a_q - a_p) <= 2e-3, (a_q, a_p)
