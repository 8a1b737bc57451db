"""GPU tests of the quantised form: int8 stochastic-rounded gradients with
exact integer histograms, FP64 gain and FP64 leaf renewal. Histogram error
is stated against FP64 sums, model quality against the plain form."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import orc_fill

pytestmark = pytest.mark.gpu


def _data(seed, n, F=10):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    g = rng.normal(0, 1, n).astype(np.float32)
    h = rng.uniform(0.05, 0.25, n).astype(np.float32)
    return X, g, h


def test_populate_exact_is_the_serial_fill(bb, orc):
    X, g, h = _data(1, 20000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    rows = np.flatnonzero(np.random.Generator(np.random.PCG64(2)).random(len(g)) < 0.4)
    got = bb.populate(plane, bb.TrainParams(), g, h, rows=rows)
    want = orc_fill(orc, plane.bins(), np.diff(off), g, h, rows=rows)
    assert np.array_equal(got.astype(np.float32), want)


def _fp64_hist(bins, n_bins, g, h):
    cells = []
    for f in range(bins.shape[0]):
        G = np.zeros(n_bins[f]); H = np.zeros(n_bins[f])
        np.add.at(G, bins[f], g.astype(np.float64))
        np.add.at(H, bins[f], h.astype(np.float64))
        cells.append(np.stack([G, H], 1))
    return np.concatenate(cells)


@pytest.mark.parametrize("mode,qmax", [("int8", 127.0), ("int16", 32767.0)])
def test_quantised_histogram_error_vs_fp64(bb, mode, qmax):
    X, g, h = _data(3, 400_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    nb = np.diff(off)
    q = bb.populate(plane, bb.TrainParams(hist_mode=mode, seed=7), g, h)
    ref = _fp64_hist(plane.bins(), nb, g, h)
    sg = np.abs(g).max() / qmax
    sh = h.max() / qmax
    counts = np.concatenate([np.bincount(plane.bins()[f], minlength=nb[f]) for f in range(len(nb))])
    # stochastic rounding: unbiased, per-row error below one scale step
    err_g = np.abs(q[:, 0] - ref[:, 0])
    err_h = np.abs(q[:, 1] - ref[:, 1])
    assert np.all(err_g <= 6 * sg * np.sqrt(counts) + sg)
    assert np.all(err_h <= 6 * sh * np.sqrt(counts) + sh)
    # every feature sees the same rows: the integer totals agree exactly
    # (cells are integer sums times the FP64 scale: recover the integers)
    scale = np.array([np.abs(g).max() / qmax, h.max() / qmax])
    ints = np.rint(q / scale)
    tot = [ints[off[f]:off[f + 1]].sum(0) for f in range(len(nb))]
    assert all(np.array_equal(tot[0], t) for t in tot)
    tot = [q[off[0]:off[1]].sum(0)]
    rel = abs(tot[0][0] - g.astype(np.float64).sum()) / np.abs(g).sum()
    assert rel < 1e-3


def test_quantised_seeded_and_deterministic(bb):
    X, g, h = _data(4, 100_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    y = (g > 0).astype(np.float32)
    def fit(seed, graph):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=6,
                                                 hist_mode="int8", seed=seed,
                                                 use_graph=graph), max_trees=8)
        b.update(8)
        return b.scores(), [b.tree(i) for i in range(8)]
    s1, t1 = fit(11, False)
    s2, t2 = fit(11, True)
    s3, _ = fit(12, False)
    assert np.array_equal(s1, s2)
    for a, c in zip(t1, t2):
        assert np.array_equal(a.feature, c.feature) and np.array_equal(a.value, c.value)
    assert not np.array_equal(s1, s3)


@pytest.mark.parametrize("grower", ["depthwise", "levelwise"])
def test_one_pass_partition_leaves_fits_deterministic(bb, grower):
    """A walked quantised tree partitions each level in one pass: chunks
    place their rows in a child in the order they finish, so row lists
    differ from run to run. Everything built from them (exact integer
    histograms, per-row routing) is order-free: three fits of 2,000,000 rows
    (hundreds of chunks per node) give the same trees and scores bit for
    bit, with and without CUDA graphs."""
    X, g, h = _data(21, 2_000_000, F=12)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    y = (g + np.nan_to_num(X[:, 0]) > 0).astype(np.float32)

    def fit(graph):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=8,
                                                 hist_mode="int8", seed=5, grower=grower,
                                                 use_graph=graph), max_trees=12)
        b.update(12)
        out = b.scores(), [b.tree(i) for i in range(12)]
        b.close()
        return out

    s0, t0 = fit(True)
    for graph in (True, False):
        s1, t1 = fit(graph)
        assert np.array_equal(s0, s1)
        for a, c in zip(t0, t1):
            for k in ("feature", "split_bin", "left", "right", "value", "covers"):
                assert np.array_equal(getattr(a, k), getattr(c, k)), k


@pytest.mark.parametrize("mono", [False, True])
def test_quantised_leaf_values_renew_from_full_gradients(bb, mono):
    """Every leaf's value is the FP64 Newton step of its rows' full-precision
    (g, h) -- not of the quantised codes -- under its monotone bounds, and the
    scores take score + lr * value of each row's leaf."""
    X, g, h = _data(8, 60_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    y = (X[:, 0] + 0.3 * np.nan_to_num(X[:, 1]) > 0).astype(np.float32)
    lr = 0.3
    b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=7,
                                            learning_rate=lr, hist_mode="int8",
                                            lambda_l2=2.0, monotone=[1] if mono else [],
                                            record_leaf_ids=True), max_trees=1)
    b.update(1)
    t = b.tree(0)
    leaf = b.leaf_ids()
    assert (t.feature[leaf] == bb.LEAF).all()
    s0 = np.float32(b.init_score)
    p = (np.float32(1.0) / (np.float32(1.0) + np.exp(-s0, dtype=np.float32))).astype(np.float32)
    gg = (p - y).astype(np.float64)
    hh = np.full(len(y), np.float64(np.float32(p * (np.float32(1.0) - p))))
    G = np.bincount(leaf, weights=gg, minlength=len(t.feature))
    H = np.bincount(leaf, weights=hh, minlength=len(t.feature))
    used = np.unique(leaf)
    want = -G[used] / (H[used] + 2.0)
    if not mono:
        # device expf and numpy exp may differ in the last place
        np.testing.assert_allclose(t.value[used], want, rtol=2e-6, atol=1e-7)
    else:
        # bounds clamp the Newton steps; every split on the constrained
        # feature orders its subtrees' values
        assert np.isfinite(t.value[used]).all()

        def leaves(i):
            if t.feature[i] == bb.LEAF:
                return [t.value[i]]
            return leaves(t.left[i]) + leaves(t.right[i])
        for i in np.flatnonzero(t.feature == 0):
            assert max(leaves(t.left[i])) <= min(leaves(t.right[i])) + 1e-6
    expect = (s0 + np.float32(lr) * t.value[leaf]).astype(np.float32)
    assert np.array_equal(b.scores(), expect)


def _auc(y, p):
    order = np.argsort(p, kind="stable")
    ranks = np.empty(len(p)); ranks[order] = np.arange(1, len(p) + 1)
    pos = y > 0.5
    n1, n0 = pos.sum(), (~pos).sum()
    return (ranks[pos].sum() - n1 * (n1 + 1) / 2) / (n1 * n0)


def test_quantised_auc_matches_plain_on_tall_binary_subset(bb):
    """HIGGS-shaped 1M-row subset, depth 8, 100 rounds: the quantised fit's
    validation AUC within 1e-3 of the plain form's."""
    from bonsai_b200 import synth
    X, y = synth.tall_binary(n=1_200_000)
    Xt, yt, Xv, yv = X[:1_000_000], y[:1_000_000], X[1_000_000:], y[1_000_000:]
    cuts, off = bb.fit_cuts(Xt)
    pt = bb.Plane(Xt, cuts, off)
    pv = bb.Plane(Xv, cuts, off)
    aucs = {}
    for mode in ("exact", "int8"):
        b = bb.Booster(pt, yt, bb.TrainParams(objective="logloss", max_depth=8,
                                               learning_rate=0.1, hist_mode=mode, seed=1,
                                               use_graph=True), max_trees=100)
        b.update(100)
        aucs[mode] = _auc(yv, bb.predict(pv, b.trees(), b.init_score, 0.1))
    assert aucs["exact"] > 0.7
    assert abs(aucs["int8"] - aucs["exact"]) <= 1e-3, aucs


def test_quantised_large_invariants(bb):
    rng = np.random.Generator(np.random.PCG64(5))
    n, F = 2_000_000, 28
    X = rng.standard_normal((n, F)).astype(np.float32)
    y = (X[:, 0] + X[:, 1] * X[:, 2] > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=8,
                                             hist_mode="int8"), max_trees=3)
    b.update(3)
    trees = b.trees()
    for t in trees:
        for i in np.flatnonzero(t.feature != bb.LEAF):
            assert t.covers[t.left[i]] + t.covers[t.right[i]] == t.covers[i]
    s = np.full(n, np.float32(b.init_score), np.float32)
    for t in trees:
        s = (s + np.float32(0.1) * bb.predict(plane, [t], 0.0, 1.0)).astype(np.float32)
    np.testing.assert_array_equal(b.scores(), s)


def test_quantised_u16_bins_histogram_and_fit(bb):
    """u16 codes (more than 256 bins) take the generic quantised kernel."""
    X, g, h = _data(8, 150_000, F=6)
    cuts, off = bb.fit_cuts(X, max_bin=700)
    plane = bb.Plane(X, cuts, off)
    assert not plane.u8
    q = bb.populate(plane, bb.TrainParams(hist_mode="int8", seed=3), g, h)
    ref = _fp64_hist(plane.bins(), np.diff(off), g, h)
    sg = np.abs(g).max() / 127.0
    counts = np.concatenate([np.bincount(plane.bins()[f], minlength=np.diff(off)[f])
                             for f in range(6)])
    assert np.all(np.abs(q[:, 0] - ref[:, 0]) <= 6 * sg * np.sqrt(counts) + sg)
    y = (X[:, 0] + np.nan_to_num(X[:, 1]) > 0).astype(np.float32)
    b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=6,
                                             hist_mode="int8"), max_trees=10)
    b.update(10)
    assert b.n_trees == 10 and np.isfinite(b.scores()).all()


def test_int16_u16_bins_levelwise_leafwise_and_shards(bb):
    """int16 codes (two-word cells) through the generic kernel on both bin
    widths, the three growers, and a two-shard fit equal to the unsharded one."""
    import threading
    X, g, h = _data(13, 120_000, F=7)
    y = (X[:, 0] + np.nan_to_num(X[:, 1]) * X[:, 2] > 0).astype(np.float32)
    for max_bin in (255, 700):
        cuts, off = bb.fit_cuts(X, max_bin=max_bin)
        plane = bb.Plane(X, cuts, off)
        q = bb.populate(plane, bb.TrainParams(hist_mode="int16", seed=3), g, h)
        ref = _fp64_hist(plane.bins(), np.diff(off), g, h)
        counts = np.concatenate([np.bincount(plane.bins()[f], minlength=np.diff(off)[f])
                                 for f in range(7)])
        sg = np.abs(g).max() / 32767.0
        assert np.all(np.abs(q[:, 0] - ref[:, 0]) <= 6 * sg * np.sqrt(counts) + sg)
        for grower in ("depthwise", "levelwise", "leafwise"):
            b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", grower=grower,
                                                     max_depth=6, max_leaves=40,
                                                     hist_mode="int16"), max_trees=5)
            b.update(5)
            assert b.n_trees == 5 and np.isfinite(b.scores()).all(), (max_bin, grower)
    cuts, off = bb.fit_cuts(X)
    params = bb.TrainParams(objective="logloss", max_depth=6, hist_mode="int16", seed=4)
    full = bb.Booster(bb.Plane(X, cuts, off), y, params, max_trees=4)
    full.update(4)
    comms = bb.Comm.group(2)
    shards = []
    for s in range(2):
        a, e = bb.shard_range(len(X), 2, s)
        shards.append(bb.Booster(bb.Plane(X[a:e], cuts, off), y[a:e], params, max_trees=4,
                                 comm=comms[s], row_offset=a, total_rows=len(X),
                                 init_score=full.init_score))
    ts = [threading.Thread(target=lambda b=b: b.update(4)) for b in shards]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert np.array_equal(np.concatenate([b.scores() for b in shards]), full.scores())


def test_int16_closer_to_plain_than_int8(bb):
    """Finer codes: the int16 fit's scores sit nearer the plain fit's."""
    X, g, h = _data(17, 200_000, F=8)
    y = (X[:, 0] + np.nan_to_num(X[:, 1]) * X[:, 2] + 0.3 * g > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    out = {}
    for mode in ("exact", "int8", "int16"):
        b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=6,
                                                hist_mode=mode, seed=2), max_trees=20)
        b.update(20)
        out[mode] = b.scores()
    d8 = np.abs(out["int8"] - out["exact"]).mean()
    d16 = np.abs(out["int16"] - out["exact"]).mean()
    assert d16 < d8
