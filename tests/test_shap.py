"""TreeSHAP contributions (bb_pred_contribs) against the reference's own
binned TreeSHAP (pred_contribs_binned, include/bonsai/booster.hpp:887-924,
src/shap.cpp): golden contributions the reference wrote for the small
regression ensemble (100 MSE trees, depth 6) and the 20-tree logloss ensemble
over data with missing values.

The CPU test restates the device's path form in numpy (merged per-feature
conditions, a Gauss-Legendre rule from numpy rather than the library's own
nodes) and checks it against the same fixtures, so the formulation is pinned
before any GPU runs. GPU tests call the C ABI on the reference's exact trees,
on trees the B200 booster grew, on 16-bit bin codes, and check additivity
(every row's contributions sum to its margin) and run-to-run identity."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden, unpack_trees

# FP64 against FP64 with a different (division-free) summation: agreement to
# ~1e-12 relative is expected; 1e-9 leaves room without hiding a wrong term.
RTOL = 1e-9
ATOL = 1e-12
LEAF = 0xFFFFFFFF


def golden_trees(d, prefix=""):
    """The fixture's trees with each internal node's split bin recovered from
    its threshold (threshold = cuts[cut_off[f] + split_bin])."""
    from bonsai_b200 import Tree
    cuts, off = d["cuts"], d["cut_off"]
    out = []
    for t in unpack_trees(d, prefix):
        sb = np.zeros(len(t.feature), np.uint32)
        for i, f in enumerate(t.feature):
            if f == LEAF:
                continue
            row = cuts[off[f]:off[f + 1]]
            hit = np.flatnonzero(row == t.value[i])
            assert len(hit) == 1, (i, f, t.value[i])
            sb[i] = hit[0]
        out.append(Tree(feature=t.feature.astype(np.uint32), value=t.value.astype(np.float32),
                        left=t.left.astype(np.uint32), right=t.right.astype(np.uint32),
                        default_left=t.default_left.astype(np.uint8),
                        gains=t.gains.astype(np.float32), covers=t.covers.astype(np.float32),
                        split_bin=sb))
    return out


def expected_value(t, i=0):
    """tree_expected_value (src/shap.cpp:250-290)."""
    if t.feature[i] == LEAF:
        return float(t.value[i])
    c = float(t.covers[i])
    if c <= 0.0:
        return 0.0
    lc, rc = int(t.left[i]), int(t.right[i])
    return (float(t.covers[lc]) * expected_value(t, lc)
            + float(t.covers[rc]) * expected_value(t, rc)) / c


def paths(t, last):
    """Every root-to-leaf path: (leaf value, [(feature, lo, hi, miss_ok, zero)])
    with a feature's conditions merged into the non-missing bins [lo, hi]."""
    out = []

    def rec(i, conds):
        if t.feature[i] == LEAF:
            out.append((float(t.value[i]), [tuple(c) for c in conds.values()]))
            return
        f, s, dl, c = int(t.feature[i]), int(t.split_bin[i]), bool(t.default_left[i]), \
            float(t.covers[i])
        for side, child in ((0, int(t.left[i])), (1, int(t.right[i]))):
            frac = float(t.covers[child]) / c if c > 0.0 else 0.0
            old = conds.get(f)
            lo, hi, ok, z = old[1:] if old else (0, int(last[f]) - 1, True, 1.0)
            if side == 0:
                hi, ok = min(hi, s), ok and dl
            else:
                lo, ok = max(lo, s + 1), ok and not dl
            nxt = dict(conds)
            nxt[f] = (f, lo, hi, ok, z * frac)
            rec(child, nxt)

    rec(0, {})
    return out


def shap_numpy(bins, last, trees, init, lr):
    """The path form: phi[f_i] += v (o_i - z_i) int_0^1 prod_{j != i}
    (z_j + (o_j - z_j) t) dt, exact with ceil(n / 2) Gauss-Legendre nodes."""
    n, F = bins.shape
    phi = np.zeros((n, F + 1))
    bias = 0.0
    for t in trees:
        bias += expected_value(t)
        for v, els in paths(t, last):
            k = len(els)
            if k == 0:
                continue
            x, w = np.polynomial.legendre.leggauss(max(1, (k + 1) // 2))
            x, w = 0.5 * (x + 1.0), 0.5 * w
            z = np.array([e[4] for e in els])
            o = np.empty((n, k))
            for j, (f, lo, hi, ok, _) in enumerate(els):
                b = bins[:, f].astype(np.int64)
                o[:, j] = np.where(b == last[f], ok, (b >= lo) & (b <= hi))
            dz = o - z                                   # [n, k]
            fac = z[None, :, None] + dz[:, :, None] * x[None, None, :]  # [n, k, m]
            for j, e in enumerate(els):
                rest = np.prod(np.delete(fac, j, axis=1), axis=1)  # [n, m]
                phi[:, e[0]] += v * dz[:, j] * (rest @ w)
    lr = float(np.float32(lr))  # the booster's learning rate is a float
    phi[:, :F] *= lr
    phi[:, F] = (phi[:, F] + bias) * lr + float(np.float32(init))
    return phi


CASES = [
    # fixture, tree prefix, contribs key, init key, rows
    ("small_regression.npz", "", "contribs", "init", 1024),
    ("missing_values.npz", "ll_", "ll_contribs", "logloss_init", None),
]


@pytest.mark.parametrize("case", CASES, ids=["small_regression", "missing_values_logloss"])
def test_path_form_matches_reference_golden(case):
    name, prefix, key, init_key, rows = case
    d = load_golden(name)
    trees = golden_trees(d, prefix)
    bins = d["bins"].T  # fixtures hold bin codes feature-major
    bins = bins[:rows] if rows else bins
    last = np.diff(d["cut_off"]).astype(np.int64) - 1
    phi = shap_numpy(bins, last, trees, float(d[init_key]), 0.1)
    np.testing.assert_allclose(phi, d[key], rtol=RTOL, atol=ATOL)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=["small_regression", "missing_values_logloss"])
def test_device_contribs_match_reference_golden(bb, case):
    from bonsai_b200 import synth
    name, prefix, key, init_key, rows = case
    d = load_golden(name)
    X = synth.regression_small()[0] if "X" not in d else d["X"]
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    trees = golden_trees(d, prefix)
    init = float(d[init_key])
    phi = bb.pred_contribs(plane, trees, init, 0.1)
    gold = d[key]
    np.testing.assert_allclose(phi[:len(gold)], gold, rtol=RTOL, atol=ATOL)
    # additivity over every row: contributions sum to the margin
    margin = bb.predict(plane, trees, init, 0.1).astype(np.float64)
    np.testing.assert_allclose(phi.sum(axis=1), margin, rtol=0, atol=1e-5)
    # a fixed-order reduction: bit-identical run to run
    assert np.array_equal(phi, bb.pred_contribs(plane, trees, init, 0.1))


@pytest.mark.gpu
def test_device_contribs_of_booster_trees(bb):
    """Trees the B200 booster grew (bit-identical to the reference's) give the
    reference's contributions."""
    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    X, y = synth.regression_small()
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    b = bb.Booster(plane, y, bb.TrainParams(max_depth=6, learning_rate=0.1), max_trees=100)
    b.update(100)
    phi = bb.pred_contribs(plane, b.trees(), b.init_score, 0.1)
    np.testing.assert_allclose(phi[:1024], d["contribs"], rtol=RTOL, atol=ATOL)


@pytest.mark.gpu
def test_device_contribs_u16_deep_paths_and_repeats(bb):
    """16-bit bin codes, depth-8 trees (repeated features on a path, missing
    values) against the numpy path form."""
    rng = np.random.Generator(np.random.PCG64(29))
    n, F = 3000, 5
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random(n) < 0.15, 1] = np.nan
    y = (X[:, 0] * X[:, 1] + np.sin(3 * X[:, 2]) > 0).astype(np.float32)
    y = np.where(np.isnan(y), 0.0, y).astype(np.float32)
    cuts, off = bb.fit_cuts(X, max_bin=700)
    plane = bb.Plane(X, cuts, off)
    assert not plane.u8
    b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=8,
                                            learning_rate=0.3, min_data_in_leaf=2),
                   max_trees=6)
    b.update(6)
    trees = b.trees()
    phi = bb.pred_contribs(plane, trees, b.init_score, 0.3)
    last = np.diff(off).astype(np.int64) - 1
    ref = shap_numpy(plane.bins().T.astype(np.int64), last, trees, b.init_score, 0.3)
    np.testing.assert_allclose(phi, ref, rtol=RTOL, atol=1e-11)


@pytest.mark.gpu
def test_device_contribs_refuses_wide_plane(bb):
    rng = np.random.Generator(np.random.PCG64(2))
    X = rng.standard_normal((64, 129)).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    t, _, _ = bb.grow_tree(plane, bb.TrainParams(max_depth=2),
                           rng.normal(0, 1, 64).astype(np.float32), np.ones(64, np.float32))
    with pytest.raises(bb.ConfigError):
        bb.pred_contribs(plane, [t], 0.0, 1.0)


@pytest.mark.gpu
def test_shap_plan_over_batches(bb):
    """A plan packed once scores planes of 1 to 20,640 rows: the same
    contributions as the full-plane call (row tiles, path lanes and path
    splits change with the batch, so agreement is to FP64 rounding), the
    same bits on a repeated run, and a plane of another shape is refused."""
    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    X, y = synth.regression_small()
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    b = bb.Booster(plane, y, bb.TrainParams(max_depth=6, learning_rate=0.1), max_trees=100)
    b.update(100)
    trees = b.trees()
    full = bb.pred_contribs(plane, trees, b.init_score, 0.1)
    np.testing.assert_allclose(full[:1024], d["contribs"], rtol=RTOL, atol=ATOL)
    plan = bb.ShapPlan(plane, trees, b.init_score, 0.1)
    for n in (1, 37, 500, 5_000, len(X)):
        p = bb.Plane(X[:n], d["cuts"], d["cut_off"])
        phi = plan.run(p)
        np.testing.assert_allclose(phi, full[:n], rtol=RTOL, atol=ATOL)
        assert np.array_equal(phi, plan.run(p))
    other = bb.Plane(X[:, :7], d["cuts"][:d["cut_off"][7]], d["cut_off"][:8])
    with pytest.raises(bb.BonsaiError):
        plan.run(other)


def chain_tree(rng, n_bins, depth):
    """A tree whose main path splits on `depth` distinct features (each
    right child a leaf), covers splitting each parent's at random."""
    from bonsai_b200 import Tree
    feats = rng.permutation(len(n_bins))[:depth]
    feature, split, left, right, dl, value, cover = [], [], [], [], [], [], []

    def node(c):
        feature.append(LEAF)
        split.append(0)
        left.append(0)
        right.append(0)
        dl.append(0)
        value.append(float(np.float32(rng.standard_normal())))
        cover.append(c)
        return len(feature) - 1

    cur = node(1000.0)
    for f in feats:
        f = int(f)
        c = cover[cur]
        u = rng.uniform(0.2, 0.8)
        feature[cur] = f
        split[cur] = int(rng.integers(max(int(n_bins[f]) - 1, 1)))
        dl[cur] = int(rng.random() < 0.5)
        a = node(c * u)
        b = node(c - c * u)
        left[cur], right[cur] = (a, b) if rng.random() < 0.5 else (b, a)
        cur = a
    n = len(feature)
    return Tree(feature=np.array(feature, np.uint32), value=np.array(value, np.float32),
                left=np.array(left, np.uint32), right=np.array(right, np.uint32),
                default_left=np.array(dl, np.uint8), gains=np.zeros(n, np.float32),
                covers=np.array(cover, np.float32), split_bin=np.array(split, np.uint32),
                depth=depth)


@pytest.mark.gpu
@pytest.mark.parametrize("depth,n", [(12, 3), (12, 2_000), (24, 3), (24, 2_000)])
def test_shap_plan_long_paths(bb, depth, n):
    """Paths of 12 and 24 distinct features (16- and 32-element records)
    against the numpy path form, over codes with missing values."""
    rng = np.random.Generator(np.random.PCG64(91 + depth + n))
    F = 30
    nb = rng.integers(3, 200, F).astype(np.uint32)
    codes = np.empty((F, n), np.uint8)
    for f in range(F):
        c = rng.integers(0, nb[f] - 1, n)
        c[rng.random(n) < 0.1] = nb[f] - 1
        codes[f] = c
    off = np.concatenate([[0], np.cumsum(nb)]).astype(np.uint32)
    plane = bb.Plane.from_bins(codes, np.arange(off[-1], dtype=np.float32), off)
    trees = [chain_tree(rng, nb, depth) for _ in range(5)]
    phi = bb.ShapPlan(plane, trees, 0.25, 0.2).run(plane)
    ref = shap_numpy(codes.T.astype(np.int64), nb.astype(np.int64) - 1, trees, 0.25, 0.2)
    np.testing.assert_allclose(phi, ref, rtol=RTOL, atol=1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("grower,kw", [
    ("levelwise", dict(max_depth=6)),
    ("leafwise", dict(max_leaves=31, max_depth=10)),
    ("depthwise", dict(max_depth=6, subsample=0.7, feature_fraction=0.6)),
])
def test_device_contribs_match_live_reference_per_grower(bb, ref, grower, kw):
    """Against the live reference's pred_contribs_binned (include/bonsai/
    booster.hpp:887-924) on the same model: a levelwise ensemble (the reference
    explains each ObliviousTree through its preorder dense_equivalent, src/
    tree.cpp:64-117; here the level-order tree the device grew), a leafwise one,
    and a depthwise one grown over row and feature samples (covers count the
    sampled rows)."""
    from oracle import TreeCfg
    rng = np.random.Generator(np.random.PCG64(41))
    n, F = 4_000, 7
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.06] = np.nan
    x = np.nan_to_num(X)
    y = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.2 * rng.standard_normal(n)).astype(np.float32)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    tc = dict(grower=grower, learning_rate=0.1, **kw)
    m = ref.train(ds, TreeCfg(n_iters=12, **tc))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(use_graph=grower != "leafwise", **tc), max_trees=12)
    b.update(12)
    phi = bb.pred_contribs(plane, b.trees(), b.init_score, 0.1)
    want = m.contribs_binned(ds)
    np.testing.assert_allclose(phi, want, rtol=RTOL, atol=ATOL)


@pytest.mark.gpu
@pytest.mark.parametrize("grower", ["depthwise", "levelwise"])
def test_softmax_contribs_match_live_reference(bb, ref, grower):
    """A softmax ensemble's per-class contributions (n x K x (F + 1),
    MulticlassBooster's layout and composition) on the reference's own model
    (its trees, split bins recovered from their thresholds; a levelwise model
    through its preorder dense_equivalent) against the live reference's; each
    class's contributions sum to its raw score."""
    from oracle import TreeCfg
    from bonsai_b200 import synth
    from bonsai_b200.model import _split_bins
    K = 3
    X, y = synth.multiclass_onehot(n=3_000, n_classes=K)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=K, grower=grower, max_depth=4,
                              n_iters=6, learning_rate=0.1))
    trees = [bb.Tree(feature=t.feature, value=t.value, left=t.left, right=t.right,
                     default_left=t.default_left, gains=t.gains, covers=t.covers,
                     split_bin=_split_bins(t.feature, t.value, cuts, off)) for t in m.trees()]
    plane = bb.Plane(X, cuts, off)
    init = m.init_scores()
    phi = bb.pred_contribs_classes(plane, trees, init, 0.1)
    want = m.contribs_binned(ds, n_classes=K)
    np.testing.assert_allclose(phi, want, rtol=RTOL, atol=ATOL)
    raw = bb.predict_classes(plane, trees, init, 0.1).astype(np.float64)
    np.testing.assert_allclose(phi.sum(axis=2), raw, rtol=0, atol=1e-5)
