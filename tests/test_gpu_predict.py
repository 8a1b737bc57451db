"""Ensemble predict through the plan (bb_predict_plan_*, the reference's
cuda_predict_plan + cuda_predict, include/bonsai/cuda/predict.hpp:29-38)
must equal the oracle's bin-space walk bit for bit: each row's leaves summed
in float in tree order, then init + lr * sum (predict_at_binned,
include/bonsai/booster.hpp:831-845; the reference's own device pin is
tests/unit/test_cuda_predict.cpp:88-140).

The ensembles are random trees in the reference's DenseTree layout: leaves
at every depth (so the heap form pads), splits with either default
direction, split bins at and past the missing bin, a root that is a leaf;
planes with missing codes, u8 and u16 codes, one to three mirror tiles;
batches from 1 row (trees split across CTAs, summed by the warp kernel)
through 320,000 rows (1,024-row CTAs)."""

from __future__ import annotations

from collections import deque

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LEAF = 0xFFFFFFFF


def random_tree(rng, n_bins, max_depth, p_leaf=0.12, root_leaf=False):
    from bonsai_b200 import Tree
    feat, split, left, right, dl, val = [], [], [], [], [], []

    def new():
        feat.append(LEAF)
        split.append(0)
        left.append(0)
        right.append(0)
        dl.append(0)
        val.append(0.0)
        return len(feat) - 1

    queue = deque([(new(), 0)])
    while queue:
        i, d = queue.popleft()
        if d == max_depth or (d > 0 and rng.random() < p_leaf) or (d == 0 and root_leaf):
            val[i] = float(np.float32(rng.standard_normal()))
            continue
        f = int(rng.integers(len(n_bins)))
        last = int(n_bins[f]) - 1
        u = rng.random()
        if u < 0.04:
            s = last            # only the missing bin can go right
        elif u < 0.06:
            s = last + 3        # past every code
        else:
            s = int(rng.integers(max(last, 1)))
        feat[i], split[i], dl[i] = f, s, int(rng.random() < 0.5)
        a, b = new(), new()
        left[i], right[i] = a, b
        queue.append((a, d + 1))
        queue.append((b, d + 1))
    n = len(feat)
    return Tree(feature=np.array(feat, np.uint32), value=np.array(val, np.float32),
                left=np.array(left, np.uint32), right=np.array(right, np.uint32),
                default_left=np.array(dl, np.uint8), gains=np.zeros(n, np.float32),
                covers=np.ones(n, np.float32), split_bin=np.array(split, np.uint32),
                depth=max_depth)


def random_plane(bb, rng, n, n_bins, p_missing=0.07):
    F = len(n_bins)
    u16 = int(max(n_bins)) > 256
    codes = np.empty((F, n), np.uint16 if u16 else np.uint8)
    for f in range(F):
        c = rng.integers(0, n_bins[f] - 1, n)
        c[rng.random(n) < p_missing] = n_bins[f] - 1
        codes[f] = c
    off = np.concatenate([[0], np.cumsum(n_bins)]).astype(np.uint32)
    cuts = np.arange(off[-1], dtype=np.float32)
    return bb.Plane.from_bins(codes, cuts, off), codes.astype(np.uint16)


def _bins(rng, F, top=256):
    return rng.integers(2, top + 1, F).astype(np.uint32)


def _ensemble(rng, n_bins, n_trees, max_depth):
    trees = [random_tree(rng, n_bins, max_depth, root_leaf=(t == 3)) for t in range(n_trees)]
    return trees


@pytest.mark.parametrize("n", [1, 37, 5_000, 40_000, 320_000])
def test_plan_equals_oracle_u8(bb, orc, n):
    rng = np.random.Generator(np.random.PCG64(100 + n))
    nb = _bins(rng, 28)
    plane, codes = random_plane(bb, rng, n, nb)
    trees = _ensemble(rng, nb, 40, 8)
    plan = bb.PredictPlan(plane, trees, 0.37, 0.1)
    assert plan.depth == 8
    got = plan.run(plane)
    want = orc.predict_binned(codes, nb, trees, 0.37, 0.1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # a plan runs again with the same scores, and bb_predict is the same walk
    assert np.array_equal(plan.run(plane).view(np.uint32), got.view(np.uint32))
    assert np.array_equal(bb.predict(plane, trees, 0.37, 0.1).view(np.uint32),
                          got.view(np.uint32))


@pytest.mark.parametrize("F,top,n", [(20, 700, 3_000), (20, 700, 60_000), (70, 256, 9_000),
                                     (70, 256, 50_000), (40, 300, 45_000), (9, 256, 2_000)])
def test_plan_equals_oracle_widths(bb, orc, F, top, n):
    """u16 codes (bins above 256), and planes over two and three mirror tiles."""
    rng = np.random.Generator(np.random.PCG64(F * 1000 + n))
    nb = _bins(rng, F, top)
    plane, codes = random_plane(bb, rng, n, nb)
    trees = _ensemble(rng, nb, 25, 7)
    plan = bb.PredictPlan(plane, trees, -1.25, 0.3)
    assert plan.depth == 7
    want = orc.predict_binned(codes, nb, trees, -1.25, 0.3)
    assert np.array_equal(plan.run(plane).view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("depth", [1, 3, 10])
def test_plan_depths(bb, orc, depth):
    rng = np.random.Generator(np.random.PCG64(7 + depth))
    nb = _bins(rng, 12)
    plane, codes = random_plane(bb, rng, 12_345, nb)
    trees = [random_tree(rng, nb, depth, p_leaf=0.05) for _ in range(30)]
    plan = bb.PredictPlan(plane, trees, 0.0, 1.0)
    assert plan.depth == depth
    want = orc.predict_binned(codes, nb, trees, 0.0, 1.0)
    assert np.array_equal(plan.run(plane).view(np.uint32), want.view(np.uint32))


def test_plan_tree_prefix(bb, orc):
    """n_trees > 0 scores the first n_trees trees only (cuda_predict's
    n_trees, include/bonsai/cuda/predict.hpp:33-38)."""
    rng = np.random.Generator(np.random.PCG64(31))
    nb = _bins(rng, 28)
    plane, codes = random_plane(bb, rng, 20_000, nb)
    trees = _ensemble(rng, nb, 50, 6)
    plan = bb.PredictPlan(plane, trees, 0.5, 0.1)
    for k in (1, 17, 50):
        want = orc.predict_binned(codes, nb, trees[:k], 0.5, 0.1)
        assert np.array_equal(plan.run(plane, k).view(np.uint32), want.view(np.uint32))
    with pytest.raises(bb.BonsaiError):
        plan.run(plane, 51)


def test_plan_on_another_plane(bb, orc):
    """A plan runs over any plane with its features and bin counts, and
    refuses one whose shape differs."""
    rng = np.random.Generator(np.random.PCG64(41))
    nb = _bins(rng, 28)
    plane_a, _ = random_plane(bb, rng, 1_000, nb)
    plane_b, codes_b = random_plane(bb, rng, 77_777, nb)
    trees = _ensemble(rng, nb, 30, 8)
    plan = bb.PredictPlan(plane_a, trees, 0.1, 0.1)
    want = orc.predict_binned(codes_b, nb, trees, 0.1, 0.1)
    assert np.array_equal(plan.run(plane_b).view(np.uint32), want.view(np.uint32))
    nb2 = nb.copy()
    nb2[5] += 1
    plane_c, _ = random_plane(bb, rng, 1_000, nb2)
    with pytest.raises(bb.BonsaiError):
        plan.run(plane_c)
    plane_d, _ = random_plane(bb, rng, 1_000, nb[:27])
    with pytest.raises(bb.BonsaiError):
        plan.run(plane_d)


def test_node_form_for_deep_trees_and_wide_planes(bb, orc):
    """Ensembles deeper than 10 and planes over more than 8 mirror tiles keep
    the node tables; the scores are the same walk's."""
    rng = np.random.Generator(np.random.PCG64(53))
    nb = _bins(rng, 16)
    plane, codes = random_plane(bb, rng, 10_000, nb)
    trees = [random_tree(rng, nb, 14, p_leaf=0.3) for _ in range(12)]
    trees.append(random_tree(rng, nb, 13, p_leaf=0.0))
    plan = bb.PredictPlan(plane, trees, 0.2, 0.1)
    assert plan.depth == 0
    want = orc.predict_binned(codes, nb, trees, 0.2, 0.1)
    assert np.array_equal(plan.run(plane).view(np.uint32), want.view(np.uint32))
    nb = _bins(rng, 300)
    plane, codes = random_plane(bb, rng, 3_000, nb)
    trees = _ensemble(rng, nb, 10, 6)
    plan = bb.PredictPlan(plane, trees, 0.2, 0.1)
    assert plan.depth == 0
    want = orc.predict_binned(codes, nb, trees, 0.2, 0.1)
    assert np.array_equal(plan.run(plane).view(np.uint32), want.view(np.uint32))


def test_plan_launch_into_device_memory(bb):
    """bb_predict_plan_launch enqueues on the caller's stream into device
    memory: the same scores as run."""
    import torch
    rng = np.random.Generator(np.random.PCG64(67))
    nb = _bins(rng, 28)
    for n in (3, 100_000):
        plane, _ = random_plane(bb, rng, n, nb)
        trees = _ensemble(rng, nb, 64, 8)
        plan = bb.PredictPlan(plane, trees, 0.3, 0.05)
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        s = torch.cuda.Stream()
        k = plan.launch(plane, out.data_ptr(), s.cuda_stream)
        assert k == (2 if n == 3 else 1)
        s.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32),
                              plan.run(plane).view(np.uint32))


def test_plan_matches_trained_booster(bb):
    """A booster's 100 trees scored through a plan equal the reference's
    golden predictions (predict_binned of its own CPU booster)."""
    from conftest import load_golden

    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    X, y = synth.regression_small()
    plane = bb.Plane(X, d["cuts"], d["cut_off"])
    b = bb.Booster(plane, y, bb.TrainParams(max_depth=6), max_trees=100)
    b.update(100)
    plan = bb.PredictPlan(plane, b.trees(), b.init_score, 0.1)
    assert plan.depth == 6
    assert np.array_equal(plan.run(plane), d["pred"])
