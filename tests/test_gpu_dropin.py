"""The drop-in check: the reference's own Booster (include/bonsai/booster.hpp:
484-592) trained with bonsai_b200's grower shim (include/bonsai_b200_grower.hpp)
in place of its CPU DepthwiseGrower must produce the same model -- the same
trees, node for node and bit for bit -- as the reference's CPU grower under
the same booster, sampler and feature draw."""

from __future__ import annotations

import os

import numpy as np
import pytest
from conftest import assert_trees_equal

from oracle import REF_B200_SO, RefLib, TreeCfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dref(bb):
    if not os.path.exists(REF_B200_SO):
        pytest.skip("the drop-in harness is not built (make -C oracle dropin)")
    return RefLib(REF_B200_SO)


def _data(seed=5, n=12_000, F=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.08] = np.nan
    X[:, 3] = np.round(X[:, 3] * 3)
    y = (np.sin(2 * np.nan_to_num(X[:, 0])) + np.nan_to_num(X[:, 1]) * np.nan_to_num(X[:, 3])
         + rng.normal(0, 0.1, n)).astype(np.float32)
    return X, y


@pytest.mark.parametrize("cfg", [
    dict(max_depth=6, n_iters=30, learning_rate=0.1),
    dict(max_depth=5, n_iters=20, feature_fraction=0.5, lambda_l1=0.3),
    dict(max_depth=6, n_iters=20, subsample=0.8, min_data_in_leaf=5),
    dict(max_depth=4, n_iters=15, monotone=[1, 0, 0, -1, 0, 0, 0]),
    dict(max_depth=5, n_iters=10, interaction_constraints=["0,1", "1+3", "2"]),
])
def test_reference_booster_over_b200_grower_matches_cpu(dref, cfg):
    X, y = _data()
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    tc = TreeCfg(**cfg)
    cpu = dref.train(ds, tc)
    gpu = dref.train_b200(ds, tc)
    assert cpu.n_trees() == gpu.n_trees() == tc.n_iters
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")
    assert np.array_equal(gpu.predict_binned(ds), cpu.predict_binned(ds))


def test_reference_booster_over_b200_grower_logloss(dref):
    X, y = _data(seed=9)
    yb = (y > np.median(y)).astype(np.float32)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, yb, cuts, off)
    tc = TreeCfg(objective="logloss", max_depth=6, n_iters=20)
    cpu = dref.train(ds, tc)
    gpu = dref.train_b200(ds, tc)
    # host objective on both sides: the same gradients, the same trees
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")


@pytest.mark.parametrize("objective,kw", [("mae", {}), ("huber", dict(huber_delta=0.5)),
                                          ("quantile", dict(quantile_alpha=0.8))])
@pytest.mark.parametrize("subsample", [1.0, 0.8])
def test_reference_booster_over_b200_grower_renewed_leaves(dref, objective, kw, subsample):
    """The host objectives whose booster renews every leaf from its rows'
    residuals (Booster::renew_leaves, include/bonsai/booster.hpp:561-591,
    763-785: MAE and quantile take the leaf's residual quantile, Huber its
    own rule) read each row's leaf id from the grower -- sampled rows from
    their leaf segments, the rest routed through the finished tree -- so the
    renewed models agree only if every id does."""
    X, y = _data(seed=11)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    tc = TreeCfg(objective=objective, max_depth=5, n_iters=10, learning_rate=0.2,
                 subsample=subsample, **kw)
    cpu = dref.train(ds, tc)
    gpu = dref.train_b200(ds, tc)
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")
    assert np.array_equal(gpu.predict_binned(ds), cpu.predict_binned(ds))


@pytest.mark.parametrize("grower,cfg", [
    ("leafwise", dict(max_leaves=31, max_depth=12, n_iters=15)),
    ("leafwise", dict(max_leaves=63, max_depth=255, n_iters=10, subsample=0.8,
                      feature_fraction=0.5, lambda_l1=0.2)),
    ("leafwise", dict(max_leaves=31, max_depth=8, n_iters=8, objective="mae", subsample=0.8)),
    ("levelwise", dict(max_depth=6, n_iters=15)),
    ("levelwise", dict(max_depth=7, n_iters=10, subsample=0.8, feature_fraction=0.6,
                       min_child_hess=4.0)),
    ("levelwise", dict(max_depth=5, n_iters=8, objective="quantile", quantile_alpha=0.3,
                       subsample=0.8)),
])
def test_reference_booster_over_leafwise_and_levelwise_shims(dref, grower, cfg):
    """The same drop-in check for B200LeafwiseGrower and B200ObliviousGrower
    (include/bonsai_b200_grower.hpp): the reference's booster over each equals
    it over the reference's LeafwiseGrower / ObliviousGrower, tree for tree --
    a levelwise model's ObliviousTree tables too, its leaf ids being leaf-table
    indices (the quantile objective renews leaves by them)."""
    X, y = _data(seed=13)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    tc = TreeCfg(grower=grower, learning_rate=0.2, **cfg)
    cpu = dref.train(ds, tc)
    gpu = dref.train_b200(ds, tc)
    assert cpu.n_trees() == gpu.n_trees() == tc.n_iters
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")
        if grower == "levelwise":
            for a, b in zip(gpu.oblivious(i), cpu.oblivious(i)):
                assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert np.array_equal(gpu.predict_binned(ds), cpu.predict_binned(ds))


@pytest.mark.parametrize("cfg", [dict(dart_drop_rate=0.3),
                                 dict(dart_drop_rate=0.5, subsample=0.8, feature_fraction=0.7)])
def test_reference_booster_over_b200_grower_dart(dref, cfg):
    """DART (booster_config.dart_drop_rate; drop_dart_trees / apply_dart_round,
    include/bonsai/booster.hpp:535-540,700-760) runs the reference's host round
    -- trees dropped, gradients against the thinned model, dropped and new
    trees rescaled -- over the shim as over the CPU grower: the same model."""
    X, y = _data(seed=17)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    tc = TreeCfg(max_depth=5, n_iters=12, learning_rate=0.2, **cfg)
    cpu = dref.train(ds, tc)
    gpu = dref.train_b200(ds, tc)
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")
    assert np.array_equal(gpu.predict_binned(ds), cpu.predict_binned(ds))


@pytest.mark.parametrize("grower", ["depthwise", "leafwise", "levelwise"])
def test_reference_booster_over_b200_grower_goss(dref, grower):
    """GOSS (GossSampler, src/sampler.cpp:57-125: the top_rate rows by |g| and an
    amplified other_rate draw of the rest) chooses rows from the gradients and
    scales theirs, then hands both to the grower: over each shim the same
    model as over the reference's CPU grower of that kind."""
    X, y = _data(seed=19)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    tc = TreeCfg(grower=grower, max_depth=5, max_leaves=31, n_iters=10, learning_rate=0.2,
                 goss_top_rate=0.2, goss_other_rate=0.15)
    cpu = dref.train(ds, tc)
    gpu = dref.train_b200(ds, tc)
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")
    assert np.array_equal(gpu.predict_binned(ds), cpu.predict_binned(ds))
