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


def test_reference_booster_over_b200_grower_logloss(dref, monkeypatch):
    X, y = _data(seed=9)
    yb = (y > np.median(y)).astype(np.float32)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, yb, cuts, off)
    tc = TreeCfg(objective="logloss", max_depth=6, n_iters=20)
    cpu = dref.train(ds, tc)
    # the reference's own escape hatch keeps the host objective (booster.hpp:
    # 634-636): the same host gradients on both sides, the same trees
    monkeypatch.setenv("BONSAI_HOST_OBJECTIVE", "1")
    gpu = dref.train_b200(ds, tc)
    for i in range(tc.n_iters):
        assert_trees_equal(gpu.tree(i), cpu.tree(i), f"round {i}")


# ---- the resident round through the reference's own Booster seam
# (try_resident_round / resident_round, include/bonsai/booster.hpp:630-676):
# the shim arms it, so grow() runs whole device rounds (bb_booster_*).

def _bb_fit(bb, X, y, cuts, off, n_iters, **kw):
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(use_graph=True, **kw), max_trees=n_iters)
    b.update(n_iters)
    return b.trees(), plane


def _same_tree(a, t, where):
    """A reference-harvested tree against one of this package's trees."""
    for k in ("feature", "left", "right", "default_left"):
        assert np.array_equal(getattr(a, k), getattr(t, k)), f"{where} {k}"
    for k in ("value", "gains", "covers"):
        x = getattr(a, k)
        z = getattr(t, k)
        assert np.array_equal(x.view(np.uint32), z.view(np.uint32)), f"{where} {k}"


@pytest.mark.parametrize("subsample", [1.0, 0.8])
def test_resident_rounds_through_the_booster_equal_the_host_rounds(dref, monkeypatch,
                                                                  subsample):
    """Squared error: the reference's booster arms the shim's resident round
    (device gradients and fused score updates; a Bernoulli sample's rows handed
    over each round with bb_booster_set_rows) and its trees equal those of the
    same booster kept on the host objective, and the CPU grower's, bit for bit."""
    X, y = _data(seed=21)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    tc = TreeCfg(max_depth=6, n_iters=12, learning_rate=0.2, subsample=subsample,
                 feature_fraction=0.8)
    cpu = dref.train(ds, tc)
    res = dref.train_b200(ds, tc)
    monkeypatch.setenv("BONSAI_HOST_OBJECTIVE", "1")
    host = dref.train_b200(ds, tc)
    for i in range(tc.n_iters):
        assert_trees_equal(res.tree(i), cpu.tree(i), f"round {i}")
        assert_trees_equal(host.tree(i), cpu.tree(i), f"round {i}")
    assert np.array_equal(res.predict_binned(ds), cpu.predict_binned(ds))


@pytest.mark.parametrize("mode", ["int8", "int16"])
@pytest.mark.parametrize("subsample", [1.0, 0.8])
def test_quantised_resident_round_through_the_booster(bb, dref, mode, subsample):
    """The quantised form behind the reference's Booster<LogLoss, B200
    DepthwiseGrowerInt8|Int16, AllRows|Bernoulli>: the resident rounds are
    this package's quantised rounds -- the same trees as bb_booster_* fitting
    the same data with the same seed (the sampler's rows are the device
    booster's own Bernoulli draws from the same seed)."""
    X, y = _data(seed=23, n=20_000)
    yb = (y > np.median(y)).astype(np.float32)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, yb, cuts, off)
    tc = TreeCfg(objective="logloss", max_depth=6, n_iters=10, learning_rate=0.2,
                 subsample=subsample, hist_mode=mode)
    got = dref.train_b200(ds, tc)
    want, _ = _bb_fit(bb, X, yb, cuts, off, tc.n_iters, objective="logloss", max_depth=6,
                      learning_rate=0.2, hist_mode=mode, seed=0, subsample=subsample,
                      random_seed=tc.random_seed)
    assert got.n_trees() == len(want) == tc.n_iters
    for i in range(tc.n_iters):
        _same_tree(got.tree(i), want[i], f"round {i}")


@pytest.mark.parametrize("grower", ["levelwise", "leafwise"])
def test_quantised_resident_levelwise_and_leafwise(bb, dref, grower):
    X, y = _data(seed=25, n=15_000)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    kw = dict(max_depth=5) if grower == "levelwise" else dict(max_depth=10, max_leaves=31)
    tc = TreeCfg(grower=grower, n_iters=6, learning_rate=0.2, hist_mode="int8", **kw)
    got = dref.train_b200(ds, tc)
    want, _ = _bb_fit(bb, X, y, cuts, off, tc.n_iters, grower=grower, learning_rate=0.2,
                      hist_mode="int8", seed=0, **kw)
    for i in range(tc.n_iters):
        if grower == "levelwise":
            # the reference keeps ObliviousTree tables: levels and leaf table
            for a, b in zip(got.oblivious(i), bb.oblivious_tables(want[i])):
                assert np.array_equal(np.asarray(a).view(np.uint8),
                                      np.asarray(b).view(np.uint8)), f"round {i}"
        else:
            _same_tree(got.tree(i), want[i], f"round {i}")


def test_resident_validation_plane_through_the_booster(dref, monkeypatch):
    """The fit loop's device validation route (src/cli/pipeline.cpp:420-450)
    over the shim: round 0's tree is added on arming and its loss is the
    host's; every later round's loss comes from the device plane and equals
    the host route's loss (the same booster kept on the host objective and
    the host bin-space walk) within float rounding."""
    X, y = _data(seed=27, n=12_000)
    Xv, yv = _data(seed=28, n=3_000)
    cuts, off = dref.fit_cuts(X)
    ds = dref.dataset(X, y, cuts, off)
    vs = dref.dataset(Xv, yv, cuts, off)
    tc = TreeCfg(max_depth=5, n_iters=8, learning_rate=0.2)
    model, losses, dev = dref.train_b200_valid(ds, vs, tc)
    assert dev[0] == 0 and (dev[1:] == 1).all()
    cpu = dref.train(ds, tc)
    for i in range(tc.n_iters):
        assert_trees_equal(model.tree(i), cpu.tree(i), f"round {i}")
    monkeypatch.setenv("BONSAI_HOST_OBJECTIVE", "1")
    host, host_losses, host_dev = dref.train_b200_valid(ds, vs, tc)
    assert (host_dev == 0).all()
    for i in range(tc.n_iters):
        assert_trees_equal(host.tree(i), cpu.tree(i), f"round {i}")
    assert losses[0] == host_losses[0]
    np.testing.assert_allclose(losses, host_losses, rtol=1e-5)


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
