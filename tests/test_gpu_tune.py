"""The launch-shape autotuner on the device: it times every candidate CTA
count per tile on the caller's data and keeps the fastest in its cache, and
-- the quantised cells being order-free integer sums -- every launch shape
grows the same trees bit for bit, on planes of one and of ten mirror tiles."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import assert_trees_equal

pytestmark = pytest.mark.gpu


def _data(n, F, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    y = (np.nan_to_num(X[:, 0]) + np.nan_to_num(X[:, 1]) * np.nan_to_num(X[:, 2])
         > 0).astype(np.float32)
    return X, y


@pytest.mark.parametrize("n,F,grower", [(200_000, 28, "depthwise"), (40_000, 300, "leafwise")])
def test_every_launch_shape_grows_the_same_trees(bb, n, F, grower):
    X, y = _data(n, F, 3)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    base = bb.TrainParams(objective="logloss", grower=grower, max_depth=6, max_leaves=31,
                          hist_mode="int8", seed=5, use_graph=grower != "leafwise")

    def fit(ctas):
        b = bb.Booster(plane, y, bb.TrainParams(**{**base.__dict__, "hist_ctas": ctas}),
                       max_trees=4)
        b.update(4)
        return b.trees(), b.scores()

    want, ws = fit(0)
    for ctas in (1, 3, 37, 148, 500):
        got, gs = fit(ctas)
        for i, (a, c) in enumerate(zip(got, want)):
            assert_trees_equal(a, c, f"ctas {ctas} tree {i}")
        assert np.array_equal(gs, ws)


def test_tune_times_candidates_and_caches(bb, tmp_path):
    from bonsai_b200 import autotune
    X, y = _data(100_000, 28, 4)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    params = bb.TrainParams(objective="logloss", max_depth=6, hist_mode="int8", use_graph=True)
    path = str(tmp_path / "tune.json")
    got = bb.tune(plane, y, params, rounds=2, path=path)
    assert got.hist_ctas in autotune.CANDIDATES
    entries = autotune.load(path)
    (entry,) = entries.values()
    assert set(int(k) for k in entry["ms_per_round"]) == set(autotune.CANDIDATES)
    assert all(v > 0 for v in entry["ms_per_round"].values())
    again = bb.tune(plane, y, params, rounds=2, path=path, timer=lambda p: 1 / 0)
    assert again.hist_ctas == got.hist_ctas
