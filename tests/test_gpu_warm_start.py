"""Warm start (bonsai_b200.model.warm_start / continued): a model, saved and
loaded, continues training from scores rebuilt as the reference rebuilds them
(include/bonsai/booster.hpp:512-524: init + lr x the loaded trees' leaf values
summed in tree order). Against the reference's own booster loaded with the
same trees (load_state) and trained the same extra rounds: every new tree and
the joined model's predictions bit for bit for squared error; for logloss the
splits exactly and values within 1e-4 (the device's expf against the
host's)."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from bonsai_b200 import model as M
from oracle import TreeCfg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("objective", ["mse", "logloss"])
def test_warm_start_matches_reference(bb, ref, objective, tmp_path):
    rng = np.random.Generator(np.random.PCG64(23))
    n, F = 8_000, 6
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    x = np.nan_to_num(X)
    y = (x[:, 0] + x[:, 1] * x[:, 2] + 0.2 * rng.standard_normal(n)).astype(np.float32)
    if objective == "logloss":
        y = (y > 0).astype(np.float32)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    plane = bb.Plane(X, cuts, off)
    p = bb.TrainParams(objective=objective, max_depth=5, learning_rate=0.1, use_graph=True)
    first = bb.Booster(plane, y, p, max_trees=4)
    first.update(4)
    path = str(tmp_path / "first.bonsai")
    M.from_booster(first, cuts, off).save(path)
    loaded = M.load(path)
    more = M.warm_start(loaded, plane, y, p, max_trees=5)
    more.update(5)
    joined = M.continued(loaded, more)
    want = ref.warm_train(ds, TreeCfg(objective=objective, max_depth=5, learning_rate=0.1,
                                      n_iters=5), loaded.trees, loaded.init_score)
    assert want.n_trees() == len(joined.trees) == 9
    # logloss gradients go through the device's expf, which may round apart
    # from the host's in the last place (the logloss tolerance, 1e-4): exact
    # splits, leaf values and gains to that tolerance
    exact = TREE_FIELDS if objective == "mse" else ("feature", "left", "right",
                                                    "default_left", "covers")
    for i in range(9):
        a, b = joined.trees[i], want.tree(i)
        for k in exact:
            assert np.array_equal(np.asarray(getattr(a, k)).view(np.uint8),
                                  np.asarray(getattr(b, k)).view(np.uint8)), (i, k)
        for k in set(TREE_FIELDS) - set(exact):
            np.testing.assert_allclose(getattr(a, k), getattr(b, k), rtol=1e-4, atol=1e-6)
    got = bb.predict(plane, joined.trees, joined.init_score, 0.1)
    if objective == "mse":
        assert np.array_equal(got.view(np.uint32), want.predict_binned(ds).view(np.uint32))
    else:
        np.testing.assert_allclose(got, want.predict_binned(ds), rtol=1e-4, atol=1e-5)
    assert joined.config["booster_config"]["n_iters"] == 9
