"""The Bernoulli row sampler's restatement (oracle.bernoulli_keep) against
the reference's own booster: each tree's root cover is the number of rows
its draw kept (BernoulliSampler::sample, src/sampler.cpp:36-55, from the
booster's std::mt19937, include/bonsai/booster.hpp:496), over several
rounds and two seeds, for the single-output and the multiclass boosters."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import TreeCfg, bernoulli_keep


def _data(n=3_000, F=5, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    y = (X[:, 0] + 0.5 * X[:, 1] * X[:, 2] + 0.1 * rng.standard_normal(n)).astype(np.float32)
    return X, y


@pytest.mark.parametrize("seed,p", [(42, 0.8), (7, 0.35)])
def test_restated_draws_match_reference_root_covers(ref, seed, p):
    X, y = _data()
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(max_depth=3, n_iters=5, subsample=p, random_seed=seed))
    keep = bernoulli_keep(len(y), p, seed, 5)
    assert [int(t.covers[0]) for t in m.trees()] == [int(k.sum()) for k in keep]


def test_restated_draws_match_reference_multiclass(ref):
    rng = np.random.Generator(np.random.PCG64(1))
    X = rng.standard_normal((2_000, 4)).astype(np.float32)
    y = rng.integers(0, 3, 2_000).astype(np.float32)
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(objective="softmax", n_classes=3, max_depth=3, n_iters=2,
                              subsample=0.6, random_seed=5))
    keep = bernoulli_keep(len(y), 0.6, 5, 6)  # round-major: a draw per class tree
    assert [int(t.covers[0]) for t in m.trees()] == [int(k.sum()) for k in keep]
