"""Seeded synthetic stand-ins for the benchmark datasets.

The public datasets these shapes imitate (California Housing, HIGGS,
Covertype) are not available offline, so each generator draws a seeded
numpy PCG64 matrix with the named shape and value distribution. Every
matrix is float32, C-contiguous, row-major (n_rows x n_features).

  regression_small  20,640 x 8: columns 0,2,4,6 ~ U[0,1), 1,3,5,7 ~
                    LogNormal(0,1); y = sin(3 x0) + x1 x2 + 0.5 log1p(x3)
                    + N(0, 0.1^2).
  tall_binary       10,000,000 x 28: 21 N(0,1) columns plus 7 products /
                    absolute values of pairs; label ~ Bernoulli(sigmoid(
                    w.x + 0.5 x0 x1)), w ~ N(0, 0.5^2).
  wide_sparse       1,000,000 x 2,000, 90% NaN at uniform positions,
                    non-missing ~ LogNormal(0,1); y = sum of 20 products of
                    2-3 random features (NaN -> 0) + N(0, 0.1^2).
  multiclass_onehot 581,012 x 54: 10 N(0,1) columns and one-hot blocks of
                    4 and 40; 7 classes by argmax of seeded linear plus
                    interaction logits.
  ragged_many       64 regression datasets, rows log-uniform in
                    [1e3, 2e5], 28 N(0,1) features, y = sum of 8 random
                    depth-4 step trees + N(0, 0.1^2).
  serving           one dataset of the ragged_many family (the same 8 step
                    trees) to fit an ensemble on, and a matrix of request
                    rows (28 N(0,1) features) to score.
"""

from __future__ import annotations

import numpy as np

__all__ = [
    "regression_small",
    "tall_binary",
    "tall_binary_weights",
    "wide_sparse",
    "multiclass_onehot",
    "ragged_many",
    "serving",
]


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def regression_small(n: int = 20_640, seed: int = 20_640):
    rng = _rng(seed)
    X = np.empty((n, 8), dtype=np.float32)
    for j in range(8):
        if j % 2 == 0:
            X[:, j] = rng.random(n, dtype=np.float64)
        else:
            X[:, j] = rng.lognormal(0.0, 1.0, n)
    x = X.astype(np.float64)
    y = np.sin(3.0 * x[:, 0]) + x[:, 1] * x[:, 2] + 0.5 * np.log1p(x[:, 3])
    y = y + rng.normal(0.0, 0.1, n)
    return X, y.astype(np.float32)


def tall_binary_weights(seed: int = 10_000_000) -> np.ndarray:
    """The label model's weights w ~ N(0, 0.5^2) over the 28 columns."""
    return _rng(seed ^ 0x5EED).normal(0.0, 0.5, 28)


def tall_binary(n: int = 10_000_000, seed: int = 10_000_000, chunk: int = 1 << 21):
    """HIGGS-shaped binary classification; generated in row chunks so the
    float64 temporaries stay small at 10M rows."""
    w = tall_binary_weights()
    rng = _rng(seed)
    X = np.empty((n, 28), dtype=np.float32)
    y = np.empty(n, dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        b = rng.standard_normal((m, 21), dtype=np.float32)
        X[s:e, :21] = b
        X[s:e, 21] = b[:, 0] * b[:, 1]
        X[s:e, 22] = np.abs(b[:, 2])
        X[s:e, 23] = b[:, 3] * b[:, 4]
        X[s:e, 24] = np.abs(b[:, 5] * b[:, 6])
        X[s:e, 25] = b[:, 7] * b[:, 8]
        X[s:e, 26] = np.abs(b[:, 9])
        X[s:e, 27] = b[:, 10] * b[:, 11]
        z = X[s:e].astype(np.float64) @ w + 0.5 * X[s:e, 0].astype(np.float64) * X[s:e, 1]
        p = 1.0 / (1.0 + np.exp(-z))
        y[s:e] = (rng.random(m) < p).astype(np.float32)
    return X, y


def wide_sparse(n: int = 1_000_000, F: int = 2_000, seed: int = 2_000,
                missing: float = 0.9, chunk: int = 16_384):
    """Generated in row chunks (the 20 product terms drawn first), so the
    float64 temporaries stay small at 1M x 2,000."""
    rng = _rng(seed)
    terms = []
    for _ in range(20):
        k = int(rng.integers(2, 4))
        terms.append(rng.choice(F, size=k, replace=False))
    X = np.empty((n, F), dtype=np.float32)
    y = np.empty(n, dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        Xc = rng.lognormal(0.0, 1.0, (m, F)).astype(np.float32)
        Xc[rng.random((m, F)) < missing] = np.nan
        Z = np.nan_to_num(Xc, nan=0.0).astype(np.float64)
        yc = np.zeros(m)
        for cols in terms:
            yc += np.prod(Z[:, cols], axis=1)
        yc += rng.normal(0.0, 0.1, m)
        X[s:e] = Xc
        y[s:e] = yc
    return X, y


def multiclass_onehot(n: int = 581_012, seed: int = 581_012, n_classes: int = 7):
    rng = _rng(seed)
    cont = rng.standard_normal((n, 10))
    W = rng.normal(0.0, 1.0, (n_classes, 10))
    inter = np.stack([cont[:, i] * cont[:, i + 1] for i in range(n_classes)], axis=1)
    logits = cont @ W.T + 0.5 * inter
    # categorical blocks drawn from the logits' region: the block index is a
    # seeded hash of the dominant class plus noise
    a = (np.argmax(logits, axis=1) + rng.integers(0, 2, n)) % 4
    b = (np.argmax(logits[:, ::-1], axis=1) * 5 + rng.integers(0, 6, n)) % 40
    X = np.zeros((n, 54), dtype=np.float32)
    X[:, :10] = cont
    X[np.arange(n), 10 + a] = 1.0
    X[np.arange(n), 14 + b] = 1.0
    bump = rng.normal(0.0, 0.5, (n_classes, 44))
    logits = logits + X[:, 10:].astype(np.float64) @ bump.T
    y = np.argmax(logits, axis=1).astype(np.float32)
    return X, y


def _step_tree(rng, F):
    feats = rng.integers(0, F, 15)
    thr = rng.normal(0.0, 1.0, 15)
    leaves = rng.normal(0.0, 1.0, 16)
    return feats, thr, leaves


def _eval_step_tree(X, tree):
    feats, thr, leaves = tree
    idx = np.zeros(X.shape[0], dtype=np.int64)
    for _ in range(4):
        go_right = X[np.arange(X.shape[0]), feats[idx]] > thr[idx]
        idx = 2 * idx + 1 + go_right
    return leaves[idx - 15]


def ragged_many(n_sets: int = 64, seed: int = 64, F: int = 28,
                lo: float = 1e3, hi: float = 2e5):
    rng = _rng(seed)
    trees = [_step_tree(rng, F) for _ in range(8)]
    out = []
    for _ in range(n_sets):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        X = rng.standard_normal((n, F), dtype=np.float32)
        y = sum(_eval_step_tree(X, t) for t in trees) + rng.normal(0.0, 0.1, n)
        out.append((X, y.astype(np.float32)))
    return out


def serving(n_fit: int = 100_000, n_requests: int = 1_000_000, seed: int = 64, F: int = 28):
    """(X_fit, y_fit, X_requests): the fit set drawn like one ragged_many
    dataset (same step trees), the request rows from their own stream."""
    rng = _rng(seed)
    trees = [_step_tree(rng, F) for _ in range(8)]
    fr = _rng(seed + 1)
    X = fr.standard_normal((n_fit, F), dtype=np.float32)
    y = sum(_eval_step_tree(X, t) for t in trees) + fr.normal(0.0, 0.1, n_fit)
    Xr = _rng(seed + 2).standard_normal((n_requests, F), dtype=np.float32)
    return X, y.astype(np.float32), Xr
