"""Host-side cut fitting: the mappers the device ingest bins against.

Restates BinMapper::fit / create_cuts (src/bin_mapper.cpp:57-232) so that a
column's cuts are the reference's for the same working set: sort the
NaN-free sample, run-length encode it, then place at most max_bin - 2 cuts
by the lightest exact rule -- every distinct value when they fit the budget,
the count-weighted greedy walk when some value outweighs a mean bin
(greedy_weighted_cuts, :38-96), else the quantile stride -- and close with the
FLT_MAX top band and the +inf missing sentinel.

For tall data (more than n_samples rows) the reference draws one shared row
sample with libc++'s ranges::sample (src/bin_mappers.cpp:31-44), which no
other standard library reproduces; here the sample is numpy's seeded choice
of n_samples distinct rows. Cuts are an input fixed for both sides of every
parity comparison, so this affects which cuts a tall dataset gets, never
whether device and host agree on them.
"""

from __future__ import annotations

import numpy as np

FLT_MAX = np.float32(np.finfo(np.float32).max)
_MID_HI = np.float32(FLT_MAX / np.float32(2.0))                     # halving is exact
_MID_LO = np.float32(np.finfo(np.float32).tiny) * np.float32(2.0)   # 2 x smallest normal


def midpoint(a, b) -> np.float32:
    """std::midpoint for float (the greedy rule's cut, src/bin_mapper.cpp:95):
    the correctly rounded half-sum that never overflows. With both magnitudes
    at most FLT_MAX/2 the sum cannot overflow and (a + b) / 2 is exact up to
    one rounding; above that each operand is halved before the add, except one
    so small (below twice the smallest normal) that halving it would round --
    that one is added whole. These are the cases the C++ standard's midpoint
    proposal (P0811) states."""
    a = np.float32(a)
    b = np.float32(b)
    if abs(a) <= _MID_HI and abs(b) <= _MID_HI:
        return np.float32((a + b) / np.float32(2.0))
    if abs(a) < _MID_LO:
        return np.float32(a + b / np.float32(2.0))
    if abs(b) < _MID_LO:
        return np.float32(a / np.float32(2.0) + b)
    return np.float32(a / np.float32(2.0) + b / np.float32(2.0))


def _greedy(vals: np.ndarray, counts: np.ndarray, n_samples: int, budget: int,
            mean_bin: float) -> list:
    cuts: list = []
    n_groups = budget + 1
    is_big = counts.astype(np.float64) >= mean_bin
    n_big = int(is_big.sum())
    big_sum = int(counts[is_big].sum())
    rest_sum = n_samples - big_sum
    rest_groups = n_groups - n_big
    bin_size = rest_sum / rest_groups if rest_groups != 0 else mean_bin
    in_bin = 0
    i = 0
    while i + 1 < len(vals) and len(cuts) < budget:
        if not is_big[i]:
            rest_sum -= int(counts[i])
        in_bin += int(counts[i])
        if is_big[i] or in_bin >= bin_size or (is_big[i + 1] and in_bin >= bin_size / 2.0):
            mid = midpoint(vals[i], vals[i + 1])
            if not cuts or cuts[-1] < mid:
                cuts.append(mid)
            in_bin = 0
            if not is_big[i] and rest_groups > 1:
                rest_groups -= 1
                bin_size = rest_sum / rest_groups
        i += 1
    return cuts


def cuts_from_sample(sample: np.ndarray, max_bin: int = 255) -> np.ndarray:
    """BinMapper::from_sample (src/bin_mapper.cpp:240-252) on a NaN-free
    working set."""
    assert max_bin > 2
    budget = max_bin - 2
    s = np.asarray(sample, dtype=np.float32)
    if s.size >= 2048:
        # the reference's radix order (sort_floats, src/bin_mapper.cpp:115-157):
        # order-preserving keys, so a run of zeros starts with -0.0 if any
        b = s.view(np.uint32)
        key = np.where((b >> 31) != 0, ~b, b ^ np.uint32(0x80000000)).astype(np.uint32)
        key.sort()
        s = np.where((key >> 31) != 0, key ^ np.uint32(0x80000000), ~key).astype(
            np.uint32).view(np.float32)
    else:
        s = np.sort(s, kind="stable")
    if s.size:
        # run-length encode under operator<: -0.0 and +0.0 are one value
        new = np.empty(s.size, dtype=bool)
        new[0] = True
        new[1:] = s[:-1] < s[1:]
        starts = np.flatnonzero(new)
        vals = s[starts]
        counts = np.diff(np.append(starts, s.size))
    else:
        vals = s
        counts = np.zeros(0, dtype=np.int64)
    mean_bin = s.size / (budget + 1)
    if len(vals) <= budget:
        cuts = list(vals)
    elif counts.max() >= mean_bin:
        cuts = _greedy(vals, counts, s.size, budget, mean_bin)
    else:
        step = max((s.size + budget) // (budget + 1), 1)
        cuts = []
        for k in range(step, s.size, step):
            v = s[k]
            if not cuts or cuts[-1] < v:
                cuts.append(v)
    if not cuts or cuts[-1] < FLT_MAX:
        cuts.append(FLT_MAX)
    cuts.append(np.float32(np.inf))
    return np.asarray(cuts, dtype=np.float32)


def sample_rows(n_rows: int, n_samples: int = 200_000, seed: int = 0):
    """The shared row sample: None (every row) when n_rows <= n_samples."""
    if n_rows <= n_samples:
        return None
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.sort(rng.choice(n_rows, size=n_samples, replace=False))


def fit_cuts(X: np.ndarray, max_bin: int = 255, n_samples: int = 200_000, seed: int = 0):
    """Per-column cuts of row-major X: (cuts, cut_off), the column f's cuts
    being cuts[cut_off[f]:cut_off[f + 1]]."""
    X = np.asarray(X, dtype=np.float32)
    rows = sample_rows(X.shape[0], n_samples, seed)
    S = X if rows is None else X[rows]
    parts = []
    for f in range(X.shape[1]):
        col = S[:, f]
        parts.append(cuts_from_sample(col[~np.isnan(col)], max_bin))
    off = np.zeros(len(parts) + 1, dtype=np.uint32)
    off[1:] = np.cumsum([len(p) for p in parts])
    return np.concatenate(parts).astype(np.float32), off
