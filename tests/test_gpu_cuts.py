"""Cut fitting on the device (bb_fit_cuts) against the host restatement
(bonsai_b200.fit_cuts) and the reference's own BinMapper::fit (oracle/_ref):
the same cuts, bit for bit, for columns that take each of the three rules
(every distinct value, the greedy walk, the quantile stride), columns with
NaN, all-NaN and constant columns, signed zeros, infinities, budgets from 3
to 700 bins, a tall matrix through the shared row sample, device input, and
more columns than one device pass holds."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _columns(rng, n):
    cols = [
        rng.standard_normal(n),                                         # quantile stride
        rng.integers(0, 12, n),                                         # distinct values
        np.where(rng.random(n) < 0.8, 0.0, rng.standard_normal(n)),     # heavy value: greedy
        np.round(rng.lognormal(0, 1, n), 1),                            # many duplicates
        np.where(rng.random(n) < 0.3, -0.0, rng.standard_normal(n)),   # signed zeros
        np.full(n, 3.25),                                               # constant
        np.full(n, np.nan),                                             # all missing
        np.where(rng.random(n) < 0.01, -np.inf, rng.standard_normal(n) * 1e30),
        np.where(rng.random(n) < 0.5, 7.0, rng.integers(0, 400, n)),    # heavy + many distinct
    ]
    X = np.stack(cols, 1).astype(np.float32)
    m = rng.random(X.shape) < 0.1
    m[:, 5] = False
    X[m] = np.nan
    return X


def _same(a, b, what):
    (ca, oa), (cb, ob) = a, b
    assert np.array_equal(oa, ob), what
    assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32)), what


@pytest.mark.parametrize("n", [1, 500, 5_000, 60_000])
@pytest.mark.parametrize("max_bin", [3, 16, 255, 256, 700])
def test_device_cuts_equal_host_cuts(bb, n, max_bin):
    rng = np.random.Generator(np.random.PCG64(n + max_bin))
    X = _columns(rng, n)
    _same(bb.fit_cuts_device(X, max_bin=max_bin), bb.fit_cuts(X, max_bin=max_bin),
          (n, max_bin))


@pytest.mark.parametrize("max_bin", [16, 255])
def test_device_cuts_equal_reference(bb, ref, max_bin):
    rng = np.random.Generator(np.random.PCG64(7))
    X = _columns(rng, 8_000)
    _same(bb.fit_cuts_device(X, max_bin=max_bin), ref.fit_cuts(X, max_bin=max_bin), max_bin)


def test_device_cuts_tall_sample_and_device_input(bb):
    import torch
    rng = np.random.Generator(np.random.PCG64(11))
    X = _columns(rng, 250_000)            # above n_samples: the shared row sample
    want = bb.fit_cuts(X)
    _same(bb.fit_cuts_device(X), want, "host input")
    _same(bb.fit_cuts_device(torch.from_numpy(X).cuda()), want, "device input")


def test_device_cuts_many_columns(bb):
    """1,600 columns x 60,000 rows: more than one pass of the device scratch."""
    rng = np.random.Generator(np.random.PCG64(13))
    X = rng.lognormal(0, 1, (60_000, 1_600)).astype(np.float32)
    X[rng.random(X.shape) < 0.5] = np.nan
    X[:, ::7] = np.round(X[:, ::7], 0)
    _same(bb.fit_cuts_device(X), bb.fit_cuts(X), "wide")


@pytest.mark.parametrize("max_bin", [16, 255])
def test_device_cuts_extreme_magnitudes(bb, ref, max_bin):
    """Greedy-rule columns above FLT_MAX / 2, huge values next to subnormal
    ones, subnormal runs and infinities: the device midpoint is
    std::midpoint's, so device cuts equal the host restatement's and the
    reference's bit for bit."""
    from test_abi import _extreme_columns
    X = _extreme_columns(np.random.Generator(np.random.PCG64(41)))
    want = ref.fit_cuts(X, max_bin=max_bin)
    _same(bb.fit_cuts(X, max_bin=max_bin), want, "host")
    _same(bb.fit_cuts_device(X, max_bin=max_bin), want, "device")
