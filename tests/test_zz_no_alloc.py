"""bb_predict_static: ensemble predict for callers that may not allocate
device memory (a host whose device memory belongs to another allocator under
a fixed budget, or a latency-bound serving path that cannot take the
device-wide synchronisation of cudaMalloc / cudaFree). It must give the same
scores as bb_predict -- the same walk and the same float arithmetic, so the
tolerance here is zero -- on consecutive calls that reuse its one fixed
device array, and refuse ensembles larger than that array.

This file is collected last on purpose: a run that stops at the first
failure has run every other test before it."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pack(trees):
    roots = np.zeros(len(trees), np.uint32)
    parts = {k: [] for k in ("feature", "split_bin", "left", "right", "default_left", "value")}
    base = 0
    for i, t in enumerate(trees):
        roots[i] = base
        for k in parts:
            parts[k].append(getattr(t, k))
        base += len(t.feature)
    return roots, base, {k: np.ascontiguousarray(np.concatenate(v)) for k, v in parts.items()}


def _call(lib, plane, roots, n_nodes, t, init, lr, out_ptr):
    return lib.bb_predict_static(plane.h, len(roots), roots.ctypes.data, n_nodes,
                                 t["feature"].ctypes.data, t["split_bin"].ctypes.data,
                                 t["left"].ctypes.data, t["right"].ctypes.data,
                                 t["default_left"].ctypes.data, t["value"].ctypes.data,
                                 lr, init, out_ptr)


def test_predict_static_matches_predict_on_consecutive_calls(bb):
    import torch

    from bonsai_b200._lib import BB_ERR_CONFIG, check, lib
    rng = np.random.Generator(np.random.PCG64(77))
    n, F = 30_000, 9
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    y = (X[:, 0] + np.nan_to_num(X[:, 1]) * X[:, 2] > 0).astype(np.float32)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=6), max_trees=12)
    b.update(12)
    trees = b.trees()
    L = lib()
    # two calls in a row through the one fixed array, the second a larger
    # ensemble than the first
    for use in (trees[:5], trees):
        want = bb.predict(plane, use, b.init_score, 0.1)
        roots, n_nodes, t = _pack(use)
        out = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
        check(_call(L, plane, roots, n_nodes, t, b.init_score, 0.1, out.data_ptr()))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), want)
    # an ensemble beyond the array's 524,288 nodes is refused before anything runs
    roots, n_nodes, t = _pack(trees[:1])
    out = torch.zeros(n, dtype=torch.float32, device="cuda")
    rc = _call(L, plane, roots, 600_000, t, 0.0, 0.1, out.data_ptr())
    assert rc == BB_ERR_CONFIG
    assert "524,288" in L.bb_last_error().decode()


def test_predict_static_on_u16_codes_and_request_planes(bb):
    """The 16-bit code kernel (more than 256 bins per feature), and a request
    plane: before its first refill it holds no rows and the call runs
    nothing; refilled with a batch whose row count is not a multiple of 64
    (its column stride differs from an ingest plane's), the scores equal
    bb_predict's bit for bit, on two refills in a row."""
    import torch

    from bonsai_b200._lib import check, lib
    rng = np.random.Generator(np.random.PCG64(78))
    n, F = 20_000, 5
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.03] = np.nan
    y = (X[:, 0] * 2 + np.nan_to_num(X[:, 3]) > 0.5).astype(np.float32)
    cuts, off = bb.fit_cuts(X, max_bin=700)
    plane = bb.Plane(X, cuts, off)
    assert int(max(np.diff(off))) > 256                 # u16 codes
    b = bb.Booster(plane, y, bb.TrainParams(objective="logloss", max_depth=7), max_trees=6)
    b.update(6)
    trees = b.trees()
    roots, n_nodes, t = _pack(trees)
    L = lib()
    req = bb.Plane.like(plane, 9_000)
    out = torch.full((9_000,), 7.0, dtype=torch.float32, device="cuda")
    check(_call(L, req, roots, n_nodes, t, b.init_score, 0.1, out.data_ptr()))
    torch.cuda.synchronize()
    assert (out.cpu().numpy() == 7.0).all()             # nothing ran
    for batch in (None, X[:8_999], X[5:6_006]):
        use = plane if batch is None else req.refill(batch)
        m = n if batch is None else len(batch)
        want = bb.predict(use, trees, b.init_score, 0.1)
        out = torch.full((m,), float("nan"), dtype=torch.float32, device="cuda")
        check(_call(L, use, roots, n_nodes, t, b.init_score, 0.1, out.data_ptr()))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), want)
