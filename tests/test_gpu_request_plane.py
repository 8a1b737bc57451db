"""Request planes (bb_plane_create_like + bb_plane_refill): a plane sized once
and refilled with each batch -- from host or device memory, batches of any
size up to its capacity, larger then smaller then larger again -- holds the
same codes as a plane ingested from that batch alone, and predict and
TreeSHAP plans score it exactly as they score that plane."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(bb):
    from bonsai_b200 import synth
    X, y, Xr = synth.serving(n_fit=5_000, n_requests=50_000)
    Xr[::7, 3] = np.nan
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(max_depth=6, learning_rate=0.1), max_trees=20)
    b.update(20)
    return plane, b.trees(), b.init_score, Xr, cuts, off


def test_refilled_plane_equals_fresh_plane(bb):
    import torch
    plane, trees, init, Xr, cuts, off = _setup(bb)
    req = bb.Plane.like(plane, 40_000)
    pplan = bb.PredictPlan(plane, trees, init, 0.1)
    splan = bb.ShapPlan(plane, trees, init, 0.1)
    for n, device in ((1, False), (37, True), (40_000, False), (5_000, True), (40_000, True),
                      (2, False)):
        X = Xr[:n]
        if device:
            req.refill(torch.from_numpy(X).cuda(), x_on_device=True)
        else:
            req.refill(X)
        fresh = bb.Plane(X, cuts, off)
        assert req.n_rows == n
        assert np.array_equal(req.bins(), fresh.bins())
        assert np.array_equal(pplan.run(req).view(np.uint32), pplan.run(fresh).view(np.uint32))
        if n <= 5_000:
            assert np.array_equal(splan.run(req), splan.run(fresh))


def test_refill_refusals(bb):
    plane, trees, init, Xr, cuts, off = _setup(bb)
    req = bb.Plane.like(plane, 100)
    with pytest.raises(bb.ConfigError):
        req.refill(Xr[:101])
    with pytest.raises(bb.BonsaiError):
        plane.refill(Xr[:10])   # an ordinary plane has no room to refill
    # an empty request plane scores nothing
    assert bb.PredictPlan(plane, trees, init, 0.1).run(req).shape == (0,)


def test_refill_across_staging_chunks(bb):
    """A batch larger than the plane's 64 MB staging buffer goes up in chunks
    that start on tile boundaries: 650,000 rows x 28 take two."""
    from bonsai_b200 import synth
    X, _, Xr = synth.serving(n_fit=2_000, n_requests=650_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    req = bb.Plane.like(plane, 700_000)
    for n in (650_000, 3, 600_001):
        req.refill(Xr[:n])
        assert np.array_equal(req.bins(), bb.Plane(Xr[:n], cuts, off).bins())
