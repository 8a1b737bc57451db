"""Zero-copy ingest of device matrices (Plane.from_device over bb_ingest's
device input; the reference's cuda_ingest_device, include/bonsai/cuda/
histogram_engine.hpp:41-50): a torch tensor, a DLPack producer and a CUDA
array interface producer give the host ingest's codes bit for bit, including
a matrix still being written on torch's stream when it is handed over; the
matrix may be freed once the plane exists; non-contiguous, non-float32,
non-2-D and host matrices are refused."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class _DLPackOnly:
    def __init__(self, t):
        self._t = t

    def __dlpack__(self, stream=None, **kw):
        return self._t.__dlpack__(stream=stream)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


class _CAIOnly:
    def __init__(self, t):
        self._t = t
        self.__cuda_array_interface__ = t.__cuda_array_interface__


def _host(seed=5, n=70_001, F=13):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    X[:, 4] = np.round(X[:, 4])
    return X


@pytest.mark.parametrize("wrap", ["tensor", "dlpack", "cai"])
def test_device_ingest_equals_host_ingest(bb, wrap):
    import torch
    X = _host()
    cuts, off = bb.fit_cuts(X)
    want = bb.Plane(X, cuts, off).bins()
    # written on torch's stream just before the handover
    t = torch.empty(X.shape, dtype=torch.float32, device="cuda")
    t.copy_(torch.from_numpy(X), non_blocking=False)
    t.mul_(2.0).mul_(0.5)
    src = {"tensor": t, "dlpack": _DLPackOnly(t), "cai": _CAIOnly(t)}[wrap]
    plane = bb.Plane.from_device(src, cuts, off)
    del src, t
    torch.cuda.empty_cache()
    assert np.array_equal(plane.bins(), want)
    # the plane stands alone: a tree grows over it
    g = np.random.Generator(np.random.PCG64(1)).standard_normal(plane.n_rows).astype(np.float32)
    tree, _, _ = bb.grow_tree(plane, bb.TrainParams(max_depth=4), g, np.ones_like(g))
    assert tree.feature[0] != 0xFFFFFFFF


def test_device_ingest_refusals(bb):
    import torch
    X = _host(n=1_000, F=6)
    cuts, off = bb.fit_cuts(X)
    t = torch.from_numpy(X).cuda()
    with pytest.raises(ValueError):
        bb.Plane.from_device(t.t(), cuts, off)          # column-major view
    with pytest.raises(ValueError):
        bb.Plane.from_device(t.double(), cuts, off)     # float64
    with pytest.raises(ValueError):
        bb.Plane.from_device(t[:, 0], cuts, off)        # 1-D
    with pytest.raises(ValueError):
        bb.Plane.from_device(torch.from_numpy(X), cuts, off)  # host memory
    with pytest.raises(ValueError):
        bb.Plane.from_device(X, cuts, off)              # numpy: DLPack, but host memory
    with pytest.raises(TypeError):
        bb.Plane.from_device(X.tolist(), cuts, off)     # no device protocol at all
