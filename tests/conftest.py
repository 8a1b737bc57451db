"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on
CPU. The oracle libraries (oracle/_ref) are test infrastructure: the C
restatement is built on demand with gcc; the reference's own CPU grower is
built where its sources exist and otherwise used prebuilt (it travels with
the repository snapshot)."""

from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200)")


def _ensure_oracle():
    so = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "bonsai_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"],
                       check=True)


@pytest.fixture(scope="session")
def orc():
    _ensure_oracle()
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import REF_SO, RefLib
    if not os.path.exists(REF_SO):
        pytest.skip("the reference's CPU grower is not built here")
    return RefLib()


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def unpack_trees(d, prefix=""):
    from oracle import Tree
    prefix = prefix + "tree_"
    sizes = d[prefix + "sizes"]
    starts = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    out = []
    for i in range(len(sizes)):
        s, e = starts[i], starts[i + 1]
        out.append(Tree(**{k: d[prefix + k][s:e] for k in (
            "feature", "value", "left", "right", "default_left", "gains", "covers")}))
    return out


TREE_FIELDS = ("feature", "value", "left", "right", "default_left", "gains", "covers")


def level_gains(t):
    """An oblivious tree's per-level gains, read along its left spine (the perfect
    level-order tree a levelwise fit returns, or the reference's preorder
    dense_equivalent, src/tree.cpp:64-117, which puts each level's gain on every node of
    the level)."""
    out, i = [], 0
    while t.feature[i] != 0xFFFFFFFF:
        out.append(t.gains[i])
        i = int(t.left[i])
    return np.asarray(out, np.float32)


def assert_trees_equal(a, b, where=""):
    for k in TREE_FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape, f"{where} {k}: {x.shape} vs {y.shape}"
        assert np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                              y.view(np.uint32) if y.dtype == np.float32 else y), (
            f"{where} {k} differs at {np.flatnonzero(x != y)[:8]}")


@pytest.fixture(scope="session")
def bb():
    """The product library, built if stale; GPU tests only."""
    from bonsai_b200.build import build_library
    build_library()
    import bonsai_b200
    if not bonsai_b200.available():
        pytest.fail("no CUDA device: GPU tests need one (no CPU fallback exists)")
    return bonsai_b200
