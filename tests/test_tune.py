"""The launch-shape autotuner's host logic on CPU: shape keys, the choice
(fastest candidate, the default on a tie), the on-disk cache (written once,
read back without timing, refreshed on request), and the plain form left
untouched. The timing itself is replaced by a stand-in; the GPU test
(tests/test_gpu_tune.py) times real rounds."""

from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest


def _plane(n=100_000, F=28, bins=255):
    return SimpleNamespace(n_rows=n, n_feats=F, n_bins=np.full(F, bins, np.uint32))


def test_tuner_picks_the_fastest_and_caches_it(tmp_path):
    from bonsai_b200 import TrainParams
    from bonsai_b200 import autotune as T
    path = str(tmp_path / "tune.json")
    calls = []

    def timer(p):
        calls.append(p.hist_ctas)
        return {0: 5.0, 148: 5.0, 74: 4.0, 37: 3.0, 16: 3.5, 8: 6.0, 4: 7.0, 2: 9.0,
                1: 9.5}[p.hist_ctas]

    params = TrainParams(objective="logloss", hist_mode="int8", max_depth=8)
    got = T.tune(_plane(), None, params, path=path, timer=timer)
    assert got.hist_ctas == 37 and got.max_depth == 8 and got.objective == "logloss"
    assert sorted(calls) == sorted(T.CANDIDATES)
    entries = json.load(open(path))
    assert len(entries) == 1
    (key, entry), = entries.items()
    assert entry["hist_ctas"] == 37 and "int8" in key and "feats=28" in key
    # the same shape again: read from the cache, nothing timed
    calls.clear()
    assert T.tune(_plane(n=70_000), None, params, path=path, timer=timer).hist_ctas == 37
    assert calls == []
    # another shape is timed; a refresh re-times
    T.tune(_plane(F=2000), None, params, path=path, timer=timer)
    assert len(json.load(open(path))) == 2
    T.tune(_plane(), None, params, path=path, timer=lambda p: float(p.hist_ctas == 0),
           refresh=True)
    assert T.load(path)[key]["hist_ctas"] != 0


def test_ties_keep_the_default_and_exact_is_untouched(tmp_path):
    from bonsai_b200 import TrainParams
    from bonsai_b200 import autotune as T
    path = str(tmp_path / "t.json")
    params = TrainParams(hist_mode="int8")
    assert T.tune(_plane(), None, params, path=path, timer=lambda p: 1.0).hist_ctas == 0
    # within the noise margin of the default: the default stays
    assert T.pick({0: 1.00, 148: 0.99, 4: 1.5}) == 0
    assert T.pick({0: 1.00, 148: 0.97, 4: 1.5}) == 148
    exact = TrainParams(hist_mode="exact")
    assert T.tune(_plane(), None, exact, path=path, timer=lambda p: 1 / 0) is exact


@pytest.mark.parametrize("n,want", [(1, "rows<=1"), (1000, "rows<=1024"),
                                    (10_000_000, "rows<=16777216")])
def test_shape_keys_bucket_rows_by_powers_of_two(n, want):
    from bonsai_b200 import TrainParams
    from bonsai_b200 import autotune as T
    k = T.shape_key(n, 28, True, TrainParams(hist_mode="int8", subsample=0.8), "B200")
    assert want in k and "sub=0.8" in k and k.startswith("B200|")
    assert T.shape_key(n, 28, True, TrainParams(grower="leafwise", max_leaves=255,
                                                hist_mode="int8"), "B200").count("leafwise255")
