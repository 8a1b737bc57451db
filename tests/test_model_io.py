"""The reference's model file (format v7, src/io/model.cpp) read and written by
bonsai_b200.model. The reference's own byte-proof (tests/unit/
test_model_io.cpp:269-296: each committed v7 fixture, loaded and saved again,
reproduces its bytes) holds here for both fixtures (tests/golden/
model_v7_*.bonsai; make_model_fixtures.py copies them), through this
package's trees and back; the encoder takes nlohmann's forms at every size
boundary; a bad magic or version is refused; config_for writes every key the
reference persists."""

from __future__ import annotations

import os
import struct

import numpy as np
import pytest

from bonsai_b200 import TrainParams
from bonsai_b200 import model as M

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture(kind):
    with open(os.path.join(GOLDEN, f"model_v7_{kind}.bonsai"), "rb") as f:
        return f.read()


@pytest.mark.parametrize("kind", ["regressor", "softmax"])
def test_fixture_resaves_byte_identically(kind, tmp_path):
    raw = _fixture(kind)
    m = M.load(os.path.join(GOLDEN, f"model_v7_{kind}.bonsai"))
    p = tmp_path / "m.bonsai"
    m.save(str(p))
    assert p.read_bytes() == raw
    # and the document alone re-encodes to the same bytes
    assert M.packb(M.unpackb(raw)) == raw


def test_fixture_contents():
    r = M.load(os.path.join(GOLDEN, "model_v7_regressor.bonsai"))
    assert r.objective == "mse" and r.grower == "depthwise" and len(r.trees) == 5
    assert r.n_classes == 1 and len(r.feature_names) == 6
    s = M.load(os.path.join(GOLDEN, "model_v7_softmax.bonsai"))
    assert s.objective == "softmax" and s.n_classes == 3 and len(s.trees) == 15
    assert len(s.class_trees(1)) == 5
    for t in r.trees + s.trees:
        internal = t.feature != M.LEAF
        # every threshold is a cut: split bins recovered exactly
        for i in np.flatnonzero(internal):
            f = int(t.feature[i])
            assert r.cuts[r.cut_off[f] + t.split_bin[i]] == t.value[i] or \
                s.cuts[s.cut_off[f] + t.split_bin[i]] == t.value[i]


@pytest.mark.parametrize("value,expect", [
    (0, b"\x00"), (127, b"\x7f"), (128, b"\xcc\x80"), (255, b"\xcc\xff"),
    (256, b"\xcd\x01\x00"), (65535, b"\xcd\xff\xff"), (65536, b"\xce\x00\x01\x00\x00"),
    (2**32 - 1, b"\xce\xff\xff\xff\xff"), (2**32, b"\xcf" + struct.pack(">Q", 2**32)),
    (-1, b"\xff"), (-32, b"\xe0"), (-33, b"\xd0\xdf"), (-128, b"\xd0\x80"),
    (-129, b"\xd1\xff\x7f"), (-32769, b"\xd2" + struct.pack(">i", -32769)),
    (0.5, b"\xca" + struct.pack(">f", 0.5)), (0.1, b"\xcb" + struct.pack(">d", 0.1)),
    (float(np.float32(0.1)), b"\xca" + struct.pack(">f", 0.1)),
    (float("inf"), b"\xcb" + struct.pack(">d", float("inf"))),
    (float(np.finfo(np.float32).max), b"\xca\x7f\x7f\xff\xff"),
    (True, b"\xc3"), (False, b"\xc2"), (None, b"\xc0"),
    ("a" * 31, b"\xbf" + b"a" * 31), ("a" * 32, b"\xd9\x20" + b"a" * 32),
    ([1] * 15, b"\x9f" + b"\x01" * 15), ([1] * 16, b"\xdc\x00\x10" + b"\x01" * 16),
    ({"b": 1, "a": 2}, b"\x82\xa1a\x02\xa1b\x01"),
])
def test_encoder_takes_nlohmann_forms(value, expect):
    assert M.packb(value) == expect
    back = M.unpackb(expect)
    assert back == value or (isinstance(value, float) and back == value)


def test_nan_is_float64():
    b = M.packb(float("nan"))
    assert b[0] == 0xCB and np.isnan(M.unpackb(b))


def test_bad_magic_and_version_refused(tmp_path):
    doc = M.unpackb(_fixture("regressor"))
    for k, v in (("magic", "bonsai02"), ("version", 6)):
        d = dict(doc)
        d[k] = v
        p = tmp_path / f"{k}.bonsai"
        p.write_bytes(M.packb(d))
        with pytest.raises(ValueError):
            M.load(str(p))
    p = tmp_path / "garbage.bonsai"
    p.write_bytes(b"not-a-bonsai-model\x00")
    with pytest.raises(ValueError):
        M.load(str(p))


def test_config_for_writes_every_persisted_key():
    ref_cfg = M.unpackb(_fixture("regressor"))["config"]
    cfg = M.config_for(TrainParams(max_depth=3, learning_rate=0.1), n_iters=5, max_bin=63)
    assert set(cfg) == set(ref_cfg)
    for section in cfg:
        assert set(cfg[section]) == set(ref_cfg[section]), section
    # the fixture's fit, restated: the same config except parallel.n_threads
    for section in cfg:
        for k, v in ref_cfg[section].items():
            if (section, k) != ("parallel", "n_threads"):
                assert cfg[section][k] == v, (section, k)
    s = M.config_for(TrainParams(objective="softmax", n_classes=7, grower="oblivious",
                                 subsample=0.8, monotone=[1, 0, -1], feature_fraction=0.5,
                                 feature_seed=9,
                                 interaction_constraints=[[0, 1], "2,3"]), n_iters=300)
    assert s["dispatch"] == {"objective_name": "softmax", "grower_name": "levelwise",
                             "sampler_name": "bernoulli"}
    assert s["objective"]["n_classes"] == 7 and s["sampler"]["subsample"] == float(np.float32(0.8))
    assert s["tree_config"]["monotone_constraints"] == [1, 0, -1]
    assert s["tree_config"]["feature_fraction"] == 0.5 and s["tree_config"]["feature_seed"] == 9
    assert s["tree_config"]["interaction_constraints"] == ["0,1", "2,3"]
