"""The reference's model file, format v7 (src/io/model.cpp:158-387).

A model file is one msgpack document written by nlohmann::json::to_msgpack:

    {"bin_mappers": [{"cuts": [...], "name": "f0"}, ...],
     "config": {<every Config section>},
     "init_score": s   |   "init_scores": [s_0, ..., s_K-1]   (softmax),
     "magic": "bonsai01",
     "trees": [<DenseTree> | <ObliviousTree>, ...],
     "version": 7}

with a DenseTree as {"covers", "depth", "gains", "n_leaves", "nodes": [{"default_left",
"feature_id", "left", "right", "threshold_or_value"}, ...]} (model.cpp:165-181) and an
ObliviousTree (the levelwise grower's) as {"covers" (per leaf), "depth", "gains" (per level),
"leaves", "n_leaves", "splits": [{"default_left", "feature_id", "threshold"}, ...]}
(model.cpp:183-201). Softmax trees are round-major (class k of round r at r * K + k).

The bytes follow nlohmann's msgpack writer, so a file written here is the file the
reference writes for the same model: maps with their keys in sorted order (its object is a
std::map), every integer in the smallest form (non-negative values as unsigned), every
number with a fraction as float32 when float32 holds it exactly within float range, else
float64 (an infinite cut, for one), and strings, arrays and maps in their smallest forms.
Both encoder and decoder are this module's own.
"""

from __future__ import annotations

import copy
import struct
from dataclasses import dataclass, field

import numpy as np

MAGIC = "bonsai01"
VERSION = 7
LEAF = 0xFFFFFFFF

# ---- msgpack, nlohmann's forms -----------------------------------------------------------

_F32_MAX = float(np.finfo(np.float32).max)


def _enc(x, out: bytearray) -> None:
    if x is None:
        out.append(0xC0)
    elif isinstance(x, (bool, np.bool_)):
        out.append(0xC3 if x else 0xC2)
    elif isinstance(x, (int, np.integer)):
        v = int(x)
        if v >= 0:
            if v < 0x80:
                out.append(v)
            elif v <= 0xFF:
                out += b"\xcc" + struct.pack(">B", v)
            elif v <= 0xFFFF:
                out += b"\xcd" + struct.pack(">H", v)
            elif v <= 0xFFFFFFFF:
                out += b"\xce" + struct.pack(">I", v)
            else:
                out += b"\xcf" + struct.pack(">Q", v)
        elif v >= -32:
            out += struct.pack(">b", v)
        elif v >= -0x80:
            out += b"\xd0" + struct.pack(">b", v)
        elif v >= -0x8000:
            out += b"\xd1" + struct.pack(">h", v)
        elif v >= -0x80000000:
            out += b"\xd2" + struct.pack(">i", v)
        else:
            out += b"\xd3" + struct.pack(">q", v)
    elif isinstance(x, (float, np.floating)):
        v = float(x)
        if -_F32_MAX <= v <= _F32_MAX and float(np.float32(v)) == v:
            out += b"\xca" + struct.pack(">f", v)
        else:
            out += b"\xcb" + struct.pack(">d", v)
    elif isinstance(x, str):
        b = x.encode("utf-8")
        n = len(b)
        if n <= 31:
            out.append(0xA0 | n)
        elif n <= 0xFF:
            out += b"\xd9" + struct.pack(">B", n)
        elif n <= 0xFFFF:
            out += b"\xda" + struct.pack(">H", n)
        else:
            out += b"\xdb" + struct.pack(">I", n)
        out += b
    elif isinstance(x, dict):
        n = len(x)
        if n <= 15:
            out.append(0x80 | n)
        elif n <= 0xFFFF:
            out += b"\xde" + struct.pack(">H", n)
        else:
            out += b"\xdf" + struct.pack(">I", n)
        for k in sorted(x):
            _enc(k, out)
            _enc(x[k], out)
    elif isinstance(x, (list, tuple, np.ndarray)):
        n = len(x)
        if n <= 15:
            out.append(0x90 | n)
        elif n <= 0xFFFF:
            out += b"\xdc" + struct.pack(">H", n)
        else:
            out += b"\xdd" + struct.pack(">I", n)
        for v in x:
            _enc(v, out)
    else:
        raise TypeError(f"model: cannot encode {type(x).__name__}")


def packb(obj) -> bytes:
    """obj as nlohmann::json::to_msgpack writes it."""
    out = bytearray()
    _enc(obj, out)
    return bytes(out)


class _Reader:
    def __init__(self, b: bytes):
        self.b = memoryview(b)
        self.i = 0

    def take(self, n: int) -> bytes:
        if self.i + n > len(self.b):
            raise ValueError("model: truncated msgpack document")
        v = self.b[self.i:self.i + n]
        self.i += n
        return bytes(v)

    def unpack(self, fmt: str):
        return struct.unpack(fmt, self.take(struct.calcsize(fmt)))[0]

    def value(self):
        t = self.take(1)[0]
        if t < 0x80:
            return t
        if t >= 0xE0:
            return t - 0x100
        if 0x80 <= t <= 0x8F:
            return self.map(t & 0x0F)
        if 0x90 <= t <= 0x9F:
            return [self.value() for _ in range(t & 0x0F)]
        if 0xA0 <= t <= 0xBF:
            return self.take(t & 0x1F).decode("utf-8")
        simple = {0xC0: None, 0xC2: False, 0xC3: True}
        if t in simple:
            return simple[t]
        fixed = {0xCA: ">f", 0xCB: ">d", 0xCC: ">B", 0xCD: ">H", 0xCE: ">I", 0xCF: ">Q",
                 0xD0: ">b", 0xD1: ">h", 0xD2: ">i", 0xD3: ">q"}
        if t in fixed:
            return self.unpack(fixed[t])
        if t in (0xD9, 0xDA, 0xDB):
            n = self.unpack({0xD9: ">B", 0xDA: ">H", 0xDB: ">I"}[t])
            return self.take(n).decode("utf-8")
        if t in (0xC4, 0xC5, 0xC6):
            return self.take(self.unpack({0xC4: ">B", 0xC5: ">H", 0xC6: ">I"}[t]))
        if t in (0xDC, 0xDD):
            n = self.unpack(">H" if t == 0xDC else ">I")
            return [self.value() for _ in range(n)]
        if t in (0xDE, 0xDF):
            return self.map(self.unpack(">H" if t == 0xDE else ">I"))
        raise ValueError(f"model: unsupported msgpack type 0x{t:02x}")

    def map(self, n: int) -> dict:
        out = {}
        for _ in range(n):
            k = self.value()
            out[k] = self.value()
        return out


def unpackb(b: bytes):
    r = _Reader(b)
    v = r.value()
    if r.i != len(r.b):
        raise ValueError("model: trailing bytes after the msgpack document")
    return v


# ---- Config ------------------------------------------------------------------------------

# Every persisted Config key with the reference's defaults (include/bonsai/config/
# {data,bin_mapper,tree,sampler,booster,dispatch,metrics,parallel,objective}_config.hpp);
# parallel.device_id is never persisted (model.cpp:63-66), data's missing_nan and
# missing_sentinel are written with their fixed values (model.cpp:104-113).
DEFAULT_CONFIG = {
    "data": {"train": "", "valid": [], "test": "", "format": "csv", "libsvm_n_features": 0,
             "header": True, "label_column": 0, "weight_column": -1, "ignore_columns": [],
             "missing_nan": True, "missing_sentinel": None},
    "bin_mapper": {"max_bin": 255, "n_samples": 200000, "seed": 0, "min_data_in_bin": 1},
    "tree_config": {"min_child_hess": 1.0, "min_gain_to_split": 0.0, "lambda_l2": 1.0,
                    "lambda_l1": 0.0, "feature_fraction": 1.0, "max_depth": 6,
                    "min_data_in_leaf": 20, "max_leaves": 31, "feature_seed": 2,
                    "monotone_constraints": [], "interaction_constraints": []},
    "sampler": {"subsample": 1.0, "top_rate": float(np.float32(0.2)),
                "other_rate": float(np.float32(0.1))},
    "booster_config": {"n_iters": 100, "learning_rate": float(np.float32(0.05)),
                       "random_seed": 42, "log_intervals": 0, "early_stopping_rounds": 0,
                       "dart_drop_rate": 0.0},
    "dispatch": {"objective_name": "mse", "grower_name": "depthwise",
                 "sampler_name": "all_rows"},
    "metrics": {"fit": [], "eval": []},
    "parallel": {"n_threads": 0},
    "objective": {"huber_delta": 1.0, "quantile_alpha": 0.5, "n_classes": 3},
}

_F32_KEYS = {"tree_config": ("min_child_hess", "min_gain_to_split", "lambda_l2", "lambda_l1",
                             "feature_fraction"),
             "sampler": ("subsample", "top_rate", "other_rate"),
             "booster_config": ("learning_rate", "dart_drop_rate"),
             "objective": ("huber_delta", "quantile_alpha")}


def config_for(params, n_iters: int, max_bin: int = 255, **sections) -> dict:
    """The Config a fit with these TrainParams persists: the reference's defaults with the
    fit's keys set (float keys as the float the reference holds). The dispatch names are the
    reference's CPU names (depthwise / levelwise / leafwise): the model is the one those
    growers produce, so any reference build loads it. sections overrides whole keys, e.g.
    data={"label_column": 3}."""
    c = copy.deepcopy(DEFAULT_CONFIG)
    tc = c["tree_config"]
    for k in ("min_child_hess", "min_gain_to_split", "lambda_l2", "lambda_l1", "max_depth",
              "min_data_in_leaf", "max_leaves"):
        tc[k] = getattr(params, k)
    frac = params.feature_fraction
    tc["feature_fraction"] = frac if 0.0 < frac < 1.0 else 1.0
    tc["feature_seed"] = int(params.feature_seed)
    tc["monotone_constraints"] = [int(v) for v in params.monotone]
    tc["interaction_constraints"] = [
        g if isinstance(g, str) else ",".join(str(int(f)) for f in g)
        for g in params.interaction_constraints]
    c["booster_config"]["n_iters"] = int(n_iters)
    c["booster_config"]["learning_rate"] = params.learning_rate
    c["booster_config"]["random_seed"] = int(params.random_seed)
    sub = params.subsample if 0.0 < params.subsample < 1.0 else 1.0
    c["sampler"]["subsample"] = sub
    c["bin_mapper"]["max_bin"] = int(max_bin)
    grower = {"oblivious": "levelwise"}.get(params.grower, params.grower)
    c["dispatch"] = {"objective_name": params.objective, "grower_name": grower,
                     "sampler_name": "bernoulli" if sub < 1.0 else "all_rows"}
    if params.objective == "softmax":
        c["objective"]["n_classes"] = int(params.n_classes)
    for name, keys in sections.items():
        c[name].update(keys)
    for name, keys in _F32_KEYS.items():
        for k in keys:
            c[name][k] = float(np.float32(c[name][k]))
    return c


# ---- trees -------------------------------------------------------------------------------

def _split_bins(feature, value, cuts, cut_off):
    """Each internal node's bin: the index of its threshold among its feature's cuts (the
    grower's thresholds are cut values)."""
    sb = np.zeros(len(feature), np.uint32)
    for i in np.flatnonzero(feature != LEAF):
        f = int(feature[i])
        c = cuts[cut_off[f]:cut_off[f + 1]]
        j = int(np.searchsorted(c, value[i]))
        if j >= len(c) or c[j] != value[i]:
            raise ValueError(f"model: node {i}'s threshold is not a cut of feature {f}")
        sb[i] = j
    return sb


def dense_to_json(t) -> dict:
    """A DenseTree record (model.cpp:165-172)."""
    nodes = [{"default_left": bool(t.default_left[i]), "feature_id": int(t.feature[i]),
              "left": int(t.left[i]), "right": int(t.right[i]),
              "threshold_or_value": float(np.float32(t.value[i]))}
             for i in range(len(t.feature))]
    return {"covers": [float(np.float32(v)) for v in t.covers], "depth": int(t.depth),
            "gains": [float(np.float32(v)) for v in t.gains], "n_leaves": int(t.n_leaves),
            "nodes": nodes}


def oblivious_to_json(t) -> dict:
    """An ObliviousTree record (model.cpp:183-190) from the perfect tree a levelwise fit
    returns (level order; level L starts at node 2^L - 1; leaves in the reference's frontier
    order): the split, threshold, default and gain of each level's first node, then the
    leaves' values and covers."""
    d = 0
    i = 0
    splits, gains = [], []
    while t.feature[i] != LEAF:
        splits.append({"default_left": bool(t.default_left[i]), "feature_id": int(t.feature[i]),
                       "threshold": float(np.float32(t.value[i]))})
        gains.append(float(np.float32(t.gains[i])))
        i = int(t.left[i])
        d += 1
    first = (1 << d) - 1
    leaves = [float(np.float32(v)) for v in t.value[first:first + (1 << d)]]
    covers = [float(np.float32(v)) for v in t.covers[first:first + (1 << d)]]
    return {"covers": covers, "depth": d, "gains": gains, "leaves": leaves,
            "n_leaves": 1 << d, "splits": splits}


def _tree(Tree, a: dict, depth: int, n_leaves: int, cuts, cut_off):
    a["split_bin"] = _split_bins(a["feature"], a["value"], cuts, cut_off)
    return Tree(**a, depth=depth, n_leaves=n_leaves)


def dense_from_json(j: dict, cuts, cut_off):
    from . import Tree
    nodes = j["nodes"]
    a = dict(feature=np.array([n["feature_id"] for n in nodes], np.uint32),
             value=np.array([n["threshold_or_value"] for n in nodes], np.float32),
             left=np.array([n["left"] for n in nodes], np.uint32),
             right=np.array([n["right"] for n in nodes], np.uint32),
             default_left=np.array([1 if n["default_left"] else 0 for n in nodes], np.uint8),
             gains=np.array(j["gains"], np.float32), covers=np.array(j["covers"], np.float32))
    return _tree(Tree, a, int(j["depth"]), int(j["n_leaves"]), cuts, cut_off)


def oblivious_from_json(j: dict, cuts, cut_off):
    """The perfect tree in level order, as a levelwise fit returns it: internal node i at
    level L takes level L's split and gain; its cover is the sum of the leaf covers below
    it (an older model without covers loads with zero covers)."""
    from . import Tree
    splits = j["splits"]
    d = len(splits)
    n = (2 << d) - 1
    first = (1 << d) - 1
    leaves = np.array(j["leaves"], np.float32)
    lc = np.array(j.get("covers", []), np.float32)
    if len(lc) != len(leaves):
        lc = np.zeros(len(leaves), np.float32)
    lg = list(j["gains"])
    a = dict(feature=np.full(n, LEAF, np.uint32), value=np.zeros(n, np.float32),
             left=np.zeros(n, np.uint32), right=np.zeros(n, np.uint32),
             default_left=np.zeros(n, np.uint8), gains=np.zeros(n, np.float32),
             covers=np.zeros(n, np.float32))
    a["value"][first:] = leaves
    a["covers"][first:] = lc
    for i in range(first - 1, -1, -1):
        L = int(np.floor(np.log2(i + 1)))
        s = splits[L]
        a["feature"][i] = s["feature_id"]
        a["value"][i] = s["threshold"]
        a["default_left"][i] = 1 if s["default_left"] else 0
        a["left"][i], a["right"][i] = 2 * i + 1, 2 * i + 2
        a["gains"][i] = lg[L] if L < len(lg) else 0.0
        a["covers"][i] = a["covers"][2 * i + 1] + a["covers"][2 * i + 2]
    return _tree(Tree, a, d, 1 << d, cuts, cut_off)


# ---- the model ---------------------------------------------------------------------------

@dataclass
class Model:
    """A loaded (or to-be-saved) model: the Config, the bin mappers as this package's
    flattened cuts, the initial score(s) and the trees in this package's form (a levelwise
    model's trees as the perfect trees a levelwise fit returns)."""
    config: dict
    cuts: np.ndarray
    cut_off: np.ndarray
    trees: list
    init_scores: np.ndarray
    feature_names: list = field(default_factory=list)

    @property
    def objective(self) -> str:
        return self.config["dispatch"]["objective_name"]

    @property
    def grower(self) -> str:
        return self.config["dispatch"]["grower_name"]

    @property
    def learning_rate(self) -> float:
        return float(self.config["booster_config"]["learning_rate"])

    @property
    def n_classes(self) -> int:
        return len(self.init_scores) if self.objective == "softmax" else 1

    @property
    def init_score(self) -> float:
        return float(self.init_scores[0])

    def class_trees(self, k: int) -> list:
        """Class k's trees of a softmax model (round-major), else every tree."""
        return self.trees[k::self.n_classes]

    def document(self) -> dict:
        cuts = np.asarray(self.cuts, np.float32)
        off = np.asarray(self.cut_off, np.uint32)
        F = len(off) - 1
        names = self.feature_names or [f"f{i}" for i in range(F)]
        levelwise = self.grower.endswith("levelwise")
        doc = {"magic": MAGIC, "version": VERSION, "config": self.config,
               "bin_mappers": [{"name": names[f],
                                "cuts": [float(v) for v in cuts[off[f]:off[f + 1]]]}
                               for f in range(F)],
               "trees": [oblivious_to_json(t) if levelwise else dense_to_json(t)
                         for t in self.trees]}
        if self.objective == "softmax":
            doc["init_scores"] = [float(np.float32(v)) for v in self.init_scores]
        else:
            doc["init_score"] = float(np.float32(self.init_scores[0]))
        return doc

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(packb(self.document()))


def from_document(doc: dict) -> Model:
    """A Model from a decoded v7 document; the magic and version are checked as the
    reference's load_booster checks them (model.cpp:361-371)."""
    if doc.get("magic") != MAGIC:
        raise ValueError("model: bad magic")
    if doc.get("version") != VERSION:
        raise ValueError("model: unsupported format version")
    cuts_l = [np.array(m["cuts"], np.float32) for m in doc["bin_mappers"]]
    off = np.concatenate([[0], np.cumsum([len(c) for c in cuts_l])]).astype(np.uint32)
    cuts = np.concatenate(cuts_l).astype(np.float32) if cuts_l else np.zeros(0, np.float32)
    cfg = doc["config"]
    levelwise = cfg["dispatch"]["grower_name"].endswith("levelwise")
    trees = [oblivious_from_json(t, cuts, off) if levelwise else dense_from_json(t, cuts, off)
             for t in doc["trees"]]
    if "init_scores" in doc:
        init = np.array(doc["init_scores"], np.float32)
    else:
        init = np.array([doc["init_score"]], np.float32)
    return Model(config=cfg, cuts=cuts, cut_off=off, trees=trees, init_scores=init,
                 feature_names=[m["name"] for m in doc["bin_mappers"]])


def load(path: str) -> Model:
    with open(path, "rb") as f:
        return from_document(unpackb(f.read()))


def from_booster(booster, cuts, cut_off, n_iters: int | None = None, feature_names=None,
                 max_bin: int = 255, **sections) -> Model:
    """The model of a fitted Booster: its trees, initial score(s) and TrainParams, with the
    plane's cuts as the bin mappers."""
    trees = booster.trees()
    k = max(1, booster.n_classes)
    rounds = n_iters if n_iters is not None else len(trees) // k
    cfg = config_for(booster.params, rounds, max_bin=max_bin, **sections)
    return Model(config=cfg, cuts=np.asarray(cuts, np.float32),
                 cut_off=np.asarray(cut_off, np.uint32), trees=trees,
                 init_scores=np.asarray(booster.init_scores, np.float32),
                 feature_names=list(feature_names) if feature_names is not None else [])


def warm_start(model: Model, plane, labels, params, max_trees: int, weights=None):
    """A Booster that continues `model` over `plane` (the reference's warm start,
    include/bonsai/booster.hpp:512-524): every row's starting score is the
    model's init + lr x (its trees' leaf values summed in tree order), the
    reference's rebuilt training score bit for bit, and the new rounds grow
    from it. Single-output models; params.learning_rate should be the model's.
    `continued` joins the result back into one model."""
    from . import Booster, predict
    if model.objective == "softmax":
        raise ValueError("warm_start: single-output models only")
    scores = predict(plane, model.trees, model.init_score, model.learning_rate)
    return Booster(plane, labels, params, max_trees=max_trees, init_scores=scores,
                   weights=weights)


def continued(model: Model, booster) -> Model:
    """`model` with the trees a warm-started booster grew appended (its initial
    score and bin mappers kept; the config counts every round)."""
    cfg = copy.deepcopy(model.config)
    trees = list(model.trees) + booster.trees()
    cfg["booster_config"]["n_iters"] = len(trees) // max(1, model.n_classes)
    return Model(config=cfg, cuts=model.cuts, cut_off=model.cut_off, trees=trees,
                 init_scores=model.init_scores, feature_names=list(model.feature_names))
