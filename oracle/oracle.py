"""TEST INFRASTRUCTURE — Python bindings for the two oracle libraries.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this,
always as the checker, never as the thing measured or shipped.

  RefLib   oracle/_ref/libbonsai_ref.so: the reference's own CPU grower
           (src/bin_mapper.cpp, src/dataset.cpp, src/split.cpp,
           src/grower.cpp, include/bonsai/booster.hpp, src/shap.cpp ...)
           compiled from its sources by oracle/Makefile.
  Oracle   oracle/_ref/liboracle.so: the C restatement bonsai_oracle.c.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libbonsai_ref.so")
ORACLE_SO = os.path.join(HERE, "_ref", "liboracle.so")
# the reference's Booster over bonsai_b200's grower shim (the drop-in check)
REF_B200_SO = os.path.join(HERE, "_ref", "libbonsai_ref_b200.so")
LEAF = 0xFFFFFFFF


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class RefCfg(C.Structure):
    _fields_ = [
        ("grower", C.c_int32), ("objective", C.c_int32), ("n_iters", C.c_uint32),
        ("learning_rate", C.c_float), ("min_child_hess", C.c_float),
        ("min_gain_to_split", C.c_float), ("lambda_l2", C.c_float),
        ("lambda_l1", C.c_float), ("feature_fraction", C.c_float),
        ("max_depth", C.c_uint32), ("min_data_in_leaf", C.c_uint32),
        ("max_leaves", C.c_uint32), ("feature_seed", C.c_uint32),
        ("subsample", C.c_float), ("random_seed", C.c_uint32),
        ("n_threads", C.c_uint32), ("n_classes", C.c_uint32),
        ("monotone", C.POINTER(C.c_int32)), ("n_monotone", C.c_uint32),
        ("interaction", C.c_char_p), ("quantile_alpha", C.c_float), ("huber_delta", C.c_float),
        ("dart_drop_rate", C.c_float), ("goss_top_rate", C.c_float),
        ("goss_other_rate", C.c_float), ("hist_mode", C.c_int32),
    ]


GROWERS = {"depthwise": 0, "levelwise": 1, "leafwise": 2}
OBJECTIVES = {"mse": 0, "logloss": 1, "softmax": 2, "poisson": 3, "mae": 4, "huber": 5,
              "quantile": 6}


@dataclass
class TreeCfg:
    """The reference's TreeConfig + BoosterConfig knobs the hot path reads
    (include/bonsai/config/tree_config.hpp:9-29, booster_config.hpp)."""
    grower: str = "depthwise"
    objective: str = "mse"
    n_iters: int = 100
    learning_rate: float = 0.1
    min_child_hess: float = 1.0
    min_gain_to_split: float = 0.0
    lambda_l2: float = 1.0
    lambda_l1: float = 0.0
    feature_fraction: float = 1.0
    max_depth: int = 6
    min_data_in_leaf: int = 20
    max_leaves: int = 31
    feature_seed: int = 2
    subsample: float = 1.0
    random_seed: int = 42
    n_threads: int = 1
    n_classes: int = 3
    quantile_alpha: float = 0.5
    huber_delta: float = 1.0
    dart_drop_rate: float = 0.0
    goss_top_rate: float = 0.0  # > 0 selects the GOSS sampler
    goss_other_rate: float = 0.1
    monotone: list = field(default_factory=list)
    interaction_constraints: list = field(default_factory=list)  # TOML strings, "0,1"
    hist_mode: str = "exact"  # the drop-in grower's form: exact, int8, int16

    def ref(self):
        c = RefCfg()
        c.grower = GROWERS[self.grower]
        c.objective = OBJECTIVES[self.objective]
        for k in ("n_iters", "learning_rate", "min_child_hess", "min_gain_to_split",
                  "lambda_l2", "lambda_l1", "feature_fraction", "max_depth",
                  "min_data_in_leaf", "max_leaves", "feature_seed", "subsample",
                  "random_seed", "n_threads", "n_classes", "quantile_alpha", "huber_delta",
                  "dart_drop_rate", "goss_top_rate", "goss_other_rate"):
            setattr(c, k, getattr(self, k))
        c.hist_mode = {"exact": 0, "int8": 1, "int16": 2}[self.hist_mode]
        if self.monotone:
            self._mono = np.asarray(self.monotone, dtype=np.int32)
            c.monotone = _p(self._mono, C.c_int32)
            c.n_monotone = len(self.monotone)
        if self.interaction_constraints:
            self._inter = ";".join(self.interaction_constraints).encode()
            c.interaction = self._inter
        return c


@dataclass
class Tree:
    feature: np.ndarray
    value: np.ndarray
    left: np.ndarray
    right: np.ndarray
    default_left: np.ndarray
    gains: np.ndarray
    covers: np.ndarray
    split_bin: np.ndarray | None = None
    depth: int = 0
    n_leaves: int = 0


class RefLib:
    """The reference's own CPU implementation (compiled from its sources)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        L = self.L = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_dataset_create.restype = C.c_void_p
        L.ref_train.restype = C.c_void_p
        L.ref_grow_tree.restype = C.c_void_p
        L.ref_model_n_trees.restype = C.c_size_t
        L.ref_model_tree_size.restype = C.c_size_t
        L.ref_model_init_score.restype = C.c_float
        L.ref_model_oblivious_depth.restype = C.c_size_t
        for name in ("ref_dataset_destroy", "ref_model_destroy"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.ref_dataset_u8.argtypes = [C.c_void_p]
        L.ref_dataset_bins.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_model_n_trees.argtypes = [C.c_void_p]
        L.ref_model_init_score.argtypes = [C.c_void_p]
        L.ref_model_tree_size.argtypes = [C.c_void_p, C.c_size_t]
        L.ref_model_tree.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 7
        L.ref_model_oblivious_depth.argtypes = [C.c_void_p, C.c_size_t]
        L.ref_model_oblivious.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 4
        L.ref_model_predict_binned.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_model_contribs_binned.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_train.argtypes = [C.c_void_p, C.POINTER(RefCfg)]

    def err(self):
        return self.L.ref_last_error().decode()

    def fit_cuts(self, X, max_bin=255, n_samples=200_000, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        n, F = X.shape
        cap = F * (max_bin + 2)
        cuts = np.empty(cap, np.float32)
        off = np.empty(F + 1, np.uint32)
        rc = self.L.ref_fit_cuts(_p(X, C.c_float), C.c_size_t(n), C.c_size_t(F),
                                 C.c_int32(max_bin), C.c_size_t(n_samples),
                                 C.c_uint64(seed), _p(cuts, C.c_float), C.c_size_t(cap),
                                 _p(off, C.c_uint32))
        if rc:
            raise RuntimeError(self.err())
        return cuts[: off[-1]].copy(), off

    def cuts_from_sample(self, S, max_bin=255):
        S = np.ascontiguousarray(S, dtype=np.float32)
        n, F = S.shape
        cap = F * (max_bin + 2)
        cuts = np.empty(cap, np.float32)
        off = np.empty(F + 1, np.uint32)
        rc = self.L.ref_cuts_from_sample(_p(S, C.c_float), C.c_size_t(n), C.c_size_t(F),
                                         C.c_int32(max_bin), _p(cuts, C.c_float),
                                         C.c_size_t(cap), _p(off, C.c_uint32))
        if rc:
            raise RuntimeError(self.err())
        return cuts[: off[-1]].copy(), off

    def dataset(self, X, y, cuts, off, weights=None):
        return RefDataset(self, X, y, cuts, off, weights)

    def train(self, ds, cfg: TreeCfg):
        rc = cfg.ref()
        h = self.L.ref_train(C.c_void_p(ds.h), C.byref(rc))
        if not h:
            raise RuntimeError(self.err())
        return RefModel(self, h)

    def warm_train(self, ds, cfg: TreeCfg, trees, init_score):
        """The reference's depthwise booster loaded with trees and init_score
        (its warm start), trained cfg.n_iters more rounds; the model holds every
        tree."""
        off = np.concatenate([[0], np.cumsum([len(t.feature) for t in trees])]).astype(np.uint32)
        types = dict(feature=np.uint32, value=np.float32, left=np.uint32, right=np.uint32,
                     default_left=np.uint8, gains=np.float32, covers=np.float32)
        # held in names for the call: a temporary's buffer could be freed first
        cat = {k: np.ascontiguousarray(np.concatenate([np.asarray(getattr(t, k)) for t in trees]),
                                       dtype=ty) for k, ty in types.items()}
        depth = np.array([t.depth for t in trees], np.uint32)
        n_leaves = np.array([t.n_leaves for t in trees], np.uint32)
        f = self.L.ref_warm_train
        f.restype = C.c_void_p
        f.argtypes = [C.c_void_p, C.POINTER(RefCfg), C.c_uint32] + [C.c_void_p] * 10 + [C.c_float]
        rc = cfg.ref()
        h = f(C.c_void_p(ds.h), C.byref(rc), len(trees), off.ctypes.data,
              *(cat[k].ctypes.data for k in types), depth.ctypes.data, n_leaves.ctypes.data,
              float(init_score))
        if not h:
            raise RuntimeError(self.err())
        return RefModel(self, h)

    def train_b200(self, ds, cfg: TreeCfg):
        """The reference's Booster with B200DepthwiseGrower (needs REF_B200_SO)."""
        f = self.L.ref_b200_train
        f.restype = C.c_void_p
        f.argtypes = [C.c_void_p, C.POINTER(RefCfg)]
        rc = cfg.ref()
        h = f(C.c_void_p(ds.h), C.byref(rc))
        if not h:
            raise RuntimeError(self.err())
        return RefModel(self, h)

    def train_b200_valid(self, ds, valid, cfg: TreeCfg):
        """train_b200 with a validation set, routed as the reference's fit loop
        routes a device grower's: returns (model, per-round losses, per-round
        flags of losses the device plane reported)."""
        f = self.L.ref_b200_train_valid
        f.restype = C.c_void_p
        f.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(RefCfg), C.c_void_p, C.c_void_p]
        rc = cfg.ref()
        losses = np.zeros(cfg.n_iters, np.float32)
        dev = np.zeros(cfg.n_iters, np.int32)
        h = f(C.c_void_p(ds.h), C.c_void_p(valid.h), C.byref(rc), losses.ctypes.data,
              dev.ctypes.data)
        if not h:
            raise RuntimeError(self.err())
        return RefModel(self, h), losses, dev

    def grow_tree(self, ds, cfg: TreeCfg, grad, hess, rows=None):
        n = ds.n
        grad = np.ascontiguousarray(grad, np.float32)
        hess = np.ascontiguousarray(hess, np.float32)
        rows = np.arange(n, dtype=np.uint32) if rows is None else np.ascontiguousarray(rows, np.uint32)
        values = np.empty(n, np.float32)
        ids = np.empty(n, np.uint32)
        rc = cfg.ref()
        self.L.ref_grow_tree.argtypes = [C.c_void_p, C.POINTER(RefCfg)] + [C.c_void_p] * 3 + [C.c_size_t] + [C.c_void_p] * 2
        h = self.L.ref_grow_tree(C.c_void_p(ds.h), C.byref(rc), grad.ctypes.data,
                                 hess.ctypes.data, rows.ctypes.data, len(rows),
                                 values.ctypes.data, ids.ctypes.data)
        if not h:
            raise RuntimeError(self.err())
        m = RefModel(self, h)
        return m.tree(0), values, ids, m

    def find_split(self, hist, n_rows, cfg: TreeCfg):
        """hist: float32 [F, n_bins, 2]."""
        hist = np.ascontiguousarray(hist, np.float32)
        F, nb, _ = hist.shape
        gain = C.c_double()
        feat = C.c_uint32()
        b = C.c_uint32()
        dl = C.c_uint8()
        valid = C.c_uint8()
        rc = cfg.ref()
        r = self.L.ref_find_split(_p(hist, C.c_float), C.c_size_t(F), C.c_size_t(nb),
                                  C.c_size_t(n_rows), C.byref(rc), C.byref(gain),
                                  C.byref(feat), C.byref(b), C.byref(dl), C.byref(valid))
        if r:
            raise RuntimeError(self.err())
        return dict(gain=gain.value, feature=feat.value, bin=b.value,
                    default_left=dl.value, valid=valid.value)


class RefDataset:
    def __init__(self, lib, X, y, cuts, off, weights=None):
        self.lib = lib
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        self.n, self.F = X.shape
        self.cuts = np.ascontiguousarray(cuts, np.float32)
        self.off = np.ascontiguousarray(off, np.uint32)
        if weights is None:
            lib.L.ref_dataset_create.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t,
                                                 C.c_void_p, C.c_void_p]
            self.h = lib.L.ref_dataset_create(X.ctypes.data, y.ctypes.data, self.n, self.F,
                                              self.cuts.ctypes.data, self.off.ctypes.data)
        else:
            w = np.ascontiguousarray(weights, np.float32)
            f = lib.L.ref_dataset_create_weighted
            f.restype = C.c_void_p
            f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_size_t,
                          C.c_void_p, C.c_void_p]
            self.h = f(X.ctypes.data, y.ctypes.data, w.ctypes.data, self.n, self.F,
                       self.cuts.ctypes.data, self.off.ctypes.data)
        if not self.h:
            raise RuntimeError(lib.err())

    def bins(self):
        out = np.empty((self.F, self.n), np.uint16)
        if self.lib.L.ref_dataset_bins(C.c_void_p(self.h), out.ctypes.data):
            raise RuntimeError(self.lib.err())
        return out

    def u8(self):
        return bool(self.lib.L.ref_dataset_u8(C.c_void_p(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.ref_dataset_destroy(C.c_void_p(self.h))
            self.h = None


class RefModel:
    def __init__(self, lib, h):
        self.lib = lib
        self.h = h

    def n_trees(self):
        return int(self.lib.L.ref_model_n_trees(C.c_void_p(self.h)))

    def init_score(self):
        return float(self.lib.L.ref_model_init_score(C.c_void_p(self.h)))

    def tree(self, t):
        n = int(self.lib.L.ref_model_tree_size(C.c_void_p(self.h), t))
        a = dict(feature=np.empty(n, np.uint32), value=np.empty(n, np.float32),
                 left=np.empty(n, np.uint32), right=np.empty(n, np.uint32),
                 default_left=np.empty(n, np.uint8), gains=np.empty(n, np.float32),
                 covers=np.empty(n, np.float32))
        self.lib.L.ref_model_tree(C.c_void_p(self.h), t, *(a[k].ctypes.data for k in (
            "feature", "value", "left", "right", "default_left", "gains", "covers")))
        return Tree(**a)

    def trees(self):
        return [self.tree(t) for t in range(self.n_trees())]

    def oblivious(self, t):
        d = int(self.lib.L.ref_model_oblivious_depth(C.c_void_p(self.h), t))
        f = np.empty(d, np.uint32)
        thr = np.empty(d, np.float32)
        dl = np.empty(d, np.uint8)
        leaves = np.empty(1 << d, np.float32)
        self.lib.L.ref_model_oblivious(C.c_void_p(self.h), t, f.ctypes.data,
                                       thr.ctypes.data, dl.ctypes.data, leaves.ctypes.data)
        return f, thr, dl, leaves

    def predict_binned(self, ds):
        out = np.empty(ds.n, np.float32)
        if self.lib.L.ref_model_predict_binned(C.c_void_p(self.h), C.c_void_p(ds.h),
                                               out.ctypes.data):
            raise RuntimeError(self.lib.err())
        return out

    def init_scores(self):
        out = np.zeros(64, np.float32)
        L = self.lib.L
        L.ref_model_init_scores.restype = C.c_size_t
        L.ref_model_init_scores.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        n = L.ref_model_init_scores(C.c_void_p(self.h), out.ctypes.data, 64)
        return out[:n].copy()

    def contribs_binned(self, ds, n_classes: int = 1):
        """n x (F + 1), or n x n_classes x (F + 1) for a multiclass model."""
        if n_classes > 1:
            out = np.empty((ds.n, n_classes, ds.F + 1), np.float64)
            f = self.lib.L.ref_model_contribs_binned_k
            f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
            if f(C.c_void_p(self.h), C.c_void_p(ds.h), out.ctypes.data, n_classes):
                raise RuntimeError(self.lib.err())
            return out
        out = np.empty((ds.n, ds.F + 1), np.float64)
        if self.lib.L.ref_model_contribs_binned(C.c_void_p(self.h), C.c_void_p(ds.h),
                                                out.ctypes.data):
            raise RuntimeError(self.lib.err())
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.ref_model_destroy(C.c_void_p(self.h))
            self.h = None


class OrcTreeCfg(C.Structure):
    _fields_ = [
        ("min_child_hess", C.c_float), ("min_gain_to_split", C.c_float),
        ("lambda_l2", C.c_float), ("lambda_l1", C.c_float),
        ("max_depth", C.c_uint32), ("min_data_in_leaf", C.c_uint32),
        ("max_leaves", C.c_uint32), ("monotone", C.POINTER(C.c_int32)),
        ("n_monotone", C.c_uint32), ("grower", C.c_int32),
    ]


class OrcTree(C.Structure):
    _fields_ = [
        ("cap", C.c_uint32), ("feature", C.POINTER(C.c_uint32)),
        ("value", C.POINTER(C.c_float)), ("left", C.POINTER(C.c_uint32)),
        ("right", C.POINTER(C.c_uint32)), ("default_left", C.POINTER(C.c_uint8)),
        ("gains", C.POINTER(C.c_float)), ("covers", C.POINTER(C.c_float)),
        ("split_bin", C.POINTER(C.c_uint32)), ("n_nodes", C.c_uint32),
        ("depth", C.c_uint32), ("n_leaves", C.c_uint32),
    ]


class _TreeBuf:
    def __init__(self, cap):
        self.a = dict(feature=np.zeros(cap, np.uint32), value=np.zeros(cap, np.float32),
                      left=np.zeros(cap, np.uint32), right=np.zeros(cap, np.uint32),
                      default_left=np.zeros(cap, np.uint8), gains=np.zeros(cap, np.float32),
                      covers=np.zeros(cap, np.float32), split_bin=np.zeros(cap, np.uint32))
        self.s = OrcTree()
        self.s.cap = cap
        for k, v in self.a.items():
            t = {np.uint32: C.c_uint32, np.float32: C.c_float, np.uint8: C.c_uint8}[v.dtype.type]
            setattr(self.s, k, _p(v, t))

    def tree(self):
        n = self.s.n_nodes
        return Tree(**{k: v[:n].copy() for k, v in self.a.items()},
                    depth=self.s.depth, n_leaves=self.s.n_leaves)


class Oracle:
    """The C restatement (bonsai_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle oracle)")
        self.L = C.CDLL(path)
        self.L.orc_init_score.restype = C.c_float

    @staticmethod
    def cfg(tc: TreeCfg):
        c = OrcTreeCfg()
        c.min_child_hess = tc.min_child_hess
        c.min_gain_to_split = tc.min_gain_to_split
        c.lambda_l2 = tc.lambda_l2
        c.lambda_l1 = tc.lambda_l1
        c.max_depth = tc.max_depth
        c.min_data_in_leaf = tc.min_data_in_leaf
        c.max_leaves = tc.max_leaves
        c.grower = GROWERS[tc.grower]
        if tc.monotone:
            c._mono = np.asarray(tc.monotone, dtype=np.int32)
            c.monotone = _p(c._mono, C.c_int32)
            c.n_monotone = len(tc.monotone)
        return c

    def transform(self, X, cuts, off):
        X = np.ascontiguousarray(X, np.float32)
        n, F = X.shape
        bins = np.empty((F, n), np.uint16)
        self.L.orc_transform(_p(X, C.c_float), C.c_size_t(n), C.c_size_t(F),
                             _p(np.ascontiguousarray(cuts, np.float32), C.c_float),
                             _p(np.ascontiguousarray(off, np.uint32), C.c_uint32),
                             _p(bins, C.c_uint16))
        return bins

    def grow(self, bins, n_bins, cuts, off, grad, hess, tc: TreeCfg, rows=None,
             selected=None):
        F, n = bins.shape
        bins = np.ascontiguousarray(bins, np.uint16)
        rows = np.arange(n, dtype=np.uint32) if rows is None else np.ascontiguousarray(rows, np.uint32)
        selected = np.arange(F, dtype=np.uint32) if selected is None else np.ascontiguousarray(selected, np.uint32)
        nb = np.ascontiguousarray(n_bins, np.uint32)
        cap = 4 << tc.max_depth if tc.grower != "leafwise" else 4 * max(tc.max_leaves, 2)
        tb = _TreeBuf(cap)
        values = np.empty(n, np.float32)
        ids = np.empty(n, np.uint32)
        cfg = self.cfg(tc)
        grad = np.ascontiguousarray(grad, np.float32)
        hess = np.ascontiguousarray(hess, np.float32)
        cuts = np.ascontiguousarray(cuts, np.float32)
        off = np.ascontiguousarray(off, np.uint32)
        rc = self.L.orc_grow_depthwise(
            _p(bins, C.c_uint16), C.c_size_t(n), C.c_size_t(F), _p(nb, C.c_uint32),
            _p(cuts, C.c_float), _p(off, C.c_uint32), _p(grad, C.c_float),
            _p(hess, C.c_float), _p(rows, C.c_uint32), C.c_size_t(len(rows)),
            _p(selected, C.c_uint32), C.c_size_t(len(selected)), C.byref(cfg),
            C.byref(tb.s), _p(values, C.c_float), _p(ids, C.c_uint32))
        if rc:
            raise RuntimeError("oracle tree outgrew its capacity")
        return tb.tree(), values, ids

    def train(self, bins, n_bins, cuts, off, labels, tc: TreeCfg):
        F, n = bins.shape
        bufs = [_TreeBuf(4 << tc.max_depth) for _ in range(tc.n_iters)]
        arr = (OrcTree * tc.n_iters)(*[b.s for b in bufs])
        init = C.c_float()
        scores = np.empty(n, np.float32)
        cfg = self.cfg(tc)
        bins = np.ascontiguousarray(bins, np.uint16)
        labels = np.ascontiguousarray(labels, np.float32)
        rc = self.L.orc_train_depthwise(
            _p(bins, C.c_uint16), C.c_size_t(n), C.c_size_t(F),
            _p(np.ascontiguousarray(n_bins, np.uint32), C.c_uint32),
            _p(np.ascontiguousarray(cuts, np.float32), C.c_float),
            _p(np.ascontiguousarray(off, np.uint32), C.c_uint32),
            _p(labels, C.c_float), C.c_int(OBJECTIVES[tc.objective]),
            C.c_uint32(tc.n_iters), C.c_float(tc.learning_rate), C.byref(cfg),
            arr, C.byref(init), _p(scores, C.c_float))
        if rc:
            raise RuntimeError("oracle tree outgrew its capacity")
        for i, b in enumerate(bufs):
            b.s = arr[i]
        return [b.tree() for b in bufs], init.value, scores

    def predict_binned(self, bins, n_bins, trees, init, lr):
        F, n = bins.shape
        bufs = []
        for t in trees:
            b = _TreeBuf(len(t.feature))
            for k in b.a:
                b.a[k][:] = getattr(t, k)
            b.s.n_nodes = len(t.feature)
            bufs.append(b)
        arr = (OrcTree * len(bufs))(*[b.s for b in bufs])
        out = np.empty(n, np.float32)
        bins = np.ascontiguousarray(bins, np.uint16)
        self.L.orc_predict_binned(_p(bins, C.c_uint16), C.c_size_t(n),
                                  _p(np.ascontiguousarray(n_bins, np.uint32), C.c_uint32),
                                  arr, C.c_size_t(len(bufs)), C.c_float(init),
                                  C.c_float(lr), _p(out, C.c_float))
        return out


def orc_find_split(orc: "Oracle", hist, n_rows, tc: TreeCfg, tot=None, lo=-np.inf, hi=np.inf):
    """orc_find_split on a [F, n_bins, 2] float32 histogram set sharing n_bins.
    Node totals default to Histogram::totals of feature 0."""
    hist = np.ascontiguousarray(hist, np.float32)
    F, nb, _ = hist.shape
    if tot is None:
        tot = (np.float32(hist[0, :, 0].astype(np.float64).sum()),
               np.float32(hist[0, :, 1].astype(np.float64).sum()))
    rows = [np.ascontiguousarray(hist[f].reshape(-1)) for f in range(F)]
    arr = (C.POINTER(C.c_float) * F)(*[_p(r, C.c_float) for r in rows])
    nbins = np.full(F, nb, np.uint32)
    present = np.ones(F, np.uint8)

    class _Split(C.Structure):
        _fields_ = [("gain", C.c_double), ("feature", C.c_uint32), ("bin", C.c_uint32),
                    ("default_left", C.c_uint8), ("valid", C.c_uint8)]

    orc.L.orc_find_split.restype = _Split
    cfg = Oracle.cfg(tc)
    s = orc.L.orc_find_split(arr, _p(nbins, C.c_uint32), _p(present, C.c_uint8),
                             C.c_size_t(F), C.c_size_t(n_rows), C.c_float(tot[0]),
                             C.c_float(tot[1]), C.c_double(lo), C.c_double(hi),
                             C.byref(cfg))
    return dict(gain=s.gain, feature=s.feature, bin=s.bin, default_left=s.default_left,
                valid=s.valid)


def orc_fill(orc: "Oracle", bins, n_bins, grad, hess, rows=None, selected=None):
    """orc_fill: one node's serial-order float histograms, [total_bins, 2]."""
    F, n = bins.shape
    bins = np.ascontiguousarray(bins, np.uint16)
    rows = np.arange(n, dtype=np.uint32) if rows is None else np.ascontiguousarray(rows, np.uint32)
    selected = np.arange(F, dtype=np.uint32) if selected is None else np.ascontiguousarray(selected, np.uint32)
    nb = np.ascontiguousarray(n_bins, np.uint32)
    total = int(nb[selected].sum())
    out = np.zeros((total, 2), np.float32)
    grad = np.ascontiguousarray(grad, np.float32)
    hess = np.ascontiguousarray(hess, np.float32)
    orc.L.orc_fill(_p(bins, C.c_uint16), C.c_size_t(n), _p(selected, C.c_uint32),
                   C.c_size_t(len(selected)), _p(nb, C.c_uint32), _p(grad, C.c_float),
                   _p(hess, C.c_float), _p(rows, C.c_uint32), C.c_size_t(len(rows)),
                   _p(out, C.c_float))
    return out


def bernoulli_keep(n: int, p: float, seed: int, trees: int) -> list:
    """BernoulliSampler::sample (src/sampler.cpp:36-55) restated in numpy:
    the booster's std::mt19937 seeded with booster_config.random_seed
    (include/bonsai/booster.hpp:496) feeds std::bernoulli_distribution(p) row
    by row, tree by tree. libstdc++ draws the uniform with
    generate_canonical<double, 53>: two 32-bit outputs x0, x1 make
    (x0 + x1 * 2^32) rounded to double, / 2^64, and a 1.0 becomes the
    largest double below 1; the row is kept when that is below p (the float
    p widened). numpy's MT19937 with its legacy seeding is the same
    generator as std::mt19937(seed). Returns one boolean mask per tree."""
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed))
    pd = np.float64(np.float32(p))
    out = []
    for _ in range(trees):
        raw = bg.random_raw(2 * n)
        u = (raw[0::2].astype(np.float64) + raw[1::2].astype(np.float64) * 4294967296.0)
        u = u / 18446744073709551616.0
        u = np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)
        out.append(u < pd)
    return out
