"""bonsai_b200: B200-native (sm_100a) CUDA growers for bonsai.

The hot path of bonsai's CUDA growers -- bin application, per-level
histograms with sibling subtraction, split finding, stable row partition,
leaf values with the fused score update, ensemble predict -- as hand-written
CUDA behind a C ABI (include/bonsai_b200.h). This module is the Python host
side over that ABI:

    cuts, off = fit_cuts(X)                  # host mappers
    plane = Plane(X, cuts, off)              # device bin application
    b = Booster(plane, y, TrainParams(...))  # device-resident boosting
    b.update(100); trees = b.trees()
    p = predict(plane, trees, b.init_score, lr)
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import BonsaiError, ConfigError, check, lib, ptr
from .binning import cuts_from_sample, fit_cuts, sample_rows

__all__ = [
    "BonsaiError", "ConfigError", "TrainParams", "Plane", "Booster", "Tree",
    "grow_tree", "populate", "predict", "PredictPlan", "ShapPlan", "predict_classes", "pred_contribs", "pred_contribs_classes", "oblivious_tables", "fit_cuts",
    "Comm", "early_stop_round", "fit_early_stopping", "shard_range", "init_score", "label_sum", "init_score_from_sum", "cuts_from_sample", "sample_rows", "fit_cuts_device",
    "available", "LEAF", "tune", "BoosterBatch",
]

LEAF = 0xFFFFFFFF
OBJECTIVES = {"mse": 0, "logloss": 1, "softmax": 2, "poisson": 3}
GROWERS = {"depthwise": 0, "levelwise": 1, "oblivious": 1, "leafwise": 2}
HIST_MODES = {"exact": 0, "plain": 0, "int8": 1, "quant8": 1, "int16": 2, "quant16": 2}


def fit_cuts_device(X, max_bin: int = 255, n_samples: int = 200_000, seed: int = 0):
    """fit_cuts on the device (bb_fit_cuts): the same row sample as the host
    fit (sample_rows), the same cuts. X is a host array or a CUDA tensor."""
    on_device = hasattr(X, "data_ptr") and getattr(X, "is_cuda", False)
    n, F = X.shape
    rows = sample_rows(n, n_samples, seed)
    if on_device:
        import torch
        S = X if rows is None else X[torch.as_tensor(rows, device=X.device)]
        S = S.float().contiguous()
        sp = S.data_ptr()
    else:
        X = np.asarray(X, dtype=np.float32)
        S = np.ascontiguousarray(X if rows is None else X[rows])
        sp = ptr(S)
    cuts = np.empty(F * max_bin, np.float32)
    off = np.empty(F + 1, np.uint32)
    check(lib().bb_fit_cuts(sp, S.shape[0], F, 1 if on_device else 0, max_bin, ptr(cuts),
                            len(cuts), ptr(off)))
    return cuts[: off[-1]].copy(), off


def available() -> bool:
    return bool(lib().bb_available())


@dataclass
class TrainParams:
    """TreeConfig / BoosterConfig keys the device path reads (defaults are
    the reference's: include/bonsai/config/tree_config.hpp:9-29)."""
    objective: str = "mse"
    learning_rate: float = 0.1
    min_child_hess: float = 1.0
    min_gain_to_split: float = 0.0
    lambda_l2: float = 1.0
    lambda_l1: float = 0.0
    max_depth: int = 6
    min_data_in_leaf: int = 20
    hist_mode: str = "exact"
    seed: int = 0
    monotone: list = field(default_factory=list)
    selected: list | None = None
    use_graph: bool = False
    record_leaf_ids: bool = False
    grower: str = "depthwise"
    max_leaves: int = 31
    n_classes: int = 0
    # TreeConfig::interaction_constraints: feature groups, each a list of ids
    # or the reference's string form ("0,1" or "0+1")
    interaction_constraints: list = field(default_factory=list)
    # sampler.subsample and booster_config.random_seed: a resident booster
    # with subsample < 1 grows each tree over a Bernoulli row sample
    # (BernoulliSampler, src/sampler.cpp:36-55)
    subsample: float = 1.0
    random_seed: int = 42
    # tree_config.feature_fraction / feature_seed: a resident booster with
    # feature_fraction < 1 grows each tree over its own feature sample
    # (sample_features, src/grower_impl.hpp:163-180)
    feature_fraction: float = 1.0
    feature_seed: int = 2
    # the quantised histogram build's CTAs per mirror tile (0: the default
    # launch shape); bonsai_b200.autotune picks it per shape. Results do not
    # depend on it.
    hist_ctas: int = 0

    def c(self) -> _lib.TrainCfg:
        c = _lib.TrainCfg()
        c.objective = OBJECTIVES[self.objective]
        c.learning_rate = self.learning_rate
        c.min_child_hess = self.min_child_hess
        c.min_gain_to_split = self.min_gain_to_split
        c.lambda_l2 = self.lambda_l2
        c.lambda_l1 = self.lambda_l1
        c.max_depth = self.max_depth
        c.min_data_in_leaf = self.min_data_in_leaf
        c.hist_mode = HIST_MODES[self.hist_mode]
        c.seed = self.seed
        c.grower = GROWERS[self.grower]
        c.max_leaves = self.max_leaves
        c.n_classes = self.n_classes
        c.subsample = self.subsample
        c.random_seed = self.random_seed
        c.feature_fraction = self.feature_fraction
        c.feature_seed = self.feature_seed
        c.use_graph = 1 if self.use_graph else 0
        c.hist_ctas = int(self.hist_ctas)
        c.record_leaf_ids = 1 if self.record_leaf_ids else 0
        if self.monotone:
            c._mono = np.ascontiguousarray(self.monotone, dtype=np.int8)
            c.monotone = c._mono.ctypes.data_as(C.POINTER(C.c_int8))
            c.n_monotone = len(self.monotone)
        if self.interaction_constraints:
            groups = []
            for g in self.interaction_constraints:
                if isinstance(g, str):
                    g = [int(x) for x in g.replace("+", ",").split(",") if x.strip()]
                groups.append(sorted(int(x) for x in g))
            c._ifeat = np.ascontiguousarray(
                np.concatenate([np.asarray(g, np.uint32) for g in groups]) if groups
                else np.zeros(0, np.uint32), dtype=np.uint32)
            c._ioff = np.ascontiguousarray(
                np.concatenate([[0], np.cumsum([len(g) for g in groups])]), dtype=np.uint32)
            c.interaction_features = c._ifeat.ctypes.data_as(C.POINTER(C.c_uint32))
            c.interaction_offsets = c._ioff.ctypes.data_as(C.POINTER(C.c_uint32))
            c.n_interaction_groups = len(groups)
        if self.selected is not None:
            c._sel = np.ascontiguousarray(self.selected, dtype=np.uint32)
            c.selected = c._sel.ctypes.data_as(C.POINTER(C.c_uint32))
            c.n_selected = len(self.selected)
        return c


@dataclass
class Tree:
    """One tree in the reference's DenseTree layout (tree.hpp:38-45)."""
    feature: np.ndarray
    value: np.ndarray
    left: np.ndarray
    right: np.ndarray
    default_left: np.ndarray
    gains: np.ndarray
    covers: np.ndarray
    split_bin: np.ndarray
    depth: int = 0
    n_leaves: int = 0


def oblivious_tables(tree: Tree):
    """A levelwise tree as the reference's ObliviousTree keeps it
    (include/bonsai/oblivious_tree.hpp): per level the split feature,
    threshold and default direction, and the 2^depth leaf values in frontier
    order (the first level is the most significant bit of a leaf's index)."""
    feats, thr, dl = [], [], []
    i = 0
    while tree.feature[i] != LEAF:
        feats.append(int(tree.feature[i]))
        thr.append(float(tree.value[i]))
        dl.append(int(tree.default_left[i]))
        i = int(tree.left[i])
    d = len(feats)
    first = (1 << d) - 1
    leaves = tree.value[first:first + (1 << d)].astype(np.float32)
    return (np.array(feats, np.uint32), np.array(thr, np.float32), np.array(dl, np.uint8),
            leaves)


def _tree_arrays(cap: int):
    return dict(feature=np.zeros(cap, np.uint32), value=np.zeros(cap, np.float32),
                left=np.zeros(cap, np.uint32), right=np.zeros(cap, np.uint32),
                default_left=np.zeros(cap, np.uint8), gains=np.zeros(cap, np.float32),
                covers=np.zeros(cap, np.float32), split_bin=np.zeros(cap, np.uint32))


_ORDER = ("feature", "value", "left", "right", "default_left", "gains", "covers",
          "split_bin")


def _finish(a: dict, meta: np.ndarray) -> Tree:
    n = int(meta[0])
    return Tree(**{k: v[:n].copy() for k, v in a.items()}, depth=int(meta[1]),
                n_leaves=int(meta[2]))


class Plane:
    """A device-resident binned dataset (bb_ingest)."""

    def __init__(self, X, cuts, cut_off, x_on_device: bool = False):
        if x_on_device:
            # a torch CUDA tensor (or anything exposing data_ptr and shape)
            n, F = X.shape
            xp = X.data_ptr()
            self._keep = X
        else:
            X = np.ascontiguousarray(X, dtype=np.float32)
            n, F = X.shape
            xp = ptr(X)
            self._keep = X
        self.cuts = np.ascontiguousarray(cuts, dtype=np.float32)
        self.cut_off = np.ascontiguousarray(cut_off, dtype=np.uint32)
        if len(self.cut_off) != F + 1:
            raise ValueError("cut_off must hold n_features + 1 offsets")
        self.n_rows, self.n_feats = int(n), int(F)
        self.n_bins = np.diff(self.cut_off).astype(np.uint32)
        h = C.c_void_p()
        check(lib().bb_ingest(xp, n, F, 1 if x_on_device else 0, ptr(self.cuts),
                              ptr(self.cut_off), C.byref(h)))
        self.h = h.value
        self._keep = None

    @classmethod
    def from_device(cls, X, cuts, cut_off) -> "Plane":
        """Zero-copy ingest of a device-resident n x F float32 row-major matrix
        (cuda_ingest_device, include/bonsai/cuda/histogram_engine.hpp:41-50): a torch
        CUDA tensor, any producer of DLPack (__dlpack__) or of the CUDA array interface
        (CuPy, Numba, JAX ...). The bin kernel reads the matrix where it lies; the
        producer's pending writes are ordered before it (DLPack and the array interface
        hand their stream to torch's current stream, which is synchronised), and the
        matrix is not retained: it may be freed once this returns."""
        import torch
        if isinstance(X, torch.Tensor):
            t = X
        elif hasattr(X, "__dlpack__"):
            t = torch.from_dlpack(X)
        elif hasattr(X, "__cuda_array_interface__"):
            t = torch.as_tensor(X, device="cuda")
        else:
            raise TypeError("from_device: expected a CUDA tensor, a DLPack producer or an "
                            "object with __cuda_array_interface__")
        if not t.is_cuda:
            raise ValueError("from_device: the matrix is not in CUDA device memory")
        if t.dtype != torch.float32 or t.dim() != 2:
            raise ValueError("from_device: expected a 2-D float32 matrix")
        if not t.is_contiguous():
            raise ValueError("from_device: the matrix must be row-major contiguous")
        with torch.cuda.device(t.device):
            torch.cuda.current_stream(t.device).synchronize()
            return cls(t, cuts, cut_off, x_on_device=True)

    @classmethod
    def from_bins(cls, bins, cuts, cut_off) -> "Plane":
        """A plane over codes binned elsewhere (bb_plane_from_bins): bins is
        [n_feats, n_rows], uint8 (every feature <= 256 bins) or uint16, each
        code below its feature's bin count cut_off[f + 1] - cut_off[f]."""
        bins = np.ascontiguousarray(bins)
        if bins.dtype not in (np.uint8, np.uint16) or bins.ndim != 2:
            raise ValueError("bins must be a 2-D uint8 or uint16 array [n_feats, n_rows]")
        self = cls.__new__(cls)
        self.cuts = np.ascontiguousarray(cuts, dtype=np.float32)
        self.cut_off = np.ascontiguousarray(cut_off, dtype=np.uint32)
        F, n = bins.shape
        if len(self.cut_off) != F + 1:
            raise ValueError("cut_off must hold n_features + 1 offsets")
        self.n_rows, self.n_feats = int(n), int(F)
        self.n_bins = np.diff(self.cut_off).astype(np.uint32)
        self._keep = None
        h = C.c_void_p()
        check(lib().bb_plane_from_bins(ptr(bins), 1 if bins.dtype == np.uint8 else 0, n, F,
                                       ptr(self.cuts), ptr(self.cut_off), C.byref(h)))
        self.h = h.value
        return self

    @classmethod
    def like(cls, plane: "Plane", max_rows: int) -> "Plane":
        """A request plane (bb_plane_create_like): `plane`'s mappers and room
        for max_rows rows, allocated once; `refill` bins each batch into it."""
        self = cls.__new__(cls)
        self.cuts, self.cut_off, self.n_bins = plane.cuts, plane.cut_off, plane.n_bins
        self.n_feats, self.n_rows, self.max_rows = plane.n_feats, 0, int(max_rows)
        self._keep = None
        h = C.c_void_p()
        check(lib().bb_plane_create_like(plane.h, max_rows, C.byref(h)))
        self.h = h.value
        return self

    def refill(self, X, x_on_device: bool = False) -> "Plane":
        """Bins a new batch into this request plane (bb_plane_refill)."""
        if x_on_device:
            n, F = X.shape
            xp = X.data_ptr()
        else:
            X = np.ascontiguousarray(X, dtype=np.float32)
            n, F = X.shape
            xp = ptr(X)
        if F != self.n_feats:
            raise ValueError("the batch has another feature count")
        check(lib().bb_plane_refill(self.h, xp, n, 1 if x_on_device else 0))
        self.n_rows = int(n)
        return self

    @property
    def u8(self) -> bool:
        return bool(lib().bb_plane_is_u8(self.h))

    def bins(self) -> np.ndarray:
        out = np.empty((self.n_feats, self.n_rows), np.uint16)
        check(lib().bb_plane_download(self.h, ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().bb_plane_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass  # interpreter shutdown: the library may be gone already


COMM_ID_BYTES = 128


class Comm:
    """A row-shard reducer (bb_comm): NCCL across processes, or one member
    of an in-process group of shards."""

    def __init__(self, h):
        self.h = h

    @staticmethod
    def _load_nccl():
        # the process's NCCL is PyTorch's when PyTorch is present: load it
        # before the library resolves libnccl.so.2
        try:
            import torch  # noqa: F401
        except ImportError:
            pass

    @staticmethod
    def unique_id() -> bytes:
        Comm._load_nccl()
        buf = (C.c_uint8 * COMM_ID_BYTES)()
        check(lib().bb_comm_unique_id(C.cast(buf, C.c_void_p)))
        return bytes(buf)

    @classmethod
    def nccl(cls, uid: bytes, n_ranks: int, rank: int) -> "Comm":
        cls._load_nccl()
        buf = (C.c_uint8 * COMM_ID_BYTES).from_buffer_copy(uid)
        h = C.c_void_p()
        check(lib().bb_comm_create(C.cast(buf, C.c_void_p), n_ranks, rank, C.byref(h)))
        return cls(h.value)

    @classmethod
    def group(cls, n_shards: int) -> list:
        arr = (C.c_void_p * n_shards)()
        check(lib().bb_comm_group(n_shards, C.cast(arr, C.c_void_p)))
        return [cls(arr[i]) for i in range(n_shards)]

    def close(self):
        if getattr(self, "h", None):
            lib().bb_comm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shard_range(n_rows: int, n_shards: int, shard: int) -> tuple:
    """Rows [begin, end) of shard `shard`: contiguous, sizes differing by one."""
    return (n_rows * shard) // n_shards, (n_rows * (shard + 1)) // n_shards


def label_sum(labels, start: float = 0.0) -> np.float32:
    """std::accumulate over float labels: a float serial sum, continued from
    `start` (so shards can chain it in row order)."""
    s = np.float32(start)
    for v in np.asarray(labels, np.float32):
        s = np.float32(s + v)
    return s


_logf = None


def init_score_from_sum(total: float, n_rows: int, objective: str) -> np.float32:
    """The objective's initial score from the fit's float label sum: the
    mean, or its log-odds through the C library's logf as the booster does."""
    global _logf
    m = np.float32(np.float32(total) / np.float32(n_rows))
    if OBJECTIVES[objective] == 0:
        return m
    if _logf is None:
        libm = C.CDLL("libm.so.6")
        libm.logf.restype = C.c_float
        libm.logf.argtypes = [C.c_float]
        _logf = libm.logf
    return np.float32(_logf(float(np.float32(m / np.float32(np.float32(1.0) - m)))))


def init_score(labels, objective: str) -> np.float32:
    """bb_booster_create's initial score over all of `labels`."""
    if objective == "poisson":
        # PoissonObjective::init_score: an FP64 sum, the log of the mean
        y = np.asarray(labels, np.float32)
        if (y < 0).any() or np.isnan(y).any():
            raise ValueError("poisson objective requires non-negative labels")
        total = float(np.cumsum(y.astype(np.float64))[-1]) if len(y) else 0.0  # in row order
        mean = total / max(len(y), 1)
        return np.float32(np.log(max(mean, 1e-9)))
    return init_score_from_sum(label_sum(labels), len(labels), objective)


class Booster:
    """Device-resident boosting (bb_booster_*). With comm, one row shard of a
    fit: the plane and labels hold the fit's rows [row_offset, row_offset +
    plane rows) of total_rows, and init_score is the fit's."""

    def __init__(self, plane: Plane, labels, params: TrainParams, max_trees: int = 1000,
                 init_scores=None, comm: Comm | None = None, row_offset: int = 0,
                 total_rows: int | None = None, init_score: float | None = None,
                 weights=None):
        self.plane = plane
        self.params = params
        self._labels = np.ascontiguousarray(labels, dtype=np.float32)
        init = None if init_scores is None else np.ascontiguousarray(init_scores, np.float32)
        h = C.c_void_p()
        self._cfg = params.c()
        if comm is None:
            check(lib().bb_booster_create(plane.h, ptr(self._labels),
                                          None if init is None else ptr(init),
                                          C.byref(self._cfg), max_trees, C.byref(h)))
        else:
            self._comm = comm
            check(lib().bb_booster_create_sharded(
                plane.h, ptr(self._labels), None if init is None else ptr(init),
                C.byref(self._cfg), max_trees, comm.h, row_offset,
                plane.n_rows if total_rows is None else total_rows,
                float(init_score), C.byref(h)))
        self.h = h.value
        if weights is not None:
            self.set_weights(weights)

    def set_weights(self, weights):
        """Per-row sample weights scaling every round's (g, h) (bb_booster_set_weights);
        None returns to the unweighted fit. Before the first round only."""
        if weights is None:
            check(lib().bb_booster_set_weights(self.h, None))
            self._weights = None
            return
        self._weights = np.ascontiguousarray(weights, dtype=np.float32)
        if self._weights.shape != (self.plane.n_rows,):
            raise ValueError("weights: one per plane row")
        check(lib().bb_booster_set_weights(self.h, ptr(self._weights)))

    def update(self, n_iters: int = 1, sync: bool = True):
        check(lib().bb_booster_update(self.h, n_iters))
        if sync:
            self.sync()

    def sync(self):
        check(lib().bb_booster_sync(self.h))

    @property
    def last_ms(self) -> float:
        ms = C.c_float()
        check(lib().bb_booster_last_ms(self.h, C.byref(ms)))
        return ms.value

    @property
    def init_score(self) -> float:
        return float(lib().bb_booster_init_score(self.h))

    @property
    def n_trees(self) -> int:
        n = C.c_uint32()
        check(lib().bb_booster_n_trees(self.h, C.byref(n)))
        return n.value

    def tree(self, t: int) -> Tree:
        cap = int(lib().bb_booster_tree_capacity(self.h))
        a = _tree_arrays(cap)
        meta = np.zeros(3, np.uint32)
        check(lib().bb_booster_tree(self.h, t, *(ptr(a[k]) for k in _ORDER), ptr(meta)))
        return _finish(a, meta)

    def trees(self) -> list:
        """Every tree, copied from the device in one transfer per array
        (bb_booster_trees)."""
        n = self.n_trees
        if n == 0:
            return []
        cap = int(lib().bb_booster_tree_capacity(self.h))
        a = _tree_arrays(cap * n)
        meta = np.zeros(3 * n, np.uint32)
        check(lib().bb_booster_trees(self.h, 0, n, *(ptr(a[k]) for k in _ORDER), ptr(meta)))
        return [_finish({k: v[i * cap:(i + 1) * cap] for k, v in a.items()},
                        meta[3 * i:3 * i + 3]) for i in range(n)]

    @property
    def n_classes(self) -> int:
        return int(lib().bb_booster_n_classes(self.h))

    @property
    def init_scores(self) -> np.ndarray:
        """One init score per class (softmax), else the one."""
        out = np.empty(max(1, self.n_classes), np.float32)
        check(lib().bb_booster_init_scores(self.h, ptr(out)))
        return out

    def scores(self) -> np.ndarray:
        """Training scores: n_rows, or n_rows x n_classes (softmax)."""
        K = self.n_classes
        out = np.empty((self.plane.n_rows, K) if K > 1 else self.plane.n_rows, np.float32)
        check(lib().bb_booster_scores(self.h, ptr(out)))
        return out

    def eval_arm(self, valid: Plane, labels, init_scores=None):
        """Arms the device validation plane (bb_booster_eval_arm): every later
        round records its validation loss on the device. `valid` must be
        binned with the training plane's cuts and outlive the booster."""
        y = np.ascontiguousarray(labels, np.float32)
        if len(y) != valid.n_rows:
            raise ValueError("labels must hold one value per validation row")
        init = None
        if init_scores is not None:
            init = np.ascontiguousarray(init_scores, np.float32)
            if init.size != valid.n_rows * self.n_classes:
                raise ValueError("init_scores must hold n_valid x n_classes values")
            # the device keeps one column per class
            if self.n_classes > 1:
                init = np.ascontiguousarray(init.reshape(valid.n_rows, self.n_classes).T)
        check(lib().bb_booster_eval_arm(self.h, valid.h, ptr(y),
                                        None if init is None else ptr(init)))
        self.valid = valid

    def eval_losses(self) -> np.ndarray:
        """The validation loss of every round since eval_arm."""
        n = C.c_uint32()
        check(lib().bb_booster_eval_losses(self.h, None, 0, C.byref(n)))
        out = np.empty(n.value, np.float32)
        if n.value:
            check(lib().bb_booster_eval_losses(self.h, ptr(out), n.value, C.byref(n)))
        return out

    def eval_scores(self) -> np.ndarray:
        """The validation raw scores: n_valid, or n_valid x n_classes."""
        K = self.n_classes
        n = self.valid.n_rows
        out = np.empty((n, K) if K > 1 else n, np.float32)
        check(lib().bb_booster_eval_scores(self.h, ptr(out)))
        return out

    def truncate(self, n_rounds: int):
        """Keeps the first n_rounds rounds (bb_booster_truncate)."""
        check(lib().bb_booster_truncate(self.h, n_rounds))

    def leaf_ids(self) -> np.ndarray:
        out = np.empty(self.plane.n_rows, np.uint32)
        check(lib().bb_booster_leaf_ids(self.h, ptr(out)))
        return out

    def profile_round(self) -> dict:
        """One boosting round timed phase by phase (bb_booster_profile_round)."""
        p = _lib.Profile()
        check(lib().bb_booster_profile_round(self.h, C.byref(p)))
        out = {k: getattr(p, k) for k, _ in _lib.Profile._fields_}
        n = min(int(p.hist_builds), 16)
        out["build_ms"] = [float(x) for x in p.build_ms[:n]]
        out["build_rows"] = [int(x) for x in p.build_rows[:n]]
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().bb_booster_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass  # interpreter shutdown: the library may be gone already


class BoosterBatch:
    """Many boosters, one graph launch per round (bb_batch_*): every
    booster's round graph is a child of one parent graph, so a round of the
    whole batch is one launch and the boosters run concurrently. Boosters
    must use CUDA graphs, without row or feature sampling; they must outlive
    the batch. Their trees and scores read as usual afterwards."""

    def __init__(self, boosters):
        self.boosters = list(boosters)
        arr = (C.c_void_p * len(self.boosters))(*[b.h for b in self.boosters])
        h = C.c_void_p()
        check(lib().bb_batch_create(arr, len(self.boosters), C.byref(h)))
        self.h = h.value

    def update(self, n_rounds: int = 1, sync: bool = True):
        check(lib().bb_batch_update(self.h, n_rounds))
        if sync:
            check(lib().bb_batch_sync(self.h))

    @property
    def last_ms(self) -> float:
        ms = C.c_float()
        check(lib().bb_batch_last_ms(self.h, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().bb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def early_stop_round(losses, patience: int):
    """The reference's early-stopping rule over a loss record
    (src/cli/pipeline.cpp:452-462): the best round is the first with the
    lowest loss so far; the fit stops at the first round `patience` rounds
    past the best. Returns (rounds to keep, stopped)."""
    best, best_i = 0.0, 0
    for i, loss in enumerate(losses):
        if i == 0 or loss < best:
            best, best_i = float(loss), i
        elif i - best_i >= patience:
            return best_i + 1, True
    return len(losses), False


def fit_early_stopping(booster: "Booster", valid: Plane, labels, n_iters: int, patience: int,
                       check_every: int = 16) -> int:
    """Boosts up to n_iters rounds with the validation loss recorded on the
    device, reading the record every `check_every` rounds, and keeps the
    rounds the reference's early-stopping rule keeps (bb_booster_truncate).
    Rounds run past the stopping point only cost time: the kept model is the
    one the per-round rule keeps. Returns the rounds kept."""
    if patience <= 0:
        raise ValueError("patience must be positive")
    booster.eval_arm(valid, labels)
    done = 0
    while done < n_iters:
        step = min(check_every, n_iters - done)
        booster.update(step)
        done += step
        keep, stopped = early_stop_round(booster.eval_losses(), patience)
        if stopped:
            booster.truncate(keep)
            return keep
    return done


def grow_tree(plane: Plane, params: TrainParams, grad, hess, rows=None):
    """One tree from given gradients (bb_grow_tree): returns
    (tree, values, leaf_ids) over every row (unsampled rows: NaN / max)."""
    n = plane.n_rows
    grad = np.ascontiguousarray(grad, np.float32)
    hess = np.ascontiguousarray(hess, np.float32)
    cfg = params.c()
    cap = int(lib().bb_tree_capacity(C.byref(cfg)))
    a = _tree_arrays(cap)
    meta = np.zeros(3, np.uint32)
    values = np.full(n, np.nan, np.float32)
    ids = np.full(n, LEAF, np.uint32)
    r = None if rows is None else np.ascontiguousarray(rows, np.uint32)
    check(lib().bb_grow_tree(plane.h, C.byref(cfg), ptr(grad), ptr(hess),
                             None if r is None else ptr(r), 0 if r is None else len(r),
                             *(ptr(a[k]) for k in _ORDER), ptr(meta), ptr(values),
                             ptr(ids)))
    return _finish(a, meta), values, ids


def populate(plane: Plane, params: TrainParams, grad, hess, rows=None) -> np.ndarray:
    """One node's histograms (bb_populate): [total_bins, 2] FP64 (g, h) cell
    sums, features in selection order."""
    grad = np.ascontiguousarray(grad, np.float32)
    hess = np.ascontiguousarray(hess, np.float32)
    sel = params.selected if params.selected is not None else range(plane.n_feats)
    total = int(sum(int(plane.n_bins[f]) for f in sel))
    out = np.empty((total, 2), np.float64)
    r = None if rows is None else np.ascontiguousarray(rows, np.uint32)
    cfg = params.c()
    check(lib().bb_populate(plane.h, C.byref(cfg), ptr(grad), ptr(hess),
                            None if r is None else ptr(r), 0 if r is None else len(r),
                            ptr(out)))
    return out


def _concat(trees: list, keys):
    roots = np.zeros(len(trees), np.uint32)
    parts = {k: [] for k in keys}
    base = 0
    for i, t in enumerate(trees):
        roots[i] = base
        for k in parts:
            parts[k].append(getattr(t, k))
        base += len(t.feature)
    return roots, base, {k: np.ascontiguousarray(np.concatenate(v)) for k, v in parts.items()}


def predict(plane: Plane, trees: list, init: float, lr: float) -> np.ndarray:
    """Ensemble predict in bin space (bb_predict)."""
    roots, base, cat = _concat(trees, ("feature", "split_bin", "left", "right",
                                       "default_left", "value"))
    out = np.empty(plane.n_rows, np.float32)
    check(lib().bb_predict(plane.h, len(trees), ptr(roots), base, ptr(cat["feature"]),
                           ptr(cat["split_bin"]), ptr(cat["left"]), ptr(cat["right"]),
                           ptr(cat["default_left"]), ptr(cat["value"]), lr, init, ptr(out)))
    return out


class PredictPlan:
    """An ensemble packed for the device once (bb_predict_plan_*): `run`
    scores any plane with the features and bin counts of the one it was
    packed against, bit-identical to `predict`."""

    def __init__(self, plane: Plane, trees: list, init: float, lr: float):
        roots, base, cat = _concat(trees, ("feature", "split_bin", "left", "right",
                                           "default_left", "value"))
        self.n_trees = len(trees)
        h = C.c_void_p()
        check(lib().bb_predict_plan_create(plane.h, len(trees), ptr(roots), base,
                                           ptr(cat["feature"]), ptr(cat["split_bin"]),
                                           ptr(cat["left"]), ptr(cat["right"]),
                                           ptr(cat["default_left"]), ptr(cat["value"]), lr,
                                           init, C.byref(h)))
        self.h = h

    @property
    def depth(self) -> int:
        """The padded heap depth, or 0 for the node-table form."""
        d = C.c_uint32()
        check(lib().bb_predict_plan_depth(self.h, C.byref(d)))
        return d.value

    def run(self, plane: Plane, n_trees: int = 0) -> np.ndarray:
        out = np.empty(plane.n_rows, np.float32)
        check(lib().bb_predict_plan_run(self.h, plane.h, n_trees, ptr(out)))
        return out

    def launch(self, plane: Plane, out_ptr: int, stream_ptr: int = 0, n_trees: int = 0) -> int:
        """Enqueues the scores into device memory at out_ptr on a stream
        (a cudaStream_t as an int); returns the kernels launched."""
        k = C.c_uint32()
        check(lib().bb_predict_plan_launch(self.h, plane.h, n_trees, C.c_void_p(out_ptr),
                                           C.c_void_p(stream_ptr), C.byref(k)))
        return k.value

    def close(self):
        if getattr(self, "h", None):
            lib().bb_predict_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pred_contribs_classes(plane: Plane, trees: list, init_scores, lr: float) -> np.ndarray:
    """TreeSHAP of a softmax ensemble whose trees are round-major (tree r * K + k
    is class k's): n_rows x K x (n_feats + 1), class k's contributions scaled
    by lr with its initial score in the bias column, as MulticlassBooster
    composes them (include/bonsai/multiclass_booster.hpp:411-436)."""
    K = len(init_scores)
    return np.stack([pred_contribs(plane, trees[k::K], float(init_scores[k]), lr)
                     for k in range(K)], axis=1)


def predict_classes(plane: Plane, trees: list, init_scores, lr: float) -> np.ndarray:
    """Raw per-class scores (n_rows x K) of a softmax ensemble whose trees are
    round-major (tree r * K + k is class k's): each class through predict."""
    K = len(init_scores)
    return np.stack([predict(plane, trees[k::K], float(init_scores[k]), lr)
                     for k in range(K)], axis=1)


def pred_contribs(plane: Plane, trees: list, init: float, lr: float) -> np.ndarray:
    """TreeSHAP contributions in bin space (bb_pred_contribs): [n_rows,
    n_feats + 1] FP64, the last column the bias; rows sum to the margin."""
    roots, base, cat = _concat(trees, ("feature", "split_bin", "left", "right",
                                       "default_left", "value", "covers"))
    out = np.empty((plane.n_rows, plane.n_feats + 1), np.float64)
    check(lib().bb_pred_contribs(plane.h, len(trees), ptr(roots), base, ptr(cat["feature"]),
                                 ptr(cat["split_bin"]), ptr(cat["left"]), ptr(cat["right"]),
                                 ptr(cat["default_left"]), ptr(cat["value"]),
                                 ptr(cat["covers"]), lr, init, ptr(out)))
    return out


class ShapPlan:
    """An ensemble's TreeSHAP paths packed for the device once
    (bb_shap_plan_*): `run` returns [n_rows, n_feats + 1] FP64 contributions
    for any plane with the features and bin counts it was packed against."""

    def __init__(self, plane: Plane, trees: list, init: float, lr: float):
        roots, base, cat = _concat(trees, ("feature", "split_bin", "left", "right",
                                           "default_left", "value", "covers"))
        h = C.c_void_p()
        check(lib().bb_shap_plan_create(plane.h, len(trees), ptr(roots), base,
                                        ptr(cat["feature"]), ptr(cat["split_bin"]),
                                        ptr(cat["left"]), ptr(cat["right"]),
                                        ptr(cat["default_left"]), ptr(cat["value"]),
                                        ptr(cat["covers"]), lr, init, C.byref(h)))
        self.h = h

    def run(self, plane: Plane) -> np.ndarray:
        out = np.empty((plane.n_rows, plane.n_feats + 1), np.float64)
        check(lib().bb_shap_plan_run(self.h, plane.h, ptr(out)))
        return out

    def launch(self, plane: Plane, out_ptr: int, stream_ptr: int = 0) -> int:
        """Enqueues the contributions into device memory at out_ptr
        (n_rows x (n_feats + 1) doubles); returns the kernels launched."""
        k = C.c_uint32()
        check(lib().bb_shap_plan_launch(self.h, plane.h, C.c_void_p(out_ptr),
                                        C.c_void_p(stream_ptr), C.byref(k)))
        return k.value

    def close(self):
        if getattr(self, "h", None):
            lib().bb_shap_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune(plane, labels, params, **kw):
    """params with the quantised build's launch shape autotuned for this
    plane (bonsai_b200.autotune: timed once per shape, cached on disk)."""
    from .autotune import tune as _tune
    return _tune(plane, labels, params, **kw)
