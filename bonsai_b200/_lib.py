"""ctypes binding of libbonsai_b200.so (the C ABI in include/bonsai_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libbonsai_b200.so")

BB_OK, BB_ERR_CUDA, BB_ERR_CONFIG, BB_ERR_ARG, BB_DECLINED = range(5)


class BonsaiError(RuntimeError):
    """A failed call: .code is the C ABI status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class ConfigError(BonsaiError):
    """A capacity or configuration refusal (the reference's ConfigError)."""


class TrainCfg(C.Structure):
    _fields_ = [
        ("objective", C.c_int32), ("learning_rate", C.c_float),
        ("min_child_hess", C.c_float), ("min_gain_to_split", C.c_float),
        ("lambda_l2", C.c_float), ("lambda_l1", C.c_float),
        ("max_depth", C.c_uint32), ("min_data_in_leaf", C.c_uint32),
        ("hist_mode", C.c_int32), ("seed", C.c_uint64),
        ("monotone", C.POINTER(C.c_int8)), ("n_monotone", C.c_uint32),
        ("selected", C.POINTER(C.c_uint32)), ("n_selected", C.c_uint32),
        ("use_graph", C.c_int32), ("record_leaf_ids", C.c_int32),
        ("grower", C.c_int32), ("max_leaves", C.c_uint32), ("n_classes", C.c_uint32),
        ("interaction_features", C.POINTER(C.c_uint32)),
        ("interaction_offsets", C.POINTER(C.c_uint32)), ("n_interaction_groups", C.c_uint32),
        ("subsample", C.c_float), ("random_seed", C.c_uint32),
        ("feature_fraction", C.c_float), ("feature_seed", C.c_uint32),
        ("external_sample", C.c_int32), ("hist_ctas", C.c_uint32),
    ]


class Profile(C.Structure):
    _fields_ = [
        ("hist_ms", C.c_double), ("partition_ms", C.c_double), ("find_ms", C.c_double),
        ("other_ms", C.c_double), ("total_ms", C.c_double), ("hist_bytes", C.c_double),
        ("hist_rows", C.c_uint64), ("hist_builds", C.c_uint32), ("launches", C.c_uint32),
        ("build_ms", C.c_double * 16), ("build_rows", C.c_uint64 * 16),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m bonsai_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.bb_last_error.restype = C.c_char_p
        L.bb_booster_init_score.restype = C.c_float
        L.bb_booster_tree_capacity.restype = C.c_uint32
        vp = C.c_void_p
        L.bb_ingest.argtypes = [vp, C.c_uint64, C.c_uint32, C.c_int, vp, vp, C.POINTER(vp)]
        L.bb_plane_is_u8.argtypes = [vp]
        L.bb_plane_from_bins.argtypes = [vp, C.c_int, C.c_uint64, C.c_uint32, vp, vp,
                                         C.POINTER(vp)]
        L.bb_plane_download.argtypes = [vp, vp]
        L.bb_plane_destroy.argtypes = [vp]
        L.bb_booster_create.argtypes = [vp, vp, vp, C.POINTER(TrainCfg), C.c_uint32,
                                        C.POINTER(vp)]
        L.bb_booster_update.argtypes = [vp, C.c_uint32]
        L.bb_booster_set_rows.argtypes = [vp, vp, C.c_uint64]
        L.bb_batch_create.argtypes = [vp, C.c_uint32, C.POINTER(vp)]
        L.bb_batch_update.argtypes = [vp, C.c_uint32]
        L.bb_batch_sync.argtypes = [vp]
        L.bb_batch_last_ms.argtypes = [vp, C.POINTER(C.c_float)]
        L.bb_batch_destroy.argtypes = [vp]
        L.bb_batch_destroy.restype = None
        L.bb_booster_sync.argtypes = [vp]
        L.bb_booster_set_weights.argtypes = [vp, vp]
        L.bb_booster_n_trees.argtypes = [vp, C.POINTER(C.c_uint32)]
        L.bb_booster_init_score.argtypes = [vp]
        L.bb_booster_tree_capacity.argtypes = [vp]
        L.bb_booster_tree.argtypes = [vp, C.c_uint32] + [vp] * 9
        L.bb_booster_trees.argtypes = [vp, C.c_uint32, C.c_uint32] + [vp] * 9
        L.bb_booster_scores.argtypes = [vp, vp]
        L.bb_booster_leaf_ids.argtypes = [vp, vp]
        L.bb_booster_last_ms.argtypes = [vp, C.POINTER(C.c_float)]
        L.bb_booster_destroy.argtypes = [vp]
        L.bb_booster_profile_round.argtypes = [vp, C.POINTER(Profile)]
        L.bb_grow_tree.argtypes = [vp, C.POINTER(TrainCfg), vp, vp, vp, C.c_uint64] + [vp] * 11
        L.bb_predict.argtypes = [vp, C.c_uint32, vp, C.c_uint32] + [vp] * 6 + [
            C.c_float, C.c_float, vp]
        L.bb_select_device.argtypes = [C.c_uint32]
        L.bb_predict_static.argtypes = [vp, C.c_uint32, vp, C.c_uint32] + [vp] * 6 + [
            C.c_float, C.c_float, vp]
        L.bb_pred_contribs.argtypes = [vp, C.c_uint32, vp, C.c_uint32] + [vp] * 7 + [
            C.c_float, C.c_float, vp]
        L.bb_booster_n_classes.argtypes = [vp]
        L.bb_booster_n_classes.restype = C.c_uint32
        L.bb_booster_init_scores.argtypes = [vp, vp]
        L.bb_tree_capacity.argtypes = [C.POINTER(TrainCfg)]
        L.bb_tree_capacity.restype = C.c_uint32
        L.bb_comm_unique_id.argtypes = [vp]
        L.bb_comm_create.argtypes = [vp, C.c_uint32, C.c_uint32, C.POINTER(vp)]
        L.bb_comm_group.argtypes = [C.c_uint32, vp]
        L.bb_comm_destroy.argtypes = [vp]
        L.bb_comm_destroy.restype = None
        L.bb_booster_create_sharded.argtypes = [vp, vp, vp, C.POINTER(TrainCfg), C.c_uint32,
                                                vp, C.c_uint64, C.c_uint64, C.c_float,
                                                C.POINTER(vp)]
        L.bb_populate.argtypes = [vp, C.POINTER(TrainCfg), vp, vp, vp, C.c_uint64, vp]
        L.bb_predict_plan_create.argtypes = [vp, C.c_uint32, vp, C.c_uint32] + [vp] * 6 + [
            C.c_float, C.c_float, C.POINTER(vp)]
        L.bb_predict_plan_run.argtypes = [vp, vp, C.c_uint32, vp]
        L.bb_predict_plan_launch.argtypes = [vp, vp, C.c_uint32, vp, vp,
                                             C.POINTER(C.c_uint32)]
        L.bb_predict_plan_depth.argtypes = [vp, C.POINTER(C.c_uint32)]
        L.bb_predict_plan_destroy.argtypes = [vp]
        L.bb_predict_plan_destroy.restype = None
        L.bb_shap_plan_create.argtypes = [vp, C.c_uint32, vp, C.c_uint32] + [vp] * 7 + [
            C.c_float, C.c_float, C.POINTER(vp)]
        L.bb_shap_plan_run.argtypes = [vp, vp, vp]
        L.bb_shap_plan_launch.argtypes = [vp, vp, vp, vp, C.POINTER(C.c_uint32)]
        L.bb_shap_plan_destroy.argtypes = [vp]
        L.bb_shap_plan_destroy.restype = None
        L.bb_booster_eval_arm.argtypes = [vp, vp, vp, vp]
        L.bb_booster_eval_losses.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_uint32)]
        L.bb_booster_eval_scores.argtypes = [vp, vp]
        L.bb_booster_truncate.argtypes = [vp, C.c_uint32]
        L.bb_plane_create_like.argtypes = [vp, C.c_uint64, C.POINTER(vp)]
        L.bb_plane_refill.argtypes = [vp, vp, C.c_uint64, C.c_int]
        L.bb_fit_cuts.argtypes = [vp, C.c_uint64, C.c_uint32, C.c_int, C.c_uint32, vp,
                                  C.c_uint32, vp]
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != BB_OK:
        msg = lib().bb_last_error().decode()
        if rc == BB_ERR_CONFIG:
            raise ConfigError(rc, msg)
        raise BonsaiError(rc, msg)


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data
