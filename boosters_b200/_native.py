"""ctypes binding of libboosters_b200.so (declarations in include/boosters_c.h).

The shared library is built in-tree by ``python -m boosters_b200.build``.
Importing this module without it raises ImportError: there is no CPU
fallback for the engine.
"""
import ctypes
import os

from ._abi import *  # noqa: F401,F403  (types and constants of the C ABI)
from ._abi import (BST_ERR_CONFIG, BST_OK, Config, ServerStats, Split, c_f32p, c_f64p, c_i32p, c_u8p, c_u16p,
                   c_u32p, c_u64p)

_HERE = os.path.dirname(os.path.abspath(__file__))
# BST_LIBRARY=checked loads the bounds-checked build (libboosters_b200_checked.so)
_VARIANT = os.environ.get("BST_LIBRARY", "")
if _VARIANT not in ("", "checked"):
    raise ImportError(f"BST_LIBRARY={_VARIANT!r}: expected unset or 'checked'")
LIB_PATH = os.path.join(_HERE, "libboosters_b200_checked.so" if _VARIANT == "checked" else "libboosters_b200.so")

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("bst_last_error", ctypes.c_char_p, []),
    ("bst_version", ctypes.c_char_p, []),
    ("bst_release_cached_memory", None, []),
    ("bst_config_default", None, [ctypes.POINTER(Config)]),
    ("bst_config_validate", ctypes.c_int32, [ctypes.POINTER(Config)]),
    ("bst_dataset_create", ctypes.c_int32,
     [c_f32p, ctypes.c_uint64, ctypes.c_uint64, c_f32p, ctypes.c_uint32, c_f32p, c_u32p,
      ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_dataset_create_view", ctypes.c_int32,
     [c_f32p, ctypes.c_uint64, ctypes.c_uint64, c_f32p, ctypes.c_uint32, c_f32p, c_u32p,
      ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_dataset_free", None, [ctypes.c_void_p]),
    ("bst_dataset_n_samples", ctypes.c_uint64, [ctypes.c_void_p]),
    ("bst_dataset_n_features", ctypes.c_uint64, [ctypes.c_void_p]),
    ("bst_binned_create", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_binned_free", None, [ctypes.c_void_p]),
    ("bst_binned_n_columns", ctypes.c_uint32, [ctypes.c_void_p]),
    ("bst_binned_column_info", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, c_u32p, c_u32p, c_i32p, c_i32p, c_u32p]),
    ("bst_binned_column_bounds", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, c_f64p]),
    ("bst_binned_column_bins", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, c_u16p]),
    ("bst_gbdt_train", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Config), ctypes.c_uint32,
      ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_gbdt_predict", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, c_f32p]),
    ("bst_gbdt_predict_raw", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, c_f32p]),
    ("bst_gbdt_predict_device", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32,
      ctypes.c_void_p, ctypes.c_void_p]),
    ("bst_model_free", None, [ctypes.c_void_p]),
    ("bst_model_to_json", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_model_to_bstr", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_model_to_bstr_level", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
                                                 ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_model_from_bytes", ctypes.c_int32, [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_buffer_free", None, [ctypes.c_void_p]),
    ("bst_model_write_json", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]),
    ("bst_model_write_bstr", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p]),
    ("bst_model_write_bstr_level", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]),
    ("bst_model_load", ctypes.c_int32, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_crc32c", ctypes.c_uint32, [ctypes.c_char_p, ctypes.c_uint64]),
    ("bst_model_n_trees", ctypes.c_uint32, [ctypes.c_void_p]),
    ("bst_model_n_groups", ctypes.c_uint32, [ctypes.c_void_p]),
    ("bst_model_n_features", ctypes.c_uint32, [ctypes.c_void_p]),
    ("bst_model_base_scores", ctypes.c_int32, [ctypes.c_void_p, c_f32p]),
    ("bst_model_train_predictions", ctypes.c_int32, [ctypes.c_void_p, c_f32p]),
    ("bst_model_tree_info", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, c_u32p, c_u32p, c_u32p]),
    ("bst_model_tree_nodes", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, c_u32p, c_f32p, c_u32p, c_u32p, c_u8p, c_u8p, c_f32p, c_u8p,
      c_f32p, c_f32p]),
    ("bst_model_tree_categories", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, c_u32p, c_u32p, c_u32p]),
    ("bst_model_tree_train_info", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, c_u32p, c_f64p, c_f64p]),
    ("bst_model_tree_row_leaves", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, c_u32p]),
    ("bst_model_train_timings", ctypes.c_int32, [ctypes.c_void_p, c_f64p]),
    ("bst_model_train_counters", ctypes.c_int32, [ctypes.c_void_p, c_u64p, ctypes.c_uint32]),
    ("bst_model_tune_info", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_booster_create", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.POINTER(Config), ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_booster_update", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    ("bst_booster_n_rounds", ctypes.c_uint32, [ctypes.c_void_p]),
    ("bst_booster_model", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_booster_stats", ctypes.c_int32, [ctypes.c_void_p, c_f64p, c_u64p, ctypes.c_uint32]),
    ("bst_booster_free", None, [ctypes.c_void_p]),
    ("bst_tree_grow", ctypes.c_int32,
     [ctypes.c_void_p, c_f32p, c_f32p, ctypes.POINTER(Config), ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_model_create", ctypes.c_int32,
     [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, c_f32p, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_model_add_tree", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, c_u32p, c_f32p, c_u32p, c_u32p, c_u8p, c_u8p, c_f32p,
      c_u8p, c_u32p, c_u32p, c_u32p, ctypes.c_uint32]),
    ("bst_bin_values", ctypes.c_int32,
     [c_f64p, ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint32, ctypes.c_int32, c_i32p, ctypes.c_uint32,
      c_f32p, ctypes.c_uint64, c_u32p]),
    ("bst_histogram_build", ctypes.c_int32,
     [c_u16p, c_u32p, ctypes.c_uint32, ctypes.c_uint64, c_f32p, c_f32p, c_u32p, ctypes.c_uint64, c_f64p]),
    ("bst_find_split", ctypes.c_int32,
     [c_f64p, c_u32p, c_i32p, c_i32p, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_uint32,
      ctypes.POINTER(Config), ctypes.c_uint32, ctypes.POINTER(Split)]),
    ("bst_find_split_noalloc", ctypes.c_int32,
     [ctypes.c_void_p, c_u32p, c_i32p, c_i32p, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
      ctypes.c_uint32, ctypes.POINTER(Config), ctypes.c_uint32, ctypes.c_void_p, ctypes.POINTER(Split)]),
    ("bst_quantize_gradients", ctypes.c_int32,
     [c_f32p, c_f32p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
      c_i32p, c_i32p, c_f64p]),
    ("bst_server_create", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_server_submit", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_server_wait", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64),
      ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_server_stats_get", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    ("bst_server_trace", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_server_replay", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]),
    ("bst_server_free", None, [ctypes.c_void_p]),
    ("bst_synth_regression", ctypes.c_int32,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, c_f32p, c_f32p]),
    ("bst_synth_binary", ctypes.c_int32,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, c_f32p, c_f32p]),
    ("bst_synth_multiclass", ctypes.c_int32,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
      c_f32p, c_f32p]),
    ("bst_metric", ctypes.c_int32,
     [ctypes.c_int32, c_f32p, ctypes.c_uint32, ctypes.c_uint64, c_f32p, c_f32p, c_f64p]),
    ("bst_check_report", ctypes.c_int32,
     [ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32),
      ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("bst_metric_ex", ctypes.c_int32,
     [ctypes.c_int32, c_f32p, ctypes.c_uint32, ctypes.c_uint64, c_f32p, c_f32p, c_f32p, ctypes.c_uint32,
      ctypes.c_float, c_f64p]),
]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m boosters_b200.build`"
            f"{' --checked' if _VARIANT else ''} "
            "(the GBDT engine has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class BoostersError(RuntimeError):
    """Error raised by the native engine (status code + message)."""

    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


def check(status):
    """Raise for a non-OK status with the engine's thread-local message."""
    if status != BST_OK:
        msg = lib.bst_last_error().decode("utf-8", "replace")
        if status == BST_ERR_CONFIG:
            raise ValueError(msg)
        raise BoostersError(status, msg)


def ptr(arr, ctype):
    """Pointer to a C-contiguous numpy array (or None)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(ctypes.POINTER(ctype))
