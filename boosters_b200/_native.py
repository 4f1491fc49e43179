"""ctypes binding of libboosters_b200.so (declarations in include/boosters_c.h).

The shared library is built in-tree by ``python -m boosters_b200.build``.
Importing this module without it raises ImportError: there is no CPU
fallback for the engine.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libboosters_b200.so")

c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_u16p = ctypes.POINTER(ctypes.c_uint16)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_f64p = ctypes.POINTER(ctypes.c_double)

BST_OK = 0
BST_ERR_INVALID_ARGUMENT = 1
BST_ERR_CONFIG = 2
BST_ERR_EMPTY_DATASET = 3
BST_ERR_MISSING_TARGETS = 4
BST_ERR_UNSUPPORTED = 5
BST_ERR_CUDA = 6
BST_ERR_OUT_OF_MEMORY = 7
BST_ERR_TIMEOUT = 8
BST_ERR_FORMAT = 9

OBJ_SQUARED, OBJ_LOGISTIC, OBJ_SOFTMAX = 0, 1, 2
METRIC_DEFAULT, METRIC_NONE, METRIC_RMSE, METRIC_LOGLOSS, METRIC_MLOGLOSS = -1, 0, 1, 2, 3
GROWTH_DEPTHWISE, GROWTH_LEAFWISE = 0, 1
PRECISION_FP32, PRECISION_Q16, PRECISION_Q8 = 0, 1, 2


class Config(ctypes.Structure):
    """bst_config (include/boosters_c.h)."""

    _fields_ = [
        ("objective", ctypes.c_int32),
        ("n_classes", ctypes.c_uint32),
        ("metric", ctypes.c_int32),
        ("n_trees", ctypes.c_uint32),
        ("learning_rate", ctypes.c_float),
        ("growth_strategy", ctypes.c_int32),
        ("max_depth", ctypes.c_uint32),
        ("max_leaves", ctypes.c_uint32),
        ("max_onehot_cats", ctypes.c_uint32),
        ("lambda_", ctypes.c_float),
        ("alpha", ctypes.c_float),
        ("min_child_weight", ctypes.c_float),
        ("min_gain", ctypes.c_float),
        ("min_samples_leaf", ctypes.c_uint32),
        ("subsample", ctypes.c_float),
        ("colsample_bytree", ctypes.c_float),
        ("colsample_bylevel", ctypes.c_float),
        ("max_bins", ctypes.c_uint32),
        ("sparsity_threshold", ctypes.c_float),
        ("enable_bundling", ctypes.c_int32),
        ("max_categorical_cardinality", ctypes.c_uint32),
        ("binning_sample_cnt", ctypes.c_uint64),
        ("early_stopping_rounds", ctypes.c_int32),
        ("cache_size", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("verbosity", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("batched", ctypes.c_int32),
        ("cuda_graph", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("record_leaves", ctypes.c_int32),
        ("phase_timings", ctypes.c_int32),
    ]


class Split(ctypes.Structure):
    """bst_split (include/boosters_c.h)."""

    _fields_ = [
        ("feature", ctypes.c_uint32),
        ("gain", ctypes.c_float),
        ("default_left", ctypes.c_int32),
        ("is_categorical", ctypes.c_int32),
        ("bin", ctypes.c_uint32),
        ("left_cats", ctypes.c_uint64 * 4),
    ]


# (name, restype, argtypes) of every exported entry point
class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("rows", ctypes.c_uint64), ("max_rows_seen", ctypes.c_uint64), ("max_batch_rows", ctypes.c_uint64)]


SIGNATURES = [
    ("bst_last_error", ctypes.c_char_p, []),
    ("bst_version", ctypes.c_char_p, []),
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
    ("bst_model_from_bytes", ctypes.c_int32, [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("bst_buffer_free", None, [ctypes.c_void_p]),
    ("bst_model_write_json", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]),
    ("bst_model_write_bstr", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p]),
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
]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m boosters_b200.build` "
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
