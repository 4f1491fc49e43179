"""ctypes declarations of the C ABI's plain types and constants
(include/boosters_c.h): status codes, enums, bst_config, bst_split and the
server statistics. Loads no library, so the CPU checker's bridge can share
these layouts without loading the engine.
"""
import ctypes

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
OBJ_ABSOLUTE, OBJ_PINBALL, OBJ_PSEUDO_HUBER, OBJ_POISSON, OBJ_HINGE = 3, 4, 5, 6, 7
METRIC_DEFAULT, METRIC_NONE, METRIC_RMSE, METRIC_LOGLOSS, METRIC_MLOGLOSS = -1, 0, 1, 2, 3
METRIC_MAE, METRIC_MAPE, METRIC_QUANTILE, METRIC_HUBER, METRIC_POISSON, METRIC_MARGIN_ACCURACY = 4, 5, 6, 7, 8, 9
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
        ("autotune", ctypes.c_int32),
        ("autotune_cache", ctypes.c_char_p),
        ("quantile_alpha", c_f32p),
        ("n_quantiles", ctypes.c_uint32),
        ("huber_delta", ctypes.c_float),
        ("goss_top_rate", ctypes.c_float),
        ("goss_other_rate", ctypes.c_float),
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


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("rows", ctypes.c_uint64), ("max_rows_seen", ctypes.c_uint64), ("max_batch_rows", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("h2d_ns", ctypes.c_uint64)]


SERVER_PHASES = ("rows", "batch_rows", "queue_ns", "copy_ns", "to_dispatch_ns", "kernel_ns", "d2h_ns",
                 "dispatch_to_done_ns")


class ServerPhase(ctypes.Structure):
    """bst_server_phase: one completed request's phases (ns)."""

    _fields_ = [(k, ctypes.c_uint64) for k in SERVER_PHASES]
