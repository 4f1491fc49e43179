"""boosters_b200 — B200-native GBDT engine with the API of egordm/boosters.

The Python surface mirrors ``boosters`` (packages/boosters-python:
``Dataset``, ``GBDTConfig``, ``GBDTModel``, ``Objective``, ``Metric``,
``GrowthStrategy``); every call goes through the C ABI of
``libboosters_b200.so`` (include/boosters_c.h), whose hot path runs as
sm_100a CUDA kernels. There is no CPU fallback.
"""
import ctypes
import os
import enum

import numpy as np

from . import _native as _n
from ._native import BoostersError

__all__ = ["Dataset", "GBDTConfig", "GBDTModel", "Objective", "Metric", "GrowthStrategy", "ImportanceType",
           "BoostersError", "BinnedDataset", "synth", "metric"]
__version__ = _n.lib.bst_version().decode()


class ImportanceType(enum.Enum):
    """Feature importance kinds (explainability/importance.rs:43-55)."""

    Split = 0
    Gain = 1
    AverageGain = 2
    Cover = 3
    AverageCover = 4


class GrowthStrategy(enum.Enum):
    """Tree growth policy (training/gbdt/expansion.rs:46-57)."""

    Depthwise = 0
    Leafwise = 1


class Objective:
    """Loss functions (training/objectives/mod.rs:196-219) the engine trains."""

    class Squared:
        code = _n.OBJ_SQUARED
        n_outputs = 1

        def __repr__(self):
            return "Objective.Squared()"

    class Logistic:
        code = _n.OBJ_LOGISTIC
        n_outputs = 1

        def __repr__(self):
            return "Objective.Logistic()"

    class Softmax:
        code = _n.OBJ_SOFTMAX

        def __init__(self, n_classes):
            if int(n_classes) < 2:
                raise ValueError("n_classes must be >= 2")
            self.n_classes = int(n_classes)
            self.n_outputs = self.n_classes

        def __repr__(self):
            return f"Objective.Softmax(n_classes={self.n_classes})"

    class Absolute:
        """L1 loss; leaf values renewed to the leaf's median residual."""
        code = _n.OBJ_ABSOLUTE
        n_outputs = 1

        def __repr__(self):
            return "Objective.Absolute()"

    class Pinball:
        """Quantile regression, one output per alpha; leaf values renewed to
        the alpha-quantile residual."""
        code = _n.OBJ_PINBALL

        def __init__(self, alpha):
            a = [float(v) for v in (alpha if np.ndim(alpha) else [alpha])]
            if not a:
                raise ValueError("alpha must have at least one quantile")
            if any(not (0.0 < v < 1.0) for v in a):
                raise ValueError("alpha values must be in (0, 1)")
            self.alpha = a
            self.n_outputs = len(a)

        def __repr__(self):
            return f"Objective.Pinball(alpha={self.alpha})"

    class Huber:
        """Pseudo-Huber loss with transition point delta."""
        code = _n.OBJ_PSEUDO_HUBER
        n_outputs = 1

        def __init__(self, delta=1.0):
            if not float(delta) > 0.0:
                raise ValueError("delta must be positive")
            self.delta = float(delta)

        def __repr__(self):
            return f"Objective.Huber(delta={self.delta})"

    class Poisson:
        code = _n.OBJ_POISSON
        n_outputs = 1

        def __repr__(self):
            return "Objective.Poisson()"

    class Hinge:
        code = _n.OBJ_HINGE
        n_outputs = 1

        def __repr__(self):
            return "Objective.Hinge()"

    @staticmethod
    def squared():
        return Objective.Squared()

    @staticmethod
    def logistic():
        return Objective.Logistic()

    @staticmethod
    def softmax(n_classes):
        return Objective.Softmax(n_classes)

    @staticmethod
    def absolute():
        return Objective.Absolute()

    @staticmethod
    def pinball(alpha):
        return Objective.Pinball(alpha)

    @staticmethod
    def huber(delta=1.0):
        return Objective.Huber(delta)

    @staticmethod
    def poisson():
        return Objective.Poisson()

    @staticmethod
    def hinge():
        return Objective.Hinge()


class Metric:
    """Evaluation metrics (training/metrics/mod.rs)."""

    class Rmse:
        code = _n.METRIC_RMSE

    class LogLoss:
        code = _n.METRIC_LOGLOSS

    class MultiLogLoss:
        code = _n.METRIC_MLOGLOSS

    class NoMetric:
        code = _n.METRIC_NONE

    class Mae:
        code = _n.METRIC_MAE

    class Mape:
        code = _n.METRIC_MAPE

    class MarginAccuracy:
        code = _n.METRIC_MARGIN_ACCURACY

    class PoissonDeviance:
        code = _n.METRIC_POISSON

    class Quantile:
        code = _n.METRIC_QUANTILE

        def __init__(self, alpha):
            self.alpha = [float(v) for v in (alpha if np.ndim(alpha) else [alpha])]
            if not self.alpha or any(not (0.0 < v < 1.0) for v in self.alpha):
                raise ValueError("alpha values must be in (0, 1)")

    class Huber:
        code = _n.METRIC_HUBER

        def __init__(self, delta=1.0):
            if not float(delta) > 0.0:
                raise ValueError("delta must be positive")
            self.delta = float(delta)

    @staticmethod
    def rmse():
        return Metric.Rmse()

    @staticmethod
    def mae():
        return Metric.Mae()

    @staticmethod
    def mape():
        return Metric.Mape()

    @staticmethod
    def margin_accuracy():
        return Metric.MarginAccuracy()

    @staticmethod
    def poisson_deviance():
        return Metric.PoissonDeviance()

    @staticmethod
    def quantile(alpha):
        return Metric.Quantile(alpha)

    @staticmethod
    def huber(delta=1.0):
        return Metric.Huber(delta)

    @staticmethod
    def logloss():
        return Metric.LogLoss()

    @staticmethod
    def mlogloss():
        return Metric.MultiLogLoss()

    @staticmethod
    def none():
        return Metric.NoMetric()


_PRECISION = {"fp32": _n.PRECISION_FP32, "q16": _n.PRECISION_Q16, "q8": _n.PRECISION_Q8}


class GBDTConfig:
    """GBDT configuration with the reference's names and defaults
    (packages/boosters-python/src/config.rs:160-560, model/gbdt/config.rs:111-226),
    plus GPU options: precision ("fp32", "q16", "q8"), batched (depth-wise
    trees grown by a device-side level loop replayed as one CUDA graph per
    tree; False selects the host-driven loop), cuda_graph, device, autotune
    (time launch-shape candidates on the first trees) and autotune_cache (a
    file keeping the chosen shapes across runs)."""

    def __init__(self, n_estimators=100, learning_rate=0.3, objective=None, metric=None,
                 growth_strategy=GrowthStrategy.Depthwise, max_depth=6, n_leaves=31,
                 max_onehot_cats=4, l1=0.0, l2=1.0, min_gain_to_split=0.0, min_child_weight=1.0,
                 min_samples_leaf=1, subsample=1.0, colsample_bytree=1.0, colsample_bylevel=1.0,
                 max_bins=256, enable_bundling=True, sparsity_threshold=0.9,
                 max_categorical_cardinality=0, binning_sample_cnt=200000, cache_size=8,
                 early_stopping_rounds=None, seed=42, verbosity=0, precision="fp32",
                 cuda_graph=False, device=0, batched=True, phase_timings=False, autotune=True,
                 autotune_cache=None, goss_top_rate=0.0, goss_other_rate=0.0):
        self.n_estimators = n_estimators
        self.learning_rate = learning_rate
        self.objective = objective if objective is not None else Objective.Squared()
        self.metric = metric
        self.growth_strategy = growth_strategy
        self.max_depth = max_depth
        self.n_leaves = n_leaves
        self.max_onehot_cats = max_onehot_cats
        self.l1 = l1
        self.l2 = l2
        self.min_gain_to_split = min_gain_to_split
        self.min_child_weight = min_child_weight
        self.min_samples_leaf = min_samples_leaf
        self.subsample = subsample
        self.colsample_bytree = colsample_bytree
        self.colsample_bylevel = colsample_bylevel
        self.max_bins = max_bins
        self.enable_bundling = enable_bundling
        self.sparsity_threshold = sparsity_threshold
        self.max_categorical_cardinality = max_categorical_cardinality
        self.binning_sample_cnt = binning_sample_cnt
        self.cache_size = cache_size
        self.early_stopping_rounds = early_stopping_rounds
        self.seed = seed
        self.verbosity = verbosity
        self.phase_timings = phase_timings
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        self.precision = precision
        self.cuda_graph = cuda_graph
        self.device = device
        self.batched = batched
        self.autotune = autotune
        self.autotune_cache = None if autotune_cache is None else os.fspath(autotune_cache)
        # GOSS row sampling (training/sampling/row.rs:214-280): top_rate > 0 turns it on
        self.goss_top_rate = goss_top_rate
        self.goss_other_rate = goss_other_rate
        _n.check(_n.lib.bst_config_validate(ctypes.byref(self.to_c())))

    def to_c(self, record_leaves=False):
        c = _n.Config()
        _n.lib.bst_config_default(ctypes.byref(c))
        c.objective = self.objective.code
        c.n_classes = getattr(self.objective, "n_classes", 0)
        c.metric = _n.METRIC_DEFAULT if self.metric is None else self.metric.code
        c.n_trees = int(self.n_estimators)
        c.learning_rate = float(self.learning_rate)
        c.growth_strategy = GrowthStrategy(self.growth_strategy).value
        c.max_depth = int(self.max_depth)
        c.max_leaves = int(self.n_leaves)
        c.max_onehot_cats = int(self.max_onehot_cats)
        c.lambda_ = float(self.l2)
        c.alpha = float(self.l1)
        c.min_child_weight = float(self.min_child_weight)
        c.min_gain = float(self.min_gain_to_split)
        c.min_samples_leaf = int(self.min_samples_leaf)
        c.subsample = float(self.subsample)
        c.colsample_bytree = float(self.colsample_bytree)
        c.colsample_bylevel = float(self.colsample_bylevel)
        c.max_bins = int(self.max_bins)
        c.sparsity_threshold = float(self.sparsity_threshold)
        c.enable_bundling = 1 if self.enable_bundling else 0
        c.max_categorical_cardinality = int(self.max_categorical_cardinality)
        c.binning_sample_cnt = int(self.binning_sample_cnt)
        c.early_stopping_rounds = -1 if self.early_stopping_rounds is None else int(self.early_stopping_rounds)
        c.cache_size = int(self.cache_size)
        c.seed = int(self.seed)
        c.verbosity = int(self.verbosity)
        c.precision = _PRECISION[self.precision]
        c.cuda_graph = 1 if self.cuda_graph else 0
        c.batched = 1 if self.batched else 0
        c.device = int(self.device)
        c.record_leaves = 1 if record_leaves else 0
        c.phase_timings = 1 if self.phase_timings else 0
        c.autotune = 1 if self.autotune else 0
        # the struct keeps the bytes object alive as long as the struct lives
        c.autotune_cache = None if self.autotune_cache is None else os.fsencode(self.autotune_cache)
        # objective / metric parameters (the struct keeps the array alive too)
        alpha = getattr(self.objective, "alpha", None) or getattr(self.metric, "alpha", None)
        if alpha:
            c.quantile_alpha = (ctypes.c_float * len(alpha))(*alpha)
            c.n_quantiles = len(alpha)
        delta = getattr(self.objective, "delta", None) or getattr(self.metric, "delta", None)
        if delta is not None:
            c.huber_delta = float(delta)
        c.goss_top_rate = float(self.goss_top_rate)
        c.goss_other_rate = float(self.goss_other_rate)
        return c

    def __repr__(self):
        return (f"GBDTConfig(n_estimators={self.n_estimators}, learning_rate={self.learning_rate}, "
                f"objective={self.objective!r}, growth_strategy={self.growth_strategy}, "
                f"max_depth={self.max_depth}, n_leaves={self.n_leaves})")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Dataset:
    """Training / prediction data (packages/boosters-python/src/data.rs:252-294).

    ``features`` is sample-major ``(n_samples, n_features)`` like the
    reference's Python Dataset; use :meth:`from_feature_major` to pass the
    core library's feature-major ``[n_features, n_samples]`` layout directly.
    ``labels`` is ``(n_samples,)`` or ``(n_outputs, n_samples)``.
    """

    def __init__(self, features, labels=None, weights=None, feature_names=None,
                 categorical_features=None, _feature_major=False):
        x = np.asarray(features)
        if x.ndim != 2:
            raise ValueError("features must be 2-D")
        xfm = _f32(x if _feature_major else x.T)
        n_features, n_samples = xfm.shape
        y = None
        n_outputs = 0
        if labels is not None:
            y = _f32(labels)
            if y.ndim == 1:
                y = y.reshape(1, -1)
            if y.shape[1] != n_samples:
                raise ValueError("labels must have one value per sample")
            n_outputs = y.shape[0]
        w = None
        if weights is not None:
            w = _f32(weights).reshape(-1)
            if w.shape[0] != n_samples:
                raise ValueError("weights must have one value per sample")
        cats = np.ascontiguousarray(sorted(set(categorical_features or [])), dtype=np.uint32)
        h = ctypes.c_void_p()
        # the engine borrows the feature array (kept alive by this object)
        # instead of copying it
        self._x = xfm
        _n.check(_n.lib.bst_dataset_create_view(
            _n.ptr(xfm, ctypes.c_float), n_features, n_samples, _n.ptr(y, ctypes.c_float), n_outputs,
            _n.ptr(w, ctypes.c_float), _n.ptr(cats, ctypes.c_uint32) if len(cats) else None, len(cats),
            ctypes.byref(h)))
        self._h = h
        self.n_samples = int(n_samples)
        self.n_features = int(n_features)
        self.has_labels = y is not None
        self.has_weights = w is not None
        self.feature_names = list(feature_names) if feature_names is not None else None
        self.categorical_features = [int(c) for c in cats]

    @classmethod
    def from_feature_major(cls, features, labels=None, weights=None, categorical_features=None):
        """Dataset::from_array layout (data/raw/dataset.rs:139): ``[n_features, n_samples]``."""
        return cls(features, labels, weights, None, categorical_features, _feature_major=True)

    @property
    def shape(self):
        return (self.n_samples, self.n_features)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _n is not None and _n.lib is not None:  # not at interpreter exit
            _n.lib.bst_dataset_free(h)
            self._h = None

    def __repr__(self):
        return f"Dataset(n_samples={self.n_samples}, n_features={self.n_features})"


class BinnedDataset:
    """GPU-resident binned dataset (data/binned/dataset.rs:207 from_dataset)."""

    def __init__(self, dataset, config=None):
        cfg = (config or GBDTConfig()).to_c()
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_binned_create(dataset._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.n_samples = dataset.n_samples

    @property
    def n_columns(self):
        return int(_n.lib.bst_binned_n_columns(self._h))

    def column_info(self, col):
        f, nb, dflt = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        cat, miss = ctypes.c_int32(), ctypes.c_int32()
        _n.check(_n.lib.bst_binned_column_info(self._h, col, ctypes.byref(f), ctypes.byref(nb), ctypes.byref(cat),
                                               ctypes.byref(miss), ctypes.byref(dflt)))
        return {"feature": f.value, "n_bins": nb.value, "is_categorical": bool(cat.value),
                "has_missing": bool(miss.value), "default_bin": dflt.value}

    def column_bounds(self, col):
        nb = self.column_info(col)["n_bins"]
        out = np.zeros(nb, dtype=np.float64)
        _n.check(_n.lib.bst_binned_column_bounds(self._h, col, _n.ptr(out, ctypes.c_double)))
        return out

    def column_bins(self, col):
        out = np.zeros(self.n_samples, dtype=np.uint16)
        _n.check(_n.lib.bst_binned_column_bins(self._h, col, _n.ptr(out, ctypes.c_uint16)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _n is not None and _n.lib is not None:  # not at interpreter exit
            _n.lib.bst_binned_free(h)
            self._h = None


class GBDTModel:
    """Gradient-boosted trees (model/gbdt/model.rs:115-258)."""

    def __init__(self, handle, config):
        self._h = handle
        self.config = config

    @staticmethod
    def train(train, config=None, val_set=None, n_threads=0, record_leaves=False):
        """GBDTModel::train. ``n_threads`` keeps the reference's split tie-break
        semantics: 1 = sequential, otherwise the rayon reduction order."""
        config = config or GBDTConfig()
        c = config.to_c(record_leaves=record_leaves)
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_gbdt_train(train._h, val_set._h if val_set is not None else None, ctypes.byref(c),
                                       int(n_threads), ctypes.byref(h)))
        m = GBDTModel(h, config)
        m._rows = train.n_samples
        return m

    # ---- model files (packages/boosters-python/src/model/gbdt.rs:259-330) ----
    def _bytes(self, fn, *args):
        buf, n = ctypes.c_void_p(), ctypes.c_uint64()
        _n.check(fn(self._h, *args, ctypes.byref(buf), ctypes.byref(n)))
        try:
            return ctypes.string_at(buf.value, n.value) if n.value else b""
        finally:
            _n.lib.bst_buffer_free(buf)

    @property
    def tune_info(self):
        """The batched pipeline's launch shape and how it was chosen."""
        buf = ctypes.create_string_buffer(4096)
        n = ctypes.c_uint64()
        _n.check(_n.lib.bst_model_tune_info(self._h, buf, len(buf), ctypes.byref(n)))
        return buf.value.decode()

    def to_bytes(self, compression_level=3):
        """The model as a ``.bstr`` file: zstd-compressed MessagePack at
        ``compression_level`` (1-22; 3 is the reference's default), or plain
        MessagePack with 0 (persist/binary.rs:21-43)."""
        return self._bytes(_n.lib.bst_model_to_bstr_level, int(compression_level))

    def to_json_bytes(self, pretty=False):
        """The model as a ``.bstr.json`` document."""
        return self._bytes(_n.lib.bst_model_to_json, 1 if pretty else 0)

    @staticmethod
    def from_bytes(data, config=None):
        """A model from ``.bstr`` or ``.bstr.json`` bytes."""
        data = bytes(data)
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_model_from_bytes(data, len(data), ctypes.byref(h)))
        return GBDTModel(h, config or GBDTConfig())

    from_json_bytes = from_bytes

    def save(self, path, pretty=False, compression_level=3):
        """Writes ``path``: JSON when it ends in ``.json``, else ``.bstr``
        (zstd at ``compression_level``, 0 for plain MessagePack)."""
        p = os.fsencode(path)
        if p.endswith(b".json"):
            _n.check(_n.lib.bst_model_write_json(self._h, p, 1 if pretty else 0))
        else:
            _n.check(_n.lib.bst_model_write_bstr_level(self._h, p, int(compression_level)))

    @staticmethod
    def load(path, config=None):
        """Reads a ``.bstr`` or ``.bstr.json`` file (Model::load, persist/mod.rs:325)."""
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_model_load(os.fsencode(path), ctypes.byref(h)))
        return GBDTModel(h, config or GBDTConfig())

    def __reduce__(self):
        return (GBDTModel.from_bytes, (self.to_bytes(),))

    @staticmethod
    def grow_tree(dataset, grad, hess, config=None, n_threads=0):
        """TreeGrower::grow on given gradients: a one-tree model."""
        config = config or GBDTConfig()
        c = config.to_c(record_leaves=True)
        g, h = _f32(grad), _f32(hess)
        hd = ctypes.c_void_p()
        _n.check(_n.lib.bst_tree_grow(dataset._h, _n.ptr(g, ctypes.c_float), _n.ptr(h, ctypes.c_float),
                                      ctypes.byref(c), int(n_threads), ctypes.byref(hd)))
        m = GBDTModel(hd, config)
        m._rows = dataset.n_samples
        return m

    @staticmethod
    def from_trees(n_features, trees, objective=None, base_scores=(0.0,)):
        """Model from explicit tree arrays (dicts with the keys of :meth:`tree`)."""
        objective = objective or Objective.Squared()
        b = _f32(base_scores)
        hd = ctypes.c_void_p()
        _n.check(_n.lib.bst_model_create(len(b), n_features, objective.code, _n.ptr(b, ctypes.c_float),
                                         ctypes.byref(hd)))
        m = GBDTModel(hd, None)
        m._rows = 0
        P = _n.ptr
        for t in trees:
            a = {k: np.ascontiguousarray(v) for k, v in t.items() if isinstance(v, (list, tuple, np.ndarray))}
            u32 = lambda k: np.ascontiguousarray(a[k], dtype=np.uint32)
            u8 = lambda k: np.ascontiguousarray(a[k], dtype=np.uint8)
            keep = [u32("split_index"), _f32(a["threshold"]), u32("left"), u32("right"), u8("default_left"),
                    u8("is_leaf"), _f32(a["leaf_value"]),
                    u8("split_type") if "split_type" in a else None,
                    u32("seg_start") if "seg_start" in a else None,
                    u32("seg_size") if "seg_size" in a else None,
                    u32("cat_words") if len(a.get("cat_words", [])) else None]
            nw = 0 if keep[10] is None else len(keep[10])
            _n.check(_n.lib.bst_model_add_tree(
                hd, int(t.get("group", 0)), len(keep[0]), P(keep[0], ctypes.c_uint32), P(keep[1], ctypes.c_float),
                P(keep[2], ctypes.c_uint32), P(keep[3], ctypes.c_uint32), P(keep[4], ctypes.c_uint8),
                P(keep[5], ctypes.c_uint8), P(keep[6], ctypes.c_float), P(keep[7], ctypes.c_uint8),
                P(keep[8], ctypes.c_uint32), P(keep[9], ctypes.c_uint32), P(keep[10], ctypes.c_uint32), nw))
        return m

    @property
    def n_trees(self):
        return int(_n.lib.bst_model_n_trees(self._h))

    @property
    def n_groups(self):
        return int(_n.lib.bst_model_n_groups(self._h))

    @property
    def n_features(self):
        return int(_n.lib.bst_model_n_features(self._h))

    @property
    def is_fitted(self):
        return True

    def _predict(self, data, raw):
        out = np.zeros((self.n_groups, data.n_samples), dtype=np.float32)
        fn = _n.lib.bst_gbdt_predict_raw if raw else _n.lib.bst_gbdt_predict
        _n.check(fn(self._h, data._h, 0, _n.ptr(out, ctypes.c_float)))
        return out

    def predict(self, data, n_threads=0):
        """Transformed predictions, shape ``(n_samples, n_outputs)``."""
        return self._predict(data, False).T.copy()

    def predict_raw(self, data, n_threads=0):
        """Raw margins, shape ``(n_samples, n_outputs)``."""
        return self._predict(data, True).T.copy()

    def predict_group_major(self, data, raw=False):
        """Predictions in the core library's ``[n_groups, n_samples]`` layout."""
        return self._predict(data, raw)

    def base_scores(self):
        out = np.zeros(self.n_groups, dtype=np.float32)
        _n.check(_n.lib.bst_model_base_scores(self._h, _n.ptr(out, ctypes.c_float)))
        return out

    def train_predictions(self):
        """Raw training predictions ``[n_groups, n_samples]`` after the last round."""
        n = self._n_train_rows()
        out = np.zeros((self.n_groups, n), dtype=np.float32)
        _n.check(_n.lib.bst_model_train_predictions(self._h, _n.ptr(out, ctypes.c_float)))
        return out

    def _n_train_rows(self):
        return int(self._rows)

    def tree(self, i):
        """SoA arrays of tree ``i`` (repr/gbdt/tree.rs:32-47) plus training detail."""
        nn, grp, nw = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _n.check(_n.lib.bst_model_tree_info(self._h, i, ctypes.byref(nn), ctypes.byref(grp), ctypes.byref(nw)))
        n = nn.value
        t = {"n_nodes": n, "group": grp.value,
             "split_index": np.zeros(n, np.uint32), "threshold": np.zeros(n, np.float32),
             "left": np.zeros(n, np.uint32), "right": np.zeros(n, np.uint32),
             "default_left": np.zeros(n, np.uint8), "is_leaf": np.zeros(n, np.uint8),
             "leaf_value": np.zeros(n, np.float32), "split_type": np.zeros(n, np.uint8),
             "gain": np.zeros(n, np.float32), "cover": np.zeros(n, np.float32),
             "seg_start": np.zeros(n, np.uint32), "seg_size": np.zeros(n, np.uint32),
             "cat_words": np.zeros(nw.value, np.uint32), "split_bin": np.zeros(n, np.uint32),
             "grad_sum": np.zeros(n, np.float64), "hess_sum": np.zeros(n, np.float64)}
        P = _n.ptr
        _n.check(_n.lib.bst_model_tree_nodes(
            self._h, i, P(t["split_index"], ctypes.c_uint32), P(t["threshold"], ctypes.c_float),
            P(t["left"], ctypes.c_uint32), P(t["right"], ctypes.c_uint32), P(t["default_left"], ctypes.c_uint8),
            P(t["is_leaf"], ctypes.c_uint8), P(t["leaf_value"], ctypes.c_float), P(t["split_type"], ctypes.c_uint8),
            P(t["gain"], ctypes.c_float), P(t["cover"], ctypes.c_float)))
        _n.check(_n.lib.bst_model_tree_categories(self._h, i, P(t["seg_start"], ctypes.c_uint32),
                                                  P(t["seg_size"], ctypes.c_uint32),
                                                  P(t["cat_words"], ctypes.c_uint32) if nw.value else None))
        _n.check(_n.lib.bst_model_tree_train_info(self._h, i, P(t["split_bin"], ctypes.c_uint32),
                                                  P(t["grad_sum"], ctypes.c_double), P(t["hess_sum"], ctypes.c_double)))
        return t

    def feature_importance(self, importance_type=ImportanceType.Split):
        """Per-feature importance (compute_forest_importance,
        explainability/importance.rs:199-270): split counts, gains or covers
        of the split nodes summed in f32 in tree and node order; the Average
        kinds divide by each feature's split count."""
        if self.n_trees == 0:
            raise _n.BoostersError(_n.BST_ERR_INVALID_ARGUMENT, "cannot compute importance of an empty model")
        F = self.n_features
        counts = np.zeros(F, np.uint64)
        values = np.zeros(F, np.float32)
        kind = ImportanceType(importance_type)
        for i in range(self.n_trees):
            t = self.tree(i)
            split = (t["is_leaf"] == 0) & (t["split_index"] < F)
            feats = t["split_index"][split].astype(np.intp)
            np.add.at(counts, feats, 1)
            if kind == ImportanceType.Split:
                np.add.at(values, feats, np.float32(1.0))
            elif kind in (ImportanceType.Gain, ImportanceType.AverageGain):
                np.add.at(values, feats, t["gain"][split])
            else:
                np.add.at(values, feats, t["cover"][split])
        if kind in (ImportanceType.AverageGain, ImportanceType.AverageCover):
            used = counts > 0
            values[used] = values[used] / counts[used].astype(np.float32)
        return values

    def tree_row_leaves(self, i, n_rows):
        out = np.zeros(n_rows, dtype=np.uint32)
        _n.check(_n.lib.bst_model_tree_row_leaves(self._h, i, _n.ptr(out, ctypes.c_uint32)))
        return out

    def train_timings(self):
        """Device milliseconds per phase of the training call."""
        out = np.zeros(8, dtype=np.float64)
        _n.check(_n.lib.bst_model_train_timings(self._h, _n.ptr(out, ctypes.c_double)))
        keys = ["binning", "gradients", "histograms", "split_scan", "partition", "leaf_update", "other", "total"]
        return dict(zip(keys, out.tolist()))

    def train_counters(self):
        out = np.zeros(6, dtype=np.uint64)
        _n.check(_n.lib.bst_model_train_counters(self._h, _n.ptr(out, ctypes.c_uint64), 6))
        keys = ["launches", "hist_launches", "hist_rows", "hist_bytes", "scan_launches", "partition_rows"]
        return dict(zip(keys, (int(v) for v in out)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _n is not None and _n.lib is not None:  # not at interpreter exit
            _n.lib.bst_model_free(h)
            self._h = None

    def __repr__(self):
        return f"GBDTModel(n_trees={self.n_trees}, n_features={self.n_features})"


_TIMING_KEYS = ["binning", "gradients", "histograms", "split_scan", "partition", "leaf_update", "other", "total"]
_COUNTER_KEYS = ["launches", "hist_launches", "hist_rows", "hist_bytes", "scan_launches", "partition_rows"]


class Booster:
    """Incremental training on a GPU-resident binned dataset: the boosting loop
    of GBDTTrainer::train (training/gbdt/trainer.rs:242-401), ``update(k)``
    runs k more rounds."""

    def __init__(self, train, config=None, n_threads=0):
        self.config = config or GBDTConfig()
        c = self.config.to_c()
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_booster_create(train._h, ctypes.byref(c), int(n_threads), ctypes.byref(h)))
        self._h = h
        self._train = train  # the booster reads the dataset's host arrays while it lives
        self._rows = train.n_samples

    def update(self, n_rounds=1):
        _n.check(_n.lib.bst_booster_update(self._h, int(n_rounds)))

    @property
    def n_rounds(self):
        return int(_n.lib.bst_booster_n_rounds(self._h))

    def model(self):
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_booster_model(self._h, ctypes.byref(h)))
        m = GBDTModel(h, self.config)
        m._rows = self._rows
        return m

    def stats(self):
        t = np.zeros(8, np.float64)
        c = np.zeros(6, np.uint64)
        _n.check(_n.lib.bst_booster_stats(self._h, _n.ptr(t, ctypes.c_double), _n.ptr(c, ctypes.c_uint64), 6))
        return dict(zip(_TIMING_KEYS, t.tolist())), dict(zip(_COUNTER_KEYS, (int(v) for v in c)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _n is not None and _n.lib is not None:  # not at interpreter exit
            _n.lib.bst_booster_free(h)
            self._h = None


def release_cached_memory():
    """Frees the device buffers the library keeps for reuse between calls
    (bst_release_cached_memory)."""
    _n.lib.bst_release_cached_memory()


_METRIC_CODES = {"rmse": _n.METRIC_RMSE, "logloss": _n.METRIC_LOGLOSS, "mlogloss": _n.METRIC_MLOGLOSS,
                 "mae": _n.METRIC_MAE, "mape": _n.METRIC_MAPE, "quantile": _n.METRIC_QUANTILE,
                 "huber": _n.METRIC_HUBER, "poisson": _n.METRIC_POISSON,
                 "margin_accuracy": _n.METRIC_MARGIN_ACCURACY}


def metric(kind, preds_group_major, labels, weights=None, alpha=None, delta=1.0):
    """Metric value (training/metrics) of transformed predictions (raw
    margins for 'margin_accuracy'): kind in {'rmse', 'logloss', 'mlogloss',
    'mae', 'mape', 'quantile' (alpha: one per output), 'huber' (delta),
    'poisson', 'margin_accuracy'}."""
    p = _f32(preds_group_major)
    if p.ndim == 1:
        p = p.reshape(1, -1)
    y = _f32(labels).reshape(-1)
    w = None if weights is None else _f32(weights).reshape(-1)
    a = None if alpha is None else _f32(np.atleast_1d(alpha))
    out = ctypes.c_double()
    _n.check(_n.lib.bst_metric_ex(_METRIC_CODES[kind], _n.ptr(p, ctypes.c_float), p.shape[0], p.shape[1],
                                  _n.ptr(y, ctypes.c_float), _n.ptr(w, ctypes.c_float), _n.ptr(a, ctypes.c_float),
                                  0 if a is None else a.size, float(delta), ctypes.byref(out)))
    return out.value


class Ticket:
    """A queued prediction request of :class:`PredictionServer`."""

    __slots__ = ("id", "rows", "out", "submit_ns", "done_ns")

    def __init__(self, tid, rows, out):
        self.id = tid
        self.rows = rows  # kept alive until the request completes
        self.out = out
        self.submit_ns = 0
        self.done_ns = 0


class PredictionServer:
    """Continuous-batching prediction over a device-resident forest.

    Requests queue FIFO; a dispatcher coalesces waiting requests into one
    traversal launch per batch (bounded by ``mem_budget_bytes`` over three
    in-flight batches) while earlier batches run. ``submit`` returns at once;
    ``wait`` returns the ``(n_groups, n_rows)`` predictions. Row buffers from
    pinned memory (e.g. ``torch.empty(..., pin_memory=True).numpy()``) give
    asynchronous host-device copies. The model must stay alive.
    """

    def __init__(self, model, mem_budget_bytes=1 << 30, max_batch_rows=0, raw=False):
        self.model = model
        self.n_features = model.n_features
        self.n_groups = model.n_groups
        h = ctypes.c_void_p()
        _n.check(_n.lib.bst_server_create(model._h, int(mem_budget_bytes), int(max_batch_rows), 1 if raw else 0,
                                          ctypes.byref(h)))
        self._h = h

    @staticmethod
    def _buffer(a, shape, what):
        """(pointer, keep-alive) of a C-contiguous float32 array: numpy (host)
        or a CUDA tensor (device; the server copies by unified addressing)."""
        if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
            import torch
            if a.dtype != torch.float32 or not a.is_contiguous() or tuple(a.shape) != tuple(shape):
                raise ValueError(f"{what} must be a contiguous float32 tensor of shape {tuple(shape)}")
            return a.data_ptr(), a
        if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous \
                or a.shape != tuple(shape):
            raise ValueError(f"{what} must be a C-contiguous float32 array of shape {tuple(shape)}")
        return a.ctypes.data, a

    def submit(self, rows, out=None):
        """Queue sample-major rows ``(n, n_features)`` float32 (C order): a
        numpy array (pinned memory copies asynchronously) or a CUDA tensor on
        the model's GPU. ``out``: ``(n_groups, n)`` float32, numpy or CUDA."""
        if not (hasattr(rows, "data_ptr") and getattr(rows, "is_cuda", False)):
            rows = np.asarray(rows)
            if rows.dtype != np.float32 or not rows.flags.c_contiguous:
                rows = np.ascontiguousarray(rows, dtype=np.float32)
        if len(rows.shape) != 2 or rows.shape[1] != self.n_features:
            raise ValueError(f"rows must have shape (n, {self.n_features})")
        n = rows.shape[0]
        rp, rows = self._buffer(rows, (n, self.n_features), "rows")
        if out is None:
            out = np.empty((self.n_groups, n), dtype=np.float32)
        op, out = self._buffer(out, (self.n_groups, n), "out")
        t = ctypes.c_uint64()
        _n.check(_n.lib.bst_server_submit(self._h, ctypes.c_void_p(rp), n, ctypes.c_void_p(op), ctypes.byref(t)))
        return Ticket(t.value, rows, out)

    def wait(self, ticket, timeout_ms=-1):
        """Predictions ``(n_groups, n_rows)`` of a ticket; raises on timeout."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        _n.check(_n.lib.bst_server_wait(self._h, ticket.id, int(timeout_ms), ctypes.byref(a), ctypes.byref(b)))
        ticket.submit_ns, ticket.done_ns = a.value, b.value
        return ticket.out

    def replay(self, pool, arrival_s, row_off, n_rows, ring=256):
        """Replays a request schedule from a native thread: request ``i`` is
        rows ``pool[row_off[i]:row_off[i] + n_rows[i]]`` (pool: numpy, or a
        CUDA tensor for device-resident requests) arriving ``arrival_s[i]``
        seconds after the start. Returns ``(latency_s, span_s, out)``: each
        request's completion minus its scheduled arrival, the span from the
        first arrival to the last completion, and the output ring
        ``(ring, n_groups, max_rows)`` (request ``i`` in slot ``i % ring``)."""
        if not (hasattr(pool, "data_ptr") and getattr(pool, "is_cuda", False)):
            pool = np.asarray(pool)
        if len(pool.shape) != 2 or pool.shape[1] != self.n_features:
            raise ValueError(f"pool must have shape (rows, {self.n_features})")
        pp, pool = self._buffer(pool, tuple(pool.shape), "pool")
        arr = np.ascontiguousarray(np.round(np.asarray(arrival_s, np.float64) * 1e9), dtype=np.uint64)
        off = np.ascontiguousarray(row_off, dtype=np.uint64)
        cnt = np.ascontiguousarray(n_rows, dtype=np.uint64)
        n_req = len(arr)
        if len(off) != n_req or len(cnt) != n_req:
            raise ValueError("arrival_s, row_off and n_rows must have the same length")
        width = int(cnt.max()) if n_req else 1
        try:
            import torch
            out = torch.empty((ring, self.n_groups, width), dtype=torch.float32).pin_memory().numpy()
        except Exception:
            out = np.empty((ring, self.n_groups, width), dtype=np.float32)
        lat = np.zeros(n_req, np.uint64)
        span = ctypes.c_uint64()
        _n.check(_n.lib.bst_server_replay(self._h, ctypes.c_void_p(pp), pool.shape[0], n_req,
                                          ctypes.c_void_p(arr.ctypes.data), ctypes.c_void_p(off.ctypes.data),
                                          ctypes.c_void_p(cnt.ctypes.data), ctypes.c_void_p(out.ctypes.data),
                                          ring, self.n_groups * width, ctypes.c_void_p(lat.ctypes.data),
                                          ctypes.byref(span)))
        return lat.astype(np.float64) / 1e9, span.value / 1e9, out

    def stats(self):
        st = _n.ServerStats()
        _n.check(_n.lib.bst_server_stats_get(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _n.ServerStats._fields_}

    def trace(self, max_records=1 << 20):
        """Phase records of the requests completed since the last call, as a
        ``(k, 8)`` uint64 array with columns ``_n.SERVER_PHASES`` (ns)."""
        out = np.zeros((int(max_records), len(_n.SERVER_PHASES)), np.uint64)
        got = ctypes.c_uint64()
        _n.check(_n.lib.bst_server_trace(self._h, ctypes.c_void_p(out.ctypes.data), int(max_records),
                                         ctypes.byref(got)))
        return out[: got.value]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _n.lib.bst_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class synth:
    """Seeded synthetic workloads; every array is feature-major ``[F, n]``."""

    @staticmethod
    def regression(n, n_features, n_informative=20, seed=1, stream=0):
        x = np.empty((n_features, n), dtype=np.float32)
        y = np.empty(n, dtype=np.float32)
        _n.check(_n.lib.bst_synth_regression(n, n_features, n_informative, seed, stream,
                                             _n.ptr(x, ctypes.c_float), _n.ptr(y, ctypes.c_float)))
        return x, y

    @staticmethod
    def binary(n, n_features, n_nan_cols=20, seed=2, stream=0):
        x = np.empty((n_features, n), dtype=np.float32)
        y = np.empty(n, dtype=np.float32)
        _n.check(_n.lib.bst_synth_binary(n, n_features, n_nan_cols, seed, stream,
                                         _n.ptr(x, ctypes.c_float), _n.ptr(y, ctypes.c_float)))
        return x, y

    @staticmethod
    def multiclass(n, n_numeric=40, n_categorical=10, n_classes=10, seed=4, stream=0):
        x = np.empty((n_numeric + n_categorical, n), dtype=np.float32)
        y = np.empty(n, dtype=np.float32)
        _n.check(_n.lib.bst_synth_multiclass(n, n_numeric, n_categorical, n_classes, seed, stream,
                                             _n.ptr(x, ctypes.c_float), _n.ptr(y, ctypes.c_float)))
        return x, y
