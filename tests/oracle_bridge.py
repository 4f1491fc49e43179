"""ctypes bridge to the CPU restatement in oracle/ (the checker).

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs
use this module; the engine never does. It loads no engine library: the
plain C types come from ``boosters_b200/_abi.py`` (read by path when the
engine package is not imported), so a process that only times the checker
maps liboracle.so alone. ``BST_ORACLE_LIB`` selects another build of the
same source (bench.py's host-tuned build).
"""
import ctypes
import importlib.util
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.environ.get("BST_ORACLE_LIB") or os.path.join(ORACLE_DIR, "liboracle.so")


def _abi_module():
    if "boosters_b200._abi" in sys.modules:
        return sys.modules["boosters_b200._abi"]
    spec = importlib.util.spec_from_file_location("_bst_abi_for_oracle", os.path.join(ROOT, "boosters_b200", "_abi.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_abi = _abi_module()
Config, Split = _abi.Config, _abi.Split

f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)
u32p = ctypes.POINTER(ctypes.c_uint32)
u16p = ctypes.POINTER(ctypes.c_uint16)
u8p = ctypes.POINTER(ctypes.c_uint8)
i32p = ctypes.POINTER(ctypes.c_int32)
vp = ctypes.c_void_p
u64 = ctypes.c_uint64
u32 = ctypes.c_uint32

_SIGS = [
    ("orc_last_error", ctypes.c_char_p, []),
    ("orc_bin", ctypes.c_int, [f32p, u64, u64, u32p, u32, vp, ctypes.POINTER(vp)]),
    ("orc_binned_free", None, [vp]),
    ("orc_binned_n_columns", u32, [vp]),
    ("orc_binned_column_info", None, [vp, u32, u32p, u32p, i32p, i32p, u32p]),
    ("orc_binned_column_bounds", None, [vp, u32, f64p]),
    ("orc_binned_column_bins", None, [vp, u32, u16p]),
    ("orc_value_to_bin", u32, [f64p, u32, ctypes.c_int32, u32, ctypes.c_int32, i32p, u32, ctypes.c_double]),
    ("orc_gain_full", ctypes.c_double, [ctypes.c_double] * 6 + [ctypes.c_float, ctypes.c_float]),
    ("orc_leaf_weight", ctypes.c_float, [ctypes.c_double, ctypes.c_double, ctypes.c_float, ctypes.c_float]),
    ("orc_is_valid_split", ctypes.c_int,
     [ctypes.c_double, ctypes.c_double, u32, u32, ctypes.c_float, u32]),
    ("orc_histogram_build", None, [u16p, u32p, u32, u64, f32p, f32p, u32p, u64, f64p]),
    ("orc_find_split", None,
     [f64p, u32p, i32p, i32p, u32, ctypes.c_double, ctypes.c_double, u32, vp, u32,
      vp]),
    ("orc_gradients", None, [ctypes.c_int32, u32, f32p, f32p, f32p, u64, f32p, f32p]),
    ("orc_base_score", None, [ctypes.c_int32, u32, f32p, f32p, u64, f32p]),
    ("orc_transform", None, [ctypes.c_int32, f32p, u32, u64]),
    ("orc_metric", ctypes.c_double, [ctypes.c_int32, f32p, u32, u64, f32p, f32p]),
    ("orc_gradients_cfg", None, [vp, u32, f32p, f32p, f32p, u64, f32p, f32p]),
    ("orc_base_score_cfg", None, [vp, u32, f32p, f32p, u64, f32p]),
    ("orc_metric_cfg", ctypes.c_double, [ctypes.c_int32, vp, f32p, u32, u64, f32p, f32p]),
    ("orc_goss", u64, [f32p, f32p, u64, ctypes.c_float, ctypes.c_float, u64, u32, u8p]),
    ("orc_leaf_quantile", ctypes.c_float, [f32p, f32p, u64, ctypes.c_float]),
    ("orc_train_limited", ctypes.c_int,
     [f32p, u64, u64, f32p, u32, f32p, u32p, u32, vp, u32, ctypes.c_int, ctypes.c_int, u32,
      ctypes.POINTER(vp)]),
    ("orc_model_free", None, [vp]),
    ("orc_model_n_trees", u32, [vp]),
    ("orc_model_n_groups", u32, [vp]),
    ("orc_model_base_scores", None, [vp, f32p]),
    ("orc_model_train_predictions", None, [vp, f32p]),
    ("orc_tree_info", None, [vp, u32, u32p, u32p, u32p]),
    ("orc_tree_nodes", None, [vp, u32, u32p, f32p, u32p, u32p, u8p, u8p, f32p, u8p, f32p, f32p]),
    ("orc_tree_categories", None, [vp, u32, u32p, u32p, u32p]),
    ("orc_tree_train_info", None, [vp, u32, u32p, f64p, f64p]),
    ("orc_tree_row_leaves", None, [vp, u32, u32p]),
    ("orc_model_train_seconds", ctypes.c_double, [vp]),
    ("orc_model_binning_seconds", ctypes.c_double, [vp]),
    ("orc_model_tree_seconds", ctypes.c_double, [vp, u32]),
    ("orc_predict", ctypes.c_int, [vp, f32p, u64, u64, ctypes.c_int, f32p]),
    ("orc_grow_tree", ctypes.c_int, [f32p, u64, u64, f32p, f32p, vp, u32, ctypes.POINTER(vp)]),
    ("orc_model_create", ctypes.c_int, [u32, u32, ctypes.c_int32, f32p, ctypes.POINTER(vp)]),
    ("orc_model_add_tree", ctypes.c_int,
     [vp, u32, u32, u32p, f32p, u32p, u32p, u8p, u8p, f32p, u8p, u32p, u32p, u32p, u32]),
    ("orc_predict_rows", ctypes.c_int, [vp, f32p, u64, u64, ctypes.c_int, ctypes.c_int, f32p]),
    ("orc_philox4x32_10", None, [u32p, u32p, u32p]),
    ("orc_config_default", None, [vp]),
    ("orc_synth_regression", ctypes.c_int, [u64, u64, u64, u64, u64, f32p, f32p]),
    ("orc_synth_binary", ctypes.c_int, [u64, u64, u64, u64, u64, f32p, f32p]),
    ("orc_synth_multiclass", ctypes.c_int, [u64, u64, u64, u64, u64, u64, f32p, f32p]),
    ("orc_quantize", None, [f32p, f32p, u64, ctypes.c_int32, u64, u32, u32, i32p, i32p, f64p]),
]


def build_oracle():
    """Compile oracle/liboracle.so with its Makefile (g++)."""
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_LIB


def _load():
    if not os.path.exists(ORACLE_LIB) and "BST_ORACLE_LIB" not in os.environ:
        build_oracle()
    lib = ctypes.CDLL(ORACLE_LIB)
    for name, res, args in _SIGS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def P(a, t):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {lib.orc_last_error().decode()}")


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class OracleBinned:
    def __init__(self, x_fm, cfg, categorical=()):
        x = f32(x_fm)
        cats = np.ascontiguousarray(sorted(categorical), dtype=np.uint32)
        h = vp()
        _check(lib.orc_bin(P(x, ctypes.c_float), x.shape[0], x.shape[1], P(cats, ctypes.c_uint32) if len(cats) else None,
                           len(cats), ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.n = x.shape[1]

    @property
    def n_columns(self):
        return lib.orc_binned_n_columns(self._h)

    def column_info(self, col):
        f, nb, d = u32(), u32(), u32()
        c, m = ctypes.c_int32(), ctypes.c_int32()
        lib.orc_binned_column_info(self._h, col, ctypes.byref(f), ctypes.byref(nb), ctypes.byref(c), ctypes.byref(m),
                                   ctypes.byref(d))
        return {"feature": f.value, "n_bins": nb.value, "is_categorical": bool(c.value),
                "has_missing": bool(m.value), "default_bin": d.value}

    def column_bounds(self, col):
        out = np.zeros(self.column_info(col)["n_bins"], np.float64)
        lib.orc_binned_column_bounds(self._h, col, P(out, ctypes.c_double))
        return out

    def column_bins(self, col):
        out = np.zeros(self.n, np.uint16)
        lib.orc_binned_column_bins(self._h, col, P(out, ctypes.c_uint16))
        return out

    def __del__(self):
        if getattr(self, "_h", None) is not None:
            lib.orc_binned_free(self._h)
            self._h = None


class OracleModel:
    @classmethod
    def grow(cls, x_fm, grad, hess, cfg, n_threads=1):
        """TreeGrower::grow on given gradients -> one-tree model."""
        x = f32(x_fm)
        g, h = f32(grad), f32(hess)
        self = cls.__new__(cls)
        hd = vp()
        _check(lib.orc_grow_tree(P(x, ctypes.c_float), x.shape[0], x.shape[1], P(g, ctypes.c_float),
                                 P(h, ctypes.c_float), ctypes.byref(cfg), n_threads, ctypes.byref(hd)))
        self._h = hd
        self.n = x.shape[1]
        self.n_features = x.shape[0]
        return self

    @classmethod
    def from_trees(cls, n_features, trees, objective=0, base=(0.0,), n_groups=1):
        """Model from explicit tree arrays (dicts with the tree() keys)."""
        self = cls.__new__(cls)
        b = f32(base)
        hd = vp()
        _check(lib.orc_model_create(n_groups, n_features, objective, P(b, ctypes.c_float), ctypes.byref(hd)))
        self._h = hd
        self.n = 0
        self.n_features = n_features
        for t in trees:
            a = {k: np.ascontiguousarray(v) for k, v in t.items() if isinstance(v, (list, np.ndarray))}
            nw = len(a.get("cat_words", []))
            _check(lib.orc_model_add_tree(
                hd, t.get("group", 0), len(a["split_index"]), P(a["split_index"].astype(np.uint32), ctypes.c_uint32),
                P(a["threshold"].astype(np.float32), ctypes.c_float), P(a["left"].astype(np.uint32), ctypes.c_uint32),
                P(a["right"].astype(np.uint32), ctypes.c_uint32), P(a["default_left"].astype(np.uint8), ctypes.c_uint8),
                P(a["is_leaf"].astype(np.uint8), ctypes.c_uint8), P(a["leaf_value"].astype(np.float32), ctypes.c_float),
                P(a["split_type"].astype(np.uint8), ctypes.c_uint8) if "split_type" in a else None,
                P(a["seg_start"].astype(np.uint32), ctypes.c_uint32) if "seg_start" in a else None,
                P(a["seg_size"].astype(np.uint32), ctypes.c_uint32) if "seg_size" in a else None,
                P(a["cat_words"].astype(np.uint32), ctypes.c_uint32) if nw else None, nw))
        return self

    def __init__(self, x_fm, y, cfg, n_threads=1, weights=None, categorical=(), record_leaves=True,
                 omp_threads=1, max_trees=0xFFFFFFFF):
        x = f32(x_fm)
        y = f32(y).reshape(-1)
        w = None if weights is None else f32(weights)
        cats = np.ascontiguousarray(sorted(categorical), dtype=np.uint32)
        h = vp()
        _check(lib.orc_train_limited(P(x, ctypes.c_float), x.shape[0], x.shape[1], P(y, ctypes.c_float), 1,
                                     P(w, ctypes.c_float), P(cats, ctypes.c_uint32) if len(cats) else None, len(cats),
                                     ctypes.byref(cfg), n_threads, 1 if record_leaves else 0, omp_threads,
                                     max_trees, ctypes.byref(h)))
        self._h = h
        self.n = x.shape[1]
        self.n_features = x.shape[0]

    @property
    def n_trees(self):
        return lib.orc_model_n_trees(self._h)

    @property
    def n_groups(self):
        return lib.orc_model_n_groups(self._h)

    def base_scores(self):
        out = np.zeros(self.n_groups, np.float32)
        lib.orc_model_base_scores(self._h, P(out, ctypes.c_float))
        return out

    def train_predictions(self):
        out = np.zeros((self.n_groups, self.n), np.float32)
        lib.orc_model_train_predictions(self._h, P(out, ctypes.c_float))
        return out

    def tree(self, i):
        nn, g, nw = u32(), u32(), u32()
        lib.orc_tree_info(self._h, i, ctypes.byref(nn), ctypes.byref(g), ctypes.byref(nw))
        n = nn.value
        t = {"n_nodes": n, "group": g.value,
             "split_index": np.zeros(n, np.uint32), "threshold": np.zeros(n, np.float32),
             "left": np.zeros(n, np.uint32), "right": np.zeros(n, np.uint32),
             "default_left": np.zeros(n, np.uint8), "is_leaf": np.zeros(n, np.uint8),
             "leaf_value": np.zeros(n, np.float32), "split_type": np.zeros(n, np.uint8),
             "gain": np.zeros(n, np.float32), "cover": np.zeros(n, np.float32),
             "seg_start": np.zeros(n, np.uint32), "seg_size": np.zeros(n, np.uint32),
             "cat_words": np.zeros(nw.value, np.uint32), "split_bin": np.zeros(n, np.uint32),
             "grad_sum": np.zeros(n, np.float64), "hess_sum": np.zeros(n, np.float64)}
        lib.orc_tree_nodes(self._h, i, P(t["split_index"], ctypes.c_uint32), P(t["threshold"], ctypes.c_float),
                           P(t["left"], ctypes.c_uint32), P(t["right"], ctypes.c_uint32),
                           P(t["default_left"], ctypes.c_uint8), P(t["is_leaf"], ctypes.c_uint8),
                           P(t["leaf_value"], ctypes.c_float), P(t["split_type"], ctypes.c_uint8),
                           P(t["gain"], ctypes.c_float), P(t["cover"], ctypes.c_float))
        lib.orc_tree_categories(self._h, i, P(t["seg_start"], ctypes.c_uint32), P(t["seg_size"], ctypes.c_uint32),
                                P(t["cat_words"], ctypes.c_uint32) if nw.value else None)
        lib.orc_tree_train_info(self._h, i, P(t["split_bin"], ctypes.c_uint32), P(t["grad_sum"], ctypes.c_double),
                                P(t["hess_sum"], ctypes.c_double))
        return t

    def row_leaves(self, i):
        out = np.zeros(self.n, np.uint32)
        lib.orc_tree_row_leaves(self._h, i, P(out, ctypes.c_uint32))
        return out

    def predict(self, x_fm, raw=False):
        x = f32(x_fm)
        out = np.zeros((self.n_groups, x.shape[1]), np.float32)
        _check(lib.orc_predict(self._h, P(x, ctypes.c_float), x.shape[0], x.shape[1], 1 if raw else 0,
                               P(out, ctypes.c_float)))
        return out

    def predict_rows(self, x_sm, raw=False, omp_threads=1):
        x = f32(x_sm)
        out = np.zeros((self.n_groups, x.shape[0]), np.float32)
        _check(lib.orc_predict_rows(self._h, P(x, ctypes.c_float), x.shape[1], x.shape[0], 1 if raw else 0,
                                    omp_threads, P(out, ctypes.c_float)))
        return out

    @property
    def train_seconds(self):
        return lib.orc_model_train_seconds(self._h)

    def __del__(self):
        if getattr(self, "_h", None) is not None:
            lib.orc_model_free(self._h)
            self._h = None


def value_to_bin(bounds, missing, default_bin, value, cats=None):
    b = np.ascontiguousarray(bounds if bounds is not None else [], dtype=np.float64)
    c = None if cats is None else np.ascontiguousarray(cats, dtype=np.int32)
    return lib.orc_value_to_bin(P(b, ctypes.c_double) if len(b) else None, len(b), missing, default_bin,
                                1 if c is not None else 0, P(c, ctypes.c_int32), 0 if c is None else len(c),
                                float(value))


def histogram_build(bins_fm, n_bins, grad, hess, rows=None):
    bins = np.ascontiguousarray(bins_fm, dtype=np.uint16)
    nb = np.ascontiguousarray(n_bins, dtype=np.uint32)
    g, h = f32(grad), f32(hess)
    r = None if rows is None else np.ascontiguousarray(rows, dtype=np.uint32)
    out = np.zeros((int(nb.sum()), 2), np.float64)
    lib.orc_histogram_build(P(bins, ctypes.c_uint16), P(nb, ctypes.c_uint32), bins.shape[0], bins.shape[1],
                            P(g, ctypes.c_float), P(h, ctypes.c_float), P(r, ctypes.c_uint32),
                            0 if r is None else len(r), P(out, ctypes.c_double))
    return out


def find_split(hist, n_bins, is_cat, has_missing, pg, ph, pc, cfg, n_threads=1):
    hh = np.ascontiguousarray(hist, dtype=np.float64)
    nb = np.ascontiguousarray(n_bins, dtype=np.uint32)
    ic = np.ascontiguousarray(is_cat, dtype=np.int32)
    hm = np.ascontiguousarray(has_missing, dtype=np.int32)
    s = Split()
    lib.orc_find_split(P(hh, ctypes.c_double), P(nb, ctypes.c_uint32), P(ic, ctypes.c_int32), P(hm, ctypes.c_int32),
                       len(nb), pg, ph, pc, ctypes.byref(cfg), n_threads, ctypes.byref(s))
    return s


def _obj_cfg(objective, alpha, delta):
    c = config(objective=objective, huber_delta=float(delta))
    if alpha is not None:
        a = [float(v) for v in np.atleast_1d(alpha)]
        c.quantile_alpha = (ctypes.c_float * len(a))(*a)
        c.n_quantiles = len(a)
    return c


def gradients(objective, preds_gm, y, w=None, alpha=None, delta=1.0):
    p = f32(preds_gm)
    if p.ndim == 1:
        p = p.reshape(1, -1)
    G, n = p.shape
    g = np.zeros((G, n), np.float32)
    h = np.zeros((G, n), np.float32)
    c = _obj_cfg(objective, alpha, delta)
    lib.orc_gradients_cfg(ctypes.byref(c), G, P(p, ctypes.c_float), P(f32(y), ctypes.c_float),
                          P(None if w is None else f32(w), ctypes.c_float), n, P(g, ctypes.c_float),
                          P(h, ctypes.c_float))
    return g, h


def base_score(objective, n_outputs, y, w=None, alpha=None):
    out = np.zeros(n_outputs, np.float32)
    yy = f32(y)
    c = _obj_cfg(objective, alpha, 1.0)
    lib.orc_base_score_cfg(ctypes.byref(c), n_outputs, P(yy, ctypes.c_float),
                           P(None if w is None else f32(w), ctypes.c_float), len(yy), P(out, ctypes.c_float))
    return out


def metric(kind, preds_gm, y, w=None, alpha=None, delta=1.0):
    p = f32(preds_gm)
    if p.ndim == 1:
        p = p.reshape(1, -1)
    c = _obj_cfg(0, alpha, delta)
    return lib.orc_metric_cfg(kind, ctypes.byref(c), P(p, ctypes.c_float), p.shape[0], p.shape[1],
                              P(f32(y), ctypes.c_float), P(None if w is None else f32(w), ctypes.c_float))


def goss(g, h, top_rate, other_rate, seed, calls=1):
    """GOSS sampler (sampling/row.rs:214-280) called `calls` times on (g, h)
    (scaled in place each call): the last call's kept mask and count, and the
    scaled g, h."""
    g = f32(g).copy()
    h = f32(h).copy()
    mask = np.zeros(g.size, np.uint8)
    k = lib.orc_goss(P(g, ctypes.c_float), P(h, ctypes.c_float), g.size, top_rate, other_rate, seed, calls,
                     P(mask, ctypes.c_uint8))
    return mask, int(k), g, h


def leaf_quantile(values, weights, alpha):
    v = f32(values)
    w = None if weights is None else f32(weights)
    return float(lib.orc_leaf_quantile(P(v, ctypes.c_float), P(w, ctypes.c_float), v.size, alpha))


def philox4x32_10(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib.orc_philox4x32_10(P(c, ctypes.c_uint32), P(k, ctypes.c_uint32), P(out, ctypes.c_uint32))
    return out


def quantize(grad, hess, precision, seed, rnd, output=0):
    """Quantised (qg, qh, steps) of one output's gradients (int32 arrays)."""
    g, h = f32(grad), f32(hess)
    n = len(g)
    qg = np.zeros(n, np.int32)
    qh = np.zeros(n, np.int32)
    steps = np.zeros(4, np.float64)
    lib.orc_quantize(P(g, ctypes.c_float), P(h, ctypes.c_float), n, precision, seed, rnd, output,
                     P(qg, ctypes.c_int32), P(qh, ctypes.c_int32), P(steps, ctypes.c_double))
    return qg, qh, steps


def config(**fields):
    """bst_config with the reference defaults (the oracle's own statement of
    GBDTConfig's builder defaults) and the given fields set."""
    c = Config()
    lib.orc_config_default(ctypes.byref(c))
    for k, v in fields.items():
        setattr(c, k, v)
    return c


class synth:
    """The seeded workloads from the oracle's own copy of the generator
    (byte-identical to the engine's ``boosters_b200.synth``)."""

    @staticmethod
    def binary(n, n_features, n_nan_cols, seed, stream=0):
        x = np.empty((n_features, n), np.float32)
        y = np.empty(n, np.float32)
        _check(lib.orc_synth_binary(n, n_features, n_nan_cols, seed, stream, P(x, ctypes.c_float),
                                    P(y, ctypes.c_float)))
        return x, y

    @staticmethod
    def regression(n, n_features, n_informative, seed, stream=0):
        x = np.empty((n_features, n), np.float32)
        y = np.empty(n, np.float32)
        _check(lib.orc_synth_regression(n, n_features, n_informative, seed, stream, P(x, ctypes.c_float),
                                        P(y, ctypes.c_float)))
        return x, y

    @staticmethod
    def multiclass(n, n_numeric, n_categorical, n_classes, seed, stream=0):
        x = np.empty((n_numeric + n_categorical, n), np.float32)
        y = np.empty(n, np.float32)
        _check(lib.orc_synth_multiclass(n, n_numeric, n_categorical, n_classes, seed, stream,
                                        P(x, ctypes.c_float), P(y, ctypes.c_float)))
        return x, y
