"""The C-ABI boundary on CPU: every declared symbol is exported, defaults and
validation follow GBDTConfig, and host-only entry points behave."""
import ctypes
import os
import re

import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(bst_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(n.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) > 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_bindings_cover_declarations():
    bound = {name for name, _, _ in n.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_config_defaults_match_reference():
    # model/gbdt/config.rs:111-226, data/binned/feature_analysis.rs:50-63
    c = n.Config()
    n.lib.bst_config_default(ctypes.byref(c))
    assert c.n_trees == 100 and abs(c.learning_rate - 0.3) < 1e-7
    assert c.growth_strategy == n.GROWTH_DEPTHWISE and c.max_depth == 6 and c.max_leaves == 31
    assert c.max_onehot_cats == 4 and c.lambda_ == 1.0 and c.alpha == 0.0
    assert c.min_child_weight == 1.0 and c.min_gain == 0.0 and c.min_samples_leaf == 1
    assert c.max_bins == 256 and abs(c.sparsity_threshold - 0.9) < 1e-7 and c.enable_bundling == 1
    assert c.max_categorical_cardinality == 0 and c.binning_sample_cnt == 200000
    assert c.cache_size == 8 and c.seed == 42 and c.early_stopping_rounds == -1


@pytest.mark.parametrize("kw,msg", [
    ({"learning_rate": 0.0}, "learning_rate must be positive"),
    ({"n_estimators": 0}, "n_trees must be at least 1"),
    ({"subsample": 1.5}, "subsample must be in (0, 1]"),
    ({"colsample_bytree": 0.0}, "colsample_bytree must be in (0, 1]"),
    ({"l2": -1.0}, "lambda must be non-negative"),
    ({"l1": -0.5}, "alpha must be non-negative"),
    ({"min_child_weight": -1.0}, "min_child_weight must be non-negative"),
    ({"min_gain_to_split": -1.0}, "min_gain must be non-negative"),
])
def test_config_validation(kw, msg):
    # GBDTConfig::validate (model/gbdt/config.rs:252-310)
    with pytest.raises(ValueError, match=re.escape(msg)):
        bst.GBDTConfig(**kw)


def test_dataset_errors_and_shapes():
    with pytest.raises(bst.BoostersError):
        bst.Dataset.from_feature_major(np.zeros((0, 5), np.float32))
    with pytest.raises(ValueError):
        bst.Dataset(np.zeros((4, 2), np.float32), labels=np.zeros(3))
    ds = bst.Dataset(np.zeros((4, 2), np.float32), labels=np.zeros(4), categorical_features=[1])
    assert ds.shape == (4, 2) and ds.categorical_features == [1]


def test_synthetic_generators_are_deterministic():
    a = bst.synth.binary(2000, 30, n_nan_cols=20, seed=2)
    b = bst.synth.binary(2000, 30, n_nan_cols=20, seed=2)
    c = bst.synth.binary(2000, 30, n_nan_cols=20, seed=2, stream=1)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert not np.array_equal(np.nan_to_num(a[0]), np.nan_to_num(c[0]))
    nan_rate = np.isnan(a[0][:20]).mean()
    assert 0.08 < nan_rate < 0.12 and not np.isnan(a[0][20:]).any()
    x, y = bst.synth.multiclass(3000, 40, 10, 10, seed=4)
    cats = x[40:]
    assert cats.min() == 0 and cats.max() <= 63 and np.all(cats == np.floor(cats))
    assert set(np.unique(y)) <= set(range(10))


def test_metric_matches_oracle():
    import oracle_bridge as ob
    rng = np.random.default_rng(1)
    y = (rng.random(500) > 0.5).astype(np.float32)
    p = rng.random(500).astype(np.float32)
    for kind, code in (("logloss", 2), ("rmse", 1)):
        assert bst.metric(kind, p, y) == ob.metric(code, p, y)
    pm = rng.random((3, 500)).astype(np.float32)
    ym = rng.integers(0, 3, 500).astype(np.float32)
    assert bst.metric("mlogloss", pm, ym) == ob.metric(3, pm, ym)


def test_gpu_entry_points_fail_cleanly_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    x, y = bst.synth.regression(100, 5, 2)
    ds = bst.Dataset.from_feature_major(x, y)
    with pytest.raises(bst.BoostersError) as e:
        bst.GBDTModel.train(ds, bst.GBDTConfig(n_estimators=1))
    assert e.value.status == n.BST_ERR_CUDA


def test_training_rejects_unsupported_options():
    x, y = bst.synth.regression(100, 5, 2)
    ds = bst.Dataset.from_feature_major(x, y)
    with pytest.raises(bst.BoostersError) as e:
        bst.GBDTModel.train(ds, bst.GBDTConfig(max_depth=30))
    assert e.value.status == n.BST_ERR_UNSUPPORTED
    with pytest.raises(bst.BoostersError) as e:
        bst.GBDTModel.train(bst.Dataset.from_feature_major(x), bst.GBDTConfig())
    assert e.value.status == n.BST_ERR_MISSING_TARGETS


def test_checked_library_exports_and_status():
    """The bounds-checked build exports the same entry points; the normal
    build answers bst_check_report with BST_ERR_UNSUPPORTED (no device
    call), the checked build without a device with BST_ERR_CUDA."""
    checked = os.path.join(os.path.dirname(n.LIB_PATH), "libboosters_b200_checked.so")
    if not os.path.exists(checked):
        pytest.skip("libboosters_b200_checked.so is not built (python -m boosters_b200.build --checked)")
    lib = ctypes.CDLL(checked)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    v = ctypes.c_uint64(7)
    normal = ctypes.CDLL(n.LIB_PATH)
    normal.bst_check_report.restype = ctypes.c_int32
    assert normal.bst_check_report(0, ctypes.byref(v), None, None, None) == 5  # BST_ERR_UNSUPPORTED
    assert v.value == 7
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if not has_gpu:
        lib.bst_check_report.restype = ctypes.c_int32
        assert lib.bst_check_report(0, ctypes.byref(v), None, None, None) == 6  # BST_ERR_CUDA
