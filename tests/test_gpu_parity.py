"""Parity of the CUDA engine (through the C ABI) with the CPU restatement of
boosters' GBDT path on the same seeded inputs.

Bit-exact: bins, bin bounds, tree structure (split feature, split bin,
threshold, default direction, children), per-row leaf assignment.
Tolerance: leaf values and predictions within 1e-5 relative (f32 results
of f64 sums accumulated in a different order).
"""
import math

import numpy as np
import pytest

import boosters_b200 as bst
import oracle_bridge as ob

pytestmark = pytest.mark.gpu

REL = 1e-5  # leaf values / predictions vs the oracle


def _cfg(**kw):
    return bst.GBDTConfig(**kw)


def compare_binned(gb, orc):
    assert gb.n_columns == orc.n_columns
    for c in range(gb.n_columns):
        gi, oi = gb.column_info(c), orc.column_info(c)
        assert gi == oi, (c, gi, oi)
        np.testing.assert_array_equal(gb.column_bounds(c), orc.column_bounds(c), err_msg=f"bounds col {c}")
        np.testing.assert_array_equal(gb.column_bins(c), orc.column_bins(c), err_msg=f"bins col {c}")


STRUCT_KEYS = ["split_index", "left", "right", "default_left", "is_leaf", "split_type", "split_bin", "seg_start",
               "seg_size", "cat_words"]


def compare_trees(gm, om, n_rows=None, check_rows=True, sum_rtol=1e-9, sum_atol=1e-9):
    """Bit-exact structure; node sums within (sum_rtol, sum_atol): 1e-9 for
    squared loss (identical gradients), 1e-6 where gradients go through exp."""
    assert gm.n_trees == om.n_trees
    for i in range(gm.n_trees):
        g, o = gm.tree(i), om.tree(i)
        assert g["n_nodes"] == o["n_nodes"], f"tree {i}: {g['n_nodes']} vs {o['n_nodes']} nodes"
        assert g["group"] == o["group"]
        for k in STRUCT_KEYS:
            np.testing.assert_array_equal(g[k], o[k], err_msg=f"tree {i} {k}")
        split = g["is_leaf"] == 0
        np.testing.assert_array_equal(g["threshold"][split], o["threshold"][split], err_msg=f"tree {i} threshold")
        leaf = ~split
        np.testing.assert_allclose(g["leaf_value"][leaf], o["leaf_value"][leaf], rtol=REL, atol=1e-7,
                                   err_msg=f"tree {i} leaf values")
        np.testing.assert_allclose(g["gain"][split], o["gain"][split], rtol=1e-5, atol=1e-6,
                                   err_msg=f"tree {i} gains")
        np.testing.assert_allclose(g["grad_sum"], o["grad_sum"], rtol=sum_rtol, atol=sum_atol, err_msg=f"tree {i} G")
        np.testing.assert_allclose(g["hess_sum"], o["hess_sum"], rtol=sum_rtol, atol=sum_atol, err_msg=f"tree {i} H")
        if check_rows:
            np.testing.assert_array_equal(gm.tree_row_leaves(i, n_rows), om.row_leaves(i),
                                          err_msg=f"tree {i} row leaves")


def train_both(x, y, n_threads=1, categorical=(), **kw):
    ds = bst.Dataset.from_feature_major(x, y, categorical_features=list(categorical))
    cfg = _cfg(**kw)
    gm = bst.GBDTModel.train(ds, cfg, n_threads=n_threads, record_leaves=True)
    om = ob.OracleModel(x, y, cfg.to_c(), n_threads=n_threads, categorical=categorical)
    return gm, om, ds


# ---------------------------------------------------------------- KATs on GPU

def test_kat_bin_values(kats):
    import ctypes
    from boosters_b200 import _native as n
    for case in kats["value_to_bin"]:
        vals = np.array([float(v) for v in case["values"]], np.float32)
        out = np.zeros(len(vals), np.uint32)
        if "cats" in case:
            cats = np.array(case["cats"], np.int32)
            rc = n.lib.bst_bin_values(None, 0, case["missing"], case["default_bin"], 1, n.ptr(cats, ctypes.c_int32),
                                      len(cats), n.ptr(vals, ctypes.c_float), len(vals), n.ptr(out, ctypes.c_uint32))
        else:
            b = np.array([float(v) for v in case["bounds"]], np.float64)
            rc = n.lib.bst_bin_values(n.ptr(b, ctypes.c_double) if len(b) else None, len(b), case["missing"],
                                      case["default_bin"], 0, None, 0, n.ptr(vals, ctypes.c_float), len(vals),
                                      n.ptr(out, ctypes.c_uint32))
        n.check(rc)
        assert out.tolist() == case["bins"], case["src"]


def test_kat_histogram(kats):
    import ctypes
    from boosters_b200 import _native as n

    def gpu_hist(bins, n_bins, grad, hess, rows=None):
        b = np.ascontiguousarray(bins, np.uint16)
        nb = np.ascontiguousarray(n_bins, np.uint32)
        g, h = np.ascontiguousarray(grad, np.float32), np.ascontiguousarray(hess, np.float32)
        r = None if rows is None else np.ascontiguousarray(rows, np.uint32)
        out = np.zeros((int(nb.sum()), 2), np.float64)
        n.check(n.lib.bst_histogram_build(n.ptr(b, ctypes.c_uint16), n.ptr(nb, ctypes.c_uint32), b.shape[0],
                                          b.shape[1], n.ptr(g, ctypes.c_float), n.ptr(h, ctypes.c_float),
                                          n.ptr(r, ctypes.c_uint32), 0 if r is None else len(r),
                                          n.ptr(out, ctypes.c_double)))
        return out

    for c in kats["histogram"]:
        h = gpu_hist(np.array(c["bins"]), c["n_bins"], c["grad"], c["hess"], c["rows"])
        np.testing.assert_allclose(h, np.array(c["expect"]), atol=1e-10, err_msg=c["src"])
    # random case vs the oracle, mixed u8 / u16 columns and a row subset
    rng = np.random.default_rng(3)
    nb = np.array([2, 17, 256, 257, 300, 5, 256, 64] * 3, np.uint32)
    n_rows = 20011
    bins = np.stack([rng.integers(0, k, n_rows) for k in nb]).astype(np.uint16)
    g = rng.normal(size=n_rows).astype(np.float32)
    h = rng.random(n_rows).astype(np.float32)
    rows = np.sort(rng.choice(n_rows, 7777, replace=False)).astype(np.uint32)
    for rr in (None, rows):
        np.testing.assert_allclose(gpu_hist(bins, nb, g, h, rr), ob.histogram_build(bins, nb, g, h, rr),
                                   rtol=1e-12, atol=1e-9)


def test_kat_find_split(kats):
    import ctypes
    from boosters_b200 import _native as n
    for c in kats["find_split"]:
        cfg = _cfg(max_onehot_cats=c["max_onehot_cats"]).to_c()
        hist = np.ascontiguousarray(c["hist"], np.float64)
        nb = np.ascontiguousarray(c["n_bins"], np.uint32)
        ic = np.ascontiguousarray(c["is_cat"], np.int32)
        hm = np.ascontiguousarray(c["has_missing"], np.int32)
        s = n.Split()
        n.check(n.lib.bst_find_split(n.ptr(hist, ctypes.c_double), n.ptr(nb, ctypes.c_uint32),
                                     n.ptr(ic, ctypes.c_int32), n.ptr(hm, ctypes.c_int32), len(nb), c["pg"], c["ph"],
                                     c["pc"], ctypes.byref(cfg), 1, ctypes.byref(s)))
        o = ob.find_split(hist, nb, ic, hm, c["pg"], c["ph"], c["pc"], cfg)
        assert (s.gain > -math.inf) == c["expect_valid"], c["src"]
        if c["expect_valid"]:
            assert s.feature == c["expect_feature"], c["src"]
        for k in ("feature", "gain", "default_left", "is_categorical", "bin"):
            assert getattr(s, k) == getattr(o, k), (c["src"], k)
        assert list(s.left_cats) == list(o.left_cats), c["src"]


def test_kat_grower_and_threshold(kats):
    for c in kats["grower"]:
        x = np.array([c["values"]], np.float32)
        ds = bst.Dataset.from_feature_major(x)
        m = bst.GBDTModel.grow_tree(ds, c["grad"], c["hess"], _cfg(max_depth=c["max_depth"]))
        assert int(m.tree(0)["is_leaf"].sum()) == c["expect_leaves"], c["src"]
    x = np.array([[0.0, 1.0]], np.float32)
    m = bst.GBDTModel.grow_tree(bst.Dataset.from_feature_major(x), [-1.0, 1.0], [1.0, 1.0],
                                _cfg(max_depth=1, min_child_weight=0.0, learning_rate=1.0))
    t = m.tree(0)
    assert t["threshold"][0] == np.nextafter(np.float32(0.5), np.float32(np.inf))


def test_kat_traversal(kats):
    for c in kats["traversal"]:
        tree = {"split_index": [0, 0, 0], "threshold": [c["threshold"], 0, 0], "left": [1, 0, 0],
                "right": [2, 0, 0], "default_left": [1 if c["default_left"] else 0, 0, 0], "is_leaf": [0, 1, 1],
                "leaf_value": [0.0, 1.0, 2.0], "split_type": [0, 0, 0]}
        m = bst.GBDTModel.from_trees(1, [tree])
        x = np.array([[float(v)] for v in c["values"]], np.float32)
        p = m.predict_raw(bst.Dataset(x))[:, 0]
        np.testing.assert_array_equal(p, np.array(c["expect"], np.float32), c["src"])
    cat = {"split_index": [0, 0, 0], "threshold": [0, 0, 0], "left": [1, 0, 0], "right": [2, 0, 0],
           "default_left": [1, 0, 0], "is_leaf": [0, 1, 1], "leaf_value": [0.0, 10.0, 20.0],
           "split_type": [1, 0, 0], "seg_start": [0, 0, 0], "seg_size": [1, 0, 0], "cat_words": [0b1010]}
    m = bst.GBDTModel.from_trees(1, [cat])
    p = m.predict_raw(bst.Dataset(np.array([[0.0], [1.0], [2.0], [3.0], [np.nan]], np.float32)))[:, 0]
    np.testing.assert_array_equal(p, [10.0, 20.0, 10.0, 20.0, 10.0])


# ------------------------------------------------------------------- binning

def test_binning_parity_regression():
    x, _ = bst.synth.regression(5000, 100, 20, seed=1)
    cfg = _cfg()
    compare_binned(bst.BinnedDataset(bst.Dataset.from_feature_major(x), cfg), ob.OracleBinned(x, cfg.to_c()))


def test_binning_parity_sampled_with_nan():
    # > 200k rows: bounds from the splitmix64 sample (dataset.rs:598-633); NaN
    # columns get a 257th bin (u16 storage)
    x, _ = bst.synth.binary(240_000, 24, n_nan_cols=8, seed=2)
    cfg = _cfg()
    gb = bst.BinnedDataset(bst.Dataset.from_feature_major(x), cfg)
    compare_binned(gb, ob.OracleBinned(x, cfg.to_c()))
    assert gb.column_info(0)["n_bins"] == 257 and gb.column_info(0)["has_missing"]


def test_binning_parity_categorical_and_edge_columns():
    x, _ = bst.synth.multiclass(20_000, 6, 4, 3, seed=4)
    extra = np.zeros((4, x.shape[1]), np.float32)
    extra[0] = 3.0                                    # constant non-zero: one bin
    extra[1] = np.nan                                 # all missing: trivial, skipped
    extra[2, ::2] = 1.0                               # binary 0/1 (density 0.5)
    extra[3] = np.where(np.arange(x.shape[1]) % 3 == 0, np.inf, 1.0 + np.arange(x.shape[1]) % 5)
    x = np.concatenate([x, extra])
    cats = [6, 7, 8, 9]
    cfg = _cfg(max_bins=64)
    gb = bst.BinnedDataset(bst.Dataset.from_feature_major(x, categorical_features=cats), cfg)
    compare_binned(gb, ob.OracleBinned(x, cfg.to_c(), categorical=cats))


def _edge_numeric_columns(n, rng):
    """Numeric columns that reach every branch of the device bounds: signed
    zeros (one distinct value), exactly max_bins and max_bins + 1 distinct
    values, heavy ties, NaN and infinities mixed in, one distinct finite
    value beside NaN, a column of every row distinct."""
    cols = []
    z = np.where(rng.random(n) < 0.5, np.float32(-0.0), np.float32(0.0)).astype(np.float32)
    z[::7] = 1.5
    cols.append(z)                                                       # -0.0 / +0.0 merge, then 1.5
    cols.append((rng.integers(0, 32, n) * 0.25).astype(np.float32))      # 32 distinct = max_bins
    cols.append((rng.integers(0, 33, n) * 0.25).astype(np.float32))      # 33 distinct: quantiles
    t = rng.normal(size=n).astype(np.float32)
    t[rng.random(n) < 0.6] = 2.0                                         # heavy ties
    t[::11] = np.nan
    t[::13] = np.inf
    t[::17] = -np.inf
    cols.append(t)
    c = np.full(n, 4.0, np.float32)
    c[::3] = np.nan                                                      # one value + NaN: one bin
    cols.append(c)
    cols.append(np.arange(n, dtype=np.float32) * np.float32(-0.5))      # all distinct, negative
    return np.stack(cols)


@pytest.mark.parametrize("n", [100, 3000, 9000])
def test_binning_parity_device_bounds_edges(n):
    rng = np.random.default_rng(n)
    x = _edge_numeric_columns(n, rng)
    for mb in (32, 2):
        cfg = _cfg(max_bins=mb)
        gb = bst.BinnedDataset(bst.Dataset.from_feature_major(x), cfg)
        compare_binned(gb, ob.OracleBinned(x, cfg.to_c()))


def test_binning_device_bounds_pinned_equals_pageable():
    # pinned inputs go up as one asynchronous copy, pageable ones on a
    # helper thread: the same bins either way
    import torch

    x, _ = bst.synth.binary(240_000, 12, n_nan_cols=4, seed=9)
    cfg = _cfg()
    xp = torch.from_numpy(x).pin_memory().numpy()
    a = bst.BinnedDataset(bst.Dataset.from_feature_major(x), cfg)
    b = bst.BinnedDataset(bst.Dataset.from_feature_major(xp), cfg)
    assert a.n_columns == b.n_columns
    for c in range(a.n_columns):
        assert a.column_info(c) == b.column_info(c)
        np.testing.assert_array_equal(a.column_bounds(c), b.column_bounds(c))
        np.testing.assert_array_equal(a.column_bins(c), b.column_bins(c))


# ------------------------------------------------------------------ training

@pytest.mark.parametrize("n_threads", [1, 0])
def test_train_parity_regression_5k(n_threads):
    # 5,000 x 100 regression, 50 trees, depth 6, 256 bins, lr 0.1, lambda 1
    x, y = bst.synth.regression(5000, 100, 20, seed=1)
    gm, om, ds = train_both(x, y, n_threads=n_threads, n_estimators=50, learning_rate=0.1, max_depth=6)
    compare_trees(gm, om, 5000)
    np.testing.assert_array_equal(gm.base_scores(), om.base_scores())
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)
    np.testing.assert_allclose(gm.predict_group_major(ds, raw=True), om.predict(x, raw=True), rtol=REL, atol=1e-6)


@pytest.mark.parametrize("batched", [True, False])
def test_train_parity_logistic_nan(batched):
    # batched: device-side level loop in a CUDA graph; else the host-driven loop
    x, y = bst.synth.binary(40_000, 40, n_nan_cols=10, seed=2)
    gm, om, ds = train_both(x, y, objective=bst.Objective.logistic(), n_estimators=15, learning_rate=0.1,
                            max_depth=8, batched=batched)
    compare_trees(gm, om, 40_000, sum_rtol=1e-6, sum_atol=1e-6)
    xv, yv = bst.synth.binary(8_000, 40, n_nan_cols=10, seed=2, stream=1)
    pg = gm.predict_group_major(bst.Dataset.from_feature_major(xv))
    po = om.predict(xv)
    np.testing.assert_allclose(pg, po, rtol=REL, atol=1e-6)
    assert abs(bst.metric("logloss", pg, yv) - bst.metric("logloss", po, yv)) < 1e-6


@pytest.mark.parametrize("precision", ["fp32", "q16"])
@pytest.mark.parametrize("batched", [True, False])
def test_train_parity_mixed_bin_counts(precision, batched):
    # columns with up to 1024 bins (u16 rows, general shared-memory tiles)
    # beside low-cardinality u8 columns (column-lane tiles)
    rng = np.random.default_rng(12)
    n = 12_000
    x = rng.normal(size=(24, n)).astype(np.float32)
    x[:12] = np.round(x[:12] * 8.0)  # ~60 distinct values
    x[3, rng.random(n) < 0.1] = np.nan
    y = (x[0] * 0.5 + np.nan_to_num(x[3]) + x[15] * x[16] + rng.normal(size=n)).astype(np.float32)
    gm, om, _ = train_both(x, y, n_estimators=8, learning_rate=0.3, max_depth=6, max_bins=1024,
                           precision=precision, batched=batched)
    compare_trees(gm, om, n)


def test_train_parity_leafwise():
    x, y = bst.synth.binary(30_000, 30, n_nan_cols=6, seed=3)
    gm, om, _ = train_both(x, y, objective=bst.Objective.logistic(), n_estimators=6, learning_rate=0.2,
                           growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=63)
    compare_trees(gm, om, 30_000, sum_rtol=1e-6, sum_atol=1e-6)


@pytest.mark.parametrize("n_leaves,precision,batched", [(2, "fp32", True), (5, "fp32", True), (17, "fp32", True),
                                                        (255, "fp32", True), (17, "q8", True), (17, "fp32", False),
                                                        (17, "q8", False)])
def test_train_parity_leafwise_budgets(n_leaves, precision, batched):
    """Batched leaf-wise growth expands heap candidates in speculative
    batches and replays the pops (plain: one node per step); budgets from one
    split to more leaves than the data supports exercise rolled-back
    expansions, the last pop and an exhausted heap."""
    x, y = bst.synth.regression(8000, 16, 6, seed=21)
    x[2, ::7] = np.nan
    gm, om, _ = train_both(x, y, n_estimators=4, learning_rate=0.3, growth_strategy=bst.GrowthStrategy.Leafwise,
                           n_leaves=n_leaves, min_samples_leaf=20, precision=precision, batched=batched)
    compare_trees(gm, om, 8000, sum_rtol=1e-9 if precision == "fp32" else 1e-6,
                  sum_atol=1e-9 if precision == "fp32" else 1e-6)


COLSAMPLE_CASES = [
    # (colsample_bytree, colsample_bylevel, growth, batched, precision, n_threads)
    (0.5, 0.7, "depthwise", False, "fp32", 1),
    (0.5, 0.7, "depthwise", True, "fp32", 1),
    (0.6, 1.0, "depthwise", True, "q8", 1),
    (1.0, 0.6, "leafwise", True, "fp32", 1),
    (0.6, 0.8, "leafwise", False, "fp32", 1),
    (0.9, 1.0, "depthwise", True, "fp32", 0),  # 22 of 24 columns: the parallel tie rule
    (0.5, 1.0, "depthwise", True, "fp32", 0),  # 12 searched: sequential rule at any n_threads
]


@pytest.mark.parametrize("bytree,bylevel,growth,batched,precision,n_threads", COLSAMPLE_CASES)
def test_train_parity_column_sampling(bytree, bylevel, growth, batched, precision, n_threads):
    """Per-tree and per-depth column samples (training/sampling/column.rs)
    drawn identically by the engine and the oracle; only the sampled
    columns are searched."""
    x, y = bst.synth.regression(6000, 24, 8, seed=31)
    x[5, ::9] = np.nan
    strat = bst.GrowthStrategy.Leafwise if growth == "leafwise" else bst.GrowthStrategy.Depthwise
    gm, om, _ = train_both(x, y, n_threads=n_threads, n_estimators=5, learning_rate=0.3, max_depth=5,
                           growth_strategy=strat, n_leaves=20, colsample_bytree=bytree, colsample_bylevel=bylevel,
                           precision=precision, batched=batched, seed=7)
    compare_trees(gm, om, 6000, sum_rtol=1e-9 if precision == "fp32" else 1e-6,
                  sum_atol=1e-9 if precision == "fp32" else 1e-6)


ROWSAMPLE_CASES = [
    # (subsample, growth, batched, precision, objective)
    (0.5, "depthwise", False, "fp32", "squared"),
    (0.5, "depthwise", True, "fp32", "squared"),
    (0.3, "depthwise", True, "q8", "logistic"),
    (0.6, "leafwise", True, "fp32", "squared"),
    (0.6, "leafwise", False, "fp32", "logistic"),
    (0.7, "depthwise", True, "fp32", "softmax"),
]


@pytest.mark.parametrize("subsample,growth,batched,precision,objective", ROWSAMPLE_CASES)
def test_train_parity_row_sampling(subsample, growth, batched, precision, objective):
    """Uniform row sampling (training/sampling/row.rs): the same reservoir
    sample per output and round in the engine and the oracle; unsampled rows
    carry zero grad/hess and node counts are sampled counts."""
    if objective == "softmax":
        x, y = bst.synth.multiclass(5000, 10, 0, 3, seed=33)
        obj = bst.Objective.softmax(3)
    elif objective == "logistic":
        x, y = bst.synth.binary(5000, 16, 3, seed=34)
        obj = bst.Objective.logistic()
    else:
        x, y = bst.synth.regression(5000, 16, 6, seed=35)
        obj = bst.Objective.squared()
    strat = bst.GrowthStrategy.Leafwise if growth == "leafwise" else bst.GrowthStrategy.Depthwise
    gm, om, _ = train_both(x, y, objective=obj, n_estimators=5, learning_rate=0.3, max_depth=5,
                           growth_strategy=strat, n_leaves=20, subsample=subsample, min_samples_leaf=30,
                           precision=precision, batched=batched, seed=9,
                           colsample_bytree=0.8 if objective == "softmax" else 1.0)
    tol = 1e-9 if (precision == "fp32" and objective == "squared") else 1e-6
    compare_trees(gm, om, 5000, sum_rtol=tol, sum_atol=tol)
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)


def test_column_sampling_one_column_per_tree():
    # ceil(24 * 0.01) = 1 column per tree: every split of a tree uses it
    x, y = bst.synth.regression(4000, 24, 8, seed=32)
    cfg = _cfg(n_estimators=6, max_depth=4, colsample_bytree=0.01)
    m = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)
    used = set()
    for i in range(m.n_trees):
        t = m.tree(i)
        feats = set(t["split_index"][t["is_leaf"] == 0].tolist())
        assert len(feats) <= 1, feats
        used |= feats
    assert len(used) > 1  # different trees draw different columns


def test_train_parity_softmax_categorical():
    x, y = bst.synth.multiclass(20_000, 12, 5, 4, seed=4)
    cats = list(range(12, 17))
    gm, om, ds = train_both(x, y, categorical=cats, objective=bst.Objective.softmax(4), n_estimators=4,
                            learning_rate=0.3, max_depth=5, max_onehot_cats=4)
    compare_trees(gm, om, 20_000, sum_rtol=1e-6, sum_atol=1e-6)
    assert any(gm.tree(i)["split_type"].any() for i in range(gm.n_trees)), "no categorical split was chosen"
    np.testing.assert_allclose(gm.predict_group_major(ds), om.predict(x), rtol=REL, atol=1e-6)


def test_grow_tree_parity_random_gradients():
    rng = np.random.default_rng(7)
    x = rng.normal(size=(20, 3000)).astype(np.float32)
    x[3, rng.random(3000) < 0.2] = np.nan
    g = rng.normal(size=3000).astype(np.float32)
    h = (0.1 + rng.random(3000)).astype(np.float32)
    for strat in (bst.GrowthStrategy.Depthwise, bst.GrowthStrategy.Leafwise):
        cfg = _cfg(max_depth=5, n_leaves=20, growth_strategy=strat, min_child_weight=0.5)
        gm = bst.GBDTModel.grow_tree(bst.Dataset.from_feature_major(x), g, h, cfg)
        om = ob.OracleModel.grow(x, g, h, cfg.to_c())
        compare_trees(gm, om, 3000)


def test_training_is_deterministic():
    x, y = bst.synth.binary(20_000, 20, n_nan_cols=4, seed=5)
    ds = bst.Dataset.from_feature_major(x, y)
    cfg = _cfg(objective=bst.Objective.logistic(), n_estimators=5, max_depth=6)
    a = bst.GBDTModel.train(ds, cfg)
    b = bst.GBDTModel.train(ds, cfg)
    for i in range(a.n_trees):
        ta, tb = a.tree(i), b.tree(i)
        for k in STRUCT_KEYS + ["threshold", "leaf_value", "gain", "grad_sum", "hess_sum"]:
            np.testing.assert_array_equal(ta[k], tb[k])
    np.testing.assert_array_equal(a.train_predictions(), b.train_predictions())


def test_sparse_column_dense_semantics():
    """A column of density <= 1 - sparsity_threshold would go to sparse
    storage in the reference (feature_analysis.rs:655-751), which the engine
    rejects; with sparsity_threshold = 1 and bundling off it is a dense
    column, and the trees match the oracle's."""
    from boosters_b200 import _native as n
    rng = np.random.default_rng(71)
    x, y = bst.synth.regression(6000, 10, 4, seed=71)
    x[3] = np.where(rng.random(6000) < 0.05, rng.normal(size=6000), 0.0).astype(np.float32)  # 95% zeros
    with pytest.raises(n.BoostersError) as ei:
        bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), _cfg(n_estimators=2))
    assert ei.value.status == n.BST_ERR_UNSUPPORTED and "sparsity_threshold" in str(ei.value)
    gm, om, _ = train_both(x, y, n_estimators=4, learning_rate=0.3, max_depth=5, sparsity_threshold=1.0,
                           enable_bundling=False)
    compare_trees(gm, om, 6000)
    assert any(3 in gm.tree(i)["split_index"][gm.tree(i)["is_leaf"] == 0] for i in range(gm.n_trees))
