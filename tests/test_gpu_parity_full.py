"""Engine-vs-oracle parity at the benchmark workloads' full sizes.

The small-shape tests in test_gpu_parity.py cover every code path; these
cases repeat the comparison on the shapes the benchmark times, where the
FP32 form's exact fixed-point histogram sums and the oracle's sequential
f64 sums (histograms/ops.rs:171-283) are most likely to disagree in the last
bits and where deep levels hold near-tied candidates:

* 1,000,000 x 100 logistic, depth 8 (20 NaN columns, 257-bin u16 columns):
  10 trees, plain FP32, batched FP32 and batched Q8;
* 10,000,000 x 200 logistic, leaf-wise 255 leaves: 3 trees, plain FP32,
  batched FP32 and batched Q8;
* 2,000,000 x 50 softmax, 10 classes, 10 categorical columns (cardinality
  4-64, Zipf frequencies), depth 6: 2 rounds (20 trees), plain and batched
  FP32.

Structure (split feature, bin, threshold, default direction, children,
categorical sets) and every row's leaf are compared bit-exact; leaf values
within 1e-5 relative, gains within 1e-5, node sums within 1e-6 relative.
On a structural mismatch the message names the first differing node with
both sides' candidates and gains (a flip between candidates whose f32 gains
are within an ulp is a summation-order tie, any other difference a bug).
The Q8 forms are compared against the oracle's quantised mode, whose
integer sums are exact on both sides.

The oracle runs with OpenMP threads over features (results do not depend on
the thread count); the training itself keeps n_threads=1 semantics.
"""
import os
import time

import numpy as np
import pytest

import boosters_b200 as bst
import oracle_bridge as ob

pytestmark = pytest.mark.gpu

OMP = max(1, os.cpu_count() or 1)
REL = 1e-5


def _first_struct_diff(g, o):
    keys = ("split_index", "split_bin", "default_left", "is_leaf", "left", "right", "split_type")
    n = min(g["n_nodes"], o["n_nodes"])
    for j in range(n):
        if any(g[k][j] != o[k][j] for k in keys):
            return j
    return n if g["n_nodes"] != o["n_nodes"] else None


def compare_full(gm, om, n_rows, label, sum_rtol=1e-6):
    assert gm.n_trees == om.n_trees, f"{label}: {gm.n_trees} vs {om.n_trees} trees"
    for i in range(gm.n_trees):
        g, o = gm.tree(i), om.tree(i)
        j = _first_struct_diff(g, o)
        if j is not None:
            def desc(t):
                if j >= t["n_nodes"]:
                    return "absent"
                if t["is_leaf"][j]:
                    return "leaf"
                return (f"feature {t['split_index'][j]} bin {t['split_bin'][j]} default_left "
                        f"{t['default_left'][j]} gain {float(t['gain'][j])!r}")
            gap = None
            if j < min(g["n_nodes"], o["n_nodes"]) and not g["is_leaf"][j] and not o["is_leaf"][j]:
                gap = abs(float(g["gain"][j]) - float(o["gain"][j]))
                ulp = float(np.spacing(np.float32(max(abs(g["gain"][j]), abs(o["gain"][j])))))
                gap = f"gain gap {gap:.3e} ({gap / ulp:.1f} f32 ulp)"
            pytest.fail(f"{label} tree {i} node {j}: engine {desc(g)} vs oracle {desc(o)}; {gap}")
        split = g["is_leaf"] == 0
        for k in ("seg_start", "seg_size", "cat_words"):
            np.testing.assert_array_equal(g[k], o[k], err_msg=f"{label} tree {i} {k}")
        np.testing.assert_array_equal(g["threshold"][split], o["threshold"][split],
                                      err_msg=f"{label} tree {i} threshold")
        np.testing.assert_allclose(g["leaf_value"][~split], o["leaf_value"][~split], rtol=REL, atol=1e-7,
                                   err_msg=f"{label} tree {i} leaf values")
        np.testing.assert_allclose(g["gain"][split], o["gain"][split], rtol=1e-5, atol=1e-6,
                                   err_msg=f"{label} tree {i} gains")
        np.testing.assert_allclose(g["grad_sum"], o["grad_sum"], rtol=sum_rtol, atol=1e-6,
                                   err_msg=f"{label} tree {i} G")
        np.testing.assert_allclose(g["hess_sum"], o["hess_sum"], rtol=sum_rtol, atol=1e-6,
                                   err_msg=f"{label} tree {i} H")
        leaves_g = gm.tree_row_leaves(i, n_rows)
        leaves_o = om.row_leaves(i)
        bad = np.flatnonzero(leaves_g != leaves_o)
        assert bad.size == 0, f"{label} tree {i}: {bad.size} rows in other leaves (first row {bad[:5]})"


def _train_engine(ds, cfg):
    t0 = time.perf_counter()
    m = bst.GBDTModel.train(ds, cfg, n_threads=1, record_leaves=True)
    return m, time.perf_counter() - t0


def _train_oracle(x, y, cfg, categorical=()):
    t0 = time.perf_counter()
    m = ob.OracleModel(x, y, cfg.to_c(), n_threads=1, categorical=categorical, omp_threads=OMP)
    return m, time.perf_counter() - t0


FORMS = {"plain_fp32": dict(precision="fp32", batched=False),
         "batched_fp32": dict(precision="fp32", batched=True),
         "batched_q8": dict(precision="q8", batched=True)}


@pytest.fixture(scope="module")
def binary_1m():
    return bst.synth.binary(1_000_000, 100, 20, seed=2)


@pytest.mark.parametrize("form", ["plain_fp32", "batched_fp32", "batched_q8"])
def test_parity_logistic_1Mx100_depth8(binary_1m, form):
    x, y = binary_1m
    ds = bst.Dataset.from_feature_major(x, y)
    cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=10, learning_rate=0.1, max_depth=8,
                         max_bins=256, metric=bst.Metric.none(), **FORMS[form])
    gm, tg = _train_engine(ds, cfg)
    om, to = _train_oracle(x, y, cfg)
    print(f"1M x 100 {form}: engine {tg:.1f} s, oracle {to:.1f} s")
    compare_full(gm, om, x.shape[1], f"1Mx100 {form}")
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)


@pytest.fixture(scope="module")
def binary_10m():
    return bst.synth.binary(10_000_000, 200, 20, seed=3)


@pytest.mark.parametrize("form", ["plain_fp32", "batched_fp32", "batched_q8"])
def test_parity_logistic_10Mx200_leafwise255(binary_10m, form):
    x, y = binary_10m
    ds = bst.Dataset.from_feature_major(x, y)
    cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=3, learning_rate=0.1,
                         growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=255, max_bins=256,
                         metric=bst.Metric.none(), **FORMS[form])
    gm, tg = _train_engine(ds, cfg)
    om, to = _train_oracle(x, y, cfg)
    print(f"10M x 200 leaf-wise {form}: engine {tg:.1f} s, oracle {to:.1f} s")
    compare_full(gm, om, x.shape[1], f"10Mx200 {form}")


@pytest.fixture(scope="module")
def multiclass_2m():
    return bst.synth.multiclass(2_000_000, 40, 10, 10, seed=4)


@pytest.mark.parametrize("form", ["plain_fp32", "batched_fp32"])
def test_parity_softmax_categorical_2Mx50(multiclass_2m, form):
    x, y = multiclass_2m
    cats = list(range(40, 50))
    ds = bst.Dataset.from_feature_major(x, y, categorical_features=cats)
    cfg = bst.GBDTConfig(objective=bst.Objective.softmax(10), n_estimators=2, learning_rate=0.1, max_depth=6,
                         max_bins=256, max_onehot_cats=4, metric=bst.Metric.none(), **FORMS[form])
    gm, tg = _train_engine(ds, cfg)
    om, to = _train_oracle(x, y, cfg, categorical=cats)
    print(f"2M x 50 softmax {form}: engine {tg:.1f} s, oracle {to:.1f} s")
    assert gm.n_trees == 20
    compare_full(gm, om, x.shape[1], f"2Mx50 softmax {form}")
    assert any(gm.tree(i)["split_type"].any() for i in range(gm.n_trees)), "no categorical split was chosen"
