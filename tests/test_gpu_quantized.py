"""Quantised training (precision "q16" / "q8") on the GPU against the oracle's
quantised mode on the same seeded inputs.

The integers themselves are bit-exact (the same Philox4x32-10 words and the
same f64 rounding); histogram sums are exact integers on both sides, so the
chosen splits, tree structure and row->leaf assignment are bit-exact too.
Leaves are solved from the f32 gradients: exact fixed-point sums on the GPU,
f64 sums in partition order in the oracle, so leaf values and node sums agree
within a tolerance like the f32 mode's.
"""
import ctypes

import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n
import oracle_bridge as ob

from test_gpu_parity import REL, STRUCT_KEYS, compare_trees, train_both

pytestmark = pytest.mark.gpu

PREC = {"q16": n.PRECISION_Q16, "q8": n.PRECISION_Q8}


def gpu_quantize(g, h, precision, seed, rnd, output=0):
    g = np.ascontiguousarray(g, np.float32)
    h = np.ascontiguousarray(h, np.float32)
    qg = np.zeros(len(g), np.int32)
    qh = np.zeros(len(g), np.int32)
    steps = np.zeros(4, np.float64)
    n.check(n.lib.bst_quantize_gradients(n.ptr(g, ctypes.c_float), n.ptr(h, ctypes.c_float), len(g), precision,
                                         seed, rnd, output, n.ptr(qg, ctypes.c_int32), n.ptr(qh, ctypes.c_int32),
                                         n.ptr(steps, ctypes.c_double)))
    return qg, qh, steps


@pytest.mark.parametrize("precision", ["q16", "q8"])
def test_quantize_bit_exact(precision):
    rng = np.random.default_rng(11)
    m = 1 << 20
    g = (rng.standard_t(3, size=m) * 0.1).astype(np.float32)
    h = rng.uniform(1e-6, 0.25, size=m).astype(np.float32)
    g[::97] = 0.0
    g[5] = -np.abs(g).max() * 1.5  # the extreme value is negative
    for seed, rnd, out in ((42, 0, 0), (0xDEADBEEFCAFE, 123, 3)):
        want = ob.quantize(g, h, PREC[precision], seed, rnd, out)
        got = gpu_quantize(g, h, PREC[precision], seed, rnd, out)
        np.testing.assert_array_equal(got[2], want[2])
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


def test_quantize_edge_inputs():
    z = np.zeros(1000, np.float32)
    qg, qh, steps = gpu_quantize(z, z, n.PRECISION_Q8, 1, 0)
    assert not qg.any() and not qh.any() and not steps.any()
    # non-finite values do not set the scale and saturate
    v = np.array([0.5, np.inf, -np.inf, 0.25, 1.0], np.float32)
    want = ob.quantize(v, np.abs(v), n.PRECISION_Q16, 3, 1)
    got = gpu_quantize(v, np.abs(v), n.PRECISION_Q16, 3, 1)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    qg, _, _ = gpu_quantize(np.zeros(0, np.float32), np.zeros(0, np.float32), n.PRECISION_Q8, 1, 0)
    assert qg.size == 0


@pytest.mark.parametrize("precision", ["q16", "q8"])
@pytest.mark.parametrize("batched", [True, False])
def test_quantised_train_parity_logistic_nan(precision, batched):
    x, y = bst.synth.binary(40_000, 40, n_nan_cols=10, seed=2)
    gm, om, ds = train_both(x, y, objective=bst.Objective.logistic(), n_estimators=12, learning_rate=0.1,
                            max_depth=8, precision=precision, batched=batched)
    compare_trees(gm, om, 40_000, sum_rtol=1e-6, sum_atol=1e-6)
    xv, _ = bst.synth.binary(8_000, 40, n_nan_cols=10, seed=2, stream=1)
    np.testing.assert_allclose(gm.predict_group_major(bst.Dataset.from_feature_major(xv)), om.predict(xv),
                               rtol=REL, atol=1e-6)


def test_quantised_train_parity_regression_q8():
    x, y = bst.synth.regression(5000, 100, 20, seed=1)
    gm, om, _ = train_both(x, y, n_estimators=30, learning_rate=0.1, max_depth=6, precision="q8")
    compare_trees(gm, om, 5000, sum_rtol=1e-9, sum_atol=1e-9)
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)


def test_quantised_train_parity_leafwise_q8():
    x, y = bst.synth.binary(30_000, 30, n_nan_cols=6, seed=3)
    gm, om, _ = train_both(x, y, objective=bst.Objective.logistic(), n_estimators=6, learning_rate=0.2,
                           growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=63, precision="q8")
    compare_trees(gm, om, 30_000, sum_rtol=1e-6, sum_atol=1e-6)


def test_quantised_train_parity_softmax_q16():
    x, y = bst.synth.multiclass(20_000, 12, 5, 4, seed=4)
    cats = list(range(12, 17))
    gm, om, _ = train_both(x, y, categorical=cats, objective=bst.Objective.softmax(4), n_estimators=3,
                           learning_rate=0.3, max_depth=5, precision="q16")
    compare_trees(gm, om, 20_000, sum_rtol=1e-6, sum_atol=1e-6)


def test_quantised_training_is_deterministic():
    x, y = bst.synth.binary(20_000, 20, n_nan_cols=4, seed=5)
    ds = bst.Dataset.from_feature_major(x, y)
    cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=5, max_depth=6, precision="q8")
    a = bst.GBDTModel.train(ds, cfg)
    b = bst.GBDTModel.train(ds, cfg)
    for i in range(a.n_trees):
        ta, tb = a.tree(i), b.tree(i)
        for k in STRUCT_KEYS + ["threshold", "leaf_value", "gain", "grad_sum", "hess_sum"]:
            np.testing.assert_array_equal(ta[k], tb[k])
