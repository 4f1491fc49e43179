"""Engine-vs-oracle parity of the objectives beyond squared / logistic /
softmax and of GOSS row sampling:

* L1 (regression.rs:80-118) and pinball (regression.rs:129-173, three
  quantiles = three outputs) with leaf renewing (objectives/mod.rs:352-409):
  every leaf's value is the alpha-quantile of its rows' residuals;
  unweighted (rank rule) and weighted (step rule), depth-wise plain and
  batched, batched leaf-wise, with uniform row sampling;
* pseudo-Huber, Poisson and hinge gradients and base scores;
* GOSS (sampling/row.rs:214-280): warm-up rounds without sampling, then
  the top rows by |grad x hess| plus the reference's adaptive draw of the
  rest, scaled; depth-wise and leaf-wise, FP32 and Q8.

Structure and per-row leaves are compared bit-exact; leaf values within
1e-5 relative (renewed leaves are residuals of f32 predictions that both
sides compute in the same order, so they agree exactly in practice).
"""
import numpy as np
import pytest

import boosters_b200 as bst
import oracle_bridge as ob
from test_gpu_parity import REL, compare_trees

pytestmark = pytest.mark.gpu


def _train_both(x, y, weights=None, **kw):
    ds = bst.Dataset.from_feature_major(x, y, weights=weights)
    cfg = bst.GBDTConfig(**kw)
    gm = bst.GBDTModel.train(ds, cfg, n_threads=1, record_leaves=True)
    om = ob.OracleModel(x, y, cfg.to_c(), n_threads=1, weights=weights)
    return gm, om


FORMS = [("depthwise", False, "fp32"), ("depthwise", True, "fp32"), ("depthwise", True, "q8"),
         ("leafwise", True, "fp32"), ("leafwise", False, "fp32")]


def _strategy(growth):
    return bst.GrowthStrategy.Leafwise if growth == "leafwise" else bst.GrowthStrategy.Depthwise


@pytest.mark.parametrize("growth,batched,precision", FORMS)
@pytest.mark.parametrize("objective", ["absolute", "pinball"])
def test_leaf_renewing_parity(objective, growth, batched, precision):
    x, y = bst.synth.regression(7000, 12, 5, seed=41)
    y = y + np.random.default_rng(3).standard_cauchy(y.size).astype(np.float32) * 0.2  # heavy tails
    obj = bst.Objective.absolute() if objective == "absolute" else bst.Objective.pinball([0.1, 0.5, 0.9])
    gm, om = _train_both(x, y, objective=obj, n_estimators=4, learning_rate=0.5, max_depth=5,
                         growth_strategy=_strategy(growth), n_leaves=24, batched=batched, precision=precision,
                         metric=bst.Metric.none())
    assert gm.n_trees == (4 if objective == "absolute" else 12)
    np.testing.assert_array_equal(gm.base_scores(), om.base_scores())
    compare_trees(gm, om, 7000, sum_rtol=1e-9 if precision == "fp32" else 1e-6,
                  sum_atol=1e-9 if precision == "fp32" else 1e-6)
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)


@pytest.mark.parametrize("growth,batched", [("depthwise", True), ("depthwise", False), ("leafwise", True)])
def test_leaf_renewing_weighted_and_sampled(growth, batched):
    """Weighted quantiles (ties resolved in partition order) and renewing
    over the sampled rows only."""
    x, y = bst.synth.regression(5000, 10, 4, seed=43)
    w = (0.25 + np.random.default_rng(5).random(5000)).astype(np.float32)
    y = np.round(y * 4.0) / 4.0  # many tied residuals
    gm, om = _train_both(x, y, weights=w, objective=bst.Objective.pinball([0.3, 0.7]), n_estimators=3,
                         learning_rate=0.5, max_depth=4, growth_strategy=_strategy(growth), n_leaves=12,
                         batched=batched, subsample=0.6, metric=bst.Metric.none())
    compare_trees(gm, om, 5000)
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)


@pytest.mark.parametrize("objective", ["huber", "poisson", "hinge"])
def test_other_objectives_parity(objective):
    rng = np.random.default_rng(47)
    x, y = bst.synth.regression(6000, 10, 4, seed=47)
    if objective == "poisson":
        y = rng.poisson(np.exp(np.clip(y * 0.3, -2, 2))).astype(np.float32)
        obj = bst.Objective.poisson()
    elif objective == "hinge":
        y = (y > np.median(y)).astype(np.float32)
        obj = bst.Objective.hinge()
    else:
        obj = bst.Objective.huber(0.7)
    gm, om = _train_both(x, y, objective=obj, n_estimators=5, learning_rate=0.3, max_depth=5,
                         metric=bst.Metric.none())
    np.testing.assert_array_equal(gm.base_scores(), om.base_scores())
    tol = 1e-6 if objective == "poisson" else 1e-9  # exp
    compare_trees(gm, om, 6000, sum_rtol=tol, sum_atol=tol)


@pytest.mark.parametrize("growth,batched,precision", [("depthwise", True, "fp32"), ("depthwise", False, "fp32"),
                                                       ("depthwise", True, "q8"), ("leafwise", True, "fp32")])
def test_goss_parity(growth, batched, precision):
    """learning_rate 0.5: rounds 0-1 unsampled, GOSS from round 2 on."""
    x, y = bst.synth.binary(8000, 16, 3, seed=53)
    gm, om = _train_both(x, y, objective=bst.Objective.logistic(), n_estimators=5, learning_rate=0.5, max_depth=5,
                         growth_strategy=_strategy(growth), n_leaves=20, batched=batched, precision=precision,
                         goss_top_rate=0.2, goss_other_rate=0.1, min_samples_leaf=5, metric=bst.Metric.none())
    compare_trees(gm, om, 8000, sum_rtol=1e-6, sum_atol=1e-6)
    np.testing.assert_allclose(gm.train_predictions(), om.train_predictions(), rtol=REL, atol=1e-6)


def test_goss_with_renewing_l1():
    x, y = bst.synth.regression(6000, 10, 4, seed=59)
    gm, om = _train_both(x, y, objective=bst.Objective.absolute(), n_estimators=4, learning_rate=0.5, max_depth=4,
                         goss_top_rate=0.3, goss_other_rate=0.2, metric=bst.Metric.none())
    compare_trees(gm, om, 6000)


def test_default_metrics_and_early_stopping():
    """Default metrics of the new objectives (metrics/mod.rs:213-232) and
    the margin accuracy's higher-is-better early stopping."""
    x, y = bst.synth.regression(4000, 8, 4, seed=61)
    yb = (y > 0).astype(np.float32)
    xv, yv = bst.synth.regression(1000, 8, 4, seed=61, stream=1)
    ybv = (yv > 0).astype(np.float32)
    ds = bst.Dataset.from_feature_major(x, yb)
    dv = bst.Dataset.from_feature_major(xv, ybv)
    cfg = bst.GBDTConfig(objective=bst.Objective.hinge(), n_estimators=60, learning_rate=0.3, max_depth=3,
                         early_stopping_rounds=3)
    m = bst.GBDTModel.train(ds, cfg, val_set=dv)
    assert 0 < m.n_trees <= 60
    acc = bst.metric("margin_accuracy", m.predict_group_major(dv, raw=True), ybv)
    assert acc > 0.8, acc
    # pinball's default metric is the quantile loss of its alphas
    cfg = bst.GBDTConfig(objective=bst.Objective.pinball([0.2, 0.8]), n_estimators=8, learning_rate=0.3,
                         max_depth=3, early_stopping_rounds=50)
    m = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg,
                            val_set=bst.Dataset.from_feature_major(xv, yv))
    assert m.n_trees == 16
