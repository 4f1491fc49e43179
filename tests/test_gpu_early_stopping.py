"""Early stopping and validation evaluation (training/gbdt/trainer.rs:344-401,
callback.rs:103-136, eval.rs:218-271).

The engine's early-stopped model is checked against a replay of the
reference's rule in Python: the per-round metric comes from prefix models
(the first r rounds of a run without early stopping, cut through the
.bstr.json round trip) predicted on the same rows, so the values are the
ones the engine sees (same traversal, transform and metric code).
"""
import json

import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n


def expected_rounds(values, patience):
    """EarlyStopping::update (lower is better) and the trainer's truncation:
    returns (rounds run, rounds kept)."""
    best, best_round, cur, best_n = None, 0, 0, 0
    run = 0
    for r, v in enumerate(values):
        run = r + 1
        improved = best is None or v < best
        if improved:
            best, best_round = v, cur
        cur += 1
        if cur - best_round > patience:
            break
        if improved:
            best_n = r + 1
    kept = best_n if 0 < best_n < run else run
    return run, kept


def prefix_model(model, rounds, n_groups):
    doc = json.loads(model.to_json_bytes())
    f = doc["model"]["forest"]
    k = rounds * n_groups
    f["trees"] = f["trees"][:k]
    if "tree_groups" in f:
        f["tree_groups"] = f["tree_groups"][:k]
    return bst.GBDTModel.from_json_bytes(json.dumps(doc).encode())


def per_round_metric(full, rounds, n_groups, ds, labels, kind):
    out = []
    for r in range(1, rounds + 1):
        p = prefix_model(full, r, n_groups).predict_group_major(ds, raw=(kind == "rmse"))
        out.append(bst.metric(kind, p, labels))
    return out


def same_prefix(es, full):
    for i in range(es.n_trees):
        a, b = es.tree(i), full.tree(i)
        for k in ("split_index", "left", "right", "is_leaf", "split_bin"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"tree {i} {k}")
        np.testing.assert_array_equal(a["leaf_value"], b["leaf_value"], err_msg=f"tree {i} leaves")


CASES = {
    "regression": dict(objective=None, kind="rmse", groups=1, patience=3),
    "logistic": dict(objective="logistic", kind="logloss", groups=1, patience=2),
    "logistic_q8": dict(objective="logistic", kind="logloss", groups=1, patience=2, precision="q8"),
    "softmax": dict(objective="softmax", kind="mlogloss", groups=3, patience=2),
}


def _data(case):
    if case["objective"] is None:
        x, y = bst.synth.regression(600, 10, 3, seed=5)
        xv, yv = bst.synth.regression(600, 10, 3, seed=5, stream=1)
        return x, y, xv, yv, bst.Objective.squared()
    if case["objective"] == "logistic":
        x, y = bst.synth.binary(2000, 10, 2, seed=6)
        xv, yv = bst.synth.binary(2000, 10, 2, seed=6, stream=1)
        return x, y, xv, yv, bst.Objective.logistic()
    x, y = bst.synth.multiclass(3000, 8, 0, 3, seed=7)
    xv, yv = bst.synth.multiclass(3000, 8, 0, 3, seed=7, stream=1)
    return x, y, xv, yv, bst.Objective.softmax(3)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_early_stopping_matches_replay(name):
    case = CASES[name]
    x, y, xv, yv, obj = _data(case)
    ds = bst.Dataset.from_feature_major(x, y)
    dv = bst.Dataset.from_feature_major(xv, yv)
    kw = dict(objective=obj, n_estimators=40, max_depth=6, learning_rate=0.5,
              precision=case.get("precision", "fp32"), batched=case.get("precision") is not None)
    full = bst.GBDTModel.train(ds, bst.GBDTConfig(**kw))
    values = per_round_metric(full, 40, case["groups"], dv, yv, case["kind"])
    run, kept = expected_rounds(values, case["patience"])
    assert kept < run < 40, (values, run, kept)  # learning rate 0.5 overfits: the stop path runs
    es = bst.GBDTModel.train(ds, bst.GBDTConfig(early_stopping_rounds=case["patience"], **kw), val_set=dv)
    assert es.n_trees == kept * case["groups"], (values, run, kept)
    same_prefix(es, full)
    # the kept trees' training predictions, not the last round's
    np.testing.assert_allclose(es.train_predictions(),
                               prefix_model(full, kept, case["groups"]).predict_group_major(ds, raw=True),
                               rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_early_stopping_on_training_metric_without_validation_set():
    x, y = bst.synth.binary(2000, 10, 2, seed=6)
    ds = bst.Dataset.from_feature_major(x, y)
    kw = dict(objective=bst.Objective.logistic(), n_estimators=25, max_depth=4, learning_rate=0.3)
    full = bst.GBDTModel.train(ds, bst.GBDTConfig(**kw))
    values = per_round_metric(full, 25, 1, ds, y, "logloss")
    run, kept = expected_rounds(values, 2)
    es = bst.GBDTModel.train(ds, bst.GBDTConfig(early_stopping_rounds=2, **kw))
    assert es.n_trees == kept
    same_prefix(es, full)


@pytest.mark.gpu
def test_early_stopping_without_metric_keeps_the_first_round():
    # Metric::None gives NaN every round: the first round is the only
    # improvement, so training stops after patience + 1 rounds and keeps one
    x, y = bst.synth.regression(1000, 8, 3, seed=8)
    ds = bst.Dataset.from_feature_major(x, y)
    es = bst.GBDTModel.train(ds, bst.GBDTConfig(n_estimators=20, max_depth=3, early_stopping_rounds=3,
                                                metric=bst.Metric.none()))
    assert es.n_trees == 1
    assert expected_rounds([float("nan")] * 20, 3) == (4, 1)


def test_booster_rejects_early_stopping():
    x, y = bst.synth.regression(200, 4, 2, seed=1)
    ds = bst.Dataset.from_feature_major(x, y)
    with pytest.raises(n.BoostersError) as e:
        bst.Booster(ds, bst.GBDTConfig(early_stopping_rounds=3))
    assert e.value.status == n.BST_ERR_UNSUPPORTED


def test_validation_set_needs_targets():
    x, y = bst.synth.regression(200, 4, 2, seed=1)
    ds = bst.Dataset.from_feature_major(x, y)
    dv = bst.Dataset.from_feature_major(x)
    with pytest.raises(n.BoostersError) as e:
        bst.GBDTModel.train(ds, bst.GBDTConfig(early_stopping_rounds=3), val_set=dv)
    assert e.value.status == n.BST_ERR_MISSING_TARGETS


def test_replay_rule():
    # callback.rs tests: improving values never stop; a plateau stops after
    # `patience` more rounds and keeps the best round
    assert expected_rounds([5, 4, 3, 2, 1], 2) == (5, 5)
    assert expected_rounds([5, 4, 4.5, 4.2, 4.1, 3], 2) == (4, 2)
    assert expected_rounds([1, 2, 3], 1) == (2, 1)
