"""scikit-learn estimators (packages/boosters-python/python/boosters/sklearn/
gbdt.py) and feature importance (explainability/importance.rs:199-270)."""
import json

import numpy as np
import pytest
from sklearn.base import clone

import boosters_b200 as bst
from boosters_b200.sklearn import GBDTClassifier, GBDTRegressor


def _two_tree_model():
    """tree 0: f0 split (gain 2, cover 10) then f1 split (gain 1, cover 4);
    tree 1: f1 split (gain 3, cover 8)."""
    def tree(splits):
        # splits: list of (feature, gain, cover) on a left spine
        k = len(splits)
        n = 2 * k + 1
        left, right = [0] * n, [0] * n
        feat, gains, covers = [0] * n, [0.0] * n, [0.0] * n
        node = 0
        for i, (f, g, c) in enumerate(splits):
            left[node], right[node] = 2 * i + 1, 2 * i + 2
            feat[node], gains[node], covers[node] = f, g, c
            node = 2 * i + 1
        return {"num_nodes": n, "split_indices": feat, "thresholds": [0.5] * n, "children_left": left,
                "children_right": right, "default_left": [False] * n,
                "leaf_values": {"type": "scalar", "values": [0.0] * n}, "gains": gains, "covers": covers}
    model = {"meta": {"num_features": 3, "num_groups": 1},
             "forest": {"trees": [tree([(0, 2.0, 10.0), (1, 1.0, 4.0)]), tree([(1, 3.0, 8.0)])], "n_groups": 1,
                        "base_score": [0.0]},
             "output_transform": "identity"}
    doc = {"bstr_version": 2, "model_type": "gbdt", "model": model}
    return bst.GBDTModel.from_json_bytes(json.dumps(doc).encode())


def test_feature_importance_kinds():
    m = _two_tree_model()
    T = bst.ImportanceType
    np.testing.assert_array_equal(m.feature_importance(T.Split), np.float32([1, 2, 0]))
    np.testing.assert_array_equal(m.feature_importance(T.Gain), np.float32([2, 4, 0]))
    np.testing.assert_array_equal(m.feature_importance(T.AverageGain), np.float32([2, 2, 0]))
    np.testing.assert_array_equal(m.feature_importance(T.Cover), np.float32([10, 12, 0]))
    np.testing.assert_array_equal(m.feature_importance(T.AverageCover), np.float32([10, 6, 0]))


def test_params_clone_and_validation():
    r = GBDTRegressor(n_estimators=7, max_depth=3)
    c = clone(r)
    assert c.get_params()["n_estimators"] == 7 and c.get_params()["max_depth"] == 3
    assert r.set_params(learning_rate=0.2).learning_rate == 0.2
    X = np.zeros((10, 2), np.float32)
    y = np.arange(10) % 2
    with pytest.raises(ValueError, match="cannot train"):
        GBDTRegressor(objective=bst.Objective.logistic()).fit(X, y)
    with pytest.raises(ValueError, match="cannot train"):
        GBDTClassifier(objective=bst.Objective.squared()).fit(X, y)
    with pytest.raises(ValueError, match="labels"):
        GBDTClassifier().fit(X, y, eval_set=(X, y + 5))


@pytest.mark.gpu
def test_regressor_matches_core_api():
    x, y = bst.synth.regression(3000, 12, 4, seed=3)
    X = np.ascontiguousarray(x.T)
    est = GBDTRegressor(n_estimators=20, max_depth=5, learning_rate=0.2).fit(X, y)
    core = bst.GBDTModel.train(bst.Dataset(X, y), bst.GBDTConfig(
        n_estimators=20, max_depth=5, learning_rate=0.2, metric=bst.Metric.rmse()))
    np.testing.assert_array_equal(est.predict(X), core.predict(bst.Dataset(X))[:, 0])
    assert est.score(X, y) > 0.5  # RegressorMixin R^2
    imp = est.feature_importances_
    assert imp.shape == (12,) and imp.sum() > 0


@pytest.mark.gpu
def test_classifier_binary_and_multiclass_labels():
    x, y = bst.synth.binary(3000, 10, 0, seed=4)
    X = np.ascontiguousarray(x.T)
    names = np.where(y > 0.5, "yes", "no")
    clf = GBDTClassifier(n_estimators=15, max_depth=4, learning_rate=0.3).fit(X, names)
    assert list(clf.classes_) == ["no", "yes"]
    proba = clf.predict_proba(X)
    assert proba.shape == (3000, 2)
    np.testing.assert_allclose(proba.sum(axis=1), 1.0, rtol=1e-6)
    pred = clf.predict(X)
    assert set(pred) <= {"no", "yes"} and (pred == names).mean() > 0.6

    xm, ym = bst.synth.multiclass(3000, 8, 0, 3, seed=5)
    Xm = np.ascontiguousarray(xm.T)
    labels = np.array([10, 20, 30])[ym.astype(int)]
    mc = GBDTClassifier(n_estimators=10, max_depth=4).fit(Xm, labels)
    assert mc.n_classes_ == 3 and mc.model_.n_groups == 3
    pm = mc.predict_proba(Xm)
    np.testing.assert_allclose(pm.sum(axis=1), 1.0, rtol=1e-5)
    np.testing.assert_array_equal(mc.predict(Xm), np.array([10, 20, 30])[np.argmax(pm, axis=1)])


@pytest.mark.gpu
def test_classifier_eval_set_early_stopping():
    x, y = bst.synth.binary(2000, 10, 0, seed=6)
    xv, yv = bst.synth.binary(2000, 10, 0, seed=6, stream=1)
    X, Xv = np.ascontiguousarray(x.T), np.ascontiguousarray(xv.T)
    clf = GBDTClassifier(n_estimators=40, max_depth=6, learning_rate=0.5, early_stopping_rounds=2)
    clf.fit(X, y, eval_set=(Xv, yv))
    core = bst.GBDTModel.train(bst.Dataset(X, y), bst.GBDTConfig(
        objective=bst.Objective.logistic(), n_estimators=40, max_depth=6, learning_rate=0.5,
        early_stopping_rounds=2, metric=bst.Metric.logloss()), val_set=bst.Dataset(Xv, yv))
    assert clf.model_.n_trees == core.n_trees <= 40
