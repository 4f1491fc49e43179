"""Trained models through .bstr and .bstr.json and back: identical tree
arrays and bit-identical predictions (host and served)."""
import numpy as np
import pytest

import boosters_b200 as bst

pytestmark = pytest.mark.gpu

KEYS = ["split_index", "threshold", "left", "right", "default_left", "is_leaf", "leaf_value", "split_type",
        "seg_size", "cat_words"]


def models():
    x, y = bst.synth.binary(20_000, 16, n_nan_cols=4, seed=21)
    yield "logistic", bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), bst.GBDTConfig(
        objective=bst.Objective.logistic(), n_estimators=30, max_depth=6, precision="q8", batched=True)), x
    xr, yr = bst.synth.regression(5_000, 20, 5, seed=22)
    yield "squared", bst.GBDTModel.train(bst.Dataset.from_feature_major(xr, yr), bst.GBDTConfig(
        n_estimators=20, max_depth=5)), xr
    xm, ym = bst.synth.multiclass(8_000, 6, 3, 4, seed=23)
    yield "softmax", bst.GBDTModel.train(bst.Dataset.from_feature_major(xm, ym, categorical_features=[6, 7, 8]),
                                         bst.GBDTConfig(objective=bst.Objective.softmax(4), n_estimators=5,
                                                        max_depth=4)), xm


@pytest.mark.parametrize("fmt", ["bstr", "json"])
def test_round_trip_predicts_identically(fmt, tmp_path):
    for name, m, x in models():
        path = tmp_path / (f"{name}.bstr.json" if fmt == "json" else f"{name}.bstr")
        m.save(path)
        back = bst.GBDTModel.load(path)
        assert (back.n_trees, back.n_groups, back.n_features) == (m.n_trees, m.n_groups, m.n_features)
        for i in range(m.n_trees):
            a, b = m.tree(i), back.tree(i)
            assert a["group"] == b["group"]
            for k in KEYS:
                if k in ("seg_size", "cat_words") and not a["split_type"].any():
                    continue
                leaf = a["is_leaf"].astype(bool)
                va, vb = a[k], b[k]
                if k in ("split_index", "threshold", "left", "right", "default_left", "split_type"):
                    va, vb = va[~leaf], vb[~leaf]  # leaves carry no split in the file
                if k == "leaf_value":
                    va, vb = va[leaf], vb[leaf]
                np.testing.assert_array_equal(va, vb, err_msg=f"{name} tree {i} {k}")
        ds = bst.Dataset.from_feature_major(x)
        for raw in (False, True):
            np.testing.assert_array_equal(back.predict_group_major(ds, raw=raw), m.predict_group_major(ds, raw=raw))
        rows = np.ascontiguousarray(x[:, :3000].T)
        srv = bst.PredictionServer(back, raw=True)
        try:
            out = srv.wait(srv.submit(rows))
        finally:
            srv.close()
        np.testing.assert_array_equal(out, m.predict_group_major(bst.Dataset(rows), raw=True))
