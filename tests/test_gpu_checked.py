"""The bounds-checked library (libboosters_b200_checked.so, built with
-DBST_CHECKED) against the normal one on the GPU.

Its kernels test every index read from device memory (row ids of the
histogram gather and leaf update, partition chunks and scatter destinations,
leaf chunks, traversal node links) before the access; a violation is counted
and the access skipped, and bst_gbdt_train returns BST_ERR_CHECK. A child
process loads the checked library (BST_LIBRARY=checked), trains the growth
forms — plain FP32, batched depth-wise Q8 and FP32, batched leaf-wise Q16,
softmax with categorical columns — and predicts; the test asserts that no
check failed and that trees and predictions equal the normal library's.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import boosters_b200 as bst

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "boosters_b200", "libboosters_b200_checked.so")

CASES = {
    "plain_fp32": dict(batched=False, precision="fp32", max_depth=6),
    "batched_q8": dict(batched=True, precision="q8", max_depth=7),
    "batched_fp32": dict(batched=True, precision="fp32", max_depth=7),
    "leafwise_q16": dict(batched=True, precision="q16", growth="leafwise", n_leaves=63),
    "softmax_cat": dict(batched=True, precision="q8", max_depth=5, softmax=4),
}

CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import tests.test_gpu_checked as t
from boosters_b200 import _native as n
assert n.LIB_PATH.endswith("libboosters_b200_checked.so"), n.LIB_PATH
out = {}
for name in t.CASES:
    trees, pred = t.run_case(name)
    v, site, idx, bound = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
    rc = n.lib.bst_check_report(0, ctypes.byref(v), ctypes.byref(site), ctypes.byref(idx), ctypes.byref(bound))
    out[name] = dict(trees=trees, pred=pred.tolist(), rc=rc, violations=v.value, site=site.value,
                     index=idx.value, bound=bound.value)
json.dump(out, open(sys.argv[2], "w"))
"""


def run_case(name):
    """Trains and predicts one case; returns (tree fields, predictions)."""
    c = dict(CASES[name])
    if "softmax" in c:
        x, y = bst.synth.multiclass(12000, n_numeric=12, n_categorical=4, n_classes=c.pop("softmax"), seed=5)
        cats = list(range(12, 16))
        obj = bst.Objective.softmax(int(y.max()) + 1)
    else:
        x, y = bst.synth.binary(20000, 24, n_nan_cols=4, seed=13)
        cats = []
        obj = bst.Objective.logistic()
    kw = dict(objective=obj, n_estimators=4, learning_rate=0.3, device=0, batched=c["batched"],
              precision=c["precision"])
    if c.get("growth") == "leafwise":
        kw.update(growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=c["n_leaves"])
    else:
        kw.update(max_depth=c["max_depth"])
    ds = bst.Dataset.from_feature_major(x, y, categorical_features=cats)
    m = bst.GBDTModel.train(ds, bst.GBDTConfig(**kw), n_threads=1, record_leaves=True)
    trees = []
    for i in range(m.n_trees):
        t = m.tree(i)
        d = {k: np.asarray(t[k]).tolist() for k in ("split_index", "split_bin", "left", "right", "default_left",
                                                    "is_leaf", "split_type", "cat_words")}
        d["leaf_value"] = np.asarray(t["leaf_value"], np.float64).tolist()
        d["rows"] = np.asarray(m.tree_row_leaves(i, len(y))).tolist()
        trees.append(d)
    return trees, np.asarray(m.predict_group_major(ds), np.float64).ravel()


@pytest.fixture(scope="module")
def checked_results(tmp_path_factory):
    if not os.path.exists(CHECKED):
        pytest.fail("libboosters_b200_checked.so is not built (python -m boosters_b200.build --checked)")
    out = tmp_path_factory.mktemp("checked") / "out.json"
    env = dict(os.environ, BST_LIBRARY="checked")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(out)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return json.load(open(out))


@pytest.mark.parametrize("name", list(CASES))
def test_checked_build_matches_and_records_nothing(checked_results, name):
    got = checked_results[name]
    assert got["rc"] == 0, got
    assert got["violations"] == 0, (f"{name}: {got['violations']} bounds violations, first at site {got['site']}: "
                                    f"index {got['index']} bound {got['bound']}")
    trees, pred = run_case(name)
    assert len(trees) == len(got["trees"])
    for i, (a, b) in enumerate(zip(trees, got["trees"])):
        for k in a:
            assert a[k] == b[k], f"{name} tree {i}: {k} differs between the normal and the checked build"
    np.testing.assert_array_equal(pred, np.asarray(got["pred"]))
