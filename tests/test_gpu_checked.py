"""The bounds-checked library (libboosters_b200_checked.so, built with
-DBST_CHECKED) against the normal one on the GPU.

Its kernels test every index read from device memory (row ids of the
histogram gather and leaf update, partition chunks and scatter destinations,
leaf chunks, traversal node links) before the access; a violation is counted
and the access skipped, and bst_gbdt_train returns BST_ERR_CHECK. A child
process loads the checked library (BST_LIBRARY=checked), trains the growth
forms — plain FP32, batched depth-wise Q8 and FP32, batched leaf-wise Q16,
softmax with categorical columns, and the 1,000,000 x 100 depth-8 Q8
headline workload — and predicts; the test asserts that no
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
    # the benchmark's headline workload: 1,000,000 x 100 logistic, depth 8, Q8
    "headline_q8_1Mx100": dict(batched=True, precision="q8", max_depth=8, rows=1_000_000, features=100,
                               nan_cols=20, trees=3, lr=0.1),
}

CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import tests.test_gpu_checked as t
from boosters_b200 import _native as n
assert n.LIB_PATH.endswith("libboosters_b200_checked.so"), n.LIB_PATH
report = {}
for name in t.CASES:
    np.savez(f"{sys.argv[2]}/{name}.npz", **t.run_case(name))
    v, site, idx, bound = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
    rc = n.lib.bst_check_report(0, ctypes.byref(v), ctypes.byref(site), ctypes.byref(idx), ctypes.byref(bound))
    report[name] = dict(rc=rc, violations=v.value, site=site.value, index=idx.value, bound=bound.value)
json.dump(report, open(f"{sys.argv[2]}/report.json", "w"))
"""


def run_case(name):
    """Trains and predicts one case; returns its trees' fields (each tree's
    arrays concatenated), per-row leaves and predictions."""
    c = dict(CASES[name])
    if "softmax" in c:
        x, y = bst.synth.multiclass(12000, n_numeric=12, n_categorical=4, n_classes=c.pop("softmax"), seed=5)
        cats = list(range(12, 16))
        obj = bst.Objective.softmax(int(y.max()) + 1)
    else:
        x, y = bst.synth.binary(c.get("rows", 20000), c.get("features", 24), n_nan_cols=c.get("nan_cols", 4),
                                seed=13)
        cats = []
        obj = bst.Objective.logistic()
    kw = dict(objective=obj, n_estimators=c.get("trees", 4), learning_rate=c.get("lr", 0.3), device=0,
              batched=c["batched"], precision=c["precision"])
    if c.get("growth") == "leafwise":
        kw.update(growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=c["n_leaves"])
    else:
        kw.update(max_depth=c["max_depth"])
    ds = bst.Dataset.from_feature_major(x, y, categorical_features=cats)
    m = bst.GBDTModel.train(ds, bst.GBDTConfig(**kw), n_threads=1, record_leaves=True)
    keys = ("split_index", "split_bin", "left", "right", "default_left", "is_leaf", "split_type", "cat_words",
            "leaf_value")
    out = {k: np.concatenate([np.asarray(m.tree(i)[k]).ravel() for i in range(m.n_trees)]) for k in keys}
    out["n_nodes"] = np.array([m.tree(i)["n_nodes"] for i in range(m.n_trees)])
    out["rows"] = np.concatenate([np.asarray(m.tree_row_leaves(i, len(y))).ravel() for i in range(m.n_trees)])
    out["pred"] = np.asarray(m.predict_group_major(ds)).ravel()
    return out


@pytest.fixture(scope="module")
def checked_dir(tmp_path_factory):
    if not os.path.exists(CHECKED):
        pytest.fail("libboosters_b200_checked.so is not built (python -m boosters_b200.build --checked)")
    out = tmp_path_factory.mktemp("checked")
    env = dict(os.environ, BST_LIBRARY="checked")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(out)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_checked_build_matches_and_records_nothing(checked_dir, name):
    got = json.load(open(checked_dir / "report.json"))[name]
    assert got["rc"] == 0, got
    assert got["violations"] == 0, (f"{name}: {got['violations']} bounds violations, first at site {got['site']}: "
                                    f"index {got['index']} bound {got['bound']}")
    ref = run_case(name)
    chk = np.load(checked_dir / f"{name}.npz")
    assert set(chk.files) == set(ref)
    for k, v in ref.items():
        np.testing.assert_array_equal(chk[k], v, err_msg=f"{name}: {k} differs between the normal and the checked "
                                                         "build")
