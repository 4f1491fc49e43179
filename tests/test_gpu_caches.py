"""Buffer reuse between training calls: the device block cache and the pinned
host block cache hand the same memory to consecutive calls (their contents
are whatever the previous call left), so consecutive calls, calls after
bst_release_cached_memory, and calls of a different shape in between must
all give the same trees as the first call."""
import numpy as np
import pytest

import boosters_b200 as bst

pytestmark = pytest.mark.gpu


def _trees(m):
    out = []
    for i in range(m.n_trees):
        t = m.tree(i)
        out.append({k: np.asarray(t[k]).copy() for k in ("split_index", "split_bin", "left", "right", "is_leaf",
                                                          "leaf_value", "threshold")})
    return out


def _same(a, b):
    assert len(a) == len(b)
    for ta, tb in zip(a, b):
        for k in ta:
            np.testing.assert_array_equal(ta[k], tb[k], err_msg=k)


@pytest.mark.parametrize("precision", ["q8", "fp32"])
def test_reused_buffers_give_identical_models(precision):
    x, y = bst.synth.binary(60_000, 30, n_nan_cols=5, seed=21)
    cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=12, max_depth=7, learning_rate=0.2,
                         precision=precision, batched=True)
    first = _trees(bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg))
    _same(first, _trees(bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)))
    # a call of another shape takes (and dirties) the cached blocks
    xo, yo = bst.synth.binary(90_000, 45, n_nan_cols=3, seed=22)
    bst.GBDTModel.train(bst.Dataset.from_feature_major(xo, yo), cfg)
    _same(first, _trees(bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)))
    bst.release_cached_memory()
    _same(first, _trees(bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)))


def test_leafwise_after_depthwise_reuses_pinned_state():
    x, y = bst.synth.binary(40_000, 20, n_nan_cols=2, seed=23)
    lw = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=6,
                        growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=31,
                        learning_rate=0.2, precision="q16", batched=True)
    dw = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=6, max_depth=6, learning_rate=0.2,
                        precision="q16", batched=True)
    first = _trees(bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), lw))
    bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), dw)
    _same(first, _trees(bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), lw)))
