"""Launch-shape autotuning of the batched depth-wise pipeline: every
candidate shape grows bit-identical trees (so exploring on a run's own
first trees changes no result), the winner is kept in the cache file, and a
second run reads it instead of exploring."""
import numpy as np
import pytest

import boosters_b200 as bst
from test_gpu_parity import STRUCT_KEYS

pytestmark = pytest.mark.gpu

CANDIDATES = [f"items={i},hist={h},grid=8" for i, h in ((2, 0), (1, 0), (2, 1), (2, 2), (2, 3))] + [
    "items=2,hist=0,grid=4"]


def _trees(m):
    return [m.tree(i) for i in range(m.n_trees)]


def _same_trees(a, b):
    assert len(a) == len(b)
    for ta, tb in zip(a, b):
        for k in STRUCT_KEYS + ["threshold", "leaf_value", "gain", "grad_sum", "hess_sum"]:
            np.testing.assert_array_equal(ta[k], tb[k], err_msg=k)


@pytest.mark.parametrize("precision", ["fp32", "q8"])
def test_every_shape_grows_the_same_trees(tmp_path, precision):
    x, y = bst.synth.binary(120_000, 40, 8, seed=9)
    ds = bst.Dataset.from_feature_major(x, y)
    cache = tmp_path / "tune.txt"
    kw = dict(objective=bst.Objective.logistic(), n_estimators=20, max_depth=7, learning_rate=0.2,
              precision=precision, batched=True)
    explored = bst.GBDTModel.train(ds, bst.GBDTConfig(autotune=True, autotune_cache=cache, **kw))
    info = explored.tune_info
    assert "(explored:" in info, info
    assert all(c in info for c in CANDIDATES), info
    lines = cache.read_text().strip().split("\n")
    assert len(lines) == 1
    key, best = lines[0].split("\t")
    assert info.startswith(best)
    ref = _trees(explored)
    # a second run reads the cache
    again = bst.GBDTModel.train(ds, bst.GBDTConfig(autotune=True, autotune_cache=cache, **kw))
    assert again.tune_info == best + " (cached)"
    _same_trees(_trees(again), ref)
    # each candidate forced through the cache grows the same trees
    for shape in CANDIDATES:
        cache.write_text(f"{key}\t{shape}\n")
        m = bst.GBDTModel.train(ds, bst.GBDTConfig(autotune=True, autotune_cache=cache, **kw))
        assert m.tune_info == shape + " (cached)"
        _same_trees(_trees(m), ref)
    builtin = bst.GBDTModel.train(ds, bst.GBDTConfig(autotune=False, **kw))
    assert builtin.tune_info.endswith("(built-in)")
    _same_trees(_trees(builtin), ref)


def test_cache_with_unknown_or_bad_lines_is_ignored(tmp_path):
    x, y = bst.synth.binary(30_000, 16, 2, seed=10)
    ds = bst.Dataset.from_feature_major(x, y)
    cache = tmp_path / "tune.txt"
    cache.write_text("some other key\titems=1,hist=0,grid=4\nbroken line without tab\n")
    kw = dict(objective=bst.Objective.logistic(), n_estimators=24, max_depth=5, precision="q8", batched=True)
    m = bst.GBDTModel.train(ds, bst.GBDTConfig(autotune=True, autotune_cache=cache, **kw))
    assert "(explored:" in m.tune_info
    text = cache.read_text()
    assert "some other key\titems=1,hist=0,grid=4" in text  # other entries kept
    key = [ln for ln in text.split("\n") if ln and not ln.startswith("some other")][-1].split("\t")[0]
    cache.write_text(f"{key}\titems=oops\n")  # unparsable shape: explore again
    m2 = bst.GBDTModel.train(ds, bst.GBDTConfig(autotune=True, autotune_cache=cache, **kw))
    assert "(explored:" in m2.tune_info
