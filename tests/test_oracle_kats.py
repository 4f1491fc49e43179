"""Pins the CPU restatement (oracle/) to the reference's own unit-test
known answers (tests/golden/kats.json, transcribed from the Rust tests)."""
import math

import numpy as np
import pytest

import oracle_bridge as ob
from boosters_b200 import GBDTConfig, GrowthStrategy


def _f(v):
    return float(v)


def test_value_to_bin(kats):
    for case in kats["value_to_bin"]:
        cats = case.get("cats")
        bounds = None if cats is not None else [_f(b) for b in case["bounds"]]
        for v, want in zip(case["values"], case["bins"]):
            got = ob.value_to_bin(bounds, case["missing"], case["default_bin"], _f(v), cats=cats)
            assert got == want, (case["src"], v, got, want)


def test_gain(kats):
    for c in kats["gain"]:
        g = ob.lib.orc_gain_full(c["gl"], c["hl"], c["gr"], c["hr"], c["gp"], c["hp"], c["lambda"], c["min_gain"])
        assert abs(g - c["expect"]) < c["tol"], c["src"]


def test_valid_split(kats):
    for c in kats["valid_split"]:
        got = ob.lib.orc_is_valid_split(c["hl"], c["hr"], c["cl"], c["cr"], c["mcw"], c["msl"])
        assert bool(got) == c["expect"], c["src"]


def test_leaf_weight(kats):
    for c in kats["leaf_weight"]:
        w = ob.lib.orc_leaf_weight(c["g"], c["h"], c["lambda"], c["alpha"])
        assert abs(w - c["expect"]) <= c["tol"], c["src"]


def test_histogram(kats):
    for c in kats["histogram"]:
        h = ob.histogram_build(np.array(c["bins"]), c["n_bins"], c["grad"], c["hess"], c["rows"])
        np.testing.assert_allclose(h, np.array(c["expect"]), atol=1e-10, err_msg=c["src"])
    c = kats["histogram_multi"][0]
    n, F, nb = c["n"], c["n_features"], c["n_bins"]
    bins = np.array([[(i + k) % nb for i in range(n)] for k in range(F)])
    h = ob.histogram_build(bins, [nb] * F, np.arange(n, dtype=np.float32), np.ones(n, np.float32))
    assert abs(h[0, 0] - c["expect_f0_bin0_grad"]) < 1e-10


def test_find_split(kats):
    for c in kats["find_split"]:
        cfg = GBDTConfig(max_onehot_cats=c["max_onehot_cats"]).to_c()
        s = ob.find_split(np.array(c["hist"], dtype=np.float64), c["n_bins"], c["is_cat"], c["has_missing"],
                          c["pg"], c["ph"], c["pc"], cfg)
        valid = s.gain > -math.inf
        assert valid == c["expect_valid"], c["src"]
        if valid:
            assert s.feature == c["expect_feature"], c["src"]
            if c.get("expect_categorical"):
                assert s.is_categorical == 1, c["src"]
            for cat in c.get("expect_left_contains", []):
                assert (s.left_cats[cat >> 6] >> (cat & 63)) & 1, c["src"]


def test_objectives(kats):
    for c in kats["objective"]:
        g, h = ob.gradients(c["objective"], np.array(c["preds"]), c["y"], c["w"], alpha=c.get("alpha"),
                            delta=c.get("delta", 1.0))
        if c["grad"] is not None:
            np.testing.assert_allclose(g, np.array(c["grad"]), atol=c["tol"], err_msg=c["src"])
        if c["hess"] is not None:
            np.testing.assert_allclose(h, np.array(c["hess"]), atol=c["tol"], err_msg=c["src"])
    for c in kats["base_score"]:
        b = ob.base_score(c["objective"], c["n_outputs"], c["y"])
        np.testing.assert_allclose(b, c["expect"], atol=c["tol"], err_msg=c["src"])


def test_leaf_quantile(kats):
    for c in kats["leaf_quantile"]:
        got = ob.leaf_quantile(c["values"], c["weights"], c["alpha"])
        if c["expect"] == "nan":
            assert np.isnan(got), c["src"]
        else:
            assert abs(got - c["expect"]) < 1e-6, c["src"]


def test_softmax_gradient_signs():
    # training/objectives/classification.rs:300-341 softmax_gradient
    preds = np.array([[1.0, 0.0], [0.0, 1.0], [0.0, 0.0]], np.float32)
    g, _ = ob.gradients(2, preds, [0.0, 1.0])
    assert g[0, 0] < 0 and g[1, 0] > 0


def test_partition(kats):
    for c in kats["partition"]:
        x = np.array(c["features"], np.float32)
        b = ob.OracleBinned(x, GBDTConfig().to_c())
        bins = b.column_bins(c["split_feature"])
        left = [i for i in range(x.shape[1]) if bins[i] <= 0]
        assert left == c["expect_left_rows"], c["src"]


def test_threshold_translation(kats):
    # grower.rs:812-842: threshold = next_up(f32(upper)); the boundary value goes left
    c = kats["threshold_translation"][0]
    x = np.array([c["values"]], np.float32)
    grad = np.array([-1.0, 1.0], np.float32)
    cfg = GBDTConfig(max_depth=1, min_child_weight=0.0, learning_rate=1.0).to_c()
    m = ob.OracleModel.grow(x, grad, np.ones(2, np.float32), cfg)
    t = m.tree(0)
    assert not t["is_leaf"][0]
    upper = np.float32(c["upper"])
    assert t["threshold"][0] > upper
    assert t["threshold"][0] == np.nextafter(upper, np.float32(np.inf))
    p = m.predict(np.array([[upper, t["threshold"][0]]], np.float32), raw=True)[0]
    assert p[0] == t["leaf_value"][t["left"][0]] and p[1] == t["leaf_value"][t["right"][0]]


def test_traversal(kats):
    for c in kats["traversal"]:
        tree = {"split_index": [0, 0, 0], "threshold": [c["threshold"], 0, 0], "left": [1, 0, 0],
                "right": [2, 0, 0], "default_left": [1 if c["default_left"] else 0, 0, 0], "is_leaf": [0, 1, 1],
                "leaf_value": [0.0, 1.0, 2.0], "split_type": [0, 0, 0]}
        m = ob.OracleModel.from_trees(1, [tree])
        x = np.array([[float(v) for v in c["values"]]], np.float32)
        np.testing.assert_array_equal(m.predict(x, raw=True)[0], np.array(c["expect"], np.float32), c["src"])


def test_categorical_traversal():
    # grower.rs:844-876 / traversal.rs cat(0, [1, 3]): categories 1 and 3 go right in the stored bitset
    tree = {"split_index": [0, 0, 0], "threshold": [0, 0, 0], "left": [1, 0, 0], "right": [2, 0, 0],
            "default_left": [1, 0, 0], "is_leaf": [0, 1, 1], "leaf_value": [0.0, 10.0, 20.0],
            "split_type": [1, 0, 0], "seg_start": [0, 0, 0], "seg_size": [1, 0, 0], "cat_words": [0b1010]}
    m = ob.OracleModel.from_trees(1, [tree])
    p = m.predict(np.array([[0.0, 1.0, 2.0, 3.0, np.nan]], np.float32), raw=True)[0]
    np.testing.assert_array_equal(p, [10.0, 20.0, 10.0, 20.0, 10.0])


def test_grower(kats):
    for c in kats["grower"]:
        x = np.array([c["values"]], np.float32)
        cfg = GBDTConfig(max_depth=c["max_depth"]).to_c()
        m = ob.OracleModel.grow(x, c["grad"], c["hess"], cfg)
        t = m.tree(0)
        assert int(t["is_leaf"].sum()) == c["expect_leaves"], c["src"]


def test_categorical_grow_bitset_is_bin_indices():
    # grower.rs:844-876: categorical splits store category indices, children swapped
    x = np.array([[0.0, 1.0, 2.0, 3.0] * 5], np.float32)
    grad = np.array([1.0, -1.0, 1.0, -1.0] * 5, np.float32)
    cfg = GBDTConfig(max_depth=1, min_child_weight=0.0, max_onehot_cats=1).to_c()
    ob_m = ob.OracleModel.grow(x, grad, np.ones(20, np.float32), cfg)
    t = ob_m.tree(0)
    assert int(t["is_leaf"].sum()) == 2


def test_leafwise_and_depthwise_shapes():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(5, 400)).astype(np.float32)
    g = rng.normal(size=400).astype(np.float32)
    h = np.ones(400, np.float32)
    cfg = GBDTConfig(growth_strategy=GrowthStrategy.Leafwise, n_leaves=7).to_c()
    t = ob.OracleModel.grow(x, g, h, cfg).tree(0)
    assert int(t["is_leaf"].sum()) <= 7
    cfg = GBDTConfig(max_depth=3).to_c()
    t = ob.OracleModel.grow(x, g, h, cfg).tree(0)
    assert int(t["is_leaf"].sum()) <= 8


def test_parallel_tie_semantics():
    # find.rs:219-270: with >= 16 candidate features the rayon reduction keeps the
    # LAST of equally good features; sequential search keeps the FIRST.
    n, F = 64, 20
    col = np.repeat(np.arange(4, dtype=np.float32), n // 4)
    x = np.tile(col, (F, 1))
    g = np.where(col < 2, -1.0, 1.0).astype(np.float32)
    h = np.ones(n, np.float32)
    cfg = GBDTConfig(max_depth=1).to_c()
    seq = ob.OracleModel.grow(x, g, h, cfg, n_threads=1).tree(0)
    par = ob.OracleModel.grow(x, g, h, cfg, n_threads=0).tree(0)
    assert seq["split_index"][0] == 0
    assert par["split_index"][0] == F - 1


def test_sparse_feature_is_rejected():
    # a column with density <= 0.1 goes to sparse storage in the reference
    # (feature_analysis.rs:408-410), which neither implementation supports
    x = np.zeros((2, 100), np.float32)
    x[0] = np.arange(100)
    x[1, :5] = 1.0
    with pytest.raises(RuntimeError, match="sparse"):
        ob.OracleBinned(x, GBDTConfig().to_c())


# ---- row-sampling generator (training/sampling/row.rs) ------------------------
# The engine and the oracle each restate rand 0.8's SmallRng (Xoshiro256++
# seeded by SplitMix64) and gen_range(0..=i); these check the oracle's copy
# against values derived from the published algorithms and against a third,
# pure-Python statement of the reservoir sampler.

M64 = (1 << 64) - 1


def _rotl(v, k):
    return ((v << k) | (v >> (64 - k))) & M64


class _PySampler:
    def __init__(self, seed):
        self.s = []
        for _ in range(4):
            seed = (seed + 0x9E3779B97F4A7C15) & M64
            z = ((seed ^ (seed >> 30)) * 0xBF58476D1CE4E5B9) & M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
            self.s.append(z ^ (z >> 31))

    def next(self):
        s = self.s
        r = (_rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
        t = (s[1] << 17) & M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        return r

    def range_inclusive(self, high):
        rng = high + 1
        zone = ((rng << (64 - rng.bit_length())) & M64) - 1
        while True:
            m = self.next() * rng
            if (m & M64) <= zone:
                return m >> 64

    def sample(self, n, rate):
        k = min(max(int(np.float32(n) * np.float32(rate)), 1), n)
        idx = list(range(k))
        for i in range(k, n):
            j = self.range_inclusive(i)
            if j < k:
                idx[j] = i
        mask = np.zeros(n, np.uint8)
        mask[idx] = 1
        return mask


def test_xoshiro256pp_known_answers():
    import ctypes
    state = (ctypes.c_uint64 * 4)(1, 2, 3, 4)
    out = (ctypes.c_uint64 * 3)()
    ob.lib.orc_xoshiro256pp(state, 3, out)
    # rotl(1 + 4, 23) + 1, then the second step worked by hand
    assert list(out) == [41943041, 58720359, 3588806011781223]
    assert _PySampler(0).s[0] == 0xE220A8397B1DCDAF  # SplitMix64(0), first output


@pytest.mark.parametrize("n,rate,seed", [(50, 0.2, 42), (1000, 0.5, 7), (333, 0.9, 0), (10, 0.01, 3)])
def test_row_sampler_matches_python_statement(n, rate, seed):
    import ctypes
    draws = 3
    masks = np.zeros((draws, n), np.uint8)
    ob.lib.orc_row_sample(ctypes.c_uint64(seed), ctypes.c_uint64(n), ctypes.c_float(rate), draws,
                          masks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    py = _PySampler(seed)
    for d in range(draws):
        want = py.sample(n, rate)
        np.testing.assert_array_equal(masks[d], want, err_msg=f"draw {d}")
        assert masks[d].sum() == min(max(int(np.float32(n) * np.float32(rate)), 1), n)
