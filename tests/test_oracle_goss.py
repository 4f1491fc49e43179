"""The oracle's GOSS restatement (sampling/row.rs:214-280) on the CPU:
the sample's shape (every row at or above the |grad x hess| threshold kept,
about other_rate x n of the rest, those scaled by (n - top) / other), the
warm-up rounds (floor(1 / learning_rate)) growing the unsampled trees, and
the generator stream advancing across calls."""
import numpy as np

import oracle_bridge as ob
from boosters_b200 import GBDTConfig, Objective, synth


def test_goss_sample_shape():
    rng = np.random.default_rng(3)
    n = 10_000
    g = rng.normal(size=n).astype(np.float32)
    h = (0.1 + rng.random(n)).astype(np.float32)
    mask, k, g2, h2 = ob.goss(g, h, 0.2, 0.1, seed=42)
    mag = np.abs(g * h)
    top_k = int(np.float32(n) * np.float32(0.2))
    other_k = int(np.float32(n) * np.float32(0.1))
    thr = np.sort(mag)[n - top_k]
    big = mag >= thr
    assert mask[big].all()
    small = mask.astype(bool) & ~big
    assert k == int(mask.sum()) == big.sum() + small.sum()
    assert abs(int(small.sum()) - other_k) <= 1  # the adaptive probability lands on other_k
    mult = np.float32(n - top_k) / np.float32(other_k)
    np.testing.assert_array_equal(g2[small], g[small] * mult)
    np.testing.assert_array_equal(h2[small], h[small] * mult)
    np.testing.assert_array_equal(g2[~small], g[~small])
    # a second call on the same sampler draws from further along the stream
    m2, _, _, _ = ob.goss(g, h, 0.2, 0.1, seed=42, calls=2)
    assert (m2 != mask).any()


def test_goss_warmup_then_sampling():
    x, y = synth.binary(3000, 8, 0, seed=5)
    base = dict(objective=Objective.logistic(), n_estimators=4, learning_rate=0.5, max_depth=4)
    plain = ob.OracleModel(x, y, GBDTConfig(**base).to_c())
    goss = ob.OracleModel(x, y, GBDTConfig(goss_top_rate=0.2, goss_other_rate=0.1, **base).to_c())
    for t in range(2):  # rounds 0 and 1: warm-up, no sampling
        np.testing.assert_array_equal(plain.tree(t)["leaf_value"], goss.tree(t)["leaf_value"])
    assert any(not np.array_equal(plain.tree(t)["leaf_value"], goss.tree(t)["leaf_value"]) for t in (2, 3))
