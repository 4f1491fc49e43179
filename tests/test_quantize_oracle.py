"""The oracle's quantised-gradient mode (the engine's Q16 / Q8 training; the
reference trains on f32 gradients only, so there is no reference vector for
the rounding itself).

Philox4x32-10 is pinned to the known-answer vectors published with the
Random123 library of Salmon, Moraes, Dror and Shaw ("Parallel Random
Numbers: As Easy as 1, 2, 3", SC 2011); the stochastic rounding is checked
through its defining properties.
"""
import numpy as np
import pytest

import oracle_bridge as ob
from boosters_b200 import GBDTConfig, GrowthStrategy, Objective, synth
from boosters_b200 import _native as n

PHILOX_KAT = [
    # (counter, key, output)
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    np.testing.assert_array_equal(ob.philox4x32_10(ctr, key), np.array(want, np.uint32))


@pytest.mark.parametrize("precision,qmax", [(n.PRECISION_Q8, 127), (n.PRECISION_Q16, 32767)])
def test_stochastic_rounding_properties(precision, qmax):
    rng = np.random.default_rng(3)
    g = rng.normal(size=20000).astype(np.float32)
    h = rng.uniform(1e-6, 0.25, size=20000).astype(np.float32)
    g[:7] = 0.0
    qg, qh, steps = ob.quantize(g, h, precision, seed=42, rnd=5)
    mg, mh = np.abs(g).max(), np.abs(h).max()
    assert steps[0] == qmax / np.float64(mg) and steps[2] == np.float64(mg) / qmax
    assert steps[1] == qmax / np.float64(mh) and steps[3] == np.float64(mh) / qmax
    for q, v, inv in ((qg, g, steps[0]), (qh, h, steps[1])):
        assert np.abs(q).max() <= qmax
        x = v.astype(np.float64) * inv
        # floor(x + u), u in [0, 1): one of the two integers around x
        assert np.all((q == np.floor(x)) | (q == np.floor(x) + 1))
    assert np.all(qg[:7] == 0)
    # same (seed, round, output) -> same integers; another round -> another draw
    qg2, qh2, _ = ob.quantize(g, h, precision, seed=42, rnd=5)
    np.testing.assert_array_equal(qg, qg2)
    np.testing.assert_array_equal(qh, qh2)
    qg3, _, _ = ob.quantize(g, h, precision, seed=42, rnd=6)
    assert np.any(qg3 != qg)
    qg4, _, _ = ob.quantize(g, h, precision, seed=42, rnd=5, output=1)
    assert np.any(qg4 != qg)


def test_stochastic_rounding_is_unbiased():
    # E[floor(x + u)] = x: the mean over rounds converges to the value
    v = np.full(4000, 0.3, np.float32)
    v[0] = 1.0  # max |v| -> step 1/127
    acc = np.zeros(4000)
    rounds = 64
    for r in range(rounds):
        q, _, steps = ob.quantize(v, v, n.PRECISION_Q8, seed=7, rnd=r)
        acc += q * steps[2]
    est = acc[1:].mean() / rounds
    assert abs(est - 0.3) < 2e-4


def test_zero_gradients_quantise_to_zero():
    z = np.zeros(100, np.float32)
    qg, qh, steps = ob.quantize(z, z, n.PRECISION_Q8, seed=1, rnd=0)
    assert not qg.any() and not qh.any()
    np.testing.assert_array_equal(steps, np.zeros(4))


def _logistic_data(n_rows, seed):
    return synth.binary(n_rows, 12, n_nan_cols=4, seed=seed)


@pytest.mark.parametrize("precision", ["q16", "q8"])
@pytest.mark.parametrize("growth", ["depth", "leaf"])
def test_quantised_oracle_training_tracks_f32(precision, growth):
    x, y = _logistic_data(6000, 11)
    kw = dict(objective=Objective.logistic(), n_estimators=30, learning_rate=0.2, max_depth=5)
    if growth == "leaf":
        kw.update(growth_strategy=GrowthStrategy.Leafwise, n_leaves=24)
    base = ob.OracleModel(x, y, GBDTConfig(**kw).to_c())
    quant = ob.OracleModel(x, y, GBDTConfig(precision=precision, **kw).to_c())
    pb = 1.0 / (1.0 + np.exp(-base.train_predictions()[0].astype(np.float64)))
    pq = 1.0 / (1.0 + np.exp(-quant.train_predictions()[0].astype(np.float64)))
    ll = lambda p: -np.mean(y * np.log(np.clip(p, 1e-15, 1)) + (1 - y) * np.log(np.clip(1 - p, 1e-15, 1)))
    assert abs(ll(pq) - ll(pb)) / ll(pb) < (0.01 if precision == "q16" else 0.03)
    # leaves are solved from the f32 gradients: grad_sum of a leaf is a sum of
    # f32 values, not a multiple of the quantisation step
    t = quant.tree(0)
    assert np.isfinite(t["leaf_value"]).all()
