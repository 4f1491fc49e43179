"""Metric parity (training/metrics/regression.rs, classification.rs) between
the library's host-side evaluation (bst_metric_ex, used for per-round
metrics and early stopping) and the oracle, on seeded inputs; no GPU."""
import numpy as np
import pytest

import boosters_b200 as bst
import oracle_bridge as ob
from boosters_b200 import _native as n

CASES = [("mae", n.METRIC_MAE, 2), ("mape", n.METRIC_MAPE, 1), ("huber", n.METRIC_HUBER, 1),
         ("poisson", n.METRIC_POISSON, 1), ("margin_accuracy", n.METRIC_MARGIN_ACCURACY, 1),
         ("quantile", n.METRIC_QUANTILE, 3), ("rmse", n.METRIC_RMSE, 2)]


@pytest.mark.parametrize("kind,code,G", CASES)
@pytest.mark.parametrize("weighted", [False, True])
def test_metric_matches_oracle(kind, code, G, weighted):
    rng = np.random.default_rng(7)
    nrow = 5000
    p = rng.normal(size=(G, nrow)).astype(np.float32)
    if kind == "poisson":
        p = np.exp(p * 0.5).astype(np.float32)
        y = rng.poisson(1.5, nrow).astype(np.float32)
    elif kind == "margin_accuracy":
        y = (rng.random(nrow) > 0.5).astype(np.float32)
    else:
        y = rng.normal(size=nrow).astype(np.float32)
    w = (0.5 + rng.random(nrow)).astype(np.float32) if weighted else None
    alpha = [0.1, 0.5, 0.9] if kind == "quantile" else None
    got = bst.metric(kind, p, y, w, alpha=alpha, delta=0.8)
    want = ob.metric(code, p, y, w, alpha=alpha, delta=0.8)
    assert got == want, (got, want)


def test_quantile_metric_needs_alphas():
    with pytest.raises(n.BoostersError):
        bst.metric("quantile", np.zeros((2, 4), np.float32), np.zeros(4, np.float32), alpha=[0.5])
