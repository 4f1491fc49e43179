"""The continuous-batching prediction server: every request's result equals
the plain per-request predict bit for bit, whether it ran alone or coalesced
with concurrent requests; admission respects the memory budget. The served
forests go through the shared-memory heap traversal (depth <= 8) or, for
deeper trees, the node-list traversal; both must match the plain predict."""
import threading

import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model():
    x, y = bst.synth.binary(30_000, 24, n_nan_cols=6, seed=7)
    cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=60, learning_rate=0.2, max_depth=6)
    return bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)


def plain_predict(model, rows, raw=False):
    return model.predict_group_major(bst.Dataset(rows), raw=raw)


def request_rows(rng, n_rows, F):
    r = rng.normal(size=(n_rows, F)).astype(np.float32)
    r[rng.random(size=r.shape) < 0.05] = np.nan
    return r


@pytest.mark.parametrize("raw", [False, True])
def test_alone_and_in_the_mix_are_identical(model, raw):
    rng = np.random.default_rng(1)
    F = model.n_features
    sizes = [1, 2, 7, 100, 1000, 4096, 33, 65536, 5, 777]
    reqs = [request_rows(rng, s, F) for s in sizes]
    want = [plain_predict(model, r, raw) for r in reqs]
    srv = bst.PredictionServer(model, mem_budget_bytes=64 << 20, raw=raw)
    try:
        # alone: submit and wait one at a time
        alone = [srv.wait(srv.submit(r)).copy() for r in reqs]
        # in the mix: everything queued at once from several threads
        tickets = [None] * len(reqs)

        def go(k0):
            for k in range(k0, len(reqs), 3):
                tickets[k] = srv.submit(reqs[k])

        th = [threading.Thread(target=go, args=(k,)) for k in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    for a, b, w in zip(alone, mixed, want):
        np.testing.assert_array_equal(a, w)
        np.testing.assert_array_equal(b, w)
    assert st["completed"] == 2 * len(reqs)
    assert st["batches"] < 2 * len(reqs)  # concurrent requests were coalesced


def test_many_small_requests_stream(model):
    rng = np.random.default_rng(2)
    F = model.n_features
    pool = request_rows(rng, 20_000, F)
    want = plain_predict(model, pool)
    srv = bst.PredictionServer(model, mem_budget_bytes=16 << 20)
    try:
        ts, spans = [], []
        for _ in range(400):
            a = int(rng.integers(0, 20_000))
            b = min(20_000, a + int(np.exp(rng.uniform(0, np.log(2000)))))
            ts.append(srv.submit(pool[a:b]))
            spans.append((a, b))
        for t, (a, b) in zip(ts, spans):
            np.testing.assert_array_equal(srv.wait(t), want[:, a:b])
            assert t.done_ns >= t.submit_ns > 0
        st = srv.stats()
    finally:
        srv.close()
    assert st["submitted"] == st["completed"] == 400
    assert st["max_rows_seen"] <= st["max_batch_rows"]


def test_softmax_groups_and_categorical_splits():
    x, y = bst.synth.multiclass(8_000, 10, 3, 4, seed=4)
    m = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y, categorical_features=[10, 11, 12]),
                            bst.GBDTConfig(objective=bst.Objective.softmax(4), n_estimators=5, max_depth=4))
    rows = np.ascontiguousarray(x[:, :3000].T)
    srv = bst.PredictionServer(m)
    try:
        out = srv.wait(srv.submit(rows))
    finally:
        srv.close()
    np.testing.assert_array_equal(out, m.predict_group_major(bst.Dataset(rows)))


def test_budget_admission_limits(model):
    F = model.n_features
    per_row = (F + model.n_groups) * 4
    srv = bst.PredictionServer(model, mem_budget_bytes=3 * per_row * 100)  # under 100-row batches
    try:
        cap = srv.stats()["max_batch_rows"]
        assert 20 <= cap <= 100  # input, output and bin-tile bytes per row share the budget
        with pytest.raises(n.BoostersError, match="exceeds"):
            srv.submit(np.zeros((cap + 1, F), np.float32))
        rng = np.random.default_rng(3)
        k = cap // 2 + 1
        rows = [request_rows(rng, k, F) for _ in range(10)]
        ts = [srv.submit(r) for r in rows]
        outs = [srv.wait(t) for t in ts]
        st = srv.stats()
    finally:
        srv.close()
    for r, o in zip(rows, outs):
        np.testing.assert_array_equal(o, plain_predict(model, r))
    assert st["max_rows_seen"] <= cap  # two requests of over half a batch never share one
    with pytest.raises(n.BoostersError, match="budget"):
        bst.PredictionServer(model, mem_budget_bytes=per_row)


def test_wait_errors(model):
    srv = bst.PredictionServer(model)
    try:
        t = srv.submit(np.zeros((10, model.n_features), np.float32))
        srv.wait(t)
        with pytest.raises(n.BoostersError, match="ticket"):
            srv.wait(t)  # already retired
    finally:
        srv.close()


def test_deep_trees_use_the_node_list_traversal():
    # leaves deeper than the heap's 8 levels: the node-list kernel serves them
    x, y = bst.synth.binary(20_000, 16, n_nan_cols=4, seed=9)
    m = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y),
                            bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=8, max_depth=11,
                                           growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=200))
    rows = np.ascontiguousarray(x[:, :5000].T)
    srv = bst.PredictionServer(m)
    try:
        out = srv.wait(srv.submit(rows))
    finally:
        srv.close()
    np.testing.assert_array_equal(out, m.predict_group_major(bst.Dataset(rows)))


def test_values_on_the_thresholds(model):
    # the served traversal bins rows against the forest's own thresholds:
    # values equal to a threshold, one ulp either side, signed zeros,
    # infinities and NaN must all go the way x < threshold sends them
    F = model.n_features
    thr = [[] for _ in range(F)]
    for i in range(model.n_trees):
        t = model.tree(i)
        for k in np.flatnonzero(t["is_leaf"] == 0):
            thr[t["split_index"][k]].append(t["threshold"][k])
    rng = np.random.default_rng(5)
    cols = []
    for f in range(F):
        v = np.asarray(thr[f] or [0.0], np.float32)
        cand = np.concatenate([v, np.nextafter(v, np.float32(-np.inf)), np.nextafter(v, np.float32(np.inf)),
                               np.array([0.0, -0.0, np.inf, -np.inf, np.nan], np.float32)])
        cols.append(rng.choice(cand, size=5000))
    rows = np.ascontiguousarray(np.stack(cols, axis=1).astype(np.float32))
    srv = bst.PredictionServer(model, raw=True)
    try:
        out = srv.wait(srv.submit(rows))
    finally:
        srv.close()
    np.testing.assert_array_equal(out, plain_predict(model, rows, raw=True))


def test_large_category_ids():
    x, y = bst.synth.multiclass(6_000, 6, 2, 3, seed=8)
    m = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y, categorical_features=[6, 7]),
                            bst.GBDTConfig(objective=bst.Objective.softmax(3), n_estimators=4, max_depth=5))
    rows = np.ascontiguousarray(x[:, :2000].T).copy()
    rng = np.random.default_rng(6)
    rows[rng.random(2000) < 0.2, 6] = 70000.0   # beyond any category set
    rows[rng.random(2000) < 0.2, 7] = -3.0      # negative category -> 0
    rows[rng.random(2000) < 0.1, 7] = 2.7       # fractional category truncates
    srv = bst.PredictionServer(m, raw=True)
    try:
        out = srv.wait(srv.submit(rows))
    finally:
        srv.close()
    np.testing.assert_array_equal(out, m.predict_group_major(bst.Dataset(rows), raw=True))


def test_u16_bin_columns():
    # more than 255 distinct thresholds on a feature: the traversal bins rows
    # into u16 columns; both missing-value directions occur
    x, y = bst.synth.binary(40_000, 12, n_nan_cols=6, seed=10)
    m = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y),
                            bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=120, max_depth=7,
                                           max_bins=1024, learning_rate=0.3))
    n_thr = max(len(np.unique(np.concatenate(
        [m.tree(i)["threshold"][(m.tree(i)["is_leaf"] == 0) & (m.tree(i)["split_index"] == f)]
         for i in range(m.n_trees)]))) for f in range(12))
    assert n_thr > 255
    rows = np.ascontiguousarray(x[:, :20_000].T)
    srv = bst.PredictionServer(m, raw=True)
    try:
        out = srv.wait(srv.submit(rows))
    finally:
        srv.close()
    np.testing.assert_array_equal(out, m.predict_group_major(bst.Dataset(rows), raw=True))


def test_replay_schedule(model):
    rng = np.random.default_rng(12)
    F = model.n_features
    pool = request_rows(rng, 50_000, F)
    n_req = 300
    sizes = np.clip(np.floor(np.exp(rng.uniform(0, np.log(4097), n_req))).astype(np.int64), 1, 4096)
    offs = rng.integers(0, 50_000 - 4096, n_req)
    arrival = np.cumsum(rng.exponential(1 / 20_000, n_req))
    want = plain_predict(model, pool, raw=True)
    srv = bst.PredictionServer(model, raw=True)
    try:
        lat, span, out = srv.replay(pool, arrival, offs, sizes, ring=n_req)
        with pytest.raises(n.BoostersError, match="pool"):
            srv.replay(pool, [0.0], [49_999], [2])
        st = srv.stats()
    finally:
        srv.close()
    for i in range(n_req):
        np.testing.assert_array_equal(out[i, :, :sizes[i]], want[:, offs[i]:offs[i] + sizes[i]])
    assert (lat > 0).all() and span >= arrival[-1] - arrival[0]
    assert st["completed"] == n_req


def test_small_ring_wraps(model):
    # an input ring of three small batches: requests of random sizes wrap
    # around it many times while earlier batches are still in flight
    F = model.n_features
    per_row = (F + model.n_groups) * 4
    rng = np.random.default_rng(13)
    pool = request_rows(rng, 20_000, F)
    want = plain_predict(model, pool)
    srv = bst.PredictionServer(model, mem_budget_bytes=3 * per_row * 100)
    try:
        cap = srv.stats()["max_batch_rows"]
        spans, ts = [], []
        for _ in range(300):
            k = int(rng.integers(1, cap + 1))
            a = int(rng.integers(0, 20_000 - k))
            ts.append(srv.submit(pool[a:a + k]))
            spans.append((a, k))
        outs = [srv.wait(t) for t in ts]
    finally:
        srv.close()
    for (a, k), o in zip(spans, outs):
        np.testing.assert_array_equal(o, want[:, a:a + k])


def test_device_resident_requests(model):
    # rows already in device memory: same results, no host copy of the rows
    import torch
    rng = np.random.default_rng(14)
    F = model.n_features
    host = request_rows(rng, 30_000, F)
    dev = torch.from_numpy(host).cuda()
    want = plain_predict(model, host, raw=True)
    srv = bst.PredictionServer(model, raw=True)
    try:
        spans = [(0, 1), (5, 700), (1000, 25_000), (29_000, 1000)]
        ts = [srv.submit(dev[a:a + k]) for a, k in spans]
        outs = [srv.wait(t).copy() for t in ts]
        dout = torch.empty((model.n_groups, 500), dtype=torch.float32, device="cuda")
        srv.wait(srv.submit(dev[100:600], out=dout))
        n_req = 200
        sizes = rng.integers(1, 3000, n_req)
        offs = rng.integers(0, 27_000, n_req)
        lat, span, ring = srv.replay(dev, np.cumsum(rng.exponential(1 / 20_000, n_req)), offs, sizes, ring=n_req)
    finally:
        srv.close()
    for (a, k), o in zip(spans, outs):
        np.testing.assert_array_equal(o, want[:, a:a + k])
    np.testing.assert_array_equal(dout.cpu().numpy(), want[:, 100:600])
    for i in range(n_req):
        np.testing.assert_array_equal(ring[i, :, :sizes[i]], want[:, offs[i]:offs[i] + sizes[i]])


def test_phase_trace(model):
    """Every completed request leaves one phase record (in completion order,
    which is submission order); copies of host rows take device time and the
    copied bytes add up to the rows sent."""
    rng = np.random.default_rng(5)
    F = model.n_features
    sizes = [3, 4000, 65536, 17, 900]
    srv = bst.PredictionServer(model)
    try:
        srv.trace()
        st0 = srv.stats()
        tickets = [srv.submit(request_rows(rng, s, F)) for s in sizes]
        for t in tickets:
            srv.wait(t)
        tr = srv.trace()
        st1 = srv.stats()
    finally:
        srv.close()
    cols = dict(zip(n.SERVER_PHASES, tr.T))
    assert cols["rows"].tolist() == sizes
    assert (cols["batch_rows"] >= cols["rows"]).all()
    big = cols["rows"] >= 900  # event resolution is about 0.5 us
    assert (cols["copy_ns"][big] > 0).all() and (cols["kernel_ns"] > 0).all()
    assert st1["h2d_bytes"] - st0["h2d_bytes"] == sum(sizes) * F * 4
    assert st1["h2d_ns"] - st0["h2d_ns"] == int(cols["copy_ns"].sum())
