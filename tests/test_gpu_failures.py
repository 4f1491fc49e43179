"""Error paths of the C ABI, driven from the host (nothing here faults, traps
or hangs a GPU): a server wait that runs out of time, a server budget below
one row per slot, and device allocations refused by the library's device
memory cap (BST_DEVICE_MEMORY_LIMIT), each returning its status code with a
message and leaving the process and the library usable."""
import os
import subprocess
import sys

import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def deep_model():
    x, y = bst.synth.binary(20_000, 50, 5, seed=17)
    cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=400, max_depth=8, learning_rate=0.1,
                         precision="q8", batched=True)
    return bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)


def test_server_wait_timeout_leaves_ticket_valid(deep_model):
    import torch

    rows_n = 60_000
    srv = bst.PredictionServer(deep_model, raw=True)
    try:
        xs, _ = bst.synth.binary(rows_n, 50, 5, seed=17, stream=3)
        rows = torch.from_numpy(np.ascontiguousarray(xs.T)).pin_memory().numpy()
        # eight large requests queue behind one another: the last one is still
        # pending when the zero-timeout wait asks for it
        tickets = [srv.submit(rows) for _ in range(8)]
        with pytest.raises(n.BoostersError) as ei:
            srv.wait(tickets[-1], timeout_ms=0)
        assert ei.value.status == n.BST_ERR_TIMEOUT
        assert "timeout" in str(ei.value)
        want = deep_model.predict_group_major(bst.Dataset(rows), raw=True)
        for t in tickets:  # the timed-out ticket is still valid
            np.testing.assert_array_equal(srv.wait(t), want)
        assert srv.stats()["completed"] == 8
    finally:
        srv.close()


def test_server_budget_below_one_row_per_slot(deep_model):
    with pytest.raises(n.BoostersError) as ei:
        bst.PredictionServer(deep_model, mem_budget_bytes=64)
    assert ei.value.status == n.BST_ERR_INVALID_ARGUMENT
    assert "budget" in str(ei.value)
    srv = bst.PredictionServer(deep_model)  # the library is still usable
    srv.close()


def test_device_memory_cap_refuses_allocations_without_abort():
    """In a child process with BST_DEVICE_MEMORY_LIMIT set: training whose
    buffers pass the cap fails with BST_ERR_OUT_OF_MEMORY (no cudaMalloc is
    attempted), a smaller training under the cap then succeeds in the same
    process, and the process exits normally."""
    code = r"""
import sys
sys.path.insert(0, sys.argv[1])
import boosters_b200 as bst
from boosters_b200 import _native as n
x, y = bst.synth.binary(4_000_000, 40, 4, seed=5)  # ~400 MB of binned rows
cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=3, max_depth=6)
try:
    bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)
    print("no error")
except n.BoostersError as e:
    print("status", e.status, "BST_DEVICE_MEMORY_LIMIT" in str(e))
xs, ys = bst.synth.binary(2_000, 8, 0, seed=5)
m = bst.GBDTModel.train(bst.Dataset.from_feature_major(xs, ys), cfg)
print("small ok", m.n_trees)
"""
    env = dict(os.environ, BST_DEVICE_MEMORY_LIMIT=str(256 << 20))
    r = subprocess.run([sys.executable, "-c", code, ROOT], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    assert f"status {n.BST_ERR_OUT_OF_MEMORY} True" in lines, r.stdout
    assert "small ok 3" in lines, r.stdout
