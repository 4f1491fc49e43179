"""bst_find_split_noalloc: the split search for callers that cannot allocate
device memory per call (device memory reserved by another allocator, or
latency-critical code that cannot pay for cudaMalloc/cudaFree). It must give
the same split as bst_find_split on the same histogram, call after call,
while its working memory is a fixed array inside the library; after its
first call on a device (which loads its code and the array), calls leave
the device's free memory unchanged.

Collected last (file name) so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import boosters_b200 as bst
from boosters_b200 import _native as n
import oracle_bridge as ob

pytestmark = pytest.mark.gpu


def _histogram(seed, n_bins, n_rows=20000):
    rng = np.random.default_rng(seed)
    hist = []
    for nb in n_bins:
        counts = rng.multinomial(n_rows, rng.dirichlet(np.ones(nb)))
        g = rng.normal(size=nb) * counts * 0.1 + 0.01 * counts
        h = counts * (0.05 + 0.2 * rng.random(nb))
        hist.append(np.stack([g, h], axis=1))
    hist = np.ascontiguousarray(np.concatenate(hist), dtype=np.float64)
    pg = float(hist[: n_bins[0], 0].sum())
    ph = float(hist[: n_bins[0], 1].sum())
    return hist, pg, ph, n_rows


def _call_reference_entry(hist, nb, ic, hm, pg, ph, pc, cfg, n_threads):
    s = n.Split()
    n.check(n.lib.bst_find_split(n.ptr(hist, ctypes.c_double), n.ptr(nb, ctypes.c_uint32), n.ptr(ic, ctypes.c_int32),
                                 n.ptr(hm, ctypes.c_int32), len(nb), pg, ph, pc, ctypes.byref(cfg), n_threads,
                                 ctypes.byref(s)))
    return s


def _call_noalloc(hist_dev, nb, ic, hm, pg, ph, pc, cfg, n_threads, stream):
    s = n.Split()
    rc = n.lib.bst_find_split_noalloc(ctypes.c_void_p(hist_dev.data_ptr()), n.ptr(nb, ctypes.c_uint32),
                                      n.ptr(ic, ctypes.c_int32), n.ptr(hm, ctypes.c_int32), len(nb), pg, ph, pc,
                                      ctypes.byref(cfg), n_threads, ctypes.c_void_p(stream), ctypes.byref(s))
    assert rc == n.BST_OK, rc
    return s


def _same(a, b):
    assert (a.gain > -np.inf) == (b.gain > -np.inf)
    for k in ("feature", "default_left", "is_categorical", "bin"):
        assert getattr(a, k) == getattr(b, k), k
    assert list(a.left_cats) == list(b.left_cats)
    np.testing.assert_allclose(a.gain, b.gain, rtol=1e-6)


def test_noalloc_split_matches_allocating_entry_twice():
    import torch

    # numeric columns (with and without a NaN bin) plus one-hot and sorted categoricals
    nb = np.array([256, 257, 64, 3, 40, 256, 17, 2] * 3, dtype=np.uint32)
    ic = np.array([0, 0, 0, 1, 1, 0, 0, 0] * 3, dtype=np.int32)
    hm = np.array([0, 1, 0, 0, 0, 1, 0, 0] * 3, dtype=np.int32)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (seed, n_threads, onehot) in enumerate([(1, 1, 4), (2, 0, 8)]):
        hist, pg, ph, pc = _histogram(seed, nb)
        cfg = bst.GBDTConfig(max_onehot_cats=onehot, min_child_weight=0.5).to_c()
        want = _call_reference_entry(hist, nb, ic, hm, pg, ph, pc, cfg, n_threads)
        hist_dev = torch.from_numpy(hist).cuda()
        got = _call_noalloc(hist_dev, nb, ic, hm, pg, ph, pc, cfg, n_threads, stream)
        assert want.gain > -np.inf, "the test histogram should have a valid split"
        _same(got, want)
        # and the CPU restatement of find.rs on the same histogram
        o = ob.find_split(hist, nb, ic, hm, pg, ph, pc, cfg, n_threads=n_threads)
        _same(got, o)


def test_noalloc_calls_leave_device_memory_unchanged():
    import torch

    nb = np.array([256, 257, 64, 3, 40, 17] * 4, dtype=np.uint32)
    ic = np.array([0, 0, 0, 1, 1, 0] * 4, dtype=np.int32)
    hm = np.array([0, 1, 0, 0, 0, 0] * 4, dtype=np.int32)
    cfg = bst.GBDTConfig(min_child_weight=0.5).to_c()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [_histogram(seed, nb) for seed in (5, 6, 7)]
    devs = [torch.from_numpy(h).cuda() for h, _, _, _ in cases]
    torch.cuda.synchronize()
    _call_noalloc(devs[0], nb, ic, hm, *cases[0][1:], cfg, 1, stream)  # first call on the device: loads code
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        for d, (_, pg, ph, pc) in zip(devs, cases):
            _call_noalloc(d, nb, ic, hm, pg, ph, pc, cfg, 1, stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    cfg = bst.GBDTConfig().to_c()
    nb = np.full(1025, 2, dtype=np.uint32)
    z = np.zeros(1025, dtype=np.int32)
    hist_dev = torch.zeros((2050, 2), dtype=torch.float64, device="cuda")
    s = n.Split()
    rc = n.lib.bst_find_split_noalloc(ctypes.c_void_p(hist_dev.data_ptr()), n.ptr(nb, ctypes.c_uint32),
                                      n.ptr(z, ctypes.c_int32), n.ptr(z, ctypes.c_int32), 1025, 0.0, 1.0, 10,
                                      ctypes.byref(cfg), 1, None, ctypes.byref(s))
    assert rc == n.BST_ERR_INVALID_ARGUMENT
    assert b"1024" in n.lib.bst_last_error()
    # 65,537 bins in all: one more than the array holds
    nb = np.array([256] * 256 + [1], dtype=np.uint32)
    z = np.zeros(len(nb), dtype=np.int32)
    hist_dev = torch.zeros((int(nb.sum()), 2), dtype=torch.float64, device="cuda")
    rc = n.lib.bst_find_split_noalloc(ctypes.c_void_p(hist_dev.data_ptr()), n.ptr(nb, ctypes.c_uint32),
                                      n.ptr(z, ctypes.c_int32), n.ptr(z, ctypes.c_int32), len(nb), 0.0, 1.0, 10,
                                      ctypes.byref(cfg), 1, None, ctypes.byref(s))
    assert rc == n.BST_ERR_INVALID_ARGUMENT
    assert b"65536" in n.lib.bst_last_error()


def test_noalloc_validation_matches_allocating_entry():
    import torch

    hist_dev = torch.zeros((600, 2), dtype=torch.float64, device="cuda")
    host = np.zeros((600, 2), np.float64)

    def both(nb, ic, hm, cfg):
        nb = np.asarray(nb, np.uint32)
        ic = np.asarray(ic, np.int32)
        hm = np.asarray(hm, np.int32)
        a, b = n.Split(), n.Split()
        ra = n.lib.bst_find_split(n.ptr(host, ctypes.c_double), n.ptr(nb, ctypes.c_uint32),
                                  n.ptr(ic, ctypes.c_int32), n.ptr(hm, ctypes.c_int32), len(nb), 0.0, 1.0, 10,
                                  ctypes.byref(cfg), 1, ctypes.byref(a))
        rb = n.lib.bst_find_split_noalloc(ctypes.c_void_p(hist_dev.data_ptr()), n.ptr(nb, ctypes.c_uint32),
                                          n.ptr(ic, ctypes.c_int32), n.ptr(hm, ctypes.c_int32), len(nb), 0.0, 1.0,
                                          10, ctypes.byref(cfg), 1, None, ctypes.byref(b))
        return ra, rb, a, b

    ok = bst.GBDTConfig().to_c()
    # no features: no candidate
    ra, rb, a, b = both(np.zeros(0), np.zeros(0), np.zeros(0), ok)
    assert ra == rb == n.BST_OK and a.gain == b.gain == -np.inf
    # a categorical feature above 256 bins
    ra, rb, _, _ = both([300], [1], [0], ok)
    assert ra == rb == n.BST_ERR_UNSUPPORTED
    # the configuration is validated as bst_find_split validates it
    for field, value in (("learning_rate", 0.0), ("n_trees", 0), ("subsample", 1.5), ("lambda_", -1.0)):
        bad = bst.GBDTConfig().to_c()
        setattr(bad, field, value)
        ra, rb, _, _ = both([16], [0], [0], bad)
        assert ra == rb == n.BST_ERR_CONFIG, field
