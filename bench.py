"""Benchmark of the B200 GBDT engine.

Workload (one GPU): binary logistic GBDT on a 1,000,000 x 100 f32 matrix
(even columns N(0,1), odd U(0,1), 10% NaN on 20 columns, label from 10
pairwise products), depth 8, 256 bins, lr 0.1, FP32 grad/hess — the
reference's plain-GBDT GPU configuration. Data are seeded synthetic.

A step is one boosting round (one tree) on the GPU-resident binned matrix;
`value` is seconds per 100 trees over the whole job (all GPUs). `e2e` is the
same metric through the public C-ABI train call from host buffers (dataset
copy, H2D, binning, 100 trees, D2H of the training predictions).
With --gpus N (torchrun) every rank trains an independent replica on its own
row stream (training does not shard; no collective on the data path).

The other survey workloads (5k x 100 regression, 10M x 200 leaf-wise
logistic, 2M x 50 softmax with categorical columns) are timed after the
headline in every form, each with its held-out loss and equal-loss flag
(`configs`; --no-configs skips them).

--impl reference times the CPU restatement of the reference's path (the Rust
crate cannot be built here), compiled -O3 -march=native on the host that runs
it, with all host threads, rank 0 only; that process loads no engine library.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "train s/100 trees, predict rows/s, p99 serve ms vs plain GPU at equal loss"
UNIT = "s/100 trees"
E2E_UNIT = "s/100 trees (from host arrays, binning included)"
N_ROWS, N_FEAT, N_NAN, SEED = 1_000_000, 100, 20, 2
WORKLOAD = "binary-logistic GBDT 1,000,000x100 f32 (20 NaN cols), depth 8, 256 bins, lr 0.1, 500 trees"
DTYPES = {"plain": "f32 grad/hess, int64 fixed-point histograms",
          "batched_fp32": "f32 grad/hess, int64 fixed-point histograms",
          "batched_q16": "int16 grad/hess (stochastic rounding), integer histograms, f64 leaf solves",
          "batched_q8": "int8 grad/hess (stochastic rounding), integer histograms, f64 leaf solves"}


def cfg_kwargs():
    import boosters_b200 as bst
    return dict(objective=bst.Objective.logistic(), n_estimators=500, learning_rate=0.1, max_depth=8, max_bins=256,
                metric=bst.Metric.none())


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        # scalar barriers and maxima only (no data-path collective): gloo
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, elapsed_s, steps):
    """s/100 trees of the whole job: N replicas each grew `steps` trees; the
    job took the slowest rank's device time."""
    return 100.0 * reduce_max(world, elapsed_s) / (steps * world)


def oracle_native():
    """Build the CPU restatement at -O3 -march=native for this host (once per
    host CPU) and point the checker bridge at it. Returns a description of
    the build. Must run before `oracle_bridge` is imported."""
    import hashlib
    sig_src = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    sig_src += line
                if line.strip() == "":
                    break
    except OSError:
        pass
    sig = hashlib.sha1(sig_src.encode()).hexdigest()[:12]
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "native", f"NATIVE_DIR=_native/{sig}"],
                       capture_output=True, text=True)
    lib = os.path.join(ROOT, "oracle", "_native", sig, "liboracle.so")
    if r.returncode == 0 and os.path.exists(lib):
        os.environ["BST_ORACLE_LIB"] = lib
        return "g++ -O3 -march=native -fopenmp (built on this host)"
    return "g++ -O3 -fopenmp (portable build; the host-tuned build failed)"


def cpu_rounds(ob, n_rounds, n_threads, x, y, cfg):
    """The CPU restatement on one workload: (per-tree seconds, binning
    seconds). n_threads=0: the reference's default parallel semantics."""
    m = ob.OracleModel(x, y, cfg, n_threads=0, record_leaves=False, omp_threads=n_threads, max_trees=n_rounds)
    return ([ob.lib.orc_model_tree_seconds(m._h, t) for t in range(m.n_trees)],
            ob.lib.orc_model_binning_seconds(m._h))


def bounded_cpu_rounds(ob, budget_s, max_rounds, n_threads, x, y, cfg):
    """1 warm-up round plus as many timed rounds (at most max_rounds) as
    about budget_s of CPU work allows. Returns (timed per-tree seconds,
    binning seconds)."""
    probe, _ = cpu_rounds(ob, 1, n_threads, x, y, cfg)
    k = max(1, min(max_rounds, int(budget_s / max(probe[0], 1e-3))))
    secs, bin_s = cpu_rounds(ob, 1 + k, n_threads, x, y, cfg)
    return secs[1:], bin_s


def oracle_cfg(ob):
    return ob.config(objective=1, n_trees=500, learning_rate=0.1, max_depth=8, max_bins=256, metric=0)


def run_reference(args, world, rank):
    if rank != 0:
        return
    build = oracle_native()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bridge as ob  # noqa: E402  (after BST_ORACLE_LIB is set)
    x, y = ob.synth.binary(N_ROWS, N_FEAT, N_NAN, seed=SEED, stream=0)
    cores = os.cpu_count() or 1
    timed, bin_s = bounded_cpu_rounds(ob, 60.0, args.steps, cores, x, y, oracle_cfg(ob))
    per_tree = sum(timed) / len(timed)
    v = 100.0 * per_tree
    sample = (f"1 warm-up + {len(timed)} timed boosting rounds (of {args.steps} asked) of the {N_ROWS}x{N_FEAT} "
              f"workload, binning excluded, {cores} threads; {build}")
    e2e = bin_s + v
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * per_tree, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": "cpu threads"},
            "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": round(e2e, 4), "unit": E2E_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "includes": f"binning from host arrays ({bin_s:.2f} s, measured) + 100 trees at the timed "
                                f"per-tree rate"}}
    print(json.dumps(line), flush=True)


PLAIN = dict(precision="fp32", batched=False)  # the reference's control flow on the GPU
FORMS = [  # (name, GBDTConfig overrides); "plain" is the reference form on the GPU
    ("plain", PLAIN),
    ("batched_fp32", dict(precision="fp32", batched=True)),
    ("batched_q16", dict(precision="q16", batched=True)),
    ("batched_q8", dict(precision="q8", batched=True)),
]
EQUAL_LOSS_REL = 1e-3


TUNE_CACHE = os.path.join(__import__("tempfile").gettempdir(), f"bst_bench_autotune_{os.getpid()}.txt")


def tune_form(bst, ds, cfg):
    """Launch-shape tuning of one form before it is timed: a throwaway
    booster explores the candidate shapes on its first trees and stores the
    winner in the run's cache file, which the timed booster then reads (so
    no candidate is explored inside the timed region)."""
    import copy
    if not cfg.batched or bst.GrowthStrategy(cfg.growth_strategy) == bst.GrowthStrategy.Leafwise:
        return ""  # the tuned pipeline is the batched depth-wise one
    c = copy.copy(cfg)
    c.autotune, c.autotune_cache = True, TUNE_CACHE
    c.n_estimators = 24  # more than the exploration's 2 trees per candidate + 1
    b = bst.Booster(ds, c, n_threads=0)
    rounds = 0
    while "(explored" not in b.model().tune_info and rounds < 64:
        b.update(4)
        rounds += 4
    return b.model().tune_info


def run_form(bst, torch, ds, xv, yv, cfg, args, world):
    """W warm-up rounds, K timed rounds (one update call, device events),
    then the rest of the configured trees; held-out logloss of the result."""
    tuned = tune_form(bst, ds, cfg)
    cfg.autotune_cache = TUNE_CACHE
    booster = bst.Booster(ds, cfg, n_threads=0)
    booster.update(args.warmup)
    t0, c0 = booster.stats()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    booster.update(args.steps)  # returns with the engine's stream idle
    ev1.record()
    ev1.synchronize()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    t1, c1 = booster.stats()
    rest = max(0, cfg.n_estimators - args.warmup - args.steps)
    if rest:
        booster.update(rest)
    model = booster.model()
    pv = model.predict_group_major(bst.Dataset.from_feature_major(xv))
    return dict(elapsed=elapsed, t0=t0, t1=t1, c0=c0, c1=c1, heldout=bst.metric("logloss", pv, yv),
                trees=booster.n_rounds, model=model, shape=model.tune_info, explored=tuned)


def serve_schedule(rng, rate, n_req, n_pool, max_rows=65536):
    """Poisson arrivals at `rate` req/s (None: all at once) with row counts
    floor(exp(U ln(max_rows + 1))) in [1, max_rows] at random pool offsets."""
    sizes = np.clip(np.floor(np.exp(rng.uniform(0, np.log(max_rows + 1), n_req))).astype(np.int64), 1, max_rows)
    offs = rng.integers(0, n_pool - max_rows, n_req)
    arrival = np.cumsum(rng.exponential(1.0 / rate, n_req)) if rate else np.zeros(n_req)
    return arrival, offs, sizes


def phase_split(tr, lat):
    """p50/p99 of each traced request phase (ms) and the achieved host->device
    copy rate over the traced copies; `lat` (s) gives the slowest requests,
    whose phases are listed apart (the p99 tail's make-up)."""
    from boosters_b200 import _native as n
    col = {k: tr[:, i].astype(np.float64) for i, k in enumerate(n.SERVER_PHASES)}
    out = {}
    for k in ("queue_ns", "copy_ns", "to_dispatch_ns", "kernel_ns", "d2h_ns", "dispatch_to_done_ns"):
        v = col[k] / 1e6
        out[k[:-3] + "_ms"] = {"p50": round(float(np.percentile(v, 50)), 3), "p99": round(float(np.percentile(v, 99)), 3)}
    out["h2d_gb_per_s"] = round(float(col["rows"].sum() * N_FEAT * 4 / max(1.0, col["copy_ns"].sum())), 2)
    if len(lat) == len(tr):
        tail = np.argsort(lat)[-max(1, len(lat) // 100):]
        out["slowest_1pct_mean_ms"] = {k[:-3]: round(float(col[k][tail].mean()) / 1e6, 3)
                                       for k in ("queue_ns", "copy_ns", "to_dispatch_ns", "kernel_ns", "d2h_ns",
                                                 "dispatch_to_done_ns")}
        out["slowest_1pct_mean_rows"] = round(float(col["rows"][tail].mean()))
    return out


def run_serving(bst, torch, local, rank):
    """Serving on a 1000-tree depth-8 forest of the 100-feature workload,
    replayed from a native submitter thread (latency from each request's
    scheduled arrival to the completion of its batch)."""
    x, y = bst.synth.binary(N_ROWS, N_FEAT, N_NAN, seed=SEED, stream=rank)
    cfg = bst.GBDTConfig(device=local, **dict(cfg_kwargs(), n_estimators=1000))
    model = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)
    xv, _ = bst.synth.binary(200_000, N_FEAT, N_NAN, seed=SEED, stream=2000 + rank)
    pool = torch.from_numpy(np.ascontiguousarray(xv.T)).pin_memory().numpy()
    pool_dev = torch.from_numpy(pool).cuda()
    srv = bst.PredictionServer(model, mem_budget_bytes=4 << 30)
    rng = np.random.default_rng(7 + rank)

    def play(rate, n_req, ring=256, rows=pool, phases=False):
        arr, offs, sizes = serve_schedule(rng, rate, n_req, pool.shape[0])
        srv.trace()  # drop earlier records
        lat, span, _ = srv.replay(rows, arr, offs, sizes, ring=ring)
        r = {"p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
             "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
             "rows_per_s": round(int(sizes.sum()) / span)}
        if phases:
            r["phases"] = phase_split(srv.trace(), lat)
        return r

    try:
        play(10_000, 2_000)  # warm-up
        st0 = srv.stats()
        head = play(10_000, 20_000, phases=True)
        st1 = srv.stats()
        sweep = {str(r): play(r, 10_000, phases=r == 17_000) for r in (14_000, 17_000, 20_000, 23_000)}
        sat = play(None, 3_000, ring=1024)
        # rows already in device memory (a GPU feature pipeline): no PCIe leg
        dev = {str(r): play(r, 10_000, rows=pool_dev) for r in (10_000, 17_000, 25_000, 34_000)}
        dev["saturation"] = play(None, 3_000, ring=1024, rows=pool_dev)
    finally:
        srv.close()
    batches = st1["batches"] - st0["batches"]
    h2d_gbs = (st1["h2d_bytes"] - st0["h2d_bytes"]) / max(1, st1["h2d_ns"] - st0["h2d_ns"])
    # the link's own rate: one 256 MiB pinned host-to-device copy, best of 5
    big_h = torch.empty(64 << 20, dtype=torch.float32).pin_memory()
    big_d = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    link_gbs = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        big_d.copy_(big_h, non_blocking=True)
        e1.record()
        e1.synchronize()
        link_gbs = max(link_gbs, big_h.numel() * 4 / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del big_h, big_d
    best = max([head["rows_per_s"]] + [v["rows_per_s"] for v in sweep.values() if v["p99_ms"] <= 2.0] + [0])
    return {"forest": "1000 trees, depth 8, 100 features (binary-logistic workload)",
            "arrivals": "Poisson, rows floor(exp(U ln 65537)) in [1, 65536], pinned host rows, native submitter",
            "requests": 20_000, "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"],
            "rows_per_s_at_10k_req_s": head["rows_per_s"], "phases_at_10k_req_s": head["phases"],
            "h2d_gb_per_s_at_10k_req_s": round(h2d_gbs, 2),
            "h2d_peak_gb_per_s": round(link_gbs, 2),
            "h2d_needed_gb_per_s_at_1e8_rows_s": round(1e8 * N_FEAT * 4 / 1e9, 1),
            "mean_batch_rows": round((st1["rows"] - st0["rows"]) / max(1, batches)),
            "sweep_req_per_s": sweep, "max_rows_per_s_with_p99_le_2ms": best,
            "saturation_rows_per_s": sat["rows_per_s"],
            "device_rows_sweep_req_per_s": dev,
            "device_rows_max_rows_per_s_with_p99_le_2ms": max(
                [v["rows_per_s"] for k, v in dev.items() if k != "saturation" and v["p99_ms"] <= 2.0] + [0]),
            "latency_clock": "steady clock, scheduled arrival to completion of the request's batch"}


def run_ours(args, world, rank, local):
    import ctypes

    import boosters_b200 as bst
    from boosters_b200 import _native as n
    import torch

    torch.cuda.set_device(local)
    kw = cfg_kwargs()
    x, y = bst.synth.binary(N_ROWS, N_FEAT, N_NAN, seed=SEED, stream=rank)
    ds = bst.Dataset.from_feature_major(x, y)
    xv, yv = bst.synth.binary(200_000, N_FEAT, N_NAN, seed=SEED, stream=1000 + rank)
    t_bin0 = time.perf_counter()
    bst.BinnedDataset(ds, bst.GBDTConfig(device=local, **kw))
    binning_s = time.perf_counter() - t_bin0

    clocks = ClockSampler(local)
    clocks.start()
    res = {}
    for name, over in FORMS:
        res[name] = run_form(bst, torch, ds, xv, yv, bst.GBDTConfig(device=local, **dict(kw, **over)), args, world)
    # a short timed region may fall between two clock samples: keep training
    # load running (untimed) until a few samples exist
    t_ext = time.perf_counter()
    if len(clocks.rows) < 4:
        b = bst.Booster(ds, bst.GBDTConfig(device=local, **kw), n_threads=0)
        while len(clocks.rows) < 4 and time.perf_counter() - t_ext < 3.0:
            b.update(10)
    clk = clocks.stop()
    clk["extended_window_s"] = round(time.perf_counter() - t_ext, 3)
    barrier(world)

    # headline: the fastest form whose held-out loss is within 1e-3 relative of
    # the plain form's at the same number of trees
    plain_loss = res["plain"]["heldout"]
    forms = {}
    for name, r in res.items():
        r["value"] = whole_job_value(world, r["elapsed"], args.steps)
        r["ms"] = 10.0 * r["value"] * world  # the slowest rank's ms per tree
        r["equal_loss"] = abs(r["heldout"] - plain_loss) <= EQUAL_LOSS_REL * plain_loss
        forms[name] = {"s_per_100_trees": round(r["value"], 5), "heldout_logloss": round(r["heldout"], 6),
                       "loss_rel_vs_plain": round((r["heldout"] - plain_loss) / plain_loss, 6),
                       "equal_loss": r["equal_loss"], "trees": r["trees"]}
        if r["shape"]:
            forms[name]["launch_shape"] = r["shape"]
            forms[name]["autotune"] = r["explored"]
    ok = [k for k, r in res.items() if r["equal_loss"]]
    head = min(ok, key=lambda k: res[k]["value"])
    hr = res[head]
    value, ms_per_step = hr["value"], hr["ms"]
    model = hr["model"]
    head_over = dict(FORMS)[head]
    c0, c1 = hr["c0"], hr["c1"]
    # the phase split and the histogram kernel's time come from a second run
    # of the headline form with per-phase CUDA events (they cost ~0.3 ms per
    # tree, so the timed forms above run without them)
    timed = run_form(bst, torch, ds, xv, yv,
                     bst.GBDTConfig(device=local, **dict(kw, **head_over, phase_timings=True,
                                                         n_estimators=args.warmup + args.steps)), args, world)
    t0_stats, t1_stats = timed["t0"], timed["t1"]

    hist_ms = t1_stats["histograms"] - t0_stats["histograms"]
    hist_bytes = timed["c1"]["hist_bytes"] - timed["c0"]["hist_bytes"]
    hist_launches = max(1, timed["c1"]["hist_launches"] - timed["c0"]["hist_launches"])
    launches = c1["launches"] - c0["launches"]
    peak, peak_kind = peaks()
    achieved = hist_bytes / (hist_ms / 1e3) / 1e9 if hist_ms > 0 else 0.0
    traffic = None
    tr_file = os.path.join(ROOT, "profiles", f"hist_build_traffic_{head}.json")
    if os.path.exists(tr_file):
        with open(tr_file) as f:
            tr = json.load(f)
        # ncu DRAM bytes per algorithmic byte, scaled to this run's average launch
        traffic = round(tr["dram_bytes_per_algorithmic_byte"] * hist_bytes / hist_launches)

    # predict throughput on device-resident rows (serving kernel), rows/s
    rows_pred = None
    try:
        xs = torch.from_numpy(np.ascontiguousarray(xv.T)).cuda()
        out = torch.empty((1, xs.shape[0]), dtype=torch.float32, device="cuda")
        st = torch.cuda.current_stream()
        for _ in range(2):
            n.check(n.lib.bst_gbdt_predict_device(model._h, ctypes.c_void_p(xs.data_ptr()), xs.shape[0], N_FEAT, 1,
                                                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        reps = 5
        for _ in range(reps):
            n.check(n.lib.bst_gbdt_predict_device(model._h, ctypes.c_void_p(xs.data_ptr()), xs.shape[0], N_FEAT, 1,
                                                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
        e1.record(st)
        e1.synchronize()
        rows_pred = xs.shape[0] * reps / (e0.elapsed_time(e1) / 1e3)
    except Exception as ex:  # reported, not fatal
        rows_pred = f"error: {ex}"

    # e2e through the public API from pinned host buffers: 100 trees per step
    e2e_cfg = bst.GBDTConfig(device=local, **dict(kw, n_estimators=100, **head_over))
    xh = torch.from_numpy(x).pin_memory().numpy()
    yh = torch.from_numpy(y).pin_memory().numpy()
    e2e_steps = max(1, min(args.steps, 5))
    bst.GBDTModel.train(bst.Dataset.from_feature_major(xh, yh), e2e_cfg)  # warm-up call
    barrier(world)
    te0 = time.perf_counter()
    for _ in range(e2e_steps):
        dsh = bst.Dataset.from_feature_major(xh, yh)
        mh = bst.GBDTModel.train(dsh, e2e_cfg)
        _ = mh.train_predictions()
    te = reduce_max(world, time.perf_counter() - te0)
    e2e_value = te / (e2e_steps * world)

    serving = None
    if not args.no_serving:
        try:
            serving = run_serving(bst, torch, local, rank)
        except Exception as ex:  # reported, not fatal
            serving = {"error": str(ex)}

    extra = None
    if not args.no_configs and rank == 0 and world == 1:
        extra = run_configs(bst, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        build = oracle_native()
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_bridge as ob  # noqa: E402  (after BST_ORACLE_LIB is set)
        cores = os.cpu_count() or 1
        timed, _ = bounded_cpu_rounds(ob, 15.0, 40, cores, x, y, oracle_cfg(ob))
        cpu = {"value": round(100.0 * sum(timed) / len(timed), 3), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"1 warm-up + {len(timed)} timed boosting rounds of the {N_ROWS}x{N_FEAT} workload, "
                         f"binning excluded; {build}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPES[head],
            "data": "synthetic (seeded counter-based generator)",
            "config": {"workload": WORKLOAD, "form": head, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (128 MB binned rows + 8 MB grad/hess per round)",
                       "binning_s": round(binning_s, 3), "heldout_logloss": round(hr["heldout"], 6),
                       "heldout_rows": int(len(yv)), "equal_loss_rule": "within 1e-3 relative of plain",
                       "speedup_vs_plain": round(res["plain"]["value"] / value, 3)},
            "forms": forms,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_b_hist_part" if head != "plain" else "k_hist_build", "launches": hist_launches,
                         "avg_launch_ms": round(hist_ms / hist_launches, 5),
                         "algorithmic_bytes_per_launch": round(hist_bytes / hist_launches)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 4), "unit": E2E_UNIT,
                    "h2d_bytes_per_step": int(x.nbytes + y.nbytes), "d2h_bytes_per_step": int(N_ROWS * 4),
                    "includes": "public train call from pinned host arrays: dataset, binning, H2D, 100 trees, "
                                "D2H of the training predictions"},
            "gpu_launches": int(launches),
            "clocks": clk,
            "predict_rows_per_s": rows_pred,
            "serving": serving,
            "configs": extra,
            "phase_ms_per_step": {k: round((t1_stats[k] - t0_stats[k]) / args.steps, 4)
                                  for k in ("gradients", "histograms", "split_scan", "partition", "leaf_update",
                                            "other")},
        }
        print(json.dumps(line), flush=True)


def time_trees(bst, torch, ds, cfg, warm, steps):
    """s/100 trees of `steps` timed rounds after `warm` (CUDA events on the
    engine's stream), then the rest of cfg's rounds; returns (value, model)."""
    tune_form(bst, ds, cfg)
    cfg.autotune_cache = TUNE_CACHE
    booster = bst.Booster(ds, cfg, n_threads=0)
    booster.update(warm)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    booster.update(steps)
    e1.record()
    e1.synchronize()
    per_round = e0.elapsed_time(e1) / 1e3 / steps
    rest = max(0, cfg.n_estimators - warm - steps)
    if rest:
        booster.update(rest)
    trees_per_round = max(1, booster.model().n_trees // max(1, booster.n_rounds))
    return 100.0 * per_round / trees_per_round, booster.model()


def config_forms(bst, torch, ds, kw, forms, warm, steps, heldout):
    """Every form of one workload: s/100 trees, held-out loss, loss relative
    to the plain form and the equal-loss flag (|rel| <= 1e-3); the fast form
    is the fastest form at equal loss."""
    out = {}
    for name in forms:
        v, m = time_trees(bst, torch, ds, bst.GBDTConfig(**kw, **dict(FORMS)[name]), warm, steps)
        out[name] = {"s_per_100_trees": round(v, 5), "heldout_loss": round(heldout(m), 6), "trees": m.n_trees}
        if m.tune_info:
            out[name]["launch_shape"] = m.tune_info
        del m
    plain = out["plain"]["heldout_loss"]
    for r in out.values():
        r["loss_rel_vs_plain"] = round((r["heldout_loss"] - plain) / plain, 6)
        r["equal_loss"] = abs(r["heldout_loss"] - plain) <= EQUAL_LOSS_REL * plain
    fast = min((k for k in out if out[k]["equal_loss"]), key=lambda k: out[k]["s_per_100_trees"])
    return {"forms": out, "fast_form": fast,
            "speedup_vs_plain": round(out["plain"]["s_per_100_trees"] / out[fast]["s_per_100_trees"], 3)}


def run_configs(bst, torch):
    """The survey's other workloads in every form, each timed on the device
    (CUDA events) and evaluated on a held-out draw of the same generator:
    5,000 x 100 regression (50 trees, depth 6); 10,000,000 x 200 logistic,
    leaf-wise 255 leaves (100 trees; the workload names no tree count);
    2,000,000 x 50 softmax with 10 categorical columns, 10 classes (200
    rounds x 10 trees, depth 6)."""
    all_forms = [k for k, _ in FORMS]
    out = {}
    x, y = bst.synth.regression(5_000, 100, 20, seed=1)
    xv, yv = bst.synth.regression(1_000, 100, 20, seed=1, stream=1)
    dv = bst.Dataset.from_feature_major(xv)
    kw = dict(n_estimators=50, max_depth=6, learning_rate=0.1, metric=bst.Metric.none())
    r = config_forms(bst, torch, bst.Dataset.from_feature_major(x, y), kw, all_forms, 5, 40,
                     lambda m: bst.metric("rmse", m.predict_group_major(dv), yv))
    out["regression_5kx100_depth6_50trees"] = dict(r, loss="heldout rmse, 1,000 rows")

    x, y = bst.synth.binary(10_000_000, 200, 20, seed=3)
    xv, yv = bst.synth.binary(2_000_000, 200, 20, seed=3, stream=1)
    ds = bst.Dataset.from_feature_major(x, y)
    dv = bst.Dataset.from_feature_major(xv)
    kw = dict(objective=bst.Objective.logistic(), n_estimators=100, learning_rate=0.1,
              growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=255, metric=bst.Metric.none())
    r = config_forms(bst, torch, ds, kw, all_forms, 2, 10,
                     lambda m: bst.metric("logloss", m.predict_group_major(dv), yv))
    out["logistic_10Mx200_leafwise255_100trees"] = dict(r, loss="heldout logloss, 2,000,000 rows")
    del ds, dv, x, xv

    x, y = bst.synth.multiclass(2_000_000, 40, 10, 10, seed=4)
    xv, yv = bst.synth.multiclass(400_000, 40, 10, 10, seed=4, stream=1)
    cats = list(range(40, 50))
    ds = bst.Dataset.from_feature_major(x, y, categorical_features=cats)
    dv = bst.Dataset.from_feature_major(xv, categorical_features=cats)
    kw = dict(objective=bst.Objective.softmax(10), n_estimators=200, max_depth=6, learning_rate=0.1,
              max_onehot_cats=4, metric=bst.Metric.none())
    r = config_forms(bst, torch, ds, kw, all_forms, 3, 20,
                     lambda m: bst.metric("mlogloss", m.predict_group_major(dv), yv))
    out["softmax10_cat10_2Mx50_depth6_200rounds"] = dict(r, loss="heldout multiclass logloss, 400,000 rows")
    return out


def run_profile(args):
    """A small fixed workload for profilers (no JSON line): `train` grows
    --rounds rounds of --workload (the 1M x 100 logistic depth-8 workload,
    the 10M x 200 leaf-wise one or the 2M x 50 softmax one) in --form, after
    a launch-shape tuning pass; `predict` trains --trees trees (batched_q8)
    of the 1M x 100 workload and predicts --rows rows three times."""
    import ctypes
    import torch
    import boosters_b200 as bst
    from boosters_b200 import _native as n
    if args.profile == "train" and args.workload == "leafwise10M":
        # 10,000,000 x 200 logistic, leaf-wise 255 leaves (--train-rows: a
        # smaller row count of the same generator, for full captures)
        x, y = bst.synth.binary(args.train_rows or 10_000_000, 200, 20, seed=3)
        ds = bst.Dataset.from_feature_major(x, y)
        cfg = bst.GBDTConfig(objective=bst.Objective.logistic(), n_estimators=100, learning_rate=0.1,
                             growth_strategy=bst.GrowthStrategy.Leafwise, n_leaves=255, metric=bst.Metric.none(),
                             **dict(FORMS)[args.form])
    elif args.profile == "train" and args.workload == "softmax2M":
        # 2,000,000 x 50 (10 categorical) softmax, 10 classes, depth 6
        x, y = bst.synth.multiclass(args.train_rows or 2_000_000, 40, 10, 10, seed=4)
        ds = bst.Dataset.from_feature_major(x, y, categorical_features=list(range(40, 50)))
        cfg = bst.GBDTConfig(objective=bst.Objective.softmax(10), n_estimators=200, max_depth=6, learning_rate=0.1,
                             max_onehot_cats=4, metric=bst.Metric.none(), **dict(FORMS)[args.form])
    else:
        x, y = bst.synth.binary(N_ROWS, N_FEAT, N_NAN, seed=SEED)
        ds = bst.Dataset.from_feature_major(x, y)
        cfg = bst.GBDTConfig(**dict(cfg_kwargs(), **dict(FORMS)[args.form]))
    if args.profile == "train":
        # the launch shape: tuned first (16 trees, before the profiled ones),
        # or forced with --shape through the cache file
        if args.shape == "builtin":  # no tuning pass: the built-in shape
            cfg.autotune = False
        else:
            print(f"tuning pass: {tune_form(bst, ds, cfg)}")
        if args.shape and args.shape != "builtin" and os.path.exists(TUNE_CACHE):
            with open(TUNE_CACHE) as f:
                key = f.read().split("\t")[0]
            with open(TUNE_CACHE, "w") as f:
                f.write(f"{key}\t{args.shape}\n")
        cfg.autotune_cache = TUNE_CACHE
        booster = bst.Booster(ds, cfg, n_threads=0)
        print(f"profiled shape: {booster.model().tune_info}")
        for r in range(args.rounds):  # per round: the histogram launches' algorithmic bytes
            c0 = booster.stats()[1]
            booster.update(1)
            c1 = booster.stats()[1]
            print(f"round {r}: hist_launches {c1['hist_launches'] - c0['hist_launches']} "
                  f"hist_bytes {c1['hist_bytes'] - c0['hist_bytes']}")
        torch.cuda.synchronize()
        print(f"profile train: {booster.n_rounds} rounds ({args.form})")
        return
    cfg = bst.GBDTConfig(**dict(cfg_kwargs(), n_estimators=args.trees, precision="q8", batched=True))
    model = bst.GBDTModel.train(bst.Dataset.from_feature_major(x, y), cfg)
    xv, _ = bst.synth.binary(args.rows, N_FEAT, N_NAN, seed=SEED, stream=9)
    xs = torch.from_numpy(np.ascontiguousarray(xv.T)).cuda()
    out = torch.empty((1, args.rows), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    for _ in range(3):
        n.check(n.lib.bst_gbdt_predict_device(model._h, ctypes.c_void_p(xs.data_ptr()), args.rows, N_FEAT, 1,
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
    torch.cuda.synchronize()
    print(f"profile predict: {args.trees} trees x {args.rows} rows, 3 launches")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--profile", choices=["train", "predict"], help="run a small workload for a profiler and exit")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other survey workloads (5k x 100, 10M x 200 leaf-wise, 2M x 50 softmax)")
    ap.add_argument("--form", default="batched_q8", choices=[k for k, _ in FORMS])
    ap.add_argument("--rounds", type=int, default=4)
    ap.add_argument("--shape", default="", help="profile train: force this launch shape (items=..,hist=..,grid=..; "
                    "builtin: the built-in shape, no tuning pass)")
    ap.add_argument("--workload", default="1M", choices=["1M", "leafwise10M", "softmax2M"],
                    help="profile train: the 1M x 100 depth-8 workload, the 10M x 200 leaf-wise one or the "
                         "2M x 50 softmax one")
    ap.add_argument("--train-rows", type=int, default=0,
                    help="profile train: rows of the leafwise10M / softmax2M workloads (0: their full size)")
    ap.add_argument("--trees", type=int, default=1000)
    ap.add_argument("--rows", type=int, default=300_000)
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
