#!/usr/bin/env python
"""Benchmark: the tall binary-classification fit (10,000,000 rows x 28 float32
features, logloss, depthwise depth 8, 255 bins, lr 0.1) on B200.

The metric is the fit time for 500 rounds. `value` is the device time of a
complete 500-round fit (CUDA events on the booster's stream around its 500
rounds, the binned plane and labels already resident); `e2e` is the wall
clock of the same fit from pinned host rows (ingest, the rounds, the model and
training scores back on the host). The plain (exact) form fits the same 500
rounds on the same plane, and both forms' validation AUC and logloss are
measured on 1,000,000 rows of the generator's validation seed. A step is one
boosting round: `ms_per_step` is K device-timed rounds after W warm-up rounds
(a barrier and a synchronize on both sides, max over ranks). The bins plane
(280 MB) and the per-row state exceed the 126 MB L2, so no flush is needed
between rounds. Cut fitting is outside every timed region, on both arms.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode exact|int8|int16]
  python bench.py --impl reference      # the reference's CPU grower, timed
  python bench.py --workload serve|wide|multiclass|many [--impl reference]

The serving workload fits a 1,000-tree depth-8 ensemble (squared error, 255
bins, lr 0.1) on 20,000 rows x 28 of the ragged-many family, then scores
request batches of 1 to 1,000,000 rows x 28: predict rows/s through a
predict plan (device time per launch, L2 flushed between launches, and end
to end from pinned host rows through a request plane, refilled per batch, to
host scores) and TreeSHAP rows/s with the additivity error against an FP64
recomputation of the margin.

Multi-GPU (torchrun): the quantised fit is row-sharded -- every rank holds a
contiguous slice of the same rows and the ranks all-reduce integer histograms
over NCCL once per level (strong scaling; trees equal the one-GPU fit's).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "10M×28 fit s/500 iters: int-quantised vs plain GPU at ΔAUC≤1e-3; hist GB/s"
WORKLOAD = "tall binary logloss 10,000,000x28, depthwise depth 8, 255 bins, lr 0.1"
N_ROUNDS = 500


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_init(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier()
        torch.cuda.synchronize()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(),
                                 f"bonsai_b200_clocks_{os.getpid()}_{id(self)}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler has started up and
            # written its first sample (its start-up holds the driver)
            t_end = time.perf_counter() + 3.0
            while time.perf_counter() < t_end and self.proc.poll() is None:
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.05)
            time.sleep(0.2)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for name, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(X, y, cuts, off, steps, warmup, rows=None):
    """The reference's own CPU depthwise grower (oracle/_ref, compiled from
    its sources) on all rows (or the first `rows`), all host threads: `steps`
    timed rounds after `warmup` rounds, the per-round time x 500 (and x the
    row ratio when sampled). Falls back to the oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n_full = X.shape[0]
    rows = n_full if rows is None else min(rows, n_full)
    Xs, ys = X[:rows], y[:rows]
    threads = len(os.sched_getaffinity(0))
    tc = O.TreeCfg(objective="logloss", max_depth=8, learning_rate=0.1, n_threads=threads)
    try:
        ref = O.RefLib()
        ds = ref.dataset(Xs, ys, cuts, off)
        kind = "reference"
        tc.n_iters = warmup
        if warmup:
            ref.train(ds, tc)
        tc.n_iters = warmup + steps
        t0 = time.perf_counter()
        ref.train(ds, tc)
        t = time.perf_counter() - t0
        # the warm-up rounds are re-run inside the timed fit: remove them
        tc.n_iters = warmup
        t1 = time.perf_counter()
        if warmup:
            ref.train(ds, tc)
        t_w = time.perf_counter() - t1 if warmup else 0.0
        per_round = max(t - t_w, 1e-9) / steps
    except FileNotFoundError:
        orc = O.Oracle()
        bins = orc.transform(Xs, cuts, off)
        kind = "port"
        threads = 1
        tc.n_iters = steps
        t0 = time.perf_counter()
        orc.train(bins, np.diff(off), cuts, off, ys, tc)
        per_round = (time.perf_counter() - t0) / steps
    value = per_round * (n_full / rows) * N_ROUNDS
    return {"value": value, "unit": "s", "cores": threads, "kind": kind,
            "sample": (f"all {rows:,} rows x 28" if rows == n_full else
                       f"first {rows:,} rows x 28 (per-round time x {n_full / rows:g})") +
                      f", {steps} timed depth-8 logloss rounds after {warmup} warm-up "
                      f"rounds, per-round time x {N_ROUNDS} (rounds)"}


def make_data(rows):
    from bonsai_b200 import synth
    from bonsai_b200.binning import fit_cuts
    X, y = synth.tall_binary(n=rows)
    cuts, off = fit_cuts(X, max_bin=255)
    return X, y, cuts, off


SERVE_METRIC = ("1,000-tree depth-8 ensemble predict rows/s at a 1,000,000-row batch; "
                "TreeSHAP rows/s and additivity error vs FP64")
SERVE_WORKLOAD = ("serving: 1,000 depth-8 trees (mse, 255 bins, lr 0.1) fit on 20,000x28; "
                  "request batches of 1 to 1,000,000 rows x 28 float32")
SERVE_FIT_ROWS = 20_000
SERVE_TREES = 1000
SERVE_BATCHES = (1, 100, 10_000, 1_000_000)
SHAP_BATCHES = (1, 100, 10_000, 100_000)
LEAF = 0xFFFFFFFF


def margin64(codes, n_bins, trees, init, lr):
    """init + lr * sum of leaves in FP64 (the bin-space walk of routes_left,
    vectorised over rows)."""
    F, n = codes.shape
    last = np.asarray(n_bins, np.int64) - 1
    acc = np.zeros(n, np.float64)
    rows = np.arange(n)
    for t in trees:
        idx = np.zeros(n, np.int64)
        feat = t.feature.astype(np.int64)
        while True:
            f = feat[idx]
            live = f != LEAF
            if not live.any():
                break
            fl = np.where(live, f, 0)
            b = codes[fl, rows].astype(np.int64)
            left = np.where(b == last[fl], t.default_left[idx] != 0, b <= t.split_bin[idx])
            nxt = np.where(left, t.left[idx], t.right[idx]).astype(np.int64)
            idx = np.where(live, nxt, idx)
        acc += t.value[idx].astype(np.float64)
    # the booster's own float init and learning rate, widened
    return float(np.float32(init)) + float(np.float32(lr)) * acc


def serve_data(n_requests=max(SERVE_BATCHES)):
    from bonsai_b200 import synth
    from bonsai_b200.binning import fit_cuts
    X, y, Xr = synth.serving(n_fit=SERVE_FIT_ROWS, n_requests=n_requests)
    cuts, off = fit_cuts(X, max_bin=255)
    return X, y, Xr, cuts, off


def serve_reference(args):
    """The reference's own CPU path (oracle/_ref, all host threads): the same
    fit through its depthwise Booster, then predict_at_binned and
    pred_contribs_binned over bounded samples of each request batch."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    X, y, Xr, cuts, off = serve_data()
    threads = len(os.sched_getaffinity(0))
    ref = O.RefLib()
    tc = O.TreeCfg(objective="mse", max_depth=8, learning_rate=0.1, n_iters=SERVE_TREES,
                   n_threads=threads)
    model = ref.train(ref.dataset(X, y, cuts, off), tc)
    out = {}
    for B in SERVE_BATCHES:
        m = min(B, 50_000)
        ds = ref.dataset(Xr[:m], np.zeros(m, np.float32), cuts, off)
        model.predict_binned(ds)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            model.predict_binned(ds)
        out[B] = m * args.steps / (time.perf_counter() - t0)
    shap = {}
    for B in SHAP_BATCHES:
        m = min(B, 64)
        ds = ref.dataset(Xr[:m], np.zeros(m, np.float32), cuts, off)
        t0 = time.perf_counter()
        model.contribs_binned(ds)
        shap[B] = m / (time.perf_counter() - t0)
    big = max(SERVE_BATCHES)
    cb = {"value": out[big], "unit": "rows/s", "cores": threads, "kind": "reference",
          "sample": f"predict_at_binned over min(batch, 50,000) rows x {args.steps} calls; "
                    "pred_contribs_binned over min(batch, 64) rows"}
    line = {"metric": SERVE_METRIC, "value": out[big], "unit": "rows/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": big / out[big] * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": SERVE_WORKLOAD, "host_threads": threads},
            "predict_rows_per_s": {str(k): v for k, v in out.items()},
            "shap_rows_per_s": {str(k): v for k, v in shap.items()},
            "cpu_baseline": cb,
            "e2e": {"value": out[big], "unit": "rows/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_ours(args, local):
    import torch
    batches = [int(x) for x in args.batches.split(",")]
    shap_batches = [int(x) for x in args.shap_batches.split(",")]
    n_max = max(batches + shap_batches)

    import bonsai_b200 as bb
    X, y, Xr, cuts, off = serve_data(n_max)
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(objective="mse", max_depth=8, learning_rate=0.1,
                                            min_data_in_leaf=20, hist_mode="exact",
                                            use_graph=True), max_trees=SERVE_TREES)
    b.update(SERVE_TREES)
    trees, init = b.trees(), b.init_score
    b.close()
    plane.close()
    Xp = torch.empty((n_max, Xr.shape[1]), dtype=torch.float32, pin_memory=True).numpy()
    Xp[...] = Xr
    big = bb.Plane(Xp, cuts, off)
    plan = bb.PredictPlan(big, trees, init, 0.1)
    req = bb.Plane.like(big, n_max)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    W, K = max(3, args.warmup), max(1, args.steps)
    dev, e2e, launches = {}, {}, {}
    with Clocks(local) as clk:
        for B in batches:
            pb = bb.Plane(Xp[:B], cuts, off)
            out = torch.empty(B, dtype=torch.float32, device="cuda")
            for _ in range(W):
                plan.launch(pb, out.data_ptr(), stream.cuda_stream)
            ms, k = 0.0, 0
            for _ in range(K):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                k += plan.launch(pb, out.data_ptr(), stream.cuda_stream)
                e1.record(stream)
                e1.synchronize()
                ms += e0.elapsed_time(e1)
            dev[B] = B * K / (ms * 1e-3)
            launches[B] = k / K
            pb.close()
            # end to end: pinned host rows -> bin into a request plane sized
            # once (bb_plane_refill, no allocation) -> plan -> host scores
            for _ in range(W):
                req.refill(Xp[:B])
                plan.run(req)
            t0 = time.perf_counter()
            for _ in range(K):
                req.refill(Xp[:B])
                plan.run(req)
            e2e[B] = B * K / (time.perf_counter() - t0)
    # TreeSHAP through a plan: device time per launch, then the additivity of
    # (up to) the first 2,000 rows against an FP64 recomputation
    splan = bb.ShapPlan(big, trees, init, 0.1)
    shap, shap_e2e, additivity = {}, {}, {}
    for B in shap_batches:
        pb = bb.Plane(Xp[:B], cuts, off)
        phi_d = torch.empty((B, Xr.shape[1] + 1), dtype=torch.float64, device="cuda")
        splan.launch(pb, phi_d.data_ptr(), stream.cuda_stream)
        ms = 0.0
        ks = max(1, min(K, 3))
        for _ in range(ks):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            splan.launch(pb, phi_d.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        shap[B] = B * ks / (ms * 1e-3)
        t0 = time.perf_counter()
        req.refill(Xp[:B])
        phi = splan.run(req)
        shap_e2e[B] = B / (time.perf_counter() - t0)
        m = min(B, 2_000)
        m64 = margin64(pb.bins()[:, :m], pb.n_bins, trees, init, 0.1)
        additivity[B] = float(np.max(np.abs(phi[:m].sum(axis=1) - m64)))
        pb.close()
    splan.close()
    # the CPU baseline: the oracle's bin-space walk (C, one thread) on a sample
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    orc = O.Oracle()
    m = 20_000
    codes = big.bins()[:, :m]
    t0 = time.perf_counter()
    orc.predict_binned(codes, big.n_bins, trees, init, 0.1)
    cpu = m / (time.perf_counter() - t0)
    big.close()
    plan.close()
    depth = max(t.depth for t in trees)
    b_max = max(batches)
    line = {
        "metric": SERVE_METRIC, "value": dev[b_max], "unit": "rows/s", "n_gpus": 1,
        "steps": K, "warmup": W, "ms_per_step": b_max / dev[b_max] * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ragged-many family)",
        "config": {"workload": SERVE_WORKLOAD, "trees": len(trees), "max_depth": depth,
                   "l2": "256 MB flush written between timed launches"},
        "predict_rows_per_s": {str(k): v for k, v in dev.items()},
        "predict_e2e_rows_per_s": {str(k): v for k, v in e2e.items()},
        "shap_rows_per_s": {str(k): v for k, v in shap.items()},
        "shap_e2e_rows_per_s": {str(k): v for k, v in shap_e2e.items()},
        "shap_additivity_max_abs": {str(k): v for k, v in additivity.items()},
        "e2e": {"value": e2e[b_max], "unit": "rows/s", "h2d_bytes_per_step": b_max * 28 * 4,
                "d2h_bytes_per_step": b_max * 4},
        "gpu_launches": int(launches[b_max] * K),
        "clocks": clk.summary(),
        "cpu_baseline": {"value": cpu, "unit": "rows/s", "cores": 1, "kind": "port",
                         "sample": f"oracle bin-space walk over the first {m:,} request rows"},
    }
    print(json.dumps(line), flush=True)


CONFIGS = {
    # name: (workload text, rounds, rows)
    "wide": ("wide sparse regression 1,000,000x2,000 (90% missing), leafwise 255 leaves, "
             "256 bins, lr 0.1, Bernoulli row subsample 0.8 (seed 42)", 200, 1_000_000),
    "multiclass": ("multiclass 581,012x54 (one-hot blocks), 7-class softmax, levelwise depth 8, "
                   "255 bins, lr 0.1", 300, 581_012),
}


def config_data(name, rows):
    from bonsai_b200 import synth
    from bonsai_b200.binning import fit_cuts
    if name == "wide":
        X, y = synth.wide_sparse(n=rows)
        cuts, off = fit_cuts(X, max_bin=256)
        return X, y, cuts, off
    X, y = synth.multiclass_onehot(n=rows)
    cuts, off = fit_cuts(X, max_bin=255)
    return X, y, cuts, off


def config_tc(name, mod):
    """The fit's knobs for the booster (mod = bonsai_b200) or the oracle's
    TreeCfg (mod = oracle)."""
    if name == "wide":
        kw = dict(objective="mse", grower="leafwise", max_leaves=255, max_depth=255,
                  learning_rate=0.1, subsample=0.8, random_seed=42)
    else:
        kw = dict(objective="softmax", n_classes=7, grower="levelwise", max_depth=8,
                  learning_rate=0.1)
    return kw


def config_main(args, name):
    """Device time per round of the configuration's fit (K timed rounds after W
    warm-up rounds, CUDA events on the booster's stream), x its rounds; the
    reference's CPU booster timed on a bounded row sample beside it."""
    import bonsai_b200 as bb
    from bonsai_b200.build import build_library
    text, rounds, rows = CONFIGS[name]
    rows = args.rows if args.rows != 10_000_000 else rows
    W, K = max(3, args.warmup), max(1, args.steps)
    X, y, cuts, off = config_data(name, rows)
    if args.impl == "reference":
        cb = config_reference(name, X, y, cuts, off, rounds)
        print(json.dumps({"metric": f"{name} fit s/{rounds} iters", "value": cb["value"],
                          "unit": "s", "impl": "reference", "n_gpus": 1, "steps": K,
                          "warmup": W, "ms_per_step": cb["value"] / rounds * 1000.0,
                          "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32", "data": "synthetic",
                          "config": {"workload": text, "rows": rows}, "cpu_baseline": cb,
                          "e2e": {"value": cb["value"], "unit": "s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    build_library()
    import torch
    Xp = torch.empty(X.shape, dtype=torch.float32, pin_memory=True).numpy()
    Xp[...] = X
    t0 = time.perf_counter()
    plane = bb.Plane(Xp, cuts, off)
    params = bb.TrainParams(hist_mode=args.mode, use_graph=True, **config_tc(name, bb))
    b = bb.Booster(plane, y, params, max_trees=W + K + 2)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    b.update(W)
    with Clocks(0) as clk:
        b.update(K)
    ms = b.last_ms / K
    prof = b.profile_round()
    b.close()
    # the quantised build's launch shape for this shape (bonsai_b200.autotune),
    # then the same K rounds with it
    autotune = None
    if args.mode != "exact" and not args.no_tune:
        t0 = time.perf_counter()
        tp = bb.tune(plane, y, params, rounds=2)
        tune_s = time.perf_counter() - t0
        default_ms = ms
        if tp.hist_ctas != params.hist_ctas:
            bt = bb.Booster(plane, y, tp, max_trees=W + K + 2)
            bt.update(W)
            with Clocks(0) as clk:
                bt.update(K)
            ms = bt.last_ms / K
            prof = bt.profile_round()
            bt.close()
        autotune = {"hist_ctas": tp.hist_ctas, "tune_s": tune_s,
                    "default_ms_per_step": default_ms, "tuned_ms_per_step": ms}
    value = ms * rounds / 1000.0
    line = {"metric": f"{name} fit s/{rounds} iters", "value": value, "unit": "s", "n_gpus": 1,
            "steps": K, "warmup": W, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.mode == "exact" else args.mode,
            "data": "synthetic (seeded stand-in)",
            "config": {"workload": text, "rows": rows, "features": X.shape[1],
                       "rounds": rounds, "hist_mode": args.mode,
                       "graph": name != "wide"},
            "e2e": {"value": t_setup + value, "unit": "s",
                    "h2d_bytes_per_step": X.nbytes / rounds, "d2h_bytes_per_step": 0,
                    "setup_s": t_setup},
            "phases_ms": {k: prof[k] for k in ("hist_ms", "partition_ms", "find_ms",
                                               "other_ms", "total_ms")},
            "gpu_launches": int(prof["launches"]) * K, "clocks": clk.summary(),
            "autotune": autotune}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = config_reference(name, X, y, cuts, off, rounds)
    print(json.dumps(line), flush=True)
    plane.close()


def config_reference(name, X, y, cuts, off, rounds, sample_rows=100_000, steps=2):
    """The reference's own CPU booster (oracle/_ref, all host threads) for
    `steps` rounds on the first sample_rows rows, per-round time scaled by
    rows and rounds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m = min(sample_rows, len(y))
    threads = len(os.sched_getaffinity(0))
    ref = O.RefLib()
    ds = ref.dataset(X[:m], y[:m], cuts, off)
    tc = O.TreeCfg(n_iters=steps, n_threads=threads, **config_tc(name, O))
    t0 = time.perf_counter()
    ref.train(ds, tc)
    per_round = (time.perf_counter() - t0) / steps
    value = per_round * (len(y) / m) * rounds
    return {"value": value, "unit": "s", "cores": threads, "kind": "reference",
            "sample": f"first {m:,} rows, {steps} rounds, per-round time x "
                      f"{len(y) / m:g} (rows) x {rounds} (rounds)"}


MANY_WORKLOAD = ("64 regression datasets of 1,000-200,000 rows x 28 (ragged-many family), "
                 "mse, depthwise depth 6, 255 bins, lr 0.1, 100 rounds each, all in flight")
MANY_ROUNDS = 100


def many_main(args):
    """The many-datasets batch: every dataset's booster on its own stream, a
    round one CUDA graph; all boosters' rounds are launched before any is
    waited on. Wall time of the whole batch (synchronize on both sides: the
    fits run on 64 streams), beside the same fits run one after another."""
    import bonsai_b200 as bb
    from bonsai_b200 import synth
    from bonsai_b200.build import build_library
    sets = synth.ragged_many()
    cuts = [bb.fit_cuts(X) for X, _ in sets]
    if args.impl == "reference":
        cb = many_reference(sets, cuts)
        print(json.dumps({"metric": "64-dataset batch fit s/100 iters", "value": cb["value"],
                          "unit": "s", "impl": "reference", "n_gpus": 1, "steps": MANY_ROUNDS,
                          "warmup": 0, "ms_per_step": cb["value"] / MANY_ROUNDS * 1000.0,
                          "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32", "data": "synthetic",
                          "config": {"workload": MANY_WORKLOAD}, "cpu_baseline": cb,
                          "e2e": {"value": cb["value"], "unit": "s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    build_library()
    import torch
    params = bb.TrainParams(max_depth=6, learning_rate=0.1, hist_mode=args.mode, use_graph=True)
    W = max(3, args.warmup)

    def fits():
        planes = [bb.Plane(X, c, o) for (X, _), (c, o) in zip(sets, cuts)]
        boosters = [bb.Booster(p, y, params, max_trees=W + MANY_ROUNDS + 1)
                    for p, (_, y) in zip(planes, sets)]
        for b in boosters:
            b.update(W, sync=False)
        for b in boosters:
            b.sync()
        return planes, boosters

    planes, boosters = fits()
    torch.cuda.synchronize()
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        for b in boosters:
            b.update(MANY_ROUNDS, sync=False)
        for b in boosters:
            b.sync()
        torch.cuda.synchronize()
        batch = time.perf_counter() - t0
    launches = sum(int(b.profile_round()["launches"]) for b in boosters) * MANY_ROUNDS
    for b in boosters:
        b.close()
    # the same rounds as one graph launch per round for the whole batch
    # (bb_batch: every booster's round graph a child of one parent graph)
    one_launch = None
    if not args.no_batch:
        planes, boosters = fits()
        group = bb.BoosterBatch(boosters)
        group.update(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        group.update(MANY_ROUNDS - 1)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        one_launch = {"s_per_100_rounds": wall * MANY_ROUNDS / (MANY_ROUNDS - 1),
                      "device_ms_per_round": group.last_ms / (MANY_ROUNDS - 1),
                      "graph_launches_per_round": 1}
        group.close()
        for b in boosters:
            b.close()
    planes, boosters = fits()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for b in boosters:
        b.update(MANY_ROUNDS)
    torch.cuda.synchronize()
    serial = time.perf_counter() - t0
    rows = sum(len(y) for _, y in sets)
    line = {"metric": "64-dataset batch fit s/100 iters", "value": batch, "unit": "s",
            "n_gpus": 1, "steps": MANY_ROUNDS, "warmup": W,
            "ms_per_step": batch / MANY_ROUNDS * 1000.0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.mode == "exact" else args.mode,
            "data": "synthetic (seeded ragged-many family)",
            "config": {"workload": MANY_WORKLOAD, "datasets": len(sets), "rows": rows,
                       "hist_mode": args.mode, "timing": "wall clock, synchronized"},
            "one_at_a_time_s": serial, "concurrency_speedup": serial / batch,
            "one_graph_launch": one_launch,
            "e2e": {"value": batch, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "gpu_launches": launches, "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = many_reference(sets, cuts)
    print(json.dumps(line), flush=True)


def many_reference(sets, cuts, every=8, steps=3):
    """The reference's CPU booster (oracle/_ref, all host threads) on every
    8th dataset for `steps` rounds; per-round time summed and scaled to all
    64 datasets (by rows) and 100 rounds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ref = O.RefLib()
    threads = len(os.sched_getaffinity(0))
    tc = O.TreeCfg(max_depth=6, learning_rate=0.1, n_iters=steps, n_threads=threads)
    t, r = 0.0, 0
    for (X, y), (c, o) in list(zip(sets, cuts))[::every]:
        ds = ref.dataset(X, y, c, o)
        t0 = time.perf_counter()
        ref.train(ds, tc)
        t += (time.perf_counter() - t0) / steps
        r += len(y)
    total = sum(len(y) for _, y in sets)
    value = t * (total / r) * MANY_ROUNDS
    return {"value": value, "unit": "s", "cores": threads, "kind": "reference",
            "sample": f"every {every}th dataset ({r:,} rows), {steps} rounds, per-round time "
                      f"x {total / r:.3g} (rows) x {MANY_ROUNDS} (rounds)"}


ACC_ROUNDS = {"wide": 50, "multiclass": 300, "many": 100}


def _mse(a, b):
    return float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))


def _softmax_loss(y, S):
    S = np.asarray(S, np.float64)
    S = S - S.max(axis=1, keepdims=True)
    lse = np.log(np.exp(S).sum(axis=1))
    return float(np.mean(lse - S[np.arange(len(y)), y.astype(np.int64)]))


def _hist_err_mse(bb, plane, scores, y):
    """The int8 root histogram of the fit's final squared-error gradients
    (g = score - y, h = 1) against FP64 sums: relative L1 error of the
    gradient cells (h is constant, so its cells are exact)."""
    g = (np.asarray(scores, np.float64) - y).astype(np.float32)
    q = bb.populate(plane, bb.TrainParams(hist_mode="int8", seed=7), g,
                    np.ones_like(g))
    codes = plane.bins()
    G = np.concatenate([np.bincount(codes[f], weights=g.astype(np.float64),
                                    minlength=int(plane.n_bins[f]))
                        for f in range(codes.shape[0])])
    return {"g_rel_l1": float(np.abs(q[:, 0] - G).sum() / np.abs(G).sum())}


def accuracy_main(args):
    """The quantised form against the plain form on held-out rows of each
    configuration's generator: validation loss (and class accuracy) of both
    fits and their difference, and the int8 histogram's error against FP64
    sums. One JSON line per configuration."""
    import bonsai_b200 as bb
    from bonsai_b200 import synth
    from bonsai_b200.binning import fit_cuts
    from bonsai_b200.build import build_library
    build_library()
    out = []
    # wide sparse leafwise: 1,000,000 training rows and 100,000 held out
    X, y = synth.wide_sparse(n=1_100_000)
    Xt, yt, Xv, yv = X[:1_000_000], y[:1_000_000], X[1_000_000:], y[1_000_000:]
    cuts, off = fit_cuts(Xt, max_bin=256)
    pt, pv = bb.Plane(Xt, cuts, off), bb.Plane(Xv, cuts, off)
    R = ACC_ROUNDS["wide"]
    res = {}
    for mode in ("int8", "exact"):
        b = bb.Booster(pt, yt, bb.TrainParams(hist_mode=mode, **config_tc("wide", bb)),
                       max_trees=R)
        b.update(R)
        res[mode] = _mse(bb.predict(pv, b.trees(), b.init_score, 0.1), yv)
        if mode == "int8":
            herr = _hist_err_mse(bb, pt, b.scores(), yt)
        b.close()
    out.append({"config": "wide", "rounds": R, "valid_rows": len(yv),
                "valid_mse": res, "delta_mse": res["int8"] - res["exact"],
                "rel_delta_mse": (res["int8"] - res["exact"]) / res["exact"],
                "hist_error_vs_fp64": herr})
    del X, Xt, pt, pv
    # multiclass levelwise softmax: 581,012 training rows and 100,000 held out
    X, y = synth.multiclass_onehot(n=681_012)
    Xt, yt, Xv, yv = X[:581_012], y[:581_012], X[581_012:], y[581_012:]
    cuts, off = fit_cuts(Xt, max_bin=255)
    pt, pv = bb.Plane(Xt, cuts, off), bb.Plane(Xv, cuts, off)
    R = ACC_ROUNDS["multiclass"]
    res = {}
    for mode in ("int8", "exact"):
        b = bb.Booster(pt, yt, bb.TrainParams(hist_mode=mode, use_graph=True,
                                              **config_tc("multiclass", bb)), max_trees=R)
        b.update(R)
        S = bb.predict_classes(pv, b.trees(), b.init_scores, 0.1)
        res[mode] = {"logloss": _softmax_loss(yv, S),
                     "accuracy": float(np.mean(np.argmax(S, axis=1) == yv))}
        b.close()
    out.append({"config": "multiclass", "rounds": R, "valid_rows": len(yv), "valid": res,
                "delta_logloss": res["int8"]["logloss"] - res["exact"]["logloss"],
                "delta_accuracy": res["int8"]["accuracy"] - res["exact"]["accuracy"]})
    del X, Xt, pt, pv
    # the 64 ragged datasets: 20% of each dataset's rows held out
    R = ACC_ROUNDS["many"]
    deltas, rels = [], []
    for X, y in synth.ragged_many():
        k = int(len(y) * 0.8)
        cuts, off = fit_cuts(X[:k])
        pt, pv = bb.Plane(X[:k], cuts, off), bb.Plane(X[k:], cuts, off)
        res = {}
        for mode in ("int8", "exact"):
            b = bb.Booster(pt, y[:k], bb.TrainParams(max_depth=6, learning_rate=0.1,
                                                     hist_mode=mode, use_graph=True),
                           max_trees=R)
            b.update(R)
            res[mode] = _mse(bb.predict(pv, b.trees(), b.init_score, 0.1), y[k:])
            b.close()
        deltas.append(res["int8"] - res["exact"])
        rels.append((res["int8"] - res["exact"]) / res["exact"])
        pt.close()
        pv.close()
    out.append({"config": "many", "rounds": R, "datasets": len(deltas),
                "rel_delta_mse": {"mean": float(np.mean(rels)), "max": float(np.max(rels)),
                                  "min": float(np.min(rels))}})
    for line in out:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="int8", choices=["exact", "int8", "int16"])
    ap.add_argument("--compare-rounds", type=int, default=N_ROUNDS,
                    help="fit: rounds of the plain form's fit for the quantised/plain ratio "
                         "and the AUC delta (0 skips it)")
    ap.add_argument("--rows", type=int, default=10_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default histogram launch shape (no autotuning)")
    ap.add_argument("--no-batch", action="store_true",
                    help="many: skip the one-launch batch (bb_batch) leg")
    ap.add_argument("--eval-rows", type=int, default=1_000_000,
                    help="fit: validation rows for the AUC and logloss (0 skips)")
    ap.add_argument("--workload", default="fit",
                    choices=["fit", "serve", "wide", "multiclass", "many", "accuracy"])
    ap.add_argument("--batches", default=",".join(map(str, SERVE_BATCHES)),
                    help="serve: predict request batch sizes")
    ap.add_argument("--shap-batches", default=",".join(map(str, SHAP_BATCHES)),
                    help="serve: TreeSHAP request batch sizes")
    args = ap.parse_args()
    W = max(3, args.warmup)
    K = max(1, args.steps)

    world, rank, local = dist_init(args.gpus)
    if args.workload == "accuracy":
        if rank == 0:
            accuracy_main(args)
        barrier(world)
        return
    if args.workload == "many":
        if rank == 0:
            many_main(args)
        barrier(world)
        return
    if args.workload in CONFIGS:
        # one GPU; other ranks (if any) idle
        if rank == 0:
            config_main(args, args.workload)
        barrier(world)
        return
    if args.workload == "serve":
        # one replica per GPU; rank 0 reports
        if args.impl == "reference":
            if rank == 0:
                serve_reference(args)
            return
        import bonsai_b200 as bb
        from bonsai_b200.build import build_library
        if rank == 0:
            build_library()
        barrier(world)
        bb.lib().bb_select_device(local)
        if rank == 0:
            serve_ours(args, local)
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        if rank == 0:
            reference_main(args, W, K)
        return
    fit_main(args, world, rank, local, W, K)


def fit_config(rows):
    """The workload's config: the same dict on both arms."""
    return {"workload": WORKLOAD, "rows": rows, "features": 28, "rounds": N_ROUNDS,
            "l2": "inputs larger than L2 (bins 280 MB, gradient pairs 80 MB)",
            "excluded": "cut fitting (the same fixed cuts on both arms)"}


def reference_main(args, W, K):
    """The reference arm: the reference's own CPU depthwise grower on all
    rows, K timed rounds after W warm-up rounds."""
    X, y, cuts, off = make_data(args.rows)
    cb = cpu_reference(X, y, cuts, off, K, W)
    line = {"metric": METRIC, "value": cb["value"], "unit": "s", "impl": "reference",
            "n_gpus": args.gpus, "steps": K, "warmup": W,
            "ms_per_step": cb["value"] / N_ROUNDS * 1000.0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded HIGGS-shaped stand-in)",
            "config": fit_config(args.rows), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def auc(y, p):
    """Area under the ROC curve (ties share their mean rank)."""
    y = np.asarray(y) > 0.5
    p = np.asarray(p, np.float64)
    order = np.argsort(p, kind="stable")
    ps = p[order]
    ranks = np.empty(len(p))
    # mean rank over runs of equal scores
    starts = np.flatnonzero(np.r_[True, ps[1:] != ps[:-1]])
    ends = np.r_[starts[1:], len(p)]
    mean = (starts + ends + 1) / 2.0
    ranks[order] = np.repeat(mean, ends - starts)
    n1 = int(y.sum())
    n0 = len(y) - n1
    return float((ranks[y].sum() - n1 * (n1 + 1) / 2.0) / (n1 * n0))


def logloss(y, margin):
    m = np.asarray(margin, np.float64)
    y = np.asarray(y, np.float64)
    return float(np.mean(np.logaddexp(0.0, m) - y * m))


def hist_error(bb, plane, scores, y, seed=7):
    """The int8 histogram against FP64 sums, over the gradients of the fit's
    final scores (logloss: g = p - y, h = p (1 - p)) at the root (every row):
    relative L1 error of the gradient and hessian cells, and the largest cell
    error in units of the stochastic-rounding spread (scale x sqrt(count))."""
    s = np.asarray(scores, np.float64)
    p = 1.0 / (1.0 + np.exp(-s))
    g = (p - y).astype(np.float32)
    h = (p * (1.0 - p)).astype(np.float32)
    q = bb.populate(plane, bb.TrainParams(hist_mode="int8", seed=seed), g, h)
    codes = plane.bins()
    nb = np.asarray(plane.n_bins, np.int64)
    G, H, N = [], [], []
    for f in range(codes.shape[0]):
        c = codes[f]
        G.append(np.bincount(c, weights=g.astype(np.float64), minlength=nb[f]))
        H.append(np.bincount(c, weights=h.astype(np.float64), minlength=nb[f]))
        N.append(np.bincount(c, minlength=nb[f]))
    G, H, N = np.concatenate(G), np.concatenate(H), np.concatenate(N)
    sg = float(np.abs(g).max()) / 127.0
    sh = float(h.max()) / 127.0
    eg = np.abs(q[:, 0] - G)
    eh = np.abs(q[:, 1] - H)
    live = N > 0
    return {"where": "root of the final round's gradients, every row",
            "g_rel_l1": float(eg.sum() / np.abs(G).sum()),
            "h_rel_l1": float(eh.sum() / np.abs(H).sum()),
            "g_max_sigmas": float((eg[live] / (sg * np.sqrt(N[live]))).max()),
            "h_max_sigmas": float((eh[live] / (sh * np.sqrt(N[live]))).max())}


def fit_main(args, world, rank, local, W, K):
    """The headline: a complete 500-round fit in each form on the 10M x 28
    data (device time with inputs resident, and wall clock end to end), the
    validation AUC and logloss of both, and K device-timed rounds."""
    import torch

    import bonsai_b200 as bb
    from bonsai_b200 import synth
    from bonsai_b200.build import build_library
    if rank == 0:
        build_library()
    barrier(world)
    bb.lib().bb_select_device(local)
    X, y, cuts, off = make_data(args.rows)
    n_fit, F = X.shape
    # N > 1: the quantised fit is row-sharded -- each rank holds a contiguous
    # slice of the same rows and the ranks combine integer histograms over
    # NCCL (strong scaling; trees equal the one-GPU fit's). The exact form's
    # float cells do not combine exactly, so N > 1 runs the quantised form only.
    sharded = world > 1
    if sharded and args.mode == "exact":
        raise SystemExit("bench: a row-sharded fit needs --mode int8 or int16")
    comm = None
    row0 = 0
    init = None
    if sharded:
        from bonsai_b200 import dist as bdist
        row0, row1 = bdist.shard_range(n_fit, world, rank)
        X = np.ascontiguousarray(X[row0:row1])
        y = np.ascontiguousarray(y[row0:row1])
        init = bdist.sharded_init_score(y, n_fit, "logloss", world, rank)
        comm = bdist.open_comm(world, rank)
    n = X.shape[0]
    Xp = torch.empty((n, F), dtype=torch.float32, pin_memory=True).numpy()
    Xp[...] = X
    yp = torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
    yp[...] = y

    def params(mode, hist_ctas=0):
        return bb.TrainParams(objective="logloss", max_depth=8, learning_rate=0.1,
                              min_data_in_leaf=20, hist_mode=mode, use_graph=True,
                              hist_ctas=hist_ctas)

    tuned = {"hist_ctas": 0}

    def booster(plane, mode, max_trees):
        p = params(mode, tuned["hist_ctas"] if mode == args.mode else 0)
        if sharded:
            return bb.Booster(plane, yp, p, max_trees=max_trees, comm=comm,
                              row_offset=row0, total_rows=n_fit, init_score=init)
        return bb.Booster(plane, yp, p, max_trees=max_trees)

    # the quantised build's launch shape for this data, timed once per shape
    # (bonsai_b200.autotune; cached on disk) before anything is timed
    autotune = None
    if args.mode != "exact" and not sharded and not args.no_tune:
        tplane = bb.Plane(Xp, cuts, off)
        t0 = time.perf_counter()
        tp = bb.tune(tplane, yp, params(args.mode))
        autotune = {"hist_ctas": tp.hist_ctas, "tune_s": time.perf_counter() - t0}
        from bonsai_b200 import autotune as _at
        ent = _at.load().get(_at.shape_key(tplane.n_rows, tplane.n_feats, True, tp,
                                           _at.device_name()))
        if ent is not None:
            autotune["ms_per_round"] = ent["ms_per_round"]
        tplane.close()
        tuned["hist_ctas"] = tp.hist_ctas

    # ---- the complete fit, end to end through the C ABI with host buffers:
    # pinned X -> ingest (H2D + bin application), labels up, 500 rounds, the
    # model and the training scores down. `value` is the device time of its
    # 500 rounds (CUDA events on the booster's stream; inputs resident).
    barrier(world)
    with Clocks(local) as clk_fit:
        t0 = time.perf_counter()
        plane = bb.Plane(Xp, cuts, off)
        t_plane = time.perf_counter() - t0
        b = booster(plane, args.mode, N_ROUNDS)
        t_setup = time.perf_counter() - t0
        b.update(N_ROUNDS)
        t_fit = time.perf_counter() - t0 - t_setup
        fit_ms = b.last_ms
        t1 = time.perf_counter()
        trees = b.trees()
        scores = b.scores()
        t_down = time.perf_counter() - t1
        wall = time.perf_counter() - t0
    fit_ms = max_over_ranks(fit_ms, world)
    wall = max_over_ranks(wall, world)
    init_score = b.init_score
    b.close()
    tree_bytes = sum(t.feature.nbytes * 8 for t in trees)

    # ---- K device-timed rounds after W warm-up rounds (the per-step figure),
    # and one profiled round for the phase and per-level histogram figures
    b = booster(plane, args.mode, W + K + 4)
    b.update(W)
    barrier(world)
    with Clocks(local) as clk:
        b.update(K)
    ms = max_over_ranks(b.last_ms / K, world)
    barrier(world)
    prof = b.profile_round()
    b.close()

    # ---- the plain form: a complete 500-round fit on the same plane
    plain = None
    plain_trees = None
    if args.mode != "exact" and args.compare_rounds > 0 and not sharded:
        bp = booster(plane, "exact", args.compare_rounds)
        bp.update(args.compare_rounds)
        pms = bp.last_ms
        plain_trees = bp.trees()
        plain_init = bp.init_score
        bp.close()
        plain = {"rounds": args.compare_rounds, "device_s": pms / 1000.0,
                 "ms_per_round": pms / args.compare_rounds,
                 "quantised_speedup": (pms / args.compare_rounds) / (fit_ms / N_ROUNDS)}

    # ---- accuracy on the validation rows (the generator's seed 10,000,001)
    accuracy = None
    if rank == 0 and args.eval_rows > 0:
        Xv, yv = synth.tall_binary(n=args.eval_rows, seed=10_000_001)
        pv = bb.Plane(Xv, cuts, off)
        mq = bb.PredictPlan(pv, trees, init_score, 0.1).run(pv)
        accuracy = {"valid_rows": args.eval_rows,
                    args.mode: {"auc": auc(yv, mq), "logloss": logloss(yv, mq)}}
        if plain_trees is not None:
            mp = bb.PredictPlan(pv, plain_trees, plain_init, 0.1).run(pv)
            accuracy["exact"] = {"auc": auc(yv, mp), "logloss": logloss(yv, mp),
                                 "rounds": len(plain_trees)}
            if len(plain_trees) == len(trees):
                accuracy["delta_auc"] = accuracy[args.mode]["auc"] - accuracy["exact"]["auc"]
                accuracy["delta_logloss"] = (accuracy[args.mode]["logloss"] -
                                             accuracy["exact"]["logloss"])
        pv.close()
        if args.mode == "int8" and not sharded:
            accuracy["hist_error_vs_fp64"] = hist_error(bb, plane, scores, y)
    if comm is not None:
        comm.close()

    peak, peak_kind = peaks()
    hist_gbs = prof["hist_bytes"] / (prof["hist_ms"] * 1e-3) / 1e9
    # DRAM bytes of the build: the measured bytes per algorithmic byte of a
    # full-size tree (one ncu pass per launch, the L2 as the fit leaves it),
    # times this tree's algorithmic bytes
    traffic = traffic_ratio = None
    tpath = os.path.join(ROOT, "profiles", "qhist_t_tall_binary_int8_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            td = json.load(f)
        traffic_ratio = td.get(args.mode, {}).get("dram_per_algorithmic_byte")
        if traffic_ratio is not None:
            traffic = traffic_ratio * prof["hist_bytes"]
    per_row = F + (2.0 if args.mode == "int8" else 4.0 if args.mode == "int16" else 8.0) + 4.0
    levels = [{"rows": r, "ms": t, "gbs": (r * per_row) / (t * 1e-3) / 1e9 if t > 0 else None}
              for r, t in zip(prof["build_rows"], prof["build_ms"])]
    # partition per level: every row's id and its split-feature code read,
    # its id written; the last level (whose rows are never listed) counts
    # its left rows only
    part_levels = max(1, len(levels) - 1)
    part_bytes = part_levels * n * (4 + 1 + 4) + n * (4 + 1)
    value = fit_ms / 1000.0
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "strong" if sharded else "weak",
        "vs_baseline": None, "dtype": "f32" if args.mode == "exact" else args.mode,
        "data": "synthetic (seeded HIGGS-shaped stand-in)",
        "config": fit_config(n_fit),
        "arm": {"hist_mode": args.mode, "graph": True, "rows_per_gpu": n,
                "parallelism": (f"row shards x{world} (NCCL all-reduce of integer "
                                "histograms)" if sharded else "single"),
                "value": f"device time of a complete {N_ROUNDS}-round fit (CUDA events on "
                         "the booster's stream, plane and labels resident)",
                "ms_per_step": f"{K} device-timed rounds after {W} warm-up rounds"},
        "fit": {"rounds": len(trees), "device_s": value, "ms_per_round": fit_ms / N_ROUNDS,
                "wall_s": wall},
        "e2e": {"value": wall, "unit": "s",
                "h2d_bytes_per_step": (X.nbytes + y.nbytes) / N_ROUNDS,
                "d2h_bytes_per_step": (tree_bytes + scores.nbytes) / N_ROUNDS,
                "setup_s": t_setup, "ingest_s": t_plane, "rounds_s": t_fit,
                "download_s": t_down,
                "what": f"wall clock: pinned host X and labels -> ingest -> {N_ROUNDS} rounds "
                        "-> trees and training scores on the host"},
        "plain_form": plain,
        "accuracy": accuracy,
        "autotune": autotune,
        "roofline": {"bound": "hbm",
                     "kernel": ("histogram build (qhist_t_kernel per level)" if args.mode != "exact"
                                else "histogram build (count+offsets+scatter+chain)"),
                     "achieved": hist_gbs, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": hist_gbs / peak, "traffic": traffic,
                     "traffic_per_algorithmic_byte": traffic_ratio,
                     "algorithmic_bytes_per_tree": prof["hist_bytes"],
                     "hist_ms_per_tree": prof["hist_ms"]},
        "hist_levels": levels,
        "partition": {"ms_per_tree": prof["partition_ms"],
                      "algorithmic_bytes_per_tree": part_bytes,
                      "gbs": part_bytes / (prof["partition_ms"] * 1e-3) / 1e9,
                      "frac": part_bytes / (prof["partition_ms"] * 1e-3) / 1e9 / peak},
        "phases_ms": {k: prof[k] for k in ("hist_ms", "partition_ms", "find_ms", "other_ms",
                                           "total_ms")},
        "gpu_launches": int(prof["launches"]) * K,
        "clocks": clk.summary(),
        "clocks_fit": clk_fit.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(X, y, cuts, off, steps=K, warmup=W)
    if rank == 0:
        print(json.dumps(line), flush=True)
    plane.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
