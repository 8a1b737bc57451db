#!/usr/bin/env python
"""Benchmark: the tall binary-classification fit (10,000,000 rows x 28 float32
features, logloss, depthwise depth 8, 255 bins, lr 0.1) on B200.

A step is one boosting round (one depth-8 tree over all 10M rows, with the
resident gradient and score update). The metric is the fit time for 500
rounds, reported as ms_per_step x 500: device time of K timed rounds (CUDA
events on the booster's stream, after W warm-up rounds, a barrier and a
synchronize on both sides, max over ranks). The bins plane (280 MB) and the
per-row state exceed the 126 MB L2, so no flush is needed between rounds.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode exact|int8|int16]
  python bench.py --impl reference      # the reference's CPU grower, timed

Multi-GPU (torchrun): every rank fits its own replica of the workload (one
fit per GPU, no collective in the data path); value is the time for all
ranks' fits, i.e. the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "10M×28 fit s/500 iters: int-quantised vs plain GPU at ΔAUC≤1e-3; hist GB/s"
WORKLOAD = "tall binary logloss 10,000,000x28, depthwise depth 8, 255 bins, lr 0.1"
N_ROUNDS = 500
CPU_SAMPLE_ROWS = 1_000_000


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
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

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
            time.sleep(0.3)
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


def cpu_reference(X, y, cuts, off, steps, warmup, rows=CPU_SAMPLE_ROWS):
    """The reference's own CPU depthwise grower (oracle/_ref, compiled from
    its sources) on the first `rows` rows, all host threads; per-round time
    scaled by rows to the full workload. Falls back to the oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n_full = X.shape[0]
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
            "sample": f"first {rows:,} rows x 28, {steps} timed depth-8 logloss rounds "
                      f"({warmup} warm-up), per-round time x {n_full / rows:g} (rows) "
                      f"x {N_ROUNDS} (rounds)"}


def make_data(rows):
    from bonsai_b200 import synth
    from bonsai_b200.binning import fit_cuts
    X, y = synth.tall_binary(n=rows)
    cuts, off = fit_cuts(X, max_bin=255)
    return X, y, cuts, off


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="int8", choices=["exact", "int8", "int16"])
    ap.add_argument("--compare-steps", type=int, default=5,
                    help="timed rounds of the plain form for the quantised/plain ratio "
                         "(0 skips it)")
    ap.add_argument("--rows", type=int, default=10_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    W = max(3, args.warmup)
    K = max(1, args.steps)

    world, rank, local = dist_init(args.gpus)
    if args.impl == "reference":
        if rank != 0:
            return
        X, y, cuts, off = make_data(args.rows)
        cb = cpu_reference(X, y, cuts, off, K, W)
        line = {"metric": METRIC, "value": cb["value"], "unit": "s", "impl": "reference",
                "n_gpus": args.gpus, "steps": K, "warmup": W,
                "ms_per_step": cb["value"] / N_ROUNDS * 1000.0, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "rows": args.rows, "features": 28,
                           "rounds": N_ROUNDS, "host_threads": cb["cores"]},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import bonsai_b200 as bb
    from bonsai_b200.build import build_library
    if rank == 0:
        build_library()
    barrier(world)
    bb.lib().bb_select_device(local)
    X, y, cuts, off = make_data(args.rows)
    n_fit, F = X.shape
    # N > 1: the quantised fit is row-sharded -- each rank holds a contiguous
    # slice of the same 10M rows and the ranks combine integer histograms over
    # NCCL (strong scaling; trees equal the one-GPU fit's); the exact form's
    # float cells do not combine exactly, so it runs one replica per GPU
    sharded = world > 1 and args.mode != "exact"
    comm = None
    row0 = 0
    if sharded:
        from bonsai_b200 import dist as bdist
        row0, row1 = bdist.shard_range(n_fit, world, rank)
        X = np.ascontiguousarray(X[row0:row1])
        y = np.ascontiguousarray(y[row0:row1])
        init = bdist.sharded_init_score(y, n_fit, "logloss", world, rank)
        comm = bdist.open_comm(world, rank)
    n = X.shape[0]

    # ---- end to end through the C ABI with host buffers: ingest (H2D of the
    # raw matrix + bin application), labels up, rounds, model + scores down
    import torch
    Xp = torch.empty((n, F), dtype=torch.float32, pin_memory=True).numpy()
    Xp[...] = X
    yp = torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
    yp[...] = y
    params = bb.TrainParams(objective="logloss", max_depth=8, learning_rate=0.1,
                            min_data_in_leaf=20, hist_mode=args.mode, use_graph=True)
    barrier(world)
    t0 = time.perf_counter()
    plane = bb.Plane(Xp, cuts, off)
    if sharded:
        b = bb.Booster(plane, yp, params, max_trees=W + K + 4, comm=comm, row_offset=row0,
                       total_rows=n_fit, init_score=init)
    else:
        b = bb.Booster(plane, yp, params, max_trees=W + K + 4)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0

    # ---- device-timed rounds
    b.update(W)
    barrier(world)
    with Clocks(local) as clk:
        b.update(K)
    ms = b.last_ms / K
    ms = max_over_ranks(ms, world)
    barrier(world)

    t1 = time.perf_counter()
    trees = b.trees()
    scores = b.scores()
    t_down = (time.perf_counter() - t1) * (N_ROUNDS / max(1, len(trees)))
    tree_bytes = sum(t.feature.nbytes * 8 for t in trees) / max(1, len(trees))

    prof = b.profile_round()
    b.close()
    if comm is not None:
        comm.close()

    # the plain (exact) form on the same plane, for the headline ratio
    plain = None
    if args.mode != "exact" and args.compare_steps > 0 and not sharded:
        pp = bb.TrainParams(objective="logloss", max_depth=8, learning_rate=0.1,
                            min_data_in_leaf=20, hist_mode="exact", use_graph=True)
        bp = bb.Booster(plane, yp, pp, max_trees=W + args.compare_steps + 1)
        bp.update(W)
        barrier(world)
        bp.update(args.compare_steps)
        pms = max_over_ranks(bp.last_ms / args.compare_steps, world)
        bp.close()
        plain = {"value": pms * N_ROUNDS / 1000.0, "unit": "s", "ms_per_step": pms,
                 "steps": args.compare_steps,
                 "quantised_speedup": pms / ms}
    peak, peak_kind = peaks()
    hist_gbs = prof["hist_bytes"] / (prof["hist_ms"] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "qhist_t_tall_binary_int8_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            td = json.load(f)
        traffic = td.get(args.mode, {}).get("dram_bytes_per_tree")

    value = ms * N_ROUNDS / 1000.0
    e2e = t_setup + value + t_down
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "strong" if sharded else "weak",
        "vs_baseline": None, "dtype": "f32" if args.mode == "exact" else args.mode,
        "data": "synthetic (seeded HIGGS-shaped stand-in)",
        "config": {"workload": WORKLOAD, "rows": n_fit, "features": F, "rounds": N_ROUNDS,
                   "hist_mode": args.mode, "graph": True,
                   "parallelism": (f"row shards x{world} (NCCL all-reduce of integer "
                                   "histograms)" if sharded else
                                   f"replicas x{world}" if world > 1 else "single"),
                   "rows_per_gpu": n,
                   "l2": "inputs larger than L2 (bins 280 MB, gh 80 MB)"},
        "e2e": {"value": e2e, "unit": "s",
                "h2d_bytes_per_step": (X.nbytes + y.nbytes) / N_ROUNDS,
                "d2h_bytes_per_step": tree_bytes + scores.nbytes / N_ROUNDS,
                "setup_s": t_setup, "download_s_per_500": t_down},
        "roofline": {"bound": "hbm",
                     "kernel": ("histogram build (qhist_t_kernel per level)" if args.mode != "exact"
                                else "histogram build (count+offsets+scatter+chain)"),
                     "achieved": hist_gbs, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": hist_gbs / peak, "traffic": traffic,
                     "algorithmic_bytes_per_tree": prof["hist_bytes"],
                     "hist_ms_per_tree": prof["hist_ms"]},
        "phases_ms": {k: prof[k] for k in ("hist_ms", "partition_ms", "find_ms", "other_ms",
                                           "total_ms")},
        "plain_form": plain,
        "gpu_launches": int(prof["launches"]) * K,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(X, y, cuts, off, steps=2, warmup=1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    plane.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
