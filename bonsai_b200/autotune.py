"""Launch-shape autotuner for the quantised histogram build.

The quantised build (qhist_t_kernel) is a persistent grid over a level's
row chunks, `hist_ctas` CTAs per mirror tile of 32 feature codes. One CTA
per SM suits a plane of one tile (28 features: a level is one 148-CTA
wave); on a plane of many tiles (2,000 features: 63 tiles) every CTA zeroes
and flushes a 64 KB table per node, so fewer, longer CTAs per tile pay off,
and the default takes about two waves over all tiles. Which count is
fastest depends on the shape (rows, features, the grower's node sizes), so
`tune` times candidates on the caller's own data -- a few boosting rounds
each, device time on the booster's stream -- and keeps the fastest per
shape in a JSON cache on disk.

The knob changes the launch only: the quantised cells are order-free
integer sums, so every candidate grows the same trees. The plain (exact)
form's build does not take it, and is returned unchanged.

  params = bonsai_b200.tune(plane, labels, params)   # cached per shape
"""

from __future__ import annotations

import dataclasses
import json
import math
import os
import time

CANDIDATES = (0, 148, 74, 37, 16, 8, 4, 2, 1)


def cache_path() -> str:
    """$BONSAI_B200_TUNE_CACHE, else ~/.cache/bonsai_b200/tune.json."""
    p = os.environ.get("BONSAI_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "bonsai_b200", "tune.json")


def device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name()
    except Exception:
        pass
    return "cuda"


def shape_key(n_rows: int, n_feats: int, u8: bool, params, device: str) -> str:
    """What the fastest launch depends on: the device, the rows (to a power
    of two), the features, the code width, the grower and its size, the
    quantised form and the row sample (to a tenth)."""
    size = params.max_leaves if params.grower == "leafwise" else params.max_depth
    rows = 1 << max(0, math.ceil(math.log2(max(1, n_rows))))
    sub = round(float(params.subsample if 0.0 < params.subsample < 1.0 else 1.0), 1)
    return (f"{device}|rows<={rows}|feats={n_feats}|{'u8' if u8 else 'u16'}|{params.grower}"
            f"{size}|{params.hist_mode}|sub={sub}")


def load(path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def store(entries: dict, path: str | None = None) -> None:
    """Writes the cache atomically (a temporary file, then a rename)."""
    path = path or cache_path()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(entries, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


MARGIN = 0.02


def pick(times: dict, margin: float = MARGIN) -> int:
    """The fastest candidate, unless it beats the default (0) by less than
    `margin` of the default's time -- a few timed rounds carry that much
    noise, and the default is the shape the library was tuned by hand for.
    Ties go to the earlier candidate."""
    best = None
    for c, t in times.items():
        if best is None or t < times[best]:
            best = c
    if 0 in times and times[best] > times[0] * (1.0 - margin):
        return 0
    return int(best)


def time_rounds(plane, labels, params, rounds: int = 3, warmup: int = 1) -> float:
    """Device milliseconds per boosting round with these params."""
    from . import Booster
    b = Booster(plane, labels, params, max_trees=warmup + rounds)
    try:
        b.update(warmup)
        b.update(rounds)
        return b.last_ms / rounds
    finally:
        b.close()


def tune(plane, labels, params, candidates=CANDIDATES, rounds: int = 3,
         path: str | None = None, timer=None, refresh: bool = False):
    """params with hist_ctas set to the fastest candidate for this shape
    (from the cache when the shape was timed before). `timer(params) -> ms`
    replaces the device timing (tests)."""
    if params.hist_mode == "exact":
        return params
    key = shape_key(plane.n_rows, plane.n_feats, bool(max(plane.n_bins) <= 256), params,
                    device_name())
    entries = load(path)
    hit = entries.get(key)
    if hit is not None and not refresh:
        return dataclasses.replace(params, hist_ctas=int(hit["hist_ctas"]))
    timer = timer or (lambda p: time_rounds(plane, labels, p, rounds))
    times = {}
    for c in candidates:
        times[int(c)] = float(timer(dataclasses.replace(params, hist_ctas=int(c))))
    best = pick(times)
    entries = load(path)  # another process may have written meanwhile
    entries[key] = {"hist_ctas": best, "ms_per_round": times,
                    "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    store(entries, path)
    return dataclasses.replace(params, hist_ctas=best)
