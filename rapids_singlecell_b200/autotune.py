"""Autotuner of the persistent sweep's launch shape on the 16-bit path.

The sweep (``k_tc_sweep``) has two choices that the engine otherwise makes by fixed rules: its
layout (two 256-thread tile streams with two threads per row, or one 512-thread stream with four;
two A tiles per stream or one: ``hb_params.sweep_form``) and its CTA cap (``max_sweep_ctas``,
one CTA per SM by default).  ``tune_sweep`` times every candidate that fits on the problem itself
(1 outer x ``iters`` k-means iterations, the sweep's device time from the run profile, best of
``repeats``) and keeps the fastest, keyed by (device, precision, PCs, clusters, batches, a
half-octave bucket of the cell count, block proportion).  The choices live in memory and, with
``cache_path``, in a JSON file.  ``harmonize(..., autotune=True)`` consults it.
"""

from __future__ import annotations

import json
import math
import os
import threading
import warnings

import numpy as np
import torch

from . import _lib
from .harmony import HarmonyProblem

_cache: dict[str, dict] = {}
_lock = threading.Lock()


def shape_key(device, precision: str, n_cells: int, n_pcs: int, n_clusters: int, n_batches: int,
              block_proportion: float = 0.05) -> str:
    """The cache key of a problem shape (cells in half-octave buckets)."""
    name = torch.cuda.get_device_name(device) if torch.cuda.is_available() else "cpu"
    bucket = int(round(2 * math.log2(max(int(n_cells), 1))))
    return (f"{name}|{precision}|d{int(n_pcs)}|K{int(n_clusters)}|B{int(n_batches)}|n{bucket}"
            f"|bp{float(block_proportion):g}")


def candidates(sms: int) -> list[tuple[int, int]]:
    """(sweep_form, max_sweep_ctas) pairs: every layout, with one CTA per SM (0) or a quarter or
    half of the SMs fewer."""
    caps = sorted({0, max(1, 3 * sms // 4), max(1, sms // 2)})
    return [(f, c) for f in sorted(_lib.SWEEP_FORMS) for c in caps]


def load_cache(path: str) -> None:
    """Adds the choices stored at ``path`` (JSON) to the in-memory cache; a file that cannot be
    read as a JSON object of choices is ignored with a warning (the shapes are then re-timed and
    the file rewritten)."""
    if not os.path.exists(path):
        return
    try:
        with open(path) as f:
            data = json.load(f)
        if not isinstance(data, dict) or not all(isinstance(v, dict) and "sweep_form" in v
                                                 for v in data.values()):
            raise ValueError("not a map of sweep choices")
    except (OSError, ValueError) as e:
        warnings.warn(f"sweep autotune cache {path!r} ignored: {e}", RuntimeWarning, stacklevel=2)
        return
    with _lock:
        _cache.update(data)


def save_cache(path: str) -> None:
    with _lock:
        data = dict(_cache)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def cached(key: str) -> dict | None:
    with _lock:
        return _cache.get(key)


def remember(key: str, choice: dict) -> None:
    with _lock:
        _cache[key] = dict(choice)


def tune_sweep(X, cats, n_batches, Y0, theta, *, precision="bf16", n_clusters, block_proportion=0.05,
               iters=2, repeats=2, cache_path=None, force=False, **params) -> dict:
    """Times the sweep candidates on this problem and returns (and caches) the fastest:
    ``{"sweep_form", "max_sweep_ctas", "us_per_launch", "timings"}``.  ``X``, ``cats``, ``Y0`` and
    ``theta`` are as for ``HarmonyProblem``; ``params`` are its other keyword arguments (the
    tolerances and iteration counts are replaced by a fixed 1 x ``iters`` run)."""
    if precision not in ("bf16", "fp16"):
        raise ValueError("the sweep autotuner applies to the 16-bit paths (bf16, fp16)")
    n_cells, n_pcs = (int(v) for v in X.shape)
    key = shape_key(X.device, precision, n_cells, n_pcs, n_clusters, n_batches, block_proportion)
    if cache_path:
        load_cache(cache_path)
    hit = cached(key)
    if hit is not None and not force:
        return hit
    sms = torch.cuda.get_device_properties(X.device).multi_processor_count
    run_kw = {k: v for k, v in params.items()
              if k not in ("max_iter_harmony", "max_iter_clustering", "tol_harmony", "tol_clustering",
                           "sweep_form", "max_sweep_ctas")}
    timings = {}
    best = None
    for form, cap in candidates(sms):
        try:
            prob = HarmonyProblem(X, cats, n_batches, Y0, theta, precision=precision, n_clusters=n_clusters,
                                  block_proportion=block_proportion, max_iter_harmony=1,
                                  max_iter_clustering=int(iters), tol_harmony=-np.inf, tol_clustering=-np.inf,
                                  sweep_form=form, max_sweep_ctas=cap, **run_kw)
        except (ValueError, _lib.HarmonyLibError):
            continue
        t = math.inf
        try:
            for rep in range(int(repeats) + 1):  # the first run warms the launch up
                _, info = prob.run(profile=True)
                pr = info.profile
                if rep > 0 and pr["block_launches"] > 0:
                    t = min(t, pr["block_ms"] / pr["block_launches"] * 1e3)
        except _lib.HarmonyLibError:  # the layout does not fit this shape
            t = math.inf
        finally:
            prob.close()
        timings[f"{form}/{cap}"] = t if math.isfinite(t) else None
        if math.isfinite(t) and (best is None or t < best[2]):
            best = (form, cap, t)
    if best is None:
        choice = {"sweep_form": 0, "max_sweep_ctas": 0, "us_per_launch": None, "timings": timings}
    else:
        choice = {"sweep_form": best[0], "max_sweep_ctas": best[1], "us_per_launch": best[2], "timings": timings}
    remember(key, choice)
    if cache_path:
        save_cache(cache_path)
    return choice
