"""Harmony cell-iterations/s on B200.

One step = one full Harmony integration (fixed 10 outer x 20 k-means
iterations, tolerances -inf) of the 500,000-cell x 50-PC workload (30 cell
types, 8 batches with Dirichlet(1) sizes, per-batch shift N(0, 0.5^2) and
scale U(0.8, 1.2), K = 100, theta = 2, sigma = 0.1), synthetic and seeded.

  value   device-resident throughput of the fused 16-bit tensor-core path
          (bf16 unless --precision says otherwise): inputs already in HBM
  e2e     the same through the public ``harmonize`` call from pinned host
          memory, host->device copy of the embedding and device->host copy of
          the corrected embedding inside the timed region
  plain   the float32 plain path (the drop-in for dtype=np.float32)

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): independent replicas, one per GPU; value = all ranks'
cell-iterations / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# 32 hardware work queues instead of CUDA's default 8, set before CUDA starts in this process:
# the batched section runs 32 streams, and with 8 queues streams share queues and serialise
# (256 problems: 32 streams measured 1.1e9-1.3e9 cell-iters/s, 8 streams 0.7e9-0.9e9).  The
# single-stream measurements are unaffected.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

OUTER, INNER = 10, 20
WORKLOAD = "C2"
METRIC = "Harmony cell-iters/s & p50/p99 latency: BF16 batched vs FP32 plain on 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16", choices=["bf16", "fp16", "fp32", "fp64"],
                    help="path of the headline line (bf16, fp16, fp32); fp64 with --profile-case only")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--sections", default="wide,batched,serving,pca,knn",
                    help="extra measurements on rank 0 beside the headline line: wide (the "
                         "2M-cell x 100-PC workload), batched (256 independent problems), "
                         "serving (Poisson request stream), pca (500k x 2000 covariance PCA), "
                         "knn (500k x 50 exact kNN); empty for none")
    ap.add_argument("--serving-requests", type=int, default=64,
                    help="requests of the serving section (the configuration names 2,000)")
    ap.add_argument("--serving-rates", default="10,100", help="bf16 arrival rates (req/s), comma-separated")
    ap.add_argument("--serving-fp32-rates", default="10", help="fp32 arrival rates (req/s)")
    ap.add_argument("--profile-case", action="store_true",
                    help="one short run for ncu: the same workload for 1 outer x 2 k-means "
                         "iterations, then exit")
    ap.add_argument("--profile-cells", type=int, default=500_000,
                    help="cells of the --profile-case run")
    ap.add_argument("--profile-inner", type=int, default=2,
                    help="k-means iterations of the --profile-case run")
    return ap.parse_args()


def run_profile_case(args):
    import torch

    from rapids_singlecell_b200.harmony import HarmonyProblem
    from rapids_singlecell_b200.synthetic import make_config

    cfg = make_config(WORKLOAD, seed=0, n_cells=args.profile_cells)
    dt = torch.float64 if args.precision == "fp64" else torch.float32
    X = torch.as_tensor(cfg["Z"], device="cuda").to(dt)
    prob = HarmonyProblem(X, cfg["cats"], cfg["n_batches"], torch.as_tensor(cfg["Y0"], device="cuda").to(dt),
                          np.full(cfg["n_batches"], 2.0), precision=args.precision,
                          n_clusters=cfg["n_clusters"], max_iter_harmony=1,
                          max_iter_clustering=args.profile_inner,
                          tol_harmony=-np.inf, tol_clustering=-np.inf)
    _, info = prob.run(profile=True)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": info.profile}))


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


def workload():
    from rapids_singlecell_b200.synthetic import make_config

    cfg = make_config(WORKLOAD, seed=0)
    return cfg


def config_dict(cfg, extra=None):
    n, d = cfg["Z"].shape
    c = {"workload": f"{WORKLOAD}: {n} cells x {d} PCs, {cfg['n_batches']} batches, "
                     f"K={cfg['n_clusters']}, {OUTER} outer x {INNER} k-means iterations fixed",
         "n_cells": n, "n_pcs": d, "n_clusters": cfg["n_clusters"], "n_batches": cfg["n_batches"],
         "outer_iters": OUTER, "kmeans_iters": INNER, "block_proportion": 0.05,
         "l2": "inputs larger than L2 (R, Z_norm and X exceed 126 MB)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
class OracleKmeans:
    """The CPU oracle (NumPy port of the reference algorithm) on the workload, for timing:
    the initial state is built once (``init_s``), ``step()`` runs and times ONE k-means
    iteration of the first outer iteration (shuffle, centroids, similarities, the blocks and the
    objective) on the evolving state, and ``correction()`` times the ridge correction of the
    current state.  Cell-iterations/s = cells / the time of one k-means iteration, so neither the
    initialisation nor the correction is charged to the k-means iterations."""

    def __init__(self, cfg, dtype):
        from oracle import harmony_oracle as ho

        self.ho = ho
        dt = np.dtype(dtype)
        self.dt = dt
        self.X = np.ascontiguousarray(cfg["Z"], dtype=dt)
        self.cats = np.asarray(cfg["cats"], dtype=np.int64)
        self.B, self.K = cfg["n_batches"], cfg["n_clusters"]
        self.n = self.X.shape[0]
        t0 = time.perf_counter()
        self.N_b = np.bincount(self.cats, minlength=self.B).astype(dt)
        self.Pr_b = (self.N_b / self.n).astype(dt)
        self.th = ho.theta_array(2.0, self.B, self.N_b, self.K, 0, dt)
        self.Z_norm = ho.l2_normalize(self.X)
        self.R, self.E, self.O, _ = ho.init_state(self.Z_norm, np.asarray(cfg["Y0"]), self.cats, self.B,
                                                  self.Pr_b, self.th, 0.1, True)
        self.init_s = time.perf_counter() - t0
        self.it = 0

    def step(self):
        t0 = time.perf_counter()
        self.ho.clustering(self.Z_norm, self.R, self.E, self.O, self.Pr_b, self.cats, self.th,
                           n_batches=self.B, sigma=0.1, block_size=int(self.n * 0.05), max_iter=1,
                           tol=-np.inf, seed=self.it & 0xFFFFFFFF, stabilized=True)
        self.it += 1
        return time.perf_counter() - t0

    def correction(self):
        """Z_hat of the current state (harmonize's first outer iteration after `it` k-means
        iterations) and the wall seconds of the correction."""
        ho = self.ho
        t0 = time.perf_counter()
        lam = ho.compute_lambda_kb(self.E, self.O, self.N_b, alpha=0.2, threshold=1e-5, ridge_lambda=1.0,
                                   dynamic_lambda=True)
        Z_hat = ho.correction_batched(self.X, self.R, self.O, lam, self.cats, self.B)
        ho.l2_normalize(Z_hat)
        return Z_hat, time.perf_counter() - t0


def blas_threads():
    try:
        from threadpoolctl import threadpool_info

        return max([i.get("num_threads", 1) for i in threadpool_info()] or [1])
    except Exception:  # noqa: BLE001
        return os.cpu_count() or 1


def cpu_sample_text(n, dtype, iters, init_s, corr_s):
    return (f"NumPy {dtype} oracle of the reference algorithm (the reference has no CPU path), "
            f"{n}-cell workload: cell-iterations/s over {iters} timed k-means iteration(s) of the first outer "
            f"iteration (shuffle, centroids, similarities, 20 blocks, objective); initial state "
            f"{init_s:.1f} s and one ridge correction {corr_s:.1f} s timed separately, not charged")


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cfg = workload()
    n = cfg["Z"].shape[0]
    ok = OracleKmeans(cfg, np.float32)
    for _ in range(args.warmup):
        ok.step()
    times = [ok.step() for _ in range(args.steps)]
    _, corr_s = ok.correction()
    t = float(np.median(times))
    v = n / t
    cores = blas_threads()
    sample = cpu_sample_text(n, "float32", args.steps, ok.init_s, corr_s)
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-iters/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": config_dict(cfg, {"precision": "fp32", "parallelism": "single"}),
           "cpu_baseline": {"value": v, "unit": "cell-iters/s", "cores": cores, "kind": "port",
                            "sample": "one step = one k-means iteration; " + sample,
                            "os_cpu_count": os.cpu_count(), "init_s": ok.init_s, "correction_s": corr_s},
           "e2e": {"value": v, "unit": "cell-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.p = None

    def wait_first_sample(self, limit_s=5.0):
        """Returns once nvidia-smi has written its first line (its start-up, NVML included, is
        then over), or after `limit_s`."""
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < limit_s:
            if os.path.getsize(self.f.name) > 0 or self.p.poll() is not None:
                return
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait(timeout=10)
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4)
                          if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(name):
    """dram bytes per launch of a kernel from its committed ncu summary, if any."""
    f = ROOT / "profiles" / name
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# Extra measurements beside the headline line (rank 0, one GPU each).

def _rel(a, b):
    return float((a.double() - b.double()).abs().max().item() / max(b.double().abs().max().item(), 1e-300))


def _gpu_time(fn, reps):
    """Device time of fn() per call (CUDA events on the current stream), after one warm-up call."""
    import torch

    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def wide_section(dev):
    """The 2,000,000-cell x 100-PC workload (50 types, 32 Zipf(1.2)-sized batches,
    shift N(0, 0.7^2), K = 200, 10 outer x 20 k-means iterations fixed), device
    resident: the bf16 path against the plain fp32 path, and the error of both
    against the engine's float64 path on the same inputs (itself checked against the
    reference's float64 run by the tests)."""
    import torch

    from rapids_singlecell_b200.harmony import HarmonyProblem
    from rapids_singlecell_b200.synthetic import make_config

    cfg = make_config("C3", seed=0)
    n, d = cfg["Z"].shape
    B, K = cfg["n_batches"], cfg["n_clusters"]
    kw = dict(n_clusters=K, max_iter_harmony=OUTER, max_iter_clustering=INNER, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    theta = np.full(B, 2.0)
    X = torch.as_tensor(cfg["Z"], device=dev)
    Y0 = torch.as_tensor(cfg["Y0"], device=dev)
    out = {"workload": f"C3: {n} cells x {d} PCs, {B} batches, K={K}, {OUTER} outer x {INNER} "
                       "k-means iterations fixed, device resident"}
    res = {}
    for prec, reps in (("bf16", 2), ("fp32", 1)):
        prob = HarmonyProblem(X, cfg["cats"], B, Y0, theta, precision=prec, **kw)
        ms = _gpu_time(prob.run, reps)
        res[prec] = prob.Z_hat.clone()
        out[prec] = {"value": n * OUTER * INNER / (ms / 1e3), "unit": "cell-iters/s", "ms_per_run": ms}
        prob.close()
    out["speedup_bf16_vs_fp32"] = out["bf16"]["value"] / out["fp32"]["value"]
    prob = HarmonyProblem(X.double(), cfg["cats"], B, Y0.double(), theta, precision="fp64", **kw)
    prob.run()
    z64 = prob.Z_hat.clone()
    prob.close()
    # against the engine's float64 path of the same 10 x 20 iterations; the comparison with the
    # reference's own kernels in float64 at this size is tests/test_gpu_reference.py
    out["rel_max_abs_err_vs_engine_fp64"] = {p: _rel(res[p], z64) for p in res}
    out["max_abs_err_vs_engine_fp64"] = {p: float((res[p].double() - z64).abs().max().item()) for p in res}
    return out


def batched_section(dev, n_problems=256, streams=32):
    """Independent problems of uneven sizes on one GPU: cells log-uniform in
    [2k, 200k], d in {30, 50}, B uniform in [2, 12], K = min(100, n / 30), each
    from the mixture generator with its own seed (10 types, Dirichlet(1)
    batches); 10 outer x 20 k-means iterations fixed; inputs resident on the
    device.  All problems go through one HarmonyServer (32 streams); bf16 and
    plain fp32 runs of the same set, and the per-problem bf16 vs fp32 error."""
    import torch

    from rapids_singlecell_b200.batched import HarmonyRequest, latency_summary, run_batched
    from rapids_singlecell_b200.synthetic import MixtureSpec, initial_centroids, make_mixture

    rng = np.random.default_rng(7)
    specs = []
    for i in range(n_problems):
        n = int(np.exp(rng.uniform(np.log(2_000), np.log(200_000))))
        specs.append((n, int(rng.choice([30, 50])), int(rng.integers(2, 13))))
    data = []
    for i, (n, d, B) in enumerate(specs):
        Z, cats, _ = make_mixture(MixtureSpec(n, d, 10, B, "dirichlet", (), 0.5, (0.8, 1.2)), 1000 + i)
        K = min(100, n // 30)
        data.append((torch.as_tensor(Z, device=dev), cats, B, initial_centroids(Z, K, 5000 + i), K))
    cell_iters = sum(s[0] for s in specs) * OUTER * INNER

    def reqs(prec, sub=None):
        sel = data if sub is None else data[:sub]
        return [HarmonyRequest(Z, cats, B, Y0, np.full(B, 2.0),
                               dict(n_clusters=K, max_iter_harmony=OUTER, max_iter_clustering=INNER,
                                    tol_harmony=-np.inf, tol_clustering=-np.inf), precision=prec)
                for Z, cats, B, Y0, K in sel]

    out = {"workload": f"{n_problems} problems, cells log-uniform in [2k, 200k] (total "
                       f"{sum(s[0] for s in specs)}), d in {{30, 50}}, B in [2, 12], K = min(100, n/30), "
                       f"{OUTER} outer x {INNER} k-means iterations fixed, {streams} streams"}
    results = {}
    for prec in ("bf16", "fp32"):
        run_batched(reqs(prec, 8), streams=streams, device=dev)  # warm-up: library, plans, threads
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = run_batched(reqs(prec), streams=streams, device=dev)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        results[prec] = r
        out[prec] = {"value": cell_iters / t, "unit": "cell-iters/s", "wall_s": t,
                     **{k: v for k, v in latency_summary(r).items()}}
    out["speedup_bf16_vs_fp32"] = out["bf16"]["value"] / out["fp32"]["value"]
    errs = [_rel(a.Z_hat, b.Z_hat) for a, b in zip(results["bf16"], results["fp32"])]
    out["rel_max_abs_diff_bf16_vs_fp32"] = {"max": float(np.max(errs)), "median": float(np.median(errs))}
    return out


def serving_section(dev, n_requests=64, rates=(10.0, 100.0), fp32_rates=(10.0,), streams=8):
    """A Poisson stream of integration requests through HarmonyServer (HBM budget
    160 GB, 8 streams): cells log-uniform in [5k, 1M], d in {30, 50, 100}, B in
    [2, 32], K = min(200, n / 30), 10 outer x 20 k-means iterations fixed.  Each
    request is the first n cells of a seeded 1M-cell mixture of its d (50 types,
    32 Zipf(1.2)-sized batches, shift N(0, 0.7^2)), its batches folded to B
    (code mod B, renumbered); host input, host result (both copies inside the
    latency).  Latency is from arrival to result."""
    import torch

    from rapids_singlecell_b200.batched import HarmonyRequest, HarmonyServer, latency_summary
    from rapids_singlecell_b200.synthetic import MixtureSpec, initial_centroids, make_mixture

    base = {d: make_mixture(MixtureSpec(1_000_000, d, 50, 32, "zipf", (), 0.7, None, zipf_s=1.2,
                                        min_batch=500), 3000 + d)[:2] for d in (30, 50, 100)}
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(n_requests):
        n = int(np.exp(rng.uniform(np.log(5_000), np.log(1_000_000))))
        d = int(rng.choice([30, 50, 100]))
        B = int(rng.integers(2, 33))
        Z = base[d][0][:n]
        _, cats = np.unique(base[d][1][:n] % B, return_inverse=True)
        B = int(cats.max()) + 1
        K = min(200, n // 30)
        reqs.append((Z, cats.astype(np.int32), B, initial_centroids(Z, K, 7000 + i), K))
    total_cells = sum(r[0].shape[0] for r in reqs)

    def stream_run(prec, rate):
        gaps = rng.exponential(1.0 / rate, len(reqs))
        with HarmonyServer(streams=streams, hbm_budget_bytes=160 << 30, device=dev) as srv:
            for Z, cats, B, Y0, K in reqs[:4]:  # warm-up
                srv.submit(HarmonyRequest(Z, cats, B, Y0, np.full(B, 2.0),
                                          dict(n_clusters=K, max_iter_harmony=1, max_iter_clustering=2),
                                          precision=prec, to_host=True)).result()
            t0 = time.perf_counter()
            futs = []
            for gap, (Z, cats, B, Y0, K) in zip(gaps, reqs):
                time.sleep(gap)
                futs.append(srv.submit(HarmonyRequest(
                    Z, cats, B, Y0, np.full(B, 2.0),
                    dict(n_clusters=K, max_iter_harmony=OUTER, max_iter_clustering=INNER,
                         tol_harmony=-np.inf, tol_clustering=-np.inf), precision=prec, to_host=True)))
            res, errors = [], 0
            for f in futs:
                try:
                    res.append(f.result())
                except Exception:  # noqa: BLE001 - counted and reported
                    errors += 1
            t = time.perf_counter() - t0
        done = sum(r.Z_hat.shape[0] for r in res)
        return {"rate_req_s": rate, "requests": len(reqs), "errors": errors, "makespan_s": t,
                "cells_per_s": done / t, "cell_iters_per_s": done * OUTER * INNER / t,
                **latency_summary(res)}

    out = {"workload": f"{n_requests} Poisson arrivals, cells log-uniform in [5k, 1M] (total {total_cells}), "
                       "d in {30, 50, 100}, B in [2, 32], K = min(200, n/30), "
                       f"{OUTER} outer x {INNER} k-means iterations fixed, HBM budget 160 GB, {streams} streams",
           "bf16": [stream_run("bf16", r) for r in rates],
           "fp32": [stream_run("fp32", r) for r in fp32_rates]}
    torch.cuda.synchronize()
    return out


def _events_ms(fn, reps=3):
    """Median device time of fn() (CUDA events on the current stream) after one warm-up."""
    import torch

    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def _tensor_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def pca_section(dev, n=500_000, g=2000, n_comps=50):
    """PCA upstream of Harmony: a seeded 500,000-cell x 2,000-gene log-normalised-looking matrix
    (rank-20 gamma factor model, Poisson counts, log1p; about 14 % nonzero) generated on the
    device, dense float32 in HBM.  Times the Gram kernel (X^T X and column sums), the projection
    onto 50 components, and the whole covariance PCA; the Gram against cuBLAS float32
    (torch.matmul(X.T, X), the GEMM a dense float32 PCA runs) on the same matrix."""
    import ctypes

    import torch

    from rapids_singlecell_b200 import _lib
    from rapids_singlecell_b200.pca import pca_arrays

    lib = _lib.load()
    gen = torch.Generator(device=dev).manual_seed(11)
    F = torch.distributions.Gamma(2.0, 1.0).sample((n, 20)).to(dev)
    L = torch.rand((20, g), generator=gen, device=dev) ** 3 * 0.6
    X = torch.log1p(torch.poisson(F @ L * 0.15, generator=gen)).contiguous()
    del F, L
    density = float((X != 0).float().mean().item())
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    ws_bytes = lib.hb_pca_gram_workspace_bytes(n, g)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    G = torch.empty((g, g), dtype=torch.float64, device=dev)
    cs = torch.empty(g, dtype=torch.float64, device=dev)

    def gram():
        _lib.check(lib.hb_pca_gram(ctypes.c_void_p(X.data_ptr()), n, g, g, ctypes.c_void_p(G.data_ptr()),
                                   ctypes.c_void_p(cs.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws_bytes, st))

    ms_gram = _events_ms(gram)
    ms_cublas = _events_ms(lambda: torch.matmul(X.T, X))
    G32 = torch.matmul(X.T.double(), X.double()) if n * g <= 2_000_000_000 else None
    err = float(((G - G32).abs().max() / G32.abs().max()).item()) if G32 is not None else None
    err32 = float(((torch.matmul(X.T, X).double() - G32).abs().max() / G32.abs().max()).item()) if G32 is not None else None
    del G32, ws
    res = {}
    ms_pca = _events_ms(lambda: res.update(r=pca_arrays(X, n_comps)), reps=2)
    comps = res["r"].components
    pws_bytes = lib.hb_pca_project_workspace_bytes(g, n_comps)
    pws = torch.empty(pws_bytes, dtype=torch.uint8, device=dev)
    out = torch.empty((n, n_comps), dtype=torch.float32, device=dev)
    mean = res["r"].mean

    def project():
        _lib.check(lib.hb_pca_project(ctypes.c_void_p(X.data_ptr()), n, g, g, ctypes.c_void_p(comps.data_ptr()),
                                      n_comps, ctypes.c_void_p(mean.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(pws.data_ptr()), pws_bytes, st))

    ms_proj = _events_ms(project)
    peak_t, kind_t = _tensor_peak()
    peak_h, kind_h = measured_peaks()
    useful = float(n) * g * (g + 1)  # one multiply-add per (i <= j) entry and row
    issued = 3.0 * 2.0 * n * (128 * 128) * ((g + 127) // 128) * ((g + 127) // 128 + 1) / 2  # bf16 MMA flops
    proj_bytes = float(n) * g * 4 + float(n) * n_comps * 4
    return {"workload": f"{n} cells x {g} genes float32 (density {density:.3f}), {n_comps} components, "
                        "covariance eigendecomposition",
            "pca_ms": ms_pca,
            "gram": {"kernel": "k_pca_gram + k_pca_reduce", "ms": ms_gram,
                     "useful_tflops": useful / ms_gram / 1e9, "issued_bf16_tflops": issued / ms_gram / 1e9,
                     "roofline": {"bound": "tensor", "achieved": issued / ms_gram / 1e9, "peak": peak_t,
                                  "unit": "TFLOP/s", "frac": issued / ms_gram / 1e9 / peak_t, "peak_kind": kind_t,
                                  "note": "achieved = bf16 MMA flops issued (3 hi/lo products of the upper "
                                          "triangle of 128 x 128 blocks)"},
                     "rel_max_abs_err_vs_float64": err},
            "cublas_fp32_gram_ms": ms_cublas, "cublas_fp32_rel_max_abs_err_vs_float64": err32,
            "speedup_gram_vs_cublas_fp32": ms_cublas / ms_gram,
            "project": {"kernel": "k_pca_project", "ms": ms_proj,
                        "roofline": {"bound": "hbm", "achieved": proj_bytes / ms_proj / 1e6, "peak": peak_h,
                                     "unit": "GB/s", "frac": proj_bytes / ms_proj / 1e6 / peak_h,
                                     "peak_kind": kind_h, "algorithmic_bytes": proj_bytes}}}


def knn_section(dev, n=500_000, d=50, k=15):
    """kNN graph of the corrected embedding: the 500,000-cell x 50-PC mixture (the Harmony
    workload's input), exact brute force, k = 15, euclidean."""
    import torch

    from rapids_singlecell_b200.neighbors import knn_arrays
    from rapids_singlecell_b200.synthetic import make_config

    Z = torch.as_tensor(make_config(WORKLOAD, seed=0)["Z"][:n, :d], device=dev)
    ms = _events_ms(lambda: knn_arrays(Z, k), reps=2)
    peak_t, kind_t = _tensor_peak()
    dpad = 64 if d <= 64 else 128
    tiles = (n + 127) // 128
    issued = 3.0 * 2.0 * (tiles * 128.0) ** 2 * dpad
    return {"workload": f"{n} x {d} float32, k={k}, euclidean, exact brute force", "ms": ms,
            "queries_per_s": n / (ms / 1e3), "distances_per_s": float(n) * n / (ms / 1e3),
            "roofline": {"bound": "tensor", "achieved": issued / ms / 1e9, "peak": peak_t, "unit": "TFLOP/s",
                         "frac": issued / ms / 1e9 / peak_t, "peak_kind": kind_t,
                         "note": "achieved = bf16 MMA flops issued (3 hi/lo products of every 128 x 128 "
                                 "query-data tile pair over the padded 64 dimensions)"}}


def run_sections(args, dev):
    out = {}
    rates = tuple(float(r) for r in args.serving_rates.split(",") if r.strip())
    fp32_rates = tuple(float(r) for r in args.serving_fp32_rates.split(",") if r.strip())
    for name in [s for s in args.sections.split(",") if s]:
        fn = {"wide": wide_section, "batched": batched_section,
              "serving": lambda d: serving_section(d, n_requests=args.serving_requests, rates=rates,
                                                   fp32_rates=fp32_rates),
              "pca": pca_section, "knn": knn_section}[name]
        t0 = time.perf_counter()
        try:
            out[name] = fn(dev)
        except Exception as e:  # noqa: BLE001 - reported in the line; the headline stands
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["section_wall_s"] = time.perf_counter() - t0
    return out


def max_over_ranks_of(x, dist, device):
    """The largest `x` over the ranks of the process group (the step time of a job is its
    slowest rank's); `x` itself without a process group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, world, ms_per_step):
    """Whole-job rate: the units all ranks processed per step / the max-over-ranks step time."""
    return units_per_rank * world / (ms_per_step / 1e3)


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from rapids_singlecell_b200.harmony import HarmonyProblem, harmonize

    cfg = workload()
    Z, cats, B, K = cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["n_clusters"]
    n = Z.shape[0]
    theta = np.full(B, 2.0)
    common = dict(n_clusters=K, max_iter_harmony=OUTER, max_iter_clustering=INNER,
                  tol_harmony=-np.inf, tol_clustering=-np.inf)
    cell_iters = n * OUTER * INNER
    dev = torch.device("cuda", local)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return max_over_ranks_of(x, dist, dev)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        # as timeit does: no garbage-collector pass inside the timed steps (a collection of the
        # harness's objects once added ~95 ms to one end-to-end step)
        gc.collect()
        gc.disable()
        per = []
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(steps):
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            per.append(e0.elapsed_time(e1))
        end.record()
        torch.cuda.synchronize()
        gc.enable()
        barrier()
        total_ms = start.elapsed_time(end)
        return max_over_ranks(total_ms) / steps, per

    # ---- fused tensor-core path, device resident -----------------------------
    X = torch.as_tensor(Z, device=dev)
    prob = HarmonyProblem(X, cats, B, torch.as_tensor(cfg["Y0"], device=dev), theta,
                          precision=args.precision, **common)
    last = {}
    calls = {"n": 0}

    def step_resident():
        # the kernel spans (CUDA events around every sweep and centroid launch) are recorded on
        # the last timed step only: the events add work between the launches of a profiled run
        calls["n"] += 1
        _, info = prob.run(profile=calls["n"] == args.warmup + args.steps)
        if info.profile is not None:
            last["info"] = info

    # the clock sampler starts before the warm-up steps, so that its start-up is not timed
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.wait_first_sample()
    ms, per = timed(step_resident, args.steps, args.warmup)
    clk = clocks.stop() if clocks else None
    prof = last["info"].profile
    value = job_throughput(cell_iters, world, ms)

    # ---- end to end through the public API from pinned host memory ------------
    Z_pin = torch.from_numpy(Z).pin_memory()
    out_pin = torch.empty(Z_pin.shape, dtype=Z_pin.dtype).pin_memory()
    codes = cats.astype(np.int32)

    def step_e2e():
        out = harmonize(Z_pin, codes, None, init_centroids=cfg["Y0"], precision=args.precision,
                        device=dev, **common)
        out_pin.copy_(out)
        last["e2e"] = out_pin

    import warnings

    warnings.simplefilter("ignore")
    ms_e2e, per_e2e = timed(step_e2e, args.steps, args.warmup)
    e2e_value = job_throughput(cell_iters, world, ms_e2e)

    # ---- plain float32 path (the drop-in for dtype=np.float32) -----------------
    plain = None
    if not args.no_plain:
        prob32 = HarmonyProblem(X, cats, B, torch.as_tensor(cfg["Y0"], device=dev), theta,
                                precision="fp32", **common)
        ms32, per32 = timed(lambda: prob32.run(), max(1, min(args.steps, 3)), 1)
        # error of the 16-bit result against the plain fp32 result of the same inputs (the
        # float64 oracle is too slow for this size on the host)
        z32 = prob32.Z_hat.double()
        z16 = last["e2e"].to(dev).double()
        diff = (z16 - z32).abs().max().item()
        plain = {"value": cell_iters * world / (ms32 / 1e3), "ms_per_step": ms32,
                 "p50_ms": float(np.percentile(per32, 50)), "p99_ms": float(np.percentile(per32, 99)),
                 "max_abs_diff_16bit_vs_fp32": diff,
                 "rel_max_abs_diff_16bit_vs_fp32": diff / max(z32.abs().max().item(), 1e-300)}
        prob32.close()
        del z32, z16
        # the float64 plain path: the reference's default dtype, the drop-in of a bare
        # harmony_integrate call (one timed step after one warm-up)
        prob64 = HarmonyProblem(X.double(), cats, B, torch.as_tensor(cfg["Y0"], device=dev).double(), theta,
                                precision="fp64", **common)
        ms64, _ = timed(lambda: prob64.run(), 1, 1)
        plain["fp64"] = {"value": cell_iters * world / (ms64 / 1e3), "ms_per_step": ms64}
        prob64.close()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel (the persistent sweep) ----------------
    # algorithmic bytes per cell and launch: Z_norm row read + R row write (d and K
    # 16-bit values) + cell id and batch (8 B); one launch = one k-means iteration.
    peak, peak_kind = measured_peaks()
    achieved = prof["block_bytes"] / (prof["block_ms"] / 1e3) / 1e9 if prof["block_ms"] > 0 else 0.0
    launches = prof["block_launches"]
    cen_launches = max(1, prof["centroid_launches"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": profiled_traffic("k_tc_sweep_C2_bf16.md"),
                "peak_kind": peak_kind,
                "kernel": "k_tc_sweep (all blocks of one k-means iteration: similarity MMA, "
                          "exp/penalty, L1 normalise, R write, observed-count delta)",
                "algorithmic_bytes_per_launch": prof["block_bytes"] / max(1, launches),
                "avg_launch_us": prof["block_ms"] / max(1, launches) * 1e3,
                "time_share": prof["block_ms"] / ms,
                "centroid": {"kernel": "k_tc_centroid_stream + reductions (Y = R^T Z_norm and the "
                                       "per-(block, batch) sums, cell order)",
                             "achieved_gbs": prof["centroid_bytes"] / (prof["centroid_ms"] / 1e3) / 1e9
                             if prof["centroid_ms"] > 0 else 0.0,
                             "frac": (prof["centroid_bytes"] / (prof["centroid_ms"] / 1e3) / 1e9 / peak)
                             if prof["centroid_ms"] > 0 else 0.0,
                             "avg_launch_us": prof["centroid_ms"] / cen_launches * 1e3,
                             "traffic": profiled_traffic("k_tc_centroid_stream_C2_bf16.md"),
                             "time_share": prof["centroid_ms"] / ms}}

    h2d = Z.nbytes + codes.nbytes + cfg["Y0"].nbytes
    d2h = Z.nbytes + 8 * (OUTER + 1)
    res = {
        "metric": METRIC, "value": value, "unit": "cell-iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision if args.precision != "fp32" else "f32", "data": "synthetic",
        "config": config_dict(cfg, {"precision": args.precision,
                                    "parallelism": "replicas" if world > 1 else "single"}),
        "p50_ms": float(np.percentile(per, 50)), "p99_ms": float(np.percentile(per, 99)),
        "per_step_ms": [round(float(t), 2) for t in per],
        "e2e": {"value": e2e_value, "unit": "cell-iters/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e,
                "p50_ms": float(np.percentile(per_e2e, 50)), "p99_ms": float(np.percentile(per_e2e, 99)),
                "per_step_ms": [round(float(t), 2) for t in per_e2e]},
        "plain_fp32": plain,
        "roofline": roofline,
        "cpu_baseline": None,            # filled after the sections (host-side legs last)
        "error_vs_fp64_oracle": None,
        "clocks": clk,
        "gpu_launches": int(prof["kernel_launches"]) * args.steps,
    }
    # the extra measurements first, the host-side oracle legs last: the multi-stream sections
    # drive the GPU from many host threads and run before the BLAS pool has been used
    res.update(run_sections(args, dev))
    # ---- CPU baseline (bounded sample on the host cores) and the error of the engine against
    # the float64 oracle of the same iterations ------------------------------------------------
    cpu_iters = 2
    ok32 = OracleKmeans(cfg, np.float32)
    t32 = float(np.median([ok32.step() for _ in range(cpu_iters)]))
    _, corr32 = ok32.correction()
    ok64 = OracleKmeans(cfg, np.float64)
    t64 = float(np.median([ok64.step() for _ in range(cpu_iters)]))
    z64, corr64 = ok64.correction()
    cpu = {"value": n / t32, "unit": "cell-iters/s", "cores": blas_threads(), "kind": "port",
           "sample": cpu_sample_text(n, "float32", cpu_iters, ok32.init_s, corr32),
           "os_cpu_count": os.cpu_count(), "init_s": ok32.init_s, "correction_s": corr32,
           "float64": {"value": n / t64, "unit": "cell-iters/s", "init_s": ok64.init_s,
                       "correction_s": corr64}}
    del ok32, ok64
    # the engine on the same 1 outer x 2 k-means iterations (same seeds and block order)
    errs = {}
    z64_t = torch.as_tensor(z64, device=dev)
    for prec in (args.precision, "fp32"):
        p1 = HarmonyProblem(X, cats, B, torch.as_tensor(cfg["Y0"], device=dev), theta, precision=prec,
                            **dict(common, max_iter_harmony=1, max_iter_clustering=cpu_iters))
        p1.run()
        errs[prec] = {"rel_max_abs": _rel(p1.Z_hat, z64_t),
                      "max_abs": float((p1.Z_hat.double() - z64_t).abs().max().item())}
        p1.close()
    error_vs_oracle = {"reference": f"NumPy float64 oracle (pinned to the reference's own kernels by "
                                    f"tests/test_oracle_vs_reference.py), 1 outer x {cpu_iters} k-means "
                                    "iterations of this workload, same seeds",
                       **errs}

    res["cpu_baseline"] = cpu
    res["error_vs_fp64_oracle"] = error_vs_oracle
    print(json.dumps(res))
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.precision == "fp64" and not args.profile_case:
        raise SystemExit("--precision fp64 is for --profile-case; the line reports the float64 path "
                         "as plain_fp32.fp64")
    if args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
