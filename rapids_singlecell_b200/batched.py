"""Many independent Harmony problems on one GPU: a batched schedule and a
serving loop.

Both run each problem as its own engine plan (``HarmonyProblem``) on one of a
small pool of CUDA streams, so that the kernels of different problems overlap on
the device: the persistent sweep of a problem of n cells uses about n / 2560
SMs and the centroid pass about n / 512, so small problems leave most of the GPU
to the others.  Host work (plan creation, the per-outer-iteration readback of
the objective) runs on one host thread per stream; the engine calls release the
GIL.

Admission is by an HBM budget: a problem starts only when its workspace, inputs
and output fit into what the running problems leave of the budget.

CUDA gives a process 8 hardware work queues unless CUDA_DEVICE_MAX_CONNECTIONS is
set before CUDA starts; beyond 8 streams the streams share queues and partly
serialise.  With the variable at 32, 32 streams ran 256 small problems about 1.4x
faster than 8.

The persistent sweep of each problem is a cooperative launch whose CTAs wait
for each other at a grid barrier (one CTA per SM).  Two such grids that are both
only partly resident could each wait for SMs the other holds, so SMs are a second
admitted resource: a 16-bit problem asks for one sweep CTA per two 128-cell tiles
of a block (each CTA runs two tile streams; one per tile above 128 clusters), at
most the SM count, and is granted what the running problems leave, but never less
than its fair share min(asked, SMs / streams); the grants of the running problems
never sum above the SM count, so all their sweeps fit on the GPU together.  Asking
for one CTA per tile instead (half-empty tile streams) measured 0.9-1.0e9 against
1.4e9 cell-iters/s on the 256-problem batch.  Plain fp32 / fp64 problems have no
cooperative launch and take no SMs from the admission.
"""

from __future__ import annotations

import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np
import torch

from .harmony import HarmonyInfo, HarmonyProblem, make_params


@dataclass
class HarmonyRequest:
    """One integration: Z (cells x PCs, host or device float32), int batch codes
    ``cats`` (0 .. n_batches-1), initial centroids ``Y0`` (n_clusters x PCs),
    per-batch ``theta`` and the engine parameters of ``HarmonyProblem``
    (``n_clusters`` required)."""

    Z: object
    cats: np.ndarray
    n_batches: int
    Y0: object
    theta: np.ndarray
    params: dict = field(default_factory=dict)
    precision: str = "bf16"
    to_host: bool = False  # copy Z_hat back into a host tensor


@dataclass
class HarmonyResult:
    Z_hat: torch.Tensor
    info: HarmonyInfo
    latency_s: float   # from submit to result: admission wait + run
    run_s: float       # run only


def sweep_ctas_wanted(req: HarmonyRequest, sms: int) -> int:
    """SMs a request's persistent sweep asks for: enough CTAs for one 128-cell tile of a
    block per tile stream (two streams per CTA up to 128 clusters, one above), at most one
    per SM.  More CTAs would not shorten the sweep, whose blocks are bound by their
    dependency chain, and would keep other problems off the GPU.  The plain fp32 / fp64 paths
    have no cooperative launch and ask for none."""
    if req.precision not in ("bf16", "fp16"):
        return 0
    n = int(req.Z.shape[0])
    bs = max(1, int(n * float(req.params.get("block_proportion", 0.05))))
    tiles = -(-min(bs, n) // 128)
    streams = 2 if int(req.params.get("n_clusters", 1)) <= 128 else 1
    return max(1, min(sms, -(-tiles // streams)))


def request_bytes(req: HarmonyRequest) -> int:
    """Device bytes a request holds while it runs: the engine workspace, Z
    (float32) and Z_hat, the centroids and the batch codes."""
    n, d = (int(v) for v in req.Z.shape)
    k = int(req.params["n_clusters"])
    rest = {kk: v for kk, v in req.params.items() if kk not in ("n_clusters", "max_sweep_ctas")}
    ws = HarmonyProblem.workspace_bytes(make_params(n, d, k, req.n_batches, precision=req.precision, **rest))
    return int(ws + 2 * n * d * 4 + k * d * 4 + n * 4)


class HarmonyServer:
    """A request loop: ``submit`` returns a Future of ``HarmonyResult``.  A
    request runs once its device bytes fit into ``hbm_budget_bytes`` next to the
    running ones and its sweep CTAs fit into the SMs they leave; ``streams``
    worker threads each own a CUDA stream."""

    def __init__(self, *, streams: int = 8, hbm_budget_bytes: int = 160 << 30, device=None):
        dev = torch.device(device) if device is not None else torch.device("cuda")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.budget = int(hbm_budget_bytes)
        self.in_use = 0
        self.sms_in_use = 0
        self._cv = threading.Condition()
        self._q: queue.Queue = queue.Queue()
        self._closed = False
        self.sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.fair_ctas = max(1, self.sms // max(1, streams))
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(streams)]
        for t in self._workers:
            t.start()

    def submit(self, req: HarmonyRequest) -> Future:
        fut: Future = Future()
        need = request_bytes(req)
        if need > self.budget:
            fut.set_exception(MemoryError(f"request needs {need} bytes, the HBM budget is {self.budget}"))
            return fut
        self._q.put((req, need, fut, time.perf_counter()))
        return fut

    def _admit(self, need: int, want: int) -> int:
        """Wait until the bytes fit and at least min(want, fair share) SMs are free;
        returns the sweep CTAs granted."""
        floor = min(want, self.fair_ctas)
        with self._cv:
            while self.in_use + need > self.budget or self.sms - self.sms_in_use < floor:
                self._cv.wait()
            grant = min(want, self.sms - self.sms_in_use)
            self.in_use += need
            self.sms_in_use += grant
            return grant

    def _release(self, need: int, grant: int) -> None:
        with self._cv:
            self.in_use -= need
            self.sms_in_use -= grant
            self._cv.notify_all()

    def _work(self) -> None:
        setup_error = None
        try:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(device=self.device)
        except Exception as e:  # noqa: BLE001 - every request of this worker fails with it
            setup_error = e
        while True:
            item = self._q.get()
            if item is None:
                return
            req, need, fut, t_submit = item
            if setup_error is not None:
                fut.set_exception(setup_error)
                continue
            grant = self._admit(need, sweep_ctas_wanted(req, self.sms))  # 0 on the plain paths
            try:
                t0 = time.perf_counter()
                with torch.cuda.stream(stream):
                    X = torch.as_tensor(req.Z).to(self.device, torch.float32)
                    Y0 = torch.as_tensor(req.Y0).to(self.device, torch.float32)
                    params = dict(req.params)
                    params["max_sweep_ctas"] = min(grant, int(params.get("max_sweep_ctas") or grant))
                    prob = HarmonyProblem(X, req.cats, req.n_batches, Y0, req.theta,
                                          precision=req.precision, stream=stream, **params)
                    Z_hat, info = prob.run()
                    prob.close()
                    out = Z_hat
                    if req.to_host:  # pinned (torch's caching host allocator): no staged copy
                        out = torch.empty(Z_hat.shape, dtype=Z_hat.dtype, pin_memory=True)
                        out.copy_(Z_hat, non_blocking=True)
                stream.synchronize()
                t1 = time.perf_counter()
                fut.set_result(HarmonyResult(out, info, t1 - t_submit, t1 - t0))
            except Exception as e:  # noqa: BLE001 - delivered to the caller through the future
                fut.set_exception(e)
            finally:
                self._release(need, grant)

    def close(self) -> None:
        if self._closed:
            return
        self._closed = True
        for _ in self._workers:
            self._q.put(None)
        for t in self._workers:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_batched(requests: list[HarmonyRequest], *, streams: int = 8,
                hbm_budget_bytes: int = 160 << 30, device=None) -> list[HarmonyResult]:
    """Run all requests through a ``HarmonyServer``; results in request order."""
    with HarmonyServer(streams=streams, hbm_budget_bytes=hbm_budget_bytes, device=device) as srv:
        futs = [srv.submit(r) for r in requests]
        return [f.result() for f in futs]


def latency_summary(results: list[HarmonyResult]) -> dict:
    lat = np.array([r.latency_s for r in results]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}
