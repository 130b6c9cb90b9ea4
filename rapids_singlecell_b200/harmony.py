"""Harmony integration on B200: host-side driver over the C ABI.

``harmonize`` mirrors ``rapids_singlecell.preprocessing._harmony.harmonize``
(src/rapids_singlecell/preprocessing/_harmony/__init__.py:41-289): the same
keyword arguments, defaults, parameter resolution and error types.  The work
runs in one call into ``libharmony_b200.so`` (``hb_harmonize``) on the current
CUDA stream; device memory for the run is one workspace tensor allocated here.
"""

from __future__ import annotations

import ctypes
import warnings
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import HbOutputs, HbParams, PRECISIONS  # noqa: F401

SUPPRESS_PENALTY = 1e30


@dataclass
class HarmonyInfo:
    objectives_harmony: list
    kmeans_objectives: list = field(default_factory=list)
    converged: bool = False
    n_outer: int = 0
    n_clusters: int = 0
    precision: str = "fp32"
    profile: dict | None = None


def make_params(n_cells, n_pcs, n_clusters, n_batches, *, precision="fp32", max_iter_harmony=10,
                max_iter_clustering=200, tol_harmony=1e-4, tol_clustering=1e-5, ridge_lambda=1.0,
                sigma=0.1, block_proportion=0.05, random_state=0, stabilized_penalty=True,
                dynamic_lambda=True, alpha=0.2, batch_prune_threshold=1e-5, max_sweep_ctas=0,
                sweep_wait_ns=0, test_unmet_arrivals=0, sweep_form=0) -> HbParams:
    """The engine's plan parameters (``hb_params``) for one problem.  ``sweep_wait_ns`` bounds each
    grid-barrier wait of the 16-bit sweep (0: 2 s); ``test_unmet_arrivals`` is a test hook that
    makes those waits run out (0 in normal use); ``sweep_form`` forces a layout of the sweep
    (``HB_SWEEP_*``, 0: the engine's choice; see ``rapids_singlecell_b200.autotune``)."""
    p = HbParams()
    p.n_cells = int(n_cells)
    p.n_pcs = int(n_pcs)
    p.n_clusters = int(n_clusters)
    p.n_batches = int(n_batches)
    p.precision = PRECISIONS[precision]
    p.block_size = int(n_cells * block_proportion)
    p.max_iter_harmony = int(max_iter_harmony)
    p.max_iter_clustering = int(max_iter_clustering)
    p.tol_harmony = tol_harmony
    p.tol_clustering = tol_clustering
    p.sigma = sigma
    p.ridge_lambda = ridge_lambda
    p.alpha = alpha
    p.batch_prune_threshold = 0.0 if batch_prune_threshold is None else batch_prune_threshold
    p.prune = 0 if batch_prune_threshold is None else 1
    p.stabilized_penalty = int(bool(stabilized_penalty))
    p.dynamic_lambda = int(bool(dynamic_lambda))
    p.random_state = int(random_state) & 0xFFFFFFFFFFFFFFFF
    p.max_sweep_ctas = int(max_sweep_ctas)
    p.sweep_wait_ns = int(sweep_wait_ns)
    p.test_unmet_arrivals = int(test_unmet_arrivals)
    p.sweep_form = int(sweep_form)
    return p


class HarmonyProblem:
    """One Harmony problem resident on the GPU: the engine plan, its workspace and
    the device inputs.  ``run()`` integrates it (and can be called again, e.g. to
    time it); nothing is copied between host and device inside ``run()`` except
    the small per-batch tables and the objective values.

    ``X`` is a CUDA tensor (float32, or float64 for precision "fp64"), ``cats``
    the int32 batch code per cell (host array), ``theta`` the per-batch theta
    (tau discount applied), ``Y0`` the initial centroids on the device.
    """

    def __init__(self, X, cats, n_batches, Y0, theta, *, precision="fp32", n_clusters,
                 max_iter_harmony=10, max_iter_clustering=200, tol_harmony=1e-4,
                 tol_clustering=1e-5, ridge_lambda=1.0, sigma=0.1, block_proportion=0.05,
                 random_state=0, stabilized_penalty=True, dynamic_lambda=True, alpha=0.2,
                 batch_prune_threshold=1e-5, stream=None, max_sweep_ctas=0, sweep_wait_ns=0,
                 test_unmet_arrivals=0, counts=None, sweep_form=0):
        self.lib = _lib.load()
        self.device = X.device
        self.X = X.contiguous()
        n_cells, n_pcs = self.X.shape
        self.n_batches = int(n_batches)
        if isinstance(cats, torch.Tensor):  # codes on the device: counted and sorted there
            self.cats = cats.to(device=self.device, dtype=torch.int32).contiguous()
            N_b = None if counts is not None else \
                torch.bincount(self.cats.long(), minlength=self.n_batches).cpu().numpy().astype(np.int64)
        else:
            cats = np.asarray(cats, dtype=np.int32)
            N_b = None if counts is not None else np.bincount(cats, minlength=self.n_batches).astype(np.int64)
            self.cats = torch.as_tensor(cats, device=self.device)
        if counts is not None:  # the cells per batch, already counted by the caller
            N_b = np.asarray(counts, dtype=np.int64)
        # the engine sorts the cells by batch itself up to 4096 batches
        self.cell_index = None
        if self.n_batches > 4096:
            self.cell_index = torch.sort(self.cats, stable=True).indices.to(torch.int32)
        self.offsets = np.zeros(self.n_batches + 1, dtype=np.int64)
        self.offsets[1:] = np.cumsum(N_b)
        self.theta = np.asarray(theta, dtype=np.float64)
        self.Y0 = torch.as_tensor(Y0, device=self.device).to(self.X.dtype).contiguous()
        self.max_iter_harmony = max_iter_harmony
        self.max_iter_clustering = max_iter_clustering
        self.n_clusters = n_clusters
        self.precision = precision
        p = make_params(n_cells, n_pcs, n_clusters, self.n_batches, precision=precision,
                        max_iter_harmony=max_iter_harmony, max_iter_clustering=max_iter_clustering,
                        tol_harmony=tol_harmony, tol_clustering=tol_clustering, ridge_lambda=ridge_lambda,
                        sigma=sigma, block_proportion=block_proportion, random_state=random_state,
                        stabilized_penalty=stabilized_penalty, dynamic_lambda=dynamic_lambda, alpha=alpha,
                        batch_prune_threshold=batch_prune_threshold, max_sweep_ctas=max_sweep_ctas,
                        sweep_wait_ns=sweep_wait_ns, test_unmet_arrivals=test_unmet_arrivals,
                        sweep_form=sweep_form)
        self.params = p
        self.plan = ctypes.c_void_p()
        _lib.check(self.lib.hb_plan_create(ctypes.byref(p), ctypes.byref(self.plan)))
        self.ws_bytes = self.lib.hb_plan_workspace_bytes(self.plan)
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        self.Z_hat = torch.empty_like(self.X)
        self._off_c = (ctypes.c_int64 * (self.n_batches + 1))(*self.offsets.tolist())
        self._th_c = (ctypes.c_double * self.n_batches)(*self.theta.tolist())
        self.stream = stream

    @staticmethod
    def workspace_bytes(params: HbParams) -> int:
        lib = _lib.load()
        plan = ctypes.c_void_p()
        _lib.check(lib.hb_plan_create(ctypes.byref(params), ctypes.byref(plan)))
        try:
            return int(lib.hb_plan_workspace_bytes(plan))
        finally:
            lib.hb_plan_destroy(plan)

    def run(self, profile: bool = False):
        mih, mic = self.max_iter_harmony, self.max_iter_clustering
        objs = (ctypes.c_double * (mih + 1))()
        n_obj = ctypes.c_int32(0)
        kobjs = (ctypes.c_double * max(1, mih * mic))()
        kits = (ctypes.c_int32 * mih)()
        conv = ctypes.c_int32(0)
        prof = _lib.HbProfile()
        out = HbOutputs(objs, ctypes.pointer(n_obj), kobjs, kits, ctypes.pointer(conv),
                        ctypes.pointer(prof) if profile else None)
        st = self.stream if self.stream is not None else torch.cuda.current_stream(self.device)
        _lib.check(self.lib.hb_harmonize(
            self.plan, self.X.data_ptr(), self.cats.data_ptr(),
            None if self.cell_index is None else self.cell_index.data_ptr(),
            self._off_c, self._th_c, self.Y0.data_ptr(), self.ws.data_ptr(), self.ws_bytes,
            self.Z_hat.data_ptr(), ctypes.byref(out), ctypes.c_void_p(st.cuda_stream)))
        n_outer = n_obj.value - 1
        info = HarmonyInfo(
            objectives_harmony=[objs[i] for i in range(n_obj.value)],
            kmeans_objectives=[[kobjs[o * mic + i] for i in range(kits[o])] for o in range(n_outer)],
            converged=bool(conv.value), n_outer=n_outer, n_clusters=self.n_clusters,
            precision=self.precision,
            profile={f: getattr(prof, f) for f, _ in _lib.HbProfile._fields_} if profile else None)
        return self.Z_hat, info

    def close(self):
        if self.plan:
            self.lib.hb_plan_destroy(self.plan)
            self.plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def from_dlpack(x):
    """Arrays of other libraries that export DLPack (``__dlpack__``: CuPy, JAX, ...) as torch
    tensors sharing their memory (no copy); torch tensors, NumPy arrays, pandas objects and
    lists pass through unchanged.  The corrected embedding is returned as a torch tensor,
    which exports DLPack itself (``cupy.from_dlpack(Z_hat)`` takes it without a copy)."""
    if isinstance(x, (torch.Tensor, np.ndarray)) or not hasattr(x, "__dlpack__"):
        return x
    return torch.from_dlpack(x)


def _integer_codes(labels):
    """(codes, number of categories) of plain integer labels: ``_integer_codes_counts``
    without the counts."""
    codes, n, _ = _integer_codes_counts(labels)
    return codes, n


def _integer_codes_counts(labels):
    """Categorical codes of plain integer labels without pandas: the categories are the
    sorted distinct values, as ``astype("category")`` gives them.  Labels already on the GPU
    (a CUDA tensor, or any DLPack device array) are coded there (``torch.unique``) and stay
    there: the codes come back as an int32 CUDA tensor, as the reference keeps its ``cats``
    on the device (_utils/_multi_gpu.py:202-232).  Host labels must be non-negative and come
    back as a NumPy array, with the cells per category (int64) as the third value (None for
    device labels).  Returns (None, 0, None) for anything else."""
    labels = from_dlpack(labels)
    if isinstance(labels, torch.Tensor) and labels.is_cuda:
        if labels.dim() != 1 or labels.numel() == 0 or labels.dtype.is_floating_point or labels.dtype == torch.bool:
            return None, 0, None
        uniq, inv = torch.unique(labels, sorted=True, return_inverse=True)
        return inv.to(torch.int32), int(uniq.numel()), None
    if isinstance(labels, torch.Tensor):
        labels = labels.detach().numpy()
    if not isinstance(labels, np.ndarray) or labels.ndim != 1 or labels.dtype.kind not in "iu":
        return None, 0, None
    if labels.size == 0 or labels.min() < 0 or labels.max() > 16 * labels.size + (1 << 20):
        return None, 0, None
    counts = np.bincount(labels)
    present = counts > 0
    if present.all():  # every value 0 .. max present: the labels are their own codes
        return labels.astype(np.int32, copy=False), int(present.size), counts.astype(np.int64)
    remap = np.cumsum(present, dtype=np.int64) - 1
    return remap[labels].astype(np.int32), int(present.sum()), counts[present].astype(np.int64)


def get_batch_codes(batch_mat, batch_key):
    """Categorical batch codes (``_get_batch_codes``, _helper.py:223-236): several
    keys are joined with ","."""
    import pandas as pd

    if batch_key is None:
        # labels given directly; a pandas Categorical keeps its (possibly unused) categories
        vec = batch_mat if isinstance(batch_mat, pd.Series) else pd.Series(batch_mat)
    elif isinstance(batch_key, str):
        vec = batch_mat[batch_key]
    elif len(batch_key) == 1:
        vec = batch_mat[batch_key[0]]
    else:
        df = batch_mat[batch_key].astype("str")
        vec = df.apply(lambda row: ",".join(row), axis=1)
    return vec.astype("category")


def theta_array(theta, n_batches: int) -> np.ndarray:
    """theta per batch (``_get_theta_array``, _helper.py:277-307)."""
    if isinstance(theta, (float, int)) and not isinstance(theta, bool):
        return np.ones(n_batches, dtype=np.float64) * float(theta)
    if isinstance(theta, (list, np.ndarray)):
        arr = np.asarray(theta, dtype=np.float64)
    elif isinstance(theta, torch.Tensor):
        arr = theta.detach().cpu().numpy().astype(np.float64)
    else:
        raise ValueError(
            f"Theta must be float, int, list, numpy array, or torch tensor, got {type(theta)}"
        )
    if arr.size != n_batches:
        raise ValueError(
            f"Theta array size ({arr.size}) must match number of batches ({n_batches})"
        )
    return arr.ravel()


def default_n_clusters(n_cells: int) -> int:
    return max(int(min(100, n_cells / 30)), 2)


def seeded_centroids(Z: torch.Tensor, n_clusters: int, random_state: int) -> torch.Tensor:
    """``n_clusters`` distinct cells chosen by ``numpy.random.default_rng(random_state)``:
    the initial centroids when the k-means initialisation does not apply (more than 256
    PCs or clusters, or more than 128 of both)."""
    rng = np.random.default_rng(random_state)
    idx = rng.choice(Z.shape[0], size=n_clusters, replace=False)
    return Z[torch.as_tensor(idx, device=Z.device)].contiguous()


KMEANS_MAX_ITER = 25   # the reference's KMeans(max_iter=25) (_harmony/__init__.py:315-321)
KMEANS_TOL = 1e-4


def kmeans_centroids(X: torch.Tensor, n_clusters: int, random_state: int, *, max_iter: int = KMEANS_MAX_ITER,
                     tol: float = KMEANS_TOL, return_iters: bool = False):
    """Initial centroids by the engine's seeded k-means on the L2-normalised rows of ``X``
    (``hb_kmeans_init``): k-means++ seeding on a sample drawn from ``random_state``, then up
    to ``max_iter`` Lloyd iterations with tensor-core assignment.  This takes the place of
    the reference's cuML ``KMeans(init="k-means||", n_init=1, max_iter=25)``
    (_harmony/__init__.py:290-323); the centres are returned unnormalised, as cuML's are,
    in the dtype of ``X``."""
    lib = _lib.load()
    X32 = X.to(torch.float32).contiguous()
    n, d = X32.shape
    ws_bytes = lib.hb_kmeans_workspace_bytes(n, d, n_clusters)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=X.device)
    Y = torch.empty((n_clusters, d), dtype=torch.float32, device=X.device)
    iters = ctypes.c_int32(0)
    st = torch.cuda.current_stream(X.device).cuda_stream
    _lib.check(lib.hb_kmeans_init(X32.data_ptr(), n, d, n_clusters, int(max_iter), float(tol),
                                  int(random_state) & 0xFFFFFFFFFFFFFFFF, Y.data_ptr(), ctypes.byref(iters),
                                  ws.data_ptr(), ws_bytes, st))
    Y = Y.to(X.dtype)
    return (Y, iters.value) if return_iters else Y


def _resolve_precision(precision, dtype) -> str:
    if precision is None:
        return "fp64" if dtype == torch.float64 else "fp32"
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {precision!r}")
    return precision


def resolve_parameters(n_cells, N_b, *, n_clusters, max_iter_harmony, theta, tau,
                       block_proportion, dynamic_lambda, alpha, batch_prune_threshold,
                       correction_method, colsum_algo):
    """Host-side parameter resolution and validation, in the order of the reference
    (_harmony/__init__.py:154-200).  Returns (n_clusters, theta per batch)."""
    n_batches = len(N_b)
    if max_iter_harmony < 1:
        raise ValueError("max_iter_harmony must be >= 1")
    if n_clusters is None:
        n_clusters = default_n_clusters(n_cells)
    if colsum_algo not in ("columns", "atomics", "gemm", "benchmark", None):
        raise ValueError("colsum_algo must be 'columns', 'atomics', 'gemm', 'benchmark' or None")
    th = theta_array(theta, n_batches)
    if tau > 0:
        th = th * (1 - np.exp(-np.asarray(N_b, dtype=np.float64) / (n_clusters * tau)) ** 2)
    if not (0 < block_proportion <= 1):
        raise ValueError("block_proportion must be in (0, 1]")
    if int(n_cells * block_proportion) < 1:
        raise ValueError("block_proportion * n_cells must be >= 1")
    if dynamic_lambda:
        if not np.isfinite(alpha) or alpha <= 0:
            raise ValueError(
                f"alpha must be a finite positive number when dynamic_lambda=True, got {alpha}."
            )
        if batch_prune_threshold is not None and not (0 <= batch_prune_threshold <= 1):
            raise ValueError(
                f"batch_prune_threshold must be in [0, 1] or None, got {batch_prune_threshold}."
            )
    if correction_method is not None and correction_method not in {"fast", "original", "batched"}:
        raise ValueError("correction_method must be 'fast', 'original', or 'batched'.")
    return int(n_clusters), th


def harmonize(
    Z,
    batch_mat,
    batch_key=None,
    *,
    n_clusters: int | None = None,
    max_iter_harmony: int = 10,
    max_iter_clustering: int = 200,
    tol_harmony: float = 1e-4,
    tol_clustering: float = 1e-5,
    ridge_lambda: float = 1.0,
    sigma: float = 0.1,
    block_proportion: float = 0.05,
    theta=2.0,
    tau: int = 0,
    correction_method: str | None = None,
    colsum_algo: str | None = None,
    random_state: int = 0,
    stabilized_penalty: bool = True,
    dynamic_lambda: bool = True,
    alpha: float = 0.2,
    batch_prune_threshold: float | None = 1e-5,
    verbose: bool = False,
    init_centroids=None,
    precision: str | None = None,
    return_info: bool = False,
    device=None,
    autotune=False,
):
    """Integrate ``Z`` (cells x PCs) across the batches in ``batch_mat[batch_key]``.

    Same parameters as the reference ``harmonize``; ``correction_method`` and
    ``colsum_algo`` are accepted and validated but only select among equivalent
    implementations there, so they do not change the computation here.  Extra:
    ``init_centroids`` (n_clusters x PCs) fixes the starting centroids,
    ``precision`` is one of "fp32", "fp64" (plain paths) or "bf16"/"fp16"
    (tensor-core paths); by default it follows the dtype of ``Z``.
    ``autotune`` (16-bit paths): True times the persistent sweep's launch shapes on this
    problem once per shape (``rapids_singlecell_b200.autotune``), a path also keeps the choices
    in that JSON file.
    Returns the corrected embedding as a torch tensor on the GPU (and a
    ``HarmonyInfo`` when ``return_info``).  ``Z`` and integer ``batch_mat`` labels may
    be arrays of any library that exports DLPack; device arrays are used in place.
    """
    Z = from_dlpack(Z)
    n_cells, n_pcs = (int(v) for v in Z.shape)
    cats_np, n_batches, N_b = _integer_codes_counts(batch_mat) if batch_key is None else (None, 0, None)
    if cats_np is None:
        codes = get_batch_codes(batch_mat, batch_key)
        n_batches = int(codes.cat.categories.size)
        cats_np = np.asarray(codes.cat.codes.values, dtype=np.int32)
    if cats_np.shape[0] != n_cells:
        raise ValueError("batch labels must have one entry per cell")
    if N_b is None:  # (host labels are counted with their codes)
        if isinstance(cats_np, torch.Tensor):  # device codes: only the B counts come to the host
            N_b = torch.bincount(cats_np.long(), minlength=n_batches).cpu().numpy().astype(np.int64)
        else:
            N_b = np.bincount(cats_np, minlength=n_batches).astype(np.int64)
    n_clusters, th = resolve_parameters(
        n_cells, N_b, n_clusters=n_clusters, max_iter_harmony=max_iter_harmony, theta=theta,
        tau=tau, block_proportion=block_proportion, dynamic_lambda=dynamic_lambda, alpha=alpha,
        batch_prune_threshold=batch_prune_threshold, correction_method=correction_method,
        colsum_algo=colsum_algo)

    lib = _lib.load()
    if device is None:
        device = Z.device if isinstance(Z, torch.Tensor) and Z.is_cuda else torch.device("cuda")
    if isinstance(Z, torch.Tensor):
        X = Z.to(device)
    else:
        X = torch.as_tensor(np.asarray(Z), device=device)
    if X.dtype not in (torch.float32, torch.float64):
        X = X.to(torch.float32)
    prec = _resolve_precision(precision, X.dtype)
    X = X.to(torch.float64 if prec == "fp64" else torch.float32).contiguous()

    if init_centroids is None:
        if (n_pcs <= 128 and n_clusters <= 256) or (n_pcs <= 256 and n_clusters <= 128):
            Y0 = kmeans_centroids(X, n_clusters, random_state)
        else:
            Y0 = seeded_centroids(X, n_clusters, random_state)
    else:
        Y0 = torch.as_tensor(init_centroids, device=device)
        if tuple(Y0.shape) != (n_clusters, n_pcs):
            raise ValueError(
                f"init_centroids must have shape ({n_clusters}, {n_pcs}), got {tuple(Y0.shape)}"
            )
    tuned = {}
    if autotune and prec in ("bf16", "fp16"):
        from .autotune import tune_sweep

        choice = tune_sweep(X, cats_np, n_batches, Y0, th, precision=prec, n_clusters=n_clusters,
                            block_proportion=block_proportion, ridge_lambda=ridge_lambda, sigma=sigma,
                            random_state=random_state, stabilized_penalty=stabilized_penalty,
                            dynamic_lambda=dynamic_lambda, alpha=alpha,
                            batch_prune_threshold=batch_prune_threshold, counts=N_b,
                            cache_path=None if autotune is True else str(autotune))
        tuned = {"sweep_form": choice["sweep_form"], "max_sweep_ctas": choice["max_sweep_ctas"]}
    problem = HarmonyProblem(
        X, cats_np, n_batches, Y0, th, precision=prec, n_clusters=n_clusters,
        max_iter_harmony=max_iter_harmony, max_iter_clustering=max_iter_clustering,
        tol_harmony=tol_harmony, tol_clustering=tol_clustering, ridge_lambda=ridge_lambda,
        sigma=sigma, block_proportion=block_proportion, random_state=random_state,
        stabilized_penalty=stabilized_penalty, dynamic_lambda=dynamic_lambda, alpha=alpha,
        batch_prune_threshold=batch_prune_threshold, counts=N_b, **tuned)
    Z_hat, info = problem.run()
    problem.close()
    if info.converged and verbose:
        print(f"Harmony converged in {info.n_outer} iterations")
    if not info.converged:
        warnings.warn("Harmony did not converge. Consider increasing the number of iterations")
    return (Z_hat, info) if return_info else Z_hat
