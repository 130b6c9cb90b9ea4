"""The reference's Harmony run on a GPU with its own kernels -- TEST INFRASTRUCTURE ONLY.

``harmonize`` restates rapids_singlecell's Python driver
(src/rapids_singlecell/preprocessing/_harmony/__init__.py:41-289) with torch CUDA
tensors in place of CuPy arrays.  Every step that the reference runs in one of its
CUDA modules goes through ``oracle/_ref/libharmony_ref.so`` (built by
``oracle/Makefile`` from ``oracle/ref_shim.cu`` and the reference's unmodified
``kernels_*.cuh`` headers): L2 / L1 row normalisation, column sums, the outer
product into E, the scatter-add into O, the objective, the whole soft k-means
loop and the batched ridge correction.  The few CuPy expressions of the driver
(``cp.dot`` for the initial similarities, the ``_calc_R`` fuse, ``_compute_lambda_kb``,
``_create_category_index_mapping``) are restated with torch.

Used by ``tests/`` to pin the NumPy oracle (through the fixtures that
``tests/golden/make_ref_golden.py`` writes) and to check the engine against the
reference on the GPU.  The shipped engine never imports this module.

Initial centroids are injected (``Y0``) in place of the cuML k-means fit of
``_initialize_centroids`` (__init__.py:315-323), exactly as the oracle does.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libharmony_ref.so"
SUPPRESS_PENALTY = 1e30  # __init__.py:38

# colsum heuristic constants (_helper.py:27-34) and its rule (_helper.py:383-397), for
# compute capability "100" (B200; the data-center branch)
_COLS_SMALL, _COLS_MEDIUM, _COLS_LARGE, _COLS_XLARGE = 200, 800, 1024, 2000
_ROWS_TINY, _ROWS_SMALL, _ROWS_MEDIUM, _ROWS_LARGE = 5_000, 10_000, 20_000, 100_000
COLSUM_CODES = {"columns": 0, "atomics": 1, "gemm": 2}

_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def load():
    """The shim library (raises when it was not built: ``make -C oracle``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"reference shim not built: {LIB_PATH} (make -C oracle)")
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.ref_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what}: {load().ref_last_error().decode()}")


def colsum_heuristic(rows: int, cols: int) -> str:
    """``_colsum_heuristic`` (_helper.py:383-397) on a data-center part."""
    if cols < _COLS_SMALL and rows < _ROWS_MEDIUM:
        return "columns"
    if cols < _COLS_SMALL and rows < _ROWS_LARGE:
        return "columns"
    if cols < _COLS_MEDIUM and rows < _ROWS_SMALL:
        return "atomics"
    if cols < _COLS_LARGE and rows < _ROWS_TINY:
        return "atomics"
    if cols < _COLS_MEDIUM and rows < _ROWS_MEDIUM:
        return "atomics"
    if cols < _COLS_XLARGE and rows < _ROWS_SMALL:
        return "atomics"
    return "gemm"


def _sfx(t):
    import torch

    return "f64" if t.dtype == torch.float64 else "f32"


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def l2_normalize(X):
    """``_normalize_cp(X, p=2)`` (_helper.py:186-204): l2_row_normalize_kernel into a new array."""
    import torch

    X = X.contiguous()
    dst = torch.empty_like(X)
    _check(getattr(load(), f"ref_l2_row_normalize_{_sfx(X)}")(_p(X), _p(dst), X.shape[0], X.shape[1], _stream()),
           "l2_row_normalize")
    return dst


def l1_normalize_(X):
    """``_normalize_cp_p1`` (_helper.py:37-60): normalize_kernel in place."""
    _check(getattr(load(), f"ref_l1_normalize_{_sfx(X)}")(_p(X), ctypes.c_longlong(X.shape[0]),
                                                            ctypes.c_longlong(X.shape[1]), _stream()),
           "normalize")
    return X


def colsum(X, algo: str):
    import torch

    out = torch.empty(X.shape[1], dtype=X.dtype, device=X.device)
    _check(getattr(load(), f"ref_colsum_{_sfx(X)}")(_p(X), _p(out), X.shape[0], X.shape[1], COLSUM_CODES[algo],
                                                      _stream()), "colsum")
    return out


def outer_(E, Pr_b, R_sum, switcher: int):
    """``_outer_cp`` (_helper.py:170-183)."""
    _check(getattr(load(), f"ref_outer_{_sfx(E)}")(_p(E), _p(Pr_b), _p(R_sum), ctypes.c_longlong(E.shape[0]),
                                                     ctypes.c_longlong(E.shape[1]), ctypes.c_longlong(switcher),
                                                     _stream()), "outer")


def scatter_add_(X, out, cats, switcher: int, n_batches: int):
    """``_scatter_add_cp`` (_helper.py:63-145)."""
    _check(getattr(load(), f"ref_scatter_add_{_sfx(X)}")(_p(X), _p(out), _p(cats), X.shape[0], X.shape[1], switcher,
                                                           n_batches, _stream()), "scatter_add")


def compute_objective(S, R, theta, sigma, O, E, stabilized: bool) -> float:
    """``_compute_objective`` (__init__.py:670-719) -> compute_objective_impl."""
    out = (ctypes.c_double if _sfx(R) == "f64" else ctypes.c_float)()
    n, K = R.shape
    _check(getattr(load(), f"ref_compute_objective_{_sfx(R)}")(_p(R), _p(S), _p(O), _p(E), _p(theta),
                                                                 ctypes.c_double(sigma), n, K, O.shape[0],
                                                                 int(stabilized), ctypes.byref(out), _stream()),
           "compute_objective")
    return float(out.value)


def category_index_mapping(cats, n_batches: int):
    """``_create_category_index_mapping`` (_utils/_multi_gpu.py:202-232): CSR offsets and the
    cells ordered by (category, index)."""
    import torch

    counts = torch.bincount(cats.long(), minlength=n_batches)
    offsets = torch.zeros(n_batches + 1, dtype=torch.int32, device=cats.device)
    offsets[1:] = torch.cumsum(counts, 0).to(torch.int32)
    cell_indices = torch.sort(cats.long(), stable=True).indices.to(torch.int32)
    return offsets, cell_indices


def compute_lambda_kb(E, O, N_b, *, alpha, threshold, ridge_lambda, dynamic_lambda):
    """``_compute_lambda_kb`` (__init__.py:454-480)."""
    import torch

    sentinel = SUPPRESS_PENALTY
    if not dynamic_lambda:
        lam = torch.full_like(E, ridge_lambda)
    else:
        lam = (alpha * E).to(E.dtype)
        if threshold is not None:
            safe_N_b = torch.where(N_b > 0, N_b, torch.ones_like(N_b))
            mask = (O / safe_N_b[:, None]) < threshold
            mask |= (N_b[:, None] == 0)
            lam[mask] = sentinel
    lam[(O + lam) == 0] = sentinel
    return lam


@dataclass
class RefResult:
    Z_hat: np.ndarray
    objectives_harmony: list = field(default_factory=list)
    kmeans_objectives: list = field(default_factory=list)
    R: np.ndarray | None = None
    O: np.ndarray | None = None
    E: np.ndarray | None = None
    converged: bool = False
    n_outer: int = 0


def harmonize(Z, cats, n_batches, Y0, *, n_clusters=None, max_iter_harmony=10, max_iter_clustering=200,
              tol_harmony=1e-4, tol_clustering=1e-5, ridge_lambda=1.0, sigma=0.1, block_proportion=0.05,
              theta=2.0, tau=0, random_state=0, stabilized_penalty=True, dynamic_lambda=True, alpha=0.2,
              batch_prune_threshold=1e-5, dtype=np.float64, device="cuda") -> RefResult:
    """``harmonize`` (__init__.py:41-289) on the GPU with the reference's kernels and injected Y0.

    Z, cats, Y0 are host arrays; the result comes back to the host.  The correction is the
    reference's "batched" method, which its auto-selection picks whenever the K (B+1)^2
    inverses fit in 1 GB (__init__.py:196-200)."""
    import torch

    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    Zt = torch.as_tensor(np.ascontiguousarray(Z), device=device).to(tdt)
    n, d = Zt.shape
    Z_norm = l2_normalize(Zt)
    cats_t = torch.as_tensor(np.asarray(cats, dtype=np.int32), device=device)
    N_b = torch.bincount(cats_t.long(), minlength=n_batches).to(tdt)
    Pr_b = (N_b.reshape(-1, 1) / n).to(tdt)
    cat_offsets, cell_indices = category_index_mapping(cats_t, n_batches)
    if max_iter_harmony < 1:
        raise ValueError("max_iter_harmony must be >= 1")
    if n_clusters is None:
        n_clusters = max(int(min(100, n / 30)), 2)
    K = n_clusters
    block_size = int(n * block_proportion)
    colsum_big = colsum_heuristic(n, K)
    colsum_small = colsum_heuristic(block_size, K)
    if isinstance(theta, (int, float)):
        th = torch.ones(n_batches, dtype=tdt, device=device) * float(theta)
    else:
        th = torch.as_tensor(np.asarray(theta, dtype=np.float64), device=device).to(tdt).ravel()
    if tau > 0:
        th = th * (1 - torch.exp(-N_b / (K * tau)) ** 2)
    th = th.contiguous()
    nb1 = n_batches + 1
    assert K * nb1 * nb1 * Zt.element_size() <= (1 << 30), "batched correction only"

    # _initialize_centroids (__init__.py:292-353) with Y0 injected
    Y = torch.as_tensor(np.asarray(Y0), device=device).to(tdt)
    Y_norm = l2_normalize(Y)
    term = -2.0 / sigma
    S = Z_norm @ Y_norm.T
    R = torch.exp(term * (1 - S)).contiguous()
    l1_normalize_(R)
    R_sum = colsum(R, colsum_big)
    E = torch.zeros((n_batches, K), dtype=tdt, device=device)
    outer_(E, Pr_b, R_sum, 1)
    O = torch.zeros((n_batches, K), dtype=tdt, device=device)
    scatter_add_(R, O, cats_t, 1, n_batches)
    objectives = [compute_objective(S, R, th, sigma, O, E, stabilized_penalty)]
    del S

    km_objs = []
    converged = False
    n_outer = 0
    Z_hat = Zt
    Pr_flat = Pr_b.ravel().contiguous()
    ctype = ctypes.c_double if tdt == torch.float64 else ctypes.c_float
    for i in range(max_iter_harmony):
        # _clustering (__init__.py:387-451) -> clustering_loop
        objs = (ctype * max(max_iter_clustering, 1))()
        n_iter = ctypes.c_int(0)
        seed = (random_state + i * 1000003) & 0xFFFFFFFF
        _check(getattr(load(), f"ref_clustering_loop_{_sfx(Zt)}")(
            _p(Z_norm), _p(R), _p(E), _p(O), _p(Pr_flat), _p(cats_t), _p(th), n, d, K, n_batches, block_size,
            COLSUM_CODES[colsum_small], ctypes.c_double(sigma), ctypes.c_double(tol_clustering), max_iter_clustering,
            ctypes.c_uint(seed), int(stabilized_penalty), objs, ctypes.byref(n_iter), _stream()), "clustering_loop")
        km = [float(objs[j]) for j in range(n_iter.value)]
        km_objs.append(km)
        objectives.append(km[-1] if km else 0.0)  # last_obj (clustering.cu:390-392)
        lam = compute_lambda_kb(E, O, N_b, alpha=alpha, threshold=batch_prune_threshold,
                                ridge_lambda=ridge_lambda, dynamic_lambda=dynamic_lambda).contiguous()
        Z_hat = torch.empty_like(Zt)
        _check(getattr(load(), f"ref_correction_batched_{_sfx(Zt)}")(
            _p(Zt), _p(R), _p(O), _p(cats_t), _p(cat_offsets), _p(cell_indices), _p(lam), n, d, K, n_batches,
            _p(Z_hat), _stream()), "correction_batched")
        Z_norm = l2_normalize(Z_hat)
        n_outer = i + 1
        if len(objectives) >= 2 and (objectives[-2] - objectives[-1]) < tol_harmony * abs(objectives[-2]):
            converged = True
            break
    torch.cuda.synchronize()
    return RefResult(Z_hat=Z_hat.cpu().numpy(), objectives_harmony=objectives, kmeans_objectives=km_objs,
                     R=R.cpu().numpy(), O=O.cpu().numpy(), E=E.cpu().numpy(), converged=converged, n_outer=n_outer)
