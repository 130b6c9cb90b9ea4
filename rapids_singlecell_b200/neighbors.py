"""k nearest neighbours on the B200: the neighbour graph of ``rapids_singlecell.pp.neighbors``.

The search is the engine's exact brute-force kernel (``hb_knn``, ``csrc/hb_knn.cu``): dot
products on the tensor core, each query's candidates re-ranked with exact float32 distances.
The reference runs cuML ``NearestNeighbors(algorithm="brute")``
(src/rapids_singlecell/preprocessing/_neighbors/_algorithms/_brute.py:14-37).  Around it,
restated from the reference: the zeroed self-distance (``_fix_self_distances``,
_neighbors/_helper/__init__.py:114-129), the distance matrix (``_build_sparse_distances``,
_neighbors/_neighbors.py:95-132) and the connectivities (``_calc_connectivities``,
_neighbors.py:265-318): the adaptive Gaussian kernel (``gauss``, _neighbors.py:163-209), the
PhenoGraph Jaccard index (``jaccard``, _neighbors.py:212-262), and the UMAP fuzzy simplicial set
(``umap``; the reference calls cuML's ``fuzzy_simplicial_set``, here the published algorithm of
McInnes, Healy and Melville 2018: per-cell rho and sigma by bisection so that the memberships sum
to log2(k), then the fuzzy union W + W^T - W o W^T).  The graph arithmetic runs in torch on the
GPU; the results are returned as scipy CSR matrices, as the reference stores them.
"""

from __future__ import annotations

import ctypes
import math
from types import MappingProxyType

import numpy as np
import torch

from . import _lib

METRICS = {"sqeuclidean": _lib.HB_KNN_SQEUCLIDEAN, "euclidean": _lib.HB_KNN_EUCLIDEAN,
           "l2": _lib.HB_KNN_EUCLIDEAN, "cosine": _lib.HB_KNN_COSINE,
           "inner_product": _lib.HB_KNN_INNER_PRODUCT}
# the reference's algorithm names (_neighbors/_neighbors.py:34-42); every one of them is
# answered by the exact search, which the approximate ones (ivf, cagra, nn-descent) estimate
ALGORITHMS = ("brute", "ivfflat", "ivfpq", "cagra", "nn_descent", "all_neighbors", "mg_ivfflat", "mg_ivfpq")


def knn_arrays(X, k: int, *, metric: str = "euclidean", queries=None, device=None):
    """(indices int64 [nq, k], distances float32 [nq, k]) of the k nearest rows of X for every
    row of `queries` (X itself when None), ascending by distance then index."""
    if metric not in METRICS:
        raise NotImplementedError(f"metric {metric!r} is not supported by the B200 kNN kernel "
                                  f"(supported: {sorted(METRICS)})")
    lib = _lib.load()
    device = torch.device(device) if device is not None else (
        X.device if isinstance(X, torch.Tensor) and X.is_cuda else torch.device("cuda"))
    Xd = torch.as_tensor(X, device=device).to(torch.float32).contiguous()
    Qd = Xd if queries is None else torch.as_tensor(queries, device=device).to(torch.float32).contiguous()
    n, d = Xd.shape
    nq = Qd.shape[0]
    same = queries is None
    idx = torch.empty((nq, k), dtype=torch.int64, device=device)
    dist = torch.empty((nq, k), dtype=torch.float32, device=device)
    code = METRICS[metric]
    ws_bytes = lib.hb_knn_workspace_bytes(nq, n, d, int(same), code)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    qp = ctypes.c_void_p(Qd.data_ptr())
    _lib.check(lib.hb_knn(qp, nq, ctypes.c_void_p(Xd.data_ptr()), n, d, k, code, ctypes.c_void_p(idx.data_ptr()),
                          ctypes.c_void_p(dist.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws_bytes, st))
    return idx, dist


def fix_self_distances(dist: torch.Tensor, metric: str) -> torch.Tensor:
    """Zero self-distance in column 0 for every metric but the inner product
    (_neighbors/_helper/__init__.py:114-129)."""
    if metric not in ("inner_product",):
        dist[:, 0] = 0.0
    return dist


def _csr(rows, cols, vals, n):
    import scipy.sparse as sp

    return sp.csr_matrix((vals.cpu().numpy(), (rows.cpu().numpy(), cols.cpu().numpy())), shape=(n, n))


def build_sparse_distances(idx: torch.Tensor, dist: torch.Tensor, n_obs: int):
    """CSR [n_obs, n_obs] with the k distances of each row (_neighbors.py:95-132)."""
    import scipy.sparse as sp

    k = dist.shape[1]
    indptr = np.arange(0, n_obs * k + 1, k, dtype=np.int64)
    return sp.csr_matrix((dist.reshape(-1).cpu().numpy(), idx.reshape(-1).cpu().numpy(), indptr),
                         shape=(n_obs, n_obs))


def _sym_reduce(rows, cols, vals, n, how):
    """Entries (i, j, v) and their transposes (j, i, v) merged per position: 'max' keeps the
    larger, 'mean' averages the matrix with its transpose, 'fuzzy' is a + b - a b."""
    key = torch.cat([rows * n + cols, cols * n + rows])
    v = torch.cat([vals, vals])
    uniq, inv = torch.unique(key, return_inverse=True)
    if how == "max":
        out = torch.full((uniq.numel(),), -math.inf, dtype=v.dtype, device=v.device)
        out.scatter_reduce_(0, inv, v, reduce="amax")
    elif how == "mean":
        out = torch.zeros(uniq.numel(), dtype=v.dtype, device=v.device).index_add_(0, inv, v) / 2
    else:  # fuzzy union: each position gets a (the entry) and b (its transpose), 0 if absent
        s = torch.zeros(uniq.numel(), dtype=v.dtype, device=v.device).index_add_(0, inv, v)
        p = torch.ones(uniq.numel(), dtype=v.dtype, device=v.device)
        # a b: the product of a position's two contributions (0 when one of them is absent)
        cnt = torch.zeros(uniq.numel(), dtype=torch.int64, device=v.device).index_add_(
            0, inv, torch.ones_like(inv))
        p.scatter_reduce_(0, inv, v, reduce="prod")
        out = s - torch.where(cnt == 2, p, torch.zeros_like(p))
    return uniq // n, uniq % n, out


def connectivities_gauss(idx, dist, n_obs):
    """Adaptive Gaussian kernel (_neighbors.py:163-209)."""
    k = idx.shape[1]
    d_sq = dist.double() ** 2
    sig_sq = torch.median(d_sq[:, 1:], dim=1).values if k > 2 else d_sq[:, 1]
    sig = torch.sqrt(sig_sq)
    rows = torch.arange(n_obs, device=idx.device).repeat_interleave(k - 1)
    cols = idx[:, 1:].reshape(-1)
    dv = d_sq[:, 1:].reshape(-1)
    den = sig_sq[rows] + sig_sq[cols]
    vals = torch.sqrt(2.0 * sig[rows] * sig[cols] / den) * torch.exp(-dv / den)
    r, c, v = _sym_reduce(rows, cols, vals, n_obs, "max")
    return _csr(r, c, v.float(), n_obs)


def connectivities_jaccard(idx, n_obs, n_neighbors):
    """PhenoGraph Jaccard index of the shared neighbours of each kNN edge, symmetrised by
    averaging (_neighbors.py:212-262)."""
    kns = n_neighbors - 1
    nb = torch.sort(idx[:, 1:], dim=1).values
    rows = torch.arange(n_obs, device=idx.device).repeat_interleave(kns)
    cols = idx[:, 1:].reshape(-1)
    shared = torch.empty(rows.numel(), dtype=torch.float64, device=idx.device)
    chunk = max(1, (1 << 26) // (kns * kns))
    for s in range(0, rows.numel(), chunk):
        a = nb[rows[s:s + chunk]]
        b = nb[cols[s:s + chunk]]
        shared[s:s + chunk] = (a[:, :, None] == b[:, None, :]).sum(dim=(1, 2)).double()
    vals = shared / (2 * kns - shared)
    keep = vals != 0
    r, c, v = _sym_reduce(rows[keep], cols[keep], vals[keep], n_obs, "mean")
    return _csr(r, c, v.float(), n_obs)


def connectivities_umap(idx, dist, n_obs, n_neighbors, n_iter: int = 64, bandwidth: float = 1.0):
    """UMAP fuzzy simplicial set with set_op_mix_ratio = 1 and local_connectivity = 1 (the
    reference's settings, _neighbors.py:135-160): rho_i = the nearest non-zero distance,
    sigma_i by bisection so that sum_j exp(-max(0, d_ij - rho_i) / sigma_i) = log2(k) bandwidth,
    memberships exp(-max(0, d_ij - rho_i) / sigma_i) (1 for the nearest), fuzzy union."""
    d = dist.double()
    target = math.log2(n_neighbors) * bandwidth
    pos = torch.where(d > 0, d, torch.full_like(d, math.inf))
    rho = pos.min(dim=1).values
    rho = torch.where(torch.isfinite(rho), rho, torch.zeros_like(rho))
    lo = torch.zeros(n_obs, dtype=torch.float64, device=d.device)
    hi = torch.full_like(lo, math.inf)
    mid = torch.ones_like(lo)
    dd = (d[:, 1:] - rho[:, None]).clamp_min(0.0)
    for _ in range(n_iter):
        psum = torch.exp(-dd / mid[:, None]).sum(dim=1)
        over = psum > target
        hi = torch.where(over, mid, hi)
        lo = torch.where(over, lo, mid)
        mid = torch.where(torch.isfinite(hi), (lo + hi) / 2, mid * 2)
    mean_d = d.mean()
    sig = torch.where(rho > 0, torch.maximum(mid, 1e-3 * d.mean(dim=1)), torch.maximum(mid, 1e-3 * mean_d))
    rows = torch.arange(n_obs, device=idx.device).repeat_interleave(idx.shape[1])
    cols = idx.reshape(-1)
    w = torch.exp(-(d - rho[:, None]).clamp_min(0.0) / sig[:, None])
    w[idx == torch.arange(n_obs, device=idx.device)[:, None]] = 0.0  # no self loops
    w = w.reshape(-1)
    keep = w > 0
    r, c, v = _sym_reduce(rows[keep], cols[keep], w[keep], n_obs, "fuzzy")
    return _csr(r, c, v.float(), n_obs)


def _choose_representation(adata, use_rep, n_pcs):
    """.X for fewer than 50 variables, else X_pca (computed when missing), or `use_rep`; the
    first n_pcs columns of X_pca when given (scanpy's rule, which the reference follows)."""
    if use_rep is None:
        n_vars = adata.X.shape[1] if getattr(adata, "X", None) is not None else 0
        if n_pcs == 0 or (n_vars < 50 and "X_pca" not in adata.obsm):
            return adata.X
        use_rep = "X_pca"
        if "X_pca" not in adata.obsm:
            from .pca import pp_pca

            pp_pca(adata, n_comps=n_pcs)
    if use_rep == "X":
        return adata.X
    rep = adata.obsm[use_rep]
    if use_rep == "X_pca" and n_pcs is not None:
        rep = rep[:, :n_pcs]
    return rep


def pp_neighbors(adata, n_neighbors: int = 15, n_pcs: int | None = None, *, use_rep: str | None = None,
                 random_state=0, algorithm: str = "brute", metric: str = "euclidean",
                 metric_kwds=MappingProxyType({}), algorithm_kwds=MappingProxyType({}), method: str = "umap",
                 key_added: str | None = None, copy: bool = False):
    """Drop-in for ``rapids_singlecell.pp.neighbors`` (_neighbors/__init__.py:35-246): the kNN
    graph of the chosen representation, ``obsp['distances']`` / ``obsp['connectivities']`` and
    ``uns['neighbors']`` (or the ``key_added`` names)."""
    if algorithm not in ALGORITHMS:
        raise ValueError(f"Invalid algorithm '{algorithm}' for KNN. Valid options are: {ALGORITHMS}.")
    if method not in ("umap", "gauss", "jaccard"):
        raise ValueError(f"method {method!r} must be 'umap', 'gauss' or 'jaccard'")
    if copy:
        adata = adata.copy()
    X = _choose_representation(adata, use_rep, n_pcs)
    if hasattr(X, "toarray"):
        X = X.toarray()
    idx, dist = knn_arrays(X, n_neighbors, metric=metric)
    dist = fix_self_distances(dist, metric)
    n_obs = idx.shape[0]
    distances = build_sparse_distances(idx, dist, n_obs)
    if method == "gauss":
        conn = connectivities_gauss(idx, dist, n_obs)
    elif method == "jaccard":
        conn = connectivities_jaccard(idx, n_obs, n_neighbors)
    else:
        conn = connectivities_umap(idx, dist, n_obs, n_neighbors)
    params = dict(n_neighbors=n_neighbors, method="rapids", random_state=random_state, metric=metric,
                  **({"metric_kwds": dict(metric_kwds)} if metric_kwds else {}),
                  **({"algorithm_kwds": dict(algorithm_kwds)} if algorithm_kwds else {}),
                  **({"use_rep": use_rep} if use_rep is not None else {}),
                  **({"n_pcs": n_pcs} if n_pcs is not None else {}))
    key = "neighbors" if key_added is None else key_added
    dkey = "distances" if key_added is None else f"{key_added}_distances"
    ckey = "connectivities" if key_added is None else f"{key_added}_connectivities"
    adata.uns[key] = {"connectivities_key": ckey, "distances_key": dkey, "params": params}
    adata.obsp[dkey] = distances
    adata.obsp[ckey] = conn
    return adata if copy else None
