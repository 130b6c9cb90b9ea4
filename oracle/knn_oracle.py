"""CPU oracle for exact k nearest neighbours -- TEST INFRASTRUCTURE ONLY.

Brute force in float64 with NumPy, the exact answer that the reference's
``_brute_knn`` (src/rapids_singlecell/preprocessing/_neighbors/_algorithms/_brute.py:14-37)
obtains from cuML ``NearestNeighbors(algorithm="brute")`` -- a third-party package (cuml-cu12/13,
pyproject.toml) that is not part of the reference tree and cannot run here, so this oracle is
the published definition of each metric (scipy.spatial.distance conventions): sqeuclidean
sum (q - x)^2, euclidean its square root, cosine 1 - q.x / (|q| |x|), inner_product q.x
(largest first).  Ties are ordered by index.  Parity of the neighbour search itself is
therefore pinned to the metric definitions, not to cuML's outputs.
"""

from __future__ import annotations

import numpy as np


def knn(X, k, metric="euclidean", queries=None, chunk=2048):
    X = np.asarray(X, dtype=np.float64)
    Q = X if queries is None else np.asarray(queries, dtype=np.float64)
    if metric == "cosine":
        Xn = X / np.maximum(np.linalg.norm(X, axis=1, keepdims=True), 1e-300)
        Qn = Q / np.maximum(np.linalg.norm(Q, axis=1, keepdims=True), 1e-300)
    idx = np.empty((Q.shape[0], k), dtype=np.int64)
    dist = np.empty((Q.shape[0], k), dtype=np.float64)
    x2 = (X * X).sum(1)
    for s in range(0, Q.shape[0], chunk):
        q = Q[s:s + chunk]
        if metric in ("euclidean", "l2", "sqeuclidean"):
            D = (q * q).sum(1)[:, None] + x2[None, :] - 2.0 * q @ X.T
            np.maximum(D, 0.0, out=D)
        elif metric == "cosine":
            D = 1.0 - Qn[s:s + chunk] @ Xn.T
        elif metric == "inner_product":
            D = -(q @ X.T)
        else:
            raise ValueError(metric)
        order = np.lexsort((np.broadcast_to(np.arange(X.shape[0]), D.shape), D), axis=1)[:, :k]
        idx[s:s + chunk] = order
        dist[s:s + chunk] = np.take_along_axis(D, order, axis=1)
    if metric in ("euclidean", "l2"):
        dist = np.sqrt(dist)
    elif metric == "inner_product":
        dist = -dist
    return idx, dist


def gauss_connectivities(idx, dist, n):
    """Adaptive Gaussian kernel of the reference (_neighbors/_neighbors.py:163-209), dense."""
    k = idx.shape[1]
    d_sq = np.asarray(dist, np.float64) ** 2
    sig_sq = np.median(d_sq[:, 1:], axis=1)
    sig = np.sqrt(sig_sq)
    W = np.zeros((n, n))
    for i in range(n):
        for jj in range(1, k):
            j = idx[i, jj]
            den = sig_sq[i] + sig_sq[j]
            W[i, j] = np.sqrt(2 * sig[i] * sig[j] / den) * np.exp(-d_sq[i, jj] / den)
    return np.maximum(W, W.T)


def jaccard_connectivities(idx, n, n_neighbors):
    """PhenoGraph Jaccard connectivities of the reference (_neighbors.py:212-262), dense."""
    kns = n_neighbors - 1
    nb = [set(idx[i, 1:].tolist()) for i in range(n)]
    W = np.zeros((n, n))
    for i in range(n):
        for j in idx[i, 1:]:
            s = len(nb[i] & nb[j])
            W[i, j] = s / (2 * kns - s)
    return (W + W.T) / 2


def umap_connectivities(idx, dist, n, n_neighbors, n_iter=64):
    """UMAP fuzzy simplicial set (McInnes, Healy & Melville 2018; smooth_knn_dist with
    local_connectivity = 1, bandwidth = 1, then the fuzzy union), dense, scalar loops."""
    dist = np.asarray(dist, np.float64)
    target = np.log2(n_neighbors)
    mean_all = dist.mean()
    W = np.zeros((n, n))
    for i in range(n):
        row = dist[i]
        nz = row[row > 0]
        rho = nz.min() if nz.size else 0.0
        lo, hi, mid = 0.0, np.inf, 1.0
        for _ in range(n_iter):
            psum = sum(np.exp(-max(0.0, row[j] - rho) / mid) for j in range(1, len(row)))
            if psum > target:
                hi = mid
                mid = (lo + hi) / 2
            else:
                lo = mid
                mid = mid * 2 if hi == np.inf else (lo + hi) / 2
        sigma = max(mid, 1e-3 * (row.mean() if rho > 0 else mean_all))
        for jj in range(len(row)):
            j = idx[i, jj]
            if j == i:
                continue
            W[i, j] = 1.0 if row[jj] - rho <= 0 else np.exp(-(row[jj] - rho) / sigma)
    return W + W.T - W * W.T
