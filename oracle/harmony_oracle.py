"""CPU oracle for the Harmony integration path -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``, the
``smoke()`` entry point and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  The shipped engine (``rapids_singlecell_b200``)
never calls into this file and fails loudly when its CUDA library is missing.

It is a NumPy restatement of rapids_singlecell's Harmony, which has no CPU
path of its own (every step there is CuPy / CUDA / cuML).  Each function cites
the reference file:line it follows (paths relative to the rapids_singlecell
source tree):

* driver .................. src/rapids_singlecell/preprocessing/_harmony/__init__.py:41-289
* initial R / E / O ....... _harmony/__init__.py:292-353, _harmony/_fuses.py:6-8
* soft k-means loop ....... _cuda/harmony/clustering/clustering.cu:241-393
* PCG shuffle keys ........ _cuda/harmony/clustering/kernels_clustering.cuh:106-117
* penalty / fused R ....... _cuda/harmony/pen/kernels_pen.cuh:8-82
* L2 / L1 row normalise ... _cuda/harmony/normalize/kernels_normalize.cuh:7-108
* objective ............... clustering.cu:188-237, kernels_clustering.cuh:8-103,
                            _cuda/harmony/kmeans/kernels_kmeans.cuh:30-96
* ridge lambda ............ _harmony/__init__.py:454-480
* arrowhead inverse ....... _cuda/harmony/correction/kernels_correction_fast.cuh:24-123
* batched correction ...... _cuda/harmony/correction/correction_batched.cu:17-130,
                            _cuda/harmony/outer/kernels_outer.cuh:41-65
* original correction ..... _harmony/__init__.py:532-570 (dense inverse cross-check)
* convergence ............. clustering.cu:380-387 (window 3), __init__.py:722-734

Initial centroids are injected (``Y0``): the reference draws them from cuML
``KMeans(init="k-means||", max_iter=25)`` (``_harmony/__init__.py:315-323``), a
third-party dependency (cuml-cu12/13>=25.10) that is not part of the reference
tree, so both sides of a parity check receive the same ``Y0``.

Pinning: the component functions below are checked in ``tests/`` against every
analytical known-answer case in the reference's own tests
(tests/test_harmony.py:262-450, tests/test_harmony_kernels.py:54-484).  The
reference's dataset goldens (PBMC / IRcolitis downloads) are not available in
this environment, so end-to-end parity of the full loop is anchored on those
component pins plus the exact block permutation.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SUPPRESS_PENALTY = 1e30  # _harmony/__init__.py:38


# ---------------------------------------------------------------------------
# small kernels
# ---------------------------------------------------------------------------


def pcg_keys(n: int, seed: int) -> np.ndarray:
    """Shuffle keys ``pcg_hash(i ^ seed)`` for i in [0, n).

    Follows ``pcg_hash_kernel`` (kernels_clustering.cuh:106-117): a 32-bit LCG
    step followed by the RXS-M-XS output permutation, all mod 2**32.  The map
    i -> key is a bijection on 32-bit words, so keys of distinct cells never
    tie and the stable radix sort of the reference is a plain argsort.
    """
    i = np.arange(n, dtype=np.uint32)
    st = i ^ np.uint32(seed & 0xFFFFFFFF)
    st = st * np.uint32(747796405) + np.uint32(2891336453)
    word = ((st >> ((st >> np.uint32(28)) + np.uint32(4))) ^ st) * np.uint32(277803737)
    return (word >> np.uint32(22)) ^ word


def block_permutation(n: int, seed: int) -> np.ndarray:
    """Cell order of one k-means iteration: stable argsort of the PCG keys.

    The reference sorts (key, index) pairs with CUB ``DeviceRadixSort::SortPairs``
    over all 32 key bits (clustering.cu:292-305), which is stable.
    """
    return np.argsort(pcg_keys(n, seed), kind="stable").astype(np.int64)


def l2_normalize(X: np.ndarray) -> np.ndarray:
    """Row L2 normalisation with the inverse norm clamped to <= 1e12.

    ``l2_row_normalize_kernel`` (kernels_normalize.cuh:7-54): a zero row stays
    zero because rsqrt(0)=inf is clamped to 1e12 and multiplies zeros.
    """
    dt = X.dtype
    ss = np.sum(X * X, axis=1, dtype=dt)
    with np.errstate(divide="ignore"):
        inv = (dt.type(1) / np.sqrt(ss)).astype(dt)
    inv = np.minimum(inv, dt.type(1e12))
    return (X * inv[:, None]).astype(dt)


def l1_normalize(X: np.ndarray) -> np.ndarray:
    """Row L1 normalisation with the norm clamped to >= 1e-12.

    ``normalize_kernel`` (kernels_normalize.cuh:58-108), used on the initial R.
    """
    dt = X.dtype
    s = np.sum(np.abs(X), axis=1, dtype=dt)
    s = np.maximum(s, dt.type(1e-12))
    return (X * (dt.type(1) / s)[:, None]).astype(dt)


def penalty(E: np.ndarray, O: np.ndarray, theta: np.ndarray, stabilized: bool) -> np.ndarray:
    """Diversity penalty ``((E+1)/(O[+E]+1)) ** theta_b`` (kernels_pen.cuh:8-21)."""
    dt = E.dtype
    denom = (O + E + dt.type(1)) if stabilized else (O + dt.type(1))
    ratio = (E + dt.type(1)) / denom
    return np.power(ratio, theta.astype(dt)[:, None]).astype(dt)


def fused_pen_norm(S_rows: np.ndarray, pen: np.ndarray, cats: np.ndarray, term) -> np.ndarray:
    """New R rows: ``exp(term*(1-s)) * pen[cat]`` scaled by 1/row-sum.

    ``fused_pen_norm_kernel`` (kernels_pen.cuh:27-82); no clamp on the sum.
    """
    dt = S_rows.dtype
    val = np.exp(dt.type(term) * (dt.type(1) - S_rows)) * pen[cats]
    rs = np.sum(val, axis=1, dtype=dt)
    return (val * (dt.type(1) / rs)[:, None]).astype(dt)


def scatter_rows_by_cat(R_rows: np.ndarray, cats: np.ndarray, n_batches: int) -> np.ndarray:
    """``out[b] = sum of rows with cat == b`` (kernels_scatter.cuh:7-26,133-176)."""
    out = np.zeros((n_batches, R_rows.shape[1]), dtype=R_rows.dtype)
    for b in range(n_batches):
        m = cats == b
        if m.any():
            out[b] = R_rows[m].sum(axis=0, dtype=R_rows.dtype)
    return out


def objective(R, S, O, E, theta, sigma, stabilized) -> float:
    """Three-term Harmony objective (clustering.cu:188-237).

    kmeans error ``sum R*2*(1-S)`` (kernels_kmeans.cuh:30-96), entropy
    ``sigma * sum x*log(x+1e-12)`` with x the row-normalised R
    (kernels_clustering.cuh:8-62) and diversity
    ``sigma * sum theta_b O log((O[+E]+1)/(E+1))`` (kernels_clustering.cuh:68-103).
    Accumulated here in float64 whatever the working dtype.
    """
    R64 = R.astype(np.float64)
    km = float(np.sum(R64 * 2.0 * (1.0 - S.astype(np.float64))))
    x = R64 / R64.sum(axis=1, keepdims=True)
    ent = float(sigma * np.sum(x * np.log(x + 1e-12)))
    O64, E64 = O.astype(np.float64), E.astype(np.float64)
    num = (O64 + E64 + 1.0) if stabilized else (O64 + 1.0)
    div = float(sigma * np.sum(theta.astype(np.float64)[:, None] * O64 * np.log(num / (E64 + 1.0))))
    return km + ent + div


def compute_lambda_kb(E, O, N_b, *, alpha, threshold, ridge_lambda, dynamic_lambda):
    """Per-(batch, cluster) ridge lambda (_harmony/__init__.py:454-480)."""
    dt = E.dtype
    sentinel = dt.type(SUPPRESS_PENALTY)
    if not dynamic_lambda:
        lam = np.full_like(E, ridge_lambda)
    else:
        lam = (alpha * E).astype(dt)
        if threshold is not None:
            safe = np.where(N_b > 0, N_b, np.ones_like(N_b))
            prune = (O / safe[:, None]) < threshold
            prune |= (N_b[:, None] == 0)
            lam[prune] = sentinel
    lam[(O + lam) == 0] = sentinel
    return lam


def arrowhead_inverse(O_col: np.ndarray, lam_col: np.ndarray) -> np.ndarray:
    """Closed-form inverse of ``[[N_k, O^T], [O, diag(O+lambda)]]``.

    ``compute_inv_mats_kernel`` (kernels_correction_fast.cuh:24-123):
    f_b = 1/(O_b+lambda_b), p_b = -f_b O_b, c = N_k - sum f_b O_b^2,
    inv[0,0] = 1/c, inv[0,j] = inv[j,0] = p_j/c, inv[i,j] = p_i p_j / c + f_i delta_ij.
    """
    dt = O_col.dtype
    f = dt.type(1) / (O_col + lam_col)
    p = -f * O_col
    Nk = O_col.sum(dtype=dt)
    c = Nk - (f * O_col * O_col).sum(dtype=dt)
    cinv = dt.type(1) / c
    nb1 = O_col.shape[0] + 1
    inv = np.empty((nb1, nb1), dtype=dt)
    inv[0, 0] = cinv
    inv[0, 1:] = cinv * p
    inv[1:, 0] = p * cinv
    inv[1:, 1:] = np.outer(p, p) * cinv + np.diag(f)
    return inv


def correction_batched(X, R, O, lambda_kb, cats, n_batches):
    """Ridge (mixture-of-experts) correction over all clusters at once.

    ``correction_batched_impl`` (correction_batched.cu:17-130):
    M_k = Phi^T diag(R_k) X with row 0 = R_k^T X and row b+1 the batch-b part,
    W_k = inv_k M_k with row 0 zeroed, Z = X - sum_k R_k * W_k[cat+1]
    (``batched_correction_kernel``, kernels_outer.cuh:41-65).
    """
    dt = X.dtype
    n, d = X.shape
    K = R.shape[1]
    nb1 = n_batches + 1
    M = np.zeros((K, nb1, d), dtype=dt)
    M[:, 0, :] = R.T @ X
    masks = [cats == b for b in range(n_batches)]
    for b, m in enumerate(masks):
        if m.any():
            M[:, b + 1, :] = R[m].T @ X[m]
    inv = np.stack([arrowhead_inverse(O[:, k], lambda_kb[:, k]) for k in range(K)])
    W = np.matmul(inv, M)
    W[:, 0, :] = 0
    Z = X.copy()
    for b, m in enumerate(masks):
        if m.any():
            Z[m] = X[m] - R[m] @ W[:, b + 1, :]
    return Z.astype(dt)


def correction_original(X, R, lambda_kb, cats, n_batches):
    """Dense-inverse correction, one cluster at a time (_harmony/__init__.py:532-570)."""
    dt = X.dtype
    K = R.shape[1]
    nb1 = n_batches + 1
    Z = X.copy()
    for k in range(K):
        lam = np.zeros(nb1, dtype=dt)
        lam[1:] = lambda_kb[:, k]
        Rk = R[:, k]
        ssum = np.zeros(n_batches, dtype=dt)
        np.add.at(ssum, cats, Rk)
        A = np.zeros((nb1, nb1), dtype=dt)
        A[0, 0] = ssum.sum()
        A[0, 1:] = ssum
        A[1:, 0] = ssum
        A[1:, 1:] = np.diag(ssum)
        inv = np.linalg.inv(A + np.diag(lam))
        P = np.zeros((nb1, X.shape[1]), dtype=dt)
        P[0] = X.T @ Rk
        for b in range(n_batches):
            m = cats == b
            P[b + 1] = X[m].T @ Rk[m]
        W = inv @ P
        W[0] = 0
        Z -= Rk[:, None] * W[cats + 1]
    return Z


# ---------------------------------------------------------------------------
# the full loop
# ---------------------------------------------------------------------------


@dataclass
class OracleResult:
    Z_hat: np.ndarray
    objectives_harmony: list
    kmeans_objectives: list = field(default_factory=list)  # one list per outer iteration
    R: np.ndarray | None = None
    O: np.ndarray | None = None
    E: np.ndarray | None = None
    Y_norm: np.ndarray | None = None
    converged: bool = False
    n_outer: int = 0


def default_n_clusters(n_cells: int) -> int:
    """``max(2, int(min(100, n/30)))`` (_harmony/__init__.py:157-159)."""
    return max(int(min(100, n_cells / 30)), 2)


def theta_array(theta, n_batches, N_b, n_clusters, tau, dtype):
    """theta per batch plus the optional tau discount (_helper.py:277-307, __init__.py:172-175)."""
    if isinstance(theta, (int, float)):
        th = np.ones(n_batches, dtype=dtype) * float(theta)
    else:
        th = np.asarray(theta, dtype=dtype).ravel()
        if th.size != n_batches:
            raise ValueError(
                f"Theta array size ({th.size}) must match number of batches ({n_batches})"
            )
    if tau > 0:
        th = th * (1 - np.exp(-N_b / (n_clusters * tau)) ** 2)
    return th.astype(dtype)


def init_state(Z_norm, Y0, cats, n_batches, Pr_b, theta, sigma, stabilized):
    """Initial R, E, O and objective (_harmony/__init__.py:292-353)."""
    dt = Z_norm.dtype
    Yn = l2_normalize(Y0.astype(dt))
    term = dt.type(-2.0 / sigma)
    S = Z_norm @ Yn.T
    R = np.exp(term * (dt.type(1) - S)).astype(dt)
    R = l1_normalize(R)
    E = (Pr_b[:, None] * R.sum(axis=0, dtype=dt)[None, :]).astype(dt)
    O = scatter_rows_by_cat(R, cats, n_batches)
    obj0 = objective(R, S, O, E, theta, sigma, stabilized)
    return R, E, O, obj0


def clustering(Z_norm, R, E, O, Pr_b, cats, theta, *, n_batches, sigma, block_size,
               max_iter, tol, seed, stabilized):
    """One clustering call: ``clustering_loop_impl`` (clustering.cu:241-393).

    R, E, O are updated in place.  Returns the list of per-iteration objectives.
    """
    dt = Z_norm.dtype
    n = Z_norm.shape[0]
    term = dt.type(-2.0) / dt.type(sigma)
    objectives = []
    S = None
    Yn = None
    for it in range(max_iter):
        Y = (R.T @ Z_norm).astype(dt)
        Yn = l2_normalize(Y)
        S = (Z_norm @ Yn.T).astype(dt)
        idx = block_permutation(n, (seed + it) & 0xFFFFFFFF)
        for pos in range(0, n, block_size):
            bidx = idx[pos:pos + block_size]
            cin = cats[bidx]
            Rin = R[bidx]
            O -= scatter_rows_by_cat(Rin, cin, n_batches)
            E -= Pr_b[:, None] * Rin.sum(axis=0, dtype=dt)[None, :]
            pen = penalty(E, O, theta, stabilized)
            Rout = fused_pen_norm(S[bidx], pen, cin, term)
            R[bidx] = Rout
            O += scatter_rows_by_cat(Rout, cin, n_batches)
            E += Pr_b[:, None] * Rout.sum(axis=0, dtype=dt)[None, :]
        obj = objective(R, S, O, E, theta, sigma, stabilized)
        objectives.append(obj)
        if len(objectives) >= 4:
            old = objectives[-2] + objectives[-3] + objectives[-4]
            new = objectives[-1] + objectives[-2] + objectives[-3]
            if (old - new) < tol * abs(old):
                break
    return objectives, Yn


def harmonize(Z, cats, n_batches, Y0, *, n_clusters=None, max_iter_harmony=10,
              max_iter_clustering=200, tol_harmony=1e-4, tol_clustering=1e-5,
              ridge_lambda=1.0, sigma=0.1, block_proportion=0.05, theta=2.0, tau=0,
              random_state=0, stabilized_penalty=True, dynamic_lambda=True, alpha=0.2,
              batch_prune_threshold=1e-5, correction_method="batched",
              dtype=np.float64, timings=None) -> OracleResult:
    """Restatement of ``harmonize`` (_harmony/__init__.py:41-289) with injected Y0.

    ``timings`` (a dict, optional) receives the wall seconds of the phases: ``init`` (input
    normalisation and the initial R / E / O / objective), ``clustering`` (all k-means
    iterations, objective included) and ``correction`` (lambda, ridge correction and the
    renormalisation), summed over the outer iterations."""
    import time

    clock = time.perf_counter
    tm = {"init": 0.0, "clustering": 0.0, "correction": 0.0}
    t0 = clock()
    dt = np.dtype(dtype)
    X = np.ascontiguousarray(Z, dtype=dt)
    cats = np.asarray(cats, dtype=np.int64)
    n = X.shape[0]
    if max_iter_harmony < 1:
        raise ValueError("max_iter_harmony must be >= 1")
    K = n_clusters if n_clusters is not None else default_n_clusters(n)
    N_b = np.bincount(cats, minlength=n_batches).astype(dt)
    Pr_b = (N_b / n).astype(dt)
    th = theta_array(theta, n_batches, N_b, K, tau, dt)
    Z_norm = l2_normalize(X)
    block_size = int(n * block_proportion)
    R, E, O, obj0 = init_state(Z_norm, np.asarray(Y0), cats, n_batches, Pr_b, th, sigma,
                               stabilized_penalty)
    objs = [obj0]
    tm["init"] = clock() - t0
    km_objs = []
    converged = False
    Z_hat = X
    Yn = None
    n_outer = 0
    for i in range(max_iter_harmony):
        t0 = clock()
        km, Yn = clustering(Z_norm, R, E, O, Pr_b, cats, th, n_batches=n_batches, sigma=sigma,
                            block_size=block_size, max_iter=max_iter_clustering,
                            tol=tol_clustering,
                            seed=(random_state + i * 1000003) & 0xFFFFFFFF,
                            stabilized=stabilized_penalty)
        km_objs.append(km)
        objs.append(km[-1])
        tm["clustering"] += clock() - t0
        t0 = clock()
        lam = compute_lambda_kb(E, O, N_b, alpha=alpha, threshold=batch_prune_threshold,
                                ridge_lambda=ridge_lambda, dynamic_lambda=dynamic_lambda)
        if correction_method == "original":
            Z_hat = correction_original(X, R, lam, cats, n_batches)
        else:
            Z_hat = correction_batched(X, R, O, lam, cats, n_batches)
        Z_norm = l2_normalize(Z_hat)
        tm["correction"] += clock() - t0
        n_outer = i + 1
        if len(objs) >= 2 and (objs[-2] - objs[-1]) < tol_harmony * abs(objs[-2]):
            converged = True
            break
    if timings is not None:
        timings.update(tm)
    return OracleResult(Z_hat=Z_hat, objectives_harmony=objs, kmeans_objectives=km_objs,
                        R=R, O=O, E=E, Y_norm=Yn, converged=converged, n_outer=n_outer)
