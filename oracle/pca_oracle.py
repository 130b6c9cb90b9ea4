"""CPU oracle for PCA by the covariance eigendecomposition -- TEST INFRASTRUCTURE ONLY.

NumPy restatement of rapids_singlecell's covariance PCA (``pp.pca`` ->
``_run_covariance_pca``, src/rapids_singlecell/preprocessing/_pca.py:339-353 ->
``PCA_sparse.fit`` / ``transform``, preprocessing/_sparse_pca/_sparse_pca.py:26-127):

* zero_center:   mean = column means (preprocessing/_utils.py:88-105),
                 cov = X^T X / n - mean mean^T  (_cov_sparse, _sparse_pca.py:138-199;
                 cov_from_gram_kernel, _cuda/spca/kernels_spca.cuh:48-62)
* uncentred:     cov = X^T X, not scaled (the return_gram path, _sparse_pca.py:183-188)
* eigh, eigenvalues and vectors reversed to descending order, components = the first
  n_comps eigenvectors as rows, variance ratio over the sum of all eigenvalues
  (_sparse_pca.py:47-69)
* transform:     X C^T - mean C^T (zero_center) or X C^T (_sparse_pca.py:84-95)

Only ``tests/`` and the CPU legs of ``bench.py`` import it; the engine never does.
Pinned to the reference's own kernels through ``tests/golden/ref_pca_*.npz`` (written by
``tests/golden/make_ref_golden.py`` with ``oracle/_ref/libharmony_ref.so``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class PcaResult:
    X_pca: np.ndarray
    components: np.ndarray      # [n_comps][n_genes]
    variance: np.ndarray        # [n_comps]
    variance_ratio: np.ndarray  # [n_comps]
    mean: np.ndarray | None


def default_n_comps(n_obs: int, n_vars: int) -> int:
    """50, or min(n_obs, n_vars) - 1 when that is not larger (_pca.py:230-235)."""
    min_dim = min(n_obs, n_vars)
    return min_dim - 1 if 50 >= min_dim else 50


def covariance(X, zero_center: bool = True):
    """(cov, mean) of X in float64 (_cov_sparse, _sparse_pca.py:138-199)."""
    X = np.asarray(X, dtype=np.float64)
    n = X.shape[0]
    if not zero_center:
        return X.T @ X, None
    mean = X.mean(axis=0)
    return X.T @ X / n - np.outer(mean, mean), mean


def pca(X, n_comps: int | None = None, zero_center: bool = True) -> PcaResult:
    """PCA_sparse.fit + transform (_sparse_pca.py:26-127) in float64."""
    X = np.asarray(X, dtype=np.float64)
    if n_comps is None:
        n_comps = default_n_comps(*X.shape)
    cov, mean = covariance(X, zero_center)
    evals, evecs = np.linalg.eigh(cov)
    evals = evals[::-1]
    comps = np.flip(evecs, axis=1).T[:n_comps]
    ratio = evals / evals.sum()
    X_pca = X @ comps.T
    if zero_center:
        X_pca = X_pca - mean @ comps.T
    return PcaResult(X_pca=X_pca, components=comps, variance=evals[:n_comps].copy(),
                     variance_ratio=ratio[:n_comps].copy(), mean=mean)


def align_signs(components, reference):
    """Per-component signs (+1 / -1) that make `components` agree with `reference`: an
    eigenvector is defined up to its sign, and eigh implementations choose differently."""
    dots = np.einsum("ij,ij->i", np.asarray(components, np.float64), np.asarray(reference, np.float64))
    return np.where(dots < 0, -1.0, 1.0)
