"""PCA on the B200: the covariance eigendecomposition of ``rapids_singlecell.pp.pca``.

The reference computes PCA of a sparse matrix (and of a dense one through cuML) from
its covariance: ``_run_covariance_pca`` (src/rapids_singlecell/preprocessing/_pca.py:339-353)
-> ``PCA_sparse`` (preprocessing/_sparse_pca/_sparse_pca.py:26-127).  Here every input,
dense or CSR, takes that route on the engine's kernels (``csrc/hb_pca.cu``):

1. a sparse input is copied dense into HBM (``hb_csr_to_dense``);
2. the Gram matrix X^T X and the column sums on the tensor core (``hb_pca_gram``: float32
   values as bf16 hi + lo parts, float32 accumulation in TMEM, float64 reduction);
3. the covariance X^T X / n - mean mean^T in float64 (``hb_pca_covariance``), or the plain
   Gram for ``zero_center=False`` (the reference's uncentred path);
4. its eigendecomposition (cuSOLVER through ``torch.linalg.eigh`` in float64; the reference
   calls ``cp.linalg.eigh``), reversed to descending order;
5. the projection X C^T - mean C^T on the tensor core (``hb_pca_project``).

``pca_arrays`` is the tensor-level call; ``pp.pca`` mirrors the reference's AnnData surface.
"""

from __future__ import annotations

import ctypes
import warnings
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

_empty = object()


@dataclass
class PcaOutput:
    X_pca: torch.Tensor            # [n, n_comps] float32, on the device
    components: torch.Tensor       # [n_comps, n_genes] float32
    variance: torch.Tensor         # [n_comps] float64 (eigenvalues)
    variance_ratio: torch.Tensor   # [n_comps] float64
    mean: torch.Tensor | None      # [n_genes] float64 (zero_center)


def default_n_comps(n_obs: int, n_vars: int) -> int:
    """50, or min(n_obs, n_vars) - 1 when that is not larger (_pca.py:230-235)."""
    min_dim = min(n_obs, n_vars)
    return min_dim - 1 if 50 >= min_dim else 50


def _p(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _is_sparse(X) -> bool:
    if isinstance(X, torch.Tensor):
        return X.layout == torch.sparse_csr
    try:
        import scipy.sparse as sp

        return sp.issparse(X)
    except ImportError:  # pragma: no cover
        return False


def _csr_parts(X, device):
    """(indptr int64, indices int32, data float32, n_rows, n_cols) on the device of a CSR
    matrix given as scipy.sparse or a torch sparse CSR tensor."""
    if isinstance(X, torch.Tensor):
        n, g = X.shape
        return (X.crow_indices().to(device=device, dtype=torch.int64).contiguous(),
                X.col_indices().to(device=device, dtype=torch.int32).contiguous(),
                X.values().to(device=device, dtype=torch.float32).contiguous(), n, g)
    X = X.tocsr()
    n, g = X.shape
    return (torch.as_tensor(np.asarray(X.indptr, dtype=np.int64), device=device),
            torch.as_tensor(np.asarray(X.indices, dtype=np.int32), device=device),
            torch.as_tensor(np.asarray(X.data, dtype=np.float32), device=device), n, g)


def densify(X, device) -> torch.Tensor:
    """A dense float32 [n, g] CUDA tensor of X (dense array or tensor, or CSR)."""
    lib = _lib.load()
    if _is_sparse(X):
        indptr, indices, data, n, g = _csr_parts(X, device)
        if indices.numel() and bool((torch.bincount(indices.long(), minlength=g) == 0).any()):
            # the reference's check before its covariance path (_sparse_pca/_helper.py:35-48)
            raise ValueError("There are genes with zero expression. Please remove them before running PCA.")
        out = torch.empty((n, g), dtype=torch.float32, device=device)
        err = torch.zeros(1, dtype=torch.int32, device=device)
        _lib.check(lib.hb_csr_to_dense(_p(indptr), _p(indices), _p(data), n, g, _p(out), g, _p(err),
                                       _stream(device)))
        return out
    t = torch.as_tensor(X, device=device)
    if t.dim() != 2:
        raise ValueError("PCA input must be two-dimensional")
    return t.to(torch.float32).contiguous()


def pca_arrays(X, n_comps: int | None = None, *, zero_center: bool = True, device=None) -> PcaOutput:
    """PCA of X (cells x genes; dense, or CSR as scipy.sparse / torch sparse CSR) by the
    covariance eigendecomposition, as ``PCA_sparse.fit_transform`` (_sparse_pca.py:26-127)."""
    lib = _lib.load()
    device = torch.device(device) if device is not None else (
        X.device if isinstance(X, torch.Tensor) and X.is_cuda else torch.device("cuda"))
    Xd = densify(X, device)
    n, g = Xd.shape
    if n < 2 or g < 1:
        raise ValueError(f"PCA needs at least two observations and one variable, got {n} x {g}")
    if n_comps is None:
        n_comps = default_n_comps(n, g)
    if not 1 <= n_comps <= min(g, 256):
        raise ValueError(f"n_comps={n_comps} must be in [1, min(n_vars, 256)]")
    st = _stream(device)
    ws_bytes = lib.hb_pca_gram_workspace_bytes(n, g)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    gram = torch.empty((g, g), dtype=torch.float64, device=device)
    csum = torch.empty(g, dtype=torch.float64, device=device)
    _lib.check(lib.hb_pca_gram(_p(Xd), n, g, g, _p(gram), _p(csum), _p(ws), ws_bytes, st))
    del ws
    cov = torch.empty_like(gram)
    mean = torch.empty(g, dtype=torch.float64, device=device) if zero_center else None
    _lib.check(lib.hb_pca_covariance(_p(gram), _p(csum), n, g, int(bool(zero_center)), _p(cov),
                                     _p(mean) if mean is not None else None, st))
    del gram
    evals, evecs = torch.linalg.eigh(cov, UPLO="U")
    del cov
    evals = torch.flip(evals, dims=(0,))
    comps = torch.flip(evecs, dims=(1,)).T[:n_comps].contiguous()
    ratio = evals / evals.sum()
    comps32 = comps.to(torch.float32).contiguous()
    out = torch.empty((n, n_comps), dtype=torch.float32, device=device)
    pws_bytes = lib.hb_pca_project_workspace_bytes(g, n_comps)
    pws = torch.empty(pws_bytes, dtype=torch.uint8, device=device)
    _lib.check(lib.hb_pca_project(_p(Xd), n, g, g, _p(comps32), n_comps, _p(mean) if mean is not None else None,
                                  _p(out), _p(pws), pws_bytes, st))
    return PcaOutput(X_pca=out, components=comps32, variance=evals[:n_comps].clone(),
                     variance_ratio=ratio[:n_comps].clone(), mean=mean)


def _resolve_mask_var(adata, mask_var, *, use_highly_variable):
    """mask_var / use_highly_variable -> (parameter, boolean mask) as the reference
    (_pca.py:26-68), including its deprecation warning and errors."""
    if use_highly_variable is not None:
        warnings.warn(
            "Argument `use_highly_variable` is deprecated, use `mask_var` instead. "
            'Use mask_var="highly_variable" instead of use_highly_variable=True, '
            "and mask_var=None instead of use_highly_variable=False.",
            FutureWarning,
            stacklevel=3,
        )
        if mask_var is not _empty:
            raise ValueError("Cannot specify both `mask_var` and `use_highly_variable`.")
    var = getattr(adata, "var", None)
    columns = getattr(var, "columns", ())
    if use_highly_variable or (use_highly_variable is None and mask_var is _empty and "highly_variable" in columns):
        mask_var = "highly_variable"
    if mask_var is _empty or mask_var is None:
        return None, None
    if isinstance(mask_var, str):
        return mask_var, np.asarray(var[mask_var].to_numpy(), dtype=bool)
    mask = np.asarray(mask_var)
    n_vars = adata.X.shape[1] if getattr(adata, "X", None) is not None else mask.shape[0]
    if mask.shape != (n_vars,):
        raise ValueError(f"The shape of the mask ({mask.shape}) does not match the number of variables ({n_vars}).")
    return None, mask.astype(bool)


def pp_pca(adata, n_comps: int | None = None, *, layer: str | None = None, zero_center: bool = True,
           svd_solver: str | None = None, random_state: int | None = 0, mask_var=_empty,
           use_highly_variable: bool | None = None, dtype: str = "float32", chunked: bool = False,
           chunk_size: int | None = None, key_added: str | None = None, copy: bool = False, **kwargs):
    """Drop-in for ``rapids_singlecell.pp.pca`` (_pca.py:71-330): writes ``obsm['X_pca']``,
    ``varm['PCs']`` and ``uns['pca']`` (variance, variance_ratio, params), or the
    ``key_added`` names.  Every solver choice (``svd_solver``, ``chunked``) computes the exact
    covariance eigendecomposition, which the reference's solvers approximate or reproduce;
    ``random_state`` therefore has no effect."""
    if use_highly_variable is True and "highly_variable" not in getattr(getattr(adata, "var", None), "keys", lambda: ())():
        raise ValueError(
            "Did not find adata.var['highly_variable']. "
            "Either your data already only consists of highly-variable genes "
            "or consider running `highly_variable_genes` first."
        )
    if copy:
        adata = adata.copy()
    X = adata.layers[layer] if layer is not None else adata.X
    mask_param, mask = _resolve_mask_var(adata, mask_var, use_highly_variable=use_highly_variable)
    if mask is not None:
        X = X[:, mask] if not isinstance(X, torch.Tensor) else X[:, torch.as_tensor(mask, device=X.device)]
    res = pca_arrays(X, n_comps, zero_center=zero_center)
    X_pca = res.X_pca.cpu().numpy()
    if X_pca.dtype != np.dtype(dtype):
        X_pca = X_pca.astype(dtype)
    key_obsm, key_varm, key_uns = ("X_pca", "PCs", "pca") if key_added is None else [key_added] * 3
    adata.obsm[key_obsm] = X_pca
    adata.uns[key_uns] = {
        "params": {"zero_center": zero_center, "use_highly_variable": mask_param == "highly_variable",
                   "mask_var": mask_param, **({"layer": layer} if layer is not None else {})},
        "variance": res.variance.cpu().numpy(),
        "variance_ratio": res.variance_ratio.cpu().numpy(),
    }
    comps = res.components.double().cpu().numpy()
    if mask is not None:
        loadings = np.zeros((mask.shape[0], comps.shape[0]))
        loadings[mask] = comps.T
        adata.varm[key_varm] = loadings
    else:
        adata.varm[key_varm] = comps.T
    return adata if copy else None
