"""The reference's covariance PCA run on a GPU with its own kernels -- TEST INFRASTRUCTURE ONLY.

``pca_csr`` restates ``PCA_sparse.fit`` / ``_transform_cupy``
(src/rapids_singlecell/preprocessing/_sparse_pca/_sparse_pca.py:26-95) for a float32 CSR
matrix with torch CUDA tensors in place of CuPy arrays: the covariance comes from the
reference's own kernels (``ref_pca_cov_csr_f32`` in ``oracle/_ref/libharmony_ref.so``:
gram_csr_upper, copy_upper_to_lower, mean_var_minor, cov_from_gram), the eigendecomposition
from cuSOLVER through ``torch.linalg.eigh`` in float32 (the reference calls
``cp.linalg.eigh(covariance, UPLO="U")``), and the transform is the same float32 product
X C^T - mean C^T.  Used by ``tests/golden/make_ref_golden.py`` to write the PCA fixtures.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import ref_harmony as rh


def pca_csr(indptr, indices, data, shape, n_comps, zero_center=True, device="cuda"):
    """(X_pca, components, variance, variance_ratio, mean) as float32 host arrays."""
    import torch

    lib = rh.load()
    n, g = shape
    ip = torch.as_tensor(np.asarray(indptr, np.int32), device=device)
    ix = torch.as_tensor(np.asarray(indices, np.int32), device=device)
    dv = torch.as_tensor(np.asarray(data, np.float32), device=device)
    cov = torch.empty((g, g), dtype=torch.float32, device=device)
    mean = torch.empty(g, dtype=torch.float32, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rh._check(lib.ref_pca_cov_csr_f32(rh._p(ip), rh._p(ix), rh._p(dv), n, g, ctypes.c_longlong(dv.numel()),
                                      0 if zero_center else 1, rh._p(cov), rh._p(mean), st), "pca_cov_csr")
    evals, evecs = torch.linalg.eigh(cov, UPLO="U")
    evals = torch.flip(evals, dims=(0,))
    comps = torch.flip(evecs, dims=(1,)).T[:n_comps].contiguous()
    ratio = evals / evals.sum()
    X = torch.sparse_csr_tensor(ip.long(), ix.long(), dv, size=(n, g)).to_dense()
    X_pca = X @ comps.T
    if zero_center:
        X_pca = X_pca - (mean @ comps.T)[None, :]
    torch.cuda.synchronize()
    return (X_pca.cpu().numpy(), comps.cpu().numpy(), evals[:n_comps].cpu().numpy(),
            ratio[:n_comps].cpu().numpy(), mean.cpu().numpy() if zero_center else None)
