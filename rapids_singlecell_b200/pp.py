"""``harmony_integrate``: the drop-in for ``rapids_singlecell.pp.harmony_integrate``.

Same signature and defaults as the reference
(src/rapids_singlecell/preprocessing/_harmony_integrate.py:15-250), the same
flavor resolution, warnings and exception types; the data path is this
package's B200 engine.  ``adata`` is anything with an ``obsm`` mapping and an
``obs`` DataFrame (an ``anndata.AnnData`` works).  Extra keyword arguments:
``init_centroids`` (fixed starting centroids), ``precision`` ("fp32", "fp64",
"bf16", "fp16"; default follows ``dtype``), and the harmonypy-style aliases
``nclust`` (= n_clusters), ``lamb`` (= ridge_lambda), ``block_size``
(= block_proportion), ``max_iter_kmeans`` (= max_iter_clustering).
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from .harmony import harmonize


def harmony_integrate(
    adata,
    key,
    *,
    basis: str = "X_pca",
    adjusted_basis: str = "X_pca_harmony",
    dtype=np.float64,
    flavor: str = "harmony2",
    n_clusters: int | None = None,
    max_iter_harmony: int = 10,
    max_iter_clustering: int = 200,
    tol_harmony: float = 1e-4,
    tol_clustering: float = 1e-5,
    sigma: float = 0.1,
    theta=2.0,
    tau: int = 0,
    ridge_lambda: float = 1.0,
    alpha: float = 0.2,
    batch_prune_threshold: float | None = 1e-5,
    correction_method: str | None = None,
    colsum_algo: str | None = None,
    block_proportion: float = 0.05,
    random_state: int = 0,
    verbose: bool = False,
    init_centroids=None,
    precision: str | None = None,
    autotune=False,
    nclust: int | None = None,
    lamb: float | None = None,
    block_size: float | None = None,
    max_iter_kmeans: int | None = None,
) -> None:
    """Integrate experiments with Harmony; writes ``adata.obsm[adjusted_basis]``.

    ``precision`` and ``autotune`` are this engine's own options (see ``harmonize``); every
    other argument is the reference's (_harmony_integrate.py:15-250)."""
    if nclust is not None:
        n_clusters = nclust
    if lamb is not None:
        ridge_lambda = lamb
    if block_size is not None:
        block_proportion = block_size
    if max_iter_kmeans is not None:
        max_iter_clustering = max_iter_kmeans

    if flavor not in {"harmony1", "harmony2"}:
        raise ValueError(f"flavor must be 'harmony1' or 'harmony2', got {flavor!r}.")
    stabilized_penalty = flavor == "harmony2"
    dynamic_lambda = flavor == "harmony2"
    if flavor == "harmony2" and ridge_lambda != 1.0:
        warnings.warn(
            "ridge_lambda is ignored when flavor='harmony2'; "
            "use alpha to control regularization strength.",
            UserWarning,
            stacklevel=2,
        )
    if flavor == "harmony1":
        if alpha != 0.2:
            warnings.warn("alpha is ignored when flavor='harmony1'; use ridge_lambda instead.",
                          UserWarning, stacklevel=2)
        if batch_prune_threshold != 1e-5:
            warnings.warn("batch_prune_threshold is ignored when flavor='harmony1'.",
                          UserWarning, stacklevel=2)

    if basis not in adata.obsm:
        raise ValueError(
            f"The specified basis '{basis}' is not available in adata.obsm. "
            f"Available bases: {list(adata.obsm.keys())}"
        )
    input_data = adata.obsm[basis]
    tdtype = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    try:
        if isinstance(input_data, torch.Tensor):
            X = input_data.to(device="cuda", dtype=tdtype).contiguous()
        else:
            try:
                arr = np.ascontiguousarray(np.asarray(input_data, dtype=dtype))
            except Exception as e:  # noqa: BLE001
                raise TypeError(
                    f"Could not convert input of type {type(input_data).__name__} to an array: {e}"
                ) from e
            try:
                X = torch.as_tensor(arr, device="cuda")
            except torch.cuda.OutOfMemoryError as e:
                raise MemoryError(
                    "Not enough GPU memory to allocate array. "
                    "Try reducing the dataset size or using a GPU with more memory."
                ) from e
        if torch.isnan(X).any():
            raise ValueError(
                "Input data contains NaN values. Please handle these before running harmony_integrate."
            )
    except Exception as e:  # noqa: BLE001
        raise RuntimeError(f"Error preparing data for Harmony: {str(e)}") from e

    Z_hat = harmonize(
        X, adata.obs, key,
        n_clusters=n_clusters, max_iter_harmony=max_iter_harmony,
        max_iter_clustering=max_iter_clustering, tol_harmony=tol_harmony,
        tol_clustering=tol_clustering, ridge_lambda=ridge_lambda, sigma=sigma,
        block_proportion=block_proportion, theta=theta, tau=tau,
        correction_method=correction_method, colsum_algo=colsum_algo,
        random_state=random_state, stabilized_penalty=stabilized_penalty,
        dynamic_lambda=dynamic_lambda, alpha=alpha,
        batch_prune_threshold=batch_prune_threshold, verbose=verbose,
        init_centroids=init_centroids, precision=precision, autotune=autotune,
    )
    adata.obsm[adjusted_basis] = Z_hat.cpu().numpy()


from .pca import pp_pca as pca  # noqa: E402  (``pp.pca``, the drop-in for rapids_singlecell.pp.pca)
from .neighbors import pp_neighbors as neighbors  # noqa: E402  (``pp.neighbors``, the drop-in for rapids_singlecell.pp.neighbors)
