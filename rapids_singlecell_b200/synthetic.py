"""Seeded Gaussian-mixture embeddings that stand in for PCA tables.

No public dataset is named for the Harmony benchmarks and the reference's own
test datasets are downloads, so every workload here is synthetic.  The draw
order is fixed and documented so that any run can be regenerated exactly:

1. ``rng = numpy.random.default_rng(seed)``
2. type means ``mu = rng.normal(0, mean_scale, (n_types, d))``
3. batch sizes (exact counts from the proportions; remainder to batch 0)
4. batch shift vectors ``rng.normal(0, shift_sd, (B, d))``
5. batch scales ``rng.uniform(lo, hi, B)`` (1.0 when no scale range is given)
6. cell types ``rng.integers(0, n_types, n)``
7. cell batches: ``rng.permutation`` of the repeated batch labels
8. noise ``rng.standard_normal((n, d))``

Cell i is ``scale[b] * (mu[type_i] + noise_i) + shift[b]``, stored float32.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class MixtureSpec:
    n_cells: int
    n_pcs: int
    n_types: int
    n_batches: int
    batch_props: str = "given"      # "given" | "dirichlet" | "zipf"
    props: tuple = ()
    shift_sd: float = 0.5
    scale_range: tuple | None = None
    mean_scale: float = 4.0
    zipf_s: float = 1.2
    min_batch: int = 0


def _batch_counts(spec: MixtureSpec, rng) -> np.ndarray:
    B, n = spec.n_batches, spec.n_cells
    if spec.batch_props == "given":
        p = np.asarray(spec.props, dtype=np.float64)
    elif spec.batch_props == "dirichlet":
        p = rng.dirichlet(np.ones(B))
    elif spec.batch_props == "zipf":
        p = 1.0 / np.arange(1, B + 1, dtype=np.float64) ** spec.zipf_s
    else:
        raise ValueError(spec.batch_props)
    p = p / p.sum()
    counts = np.floor(p * n).astype(np.int64)
    if spec.min_batch:
        counts = np.maximum(counts, spec.min_batch)
    counts[0] += n - counts.sum()
    if counts.min() < 0:
        raise ValueError("batch counts do not fit n_cells")
    return counts


def make_mixture(spec: MixtureSpec, seed: int):
    """Return ``(Z float32 [n, d], cats int32 [n], cell_types int32 [n])``."""
    rng = np.random.default_rng(seed)
    d = spec.n_pcs
    mu = rng.normal(0.0, spec.mean_scale, (spec.n_types, d))
    counts = _batch_counts(spec, rng)
    shift = rng.normal(0.0, spec.shift_sd, (spec.n_batches, d))
    if spec.scale_range is not None:
        scale = rng.uniform(spec.scale_range[0], spec.scale_range[1], spec.n_batches)
    else:
        scale = np.ones(spec.n_batches)
    types = rng.integers(0, spec.n_types, spec.n_cells)
    cats = rng.permutation(np.repeat(np.arange(spec.n_batches), counts))
    noise = rng.standard_normal((spec.n_cells, d))
    Z = scale[cats][:, None] * (mu[types] + noise) + shift[cats]
    return Z.astype(np.float32), cats.astype(np.int32), types.astype(np.int32)


def initial_centroids(Z: np.ndarray, n_clusters: int, seed: int) -> np.ndarray:
    """Seeded initial centroids: ``n_clusters`` distinct cells of the L2-normalised
    embedding, chosen by ``default_rng(seed).choice(n, K, replace=False)``."""
    rng = np.random.default_rng(seed)
    idx = rng.choice(Z.shape[0], size=n_clusters, replace=False)
    Y = Z[idx].astype(np.float64)
    Y /= np.maximum(np.linalg.norm(Y, axis=1, keepdims=True), 1e-12)
    return Y.astype(np.float32)


# Benchmark configurations (cells x PCs, mixture, clustering parameters).
CONFIGS = {
    # 20k x 50, 10 types, 3 batches at 50/30/20 %, shift N(0, 0.5^2); K=100
    "C1": dict(spec=MixtureSpec(20_000, 50, 10, 3, "given", (0.5, 0.3, 0.2), 0.5),
               n_clusters=100, max_iter_harmony=10, max_iter_clustering=20),
    # 500k x 50, 30 types, 8 batches Dirichlet(1), shift N(0, 0.5^2), scale U(0.8, 1.2); K=100
    "C2": dict(spec=MixtureSpec(500_000, 50, 30, 8, "dirichlet", (), 0.5, (0.8, 1.2)),
               n_clusters=100, max_iter_harmony=10, max_iter_clustering=20),
    # 2M x 100, 50 types, 32 batches Zipf(1.2) sizes (>= 500 cells), shift N(0, 0.7^2); K=200
    "C3": dict(spec=MixtureSpec(2_000_000, 100, 50, 32, "zipf", (), 0.7, None, zipf_s=1.2,
                                min_batch=500),
               n_clusters=200, max_iter_harmony=10, max_iter_clustering=20),
}


def make_config(name: str, seed: int = 0, n_cells: int | None = None):
    """Materialise a named configuration, optionally with fewer cells (same mixture)."""
    cfg = dict(CONFIGS[name])
    spec = cfg.pop("spec")
    if n_cells is not None:
        spec = MixtureSpec(**{**spec.__dict__, "n_cells": n_cells})
    Z, cats, types = make_mixture(spec, seed)
    Y0 = initial_centroids(Z, cfg["n_clusters"], seed + 1)
    return dict(Z=Z, cats=cats, types=types, Y0=Y0, n_batches=spec.n_batches, **cfg)
