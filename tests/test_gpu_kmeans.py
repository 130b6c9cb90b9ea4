"""The engine's seeded k-means initialisation (hb_kmeans_init) against its oracle:
the k-means++ seeding bit for bit, the Lloyd iterations by inertia (the device
assigns with bf16 operands on the tensor core, the oracle in float64)."""

import ctypes

import numpy as np
import pandas as pd
import pytest
import torch

from oracle import kmeans_oracle as ko
from rapids_singlecell_b200.harmony import harmonize, kmeans_centroids
from rapids_singlecell_b200.synthetic import make_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_cells,K", [(20_000, 100), (3_000, 100)])  # sampled / every cell
def test_seeding_matches_oracle_bit_for_bit(n_cells, K):
    cfg = make_config("C1", seed=4, n_cells=n_cells)
    Z = cfg["Z"]
    Y, iters = kmeans_centroids(torch.as_tensor(Z, device="cuda"), K, 11, max_iter=0, return_iters=True)
    assert iters == 0
    ref = ko.seed_centres(Z, K, 11)
    assert np.array_equal(Y.cpu().numpy(), ref)


@pytest.mark.parametrize("cfg_name,n_cells,K", [("C1", 20_000, 100), ("C2", 60_000, 100), ("C3", 30_000, 200)])
def test_lloyd_reaches_the_oracle_inertia(cfg_name, n_cells, K):
    cfg = make_config(cfg_name, seed=2, n_cells=n_cells)
    Z = cfg["Z"]
    Y, iters = kmeans_centroids(torch.as_tensor(Z, device="cuda"), K, 3, return_iters=True)
    Y = Y.cpu().numpy()
    Y0 = ko.seed_centres(Z, K, 3)
    Yr, it_r = ko.lloyd(Z, Y0, 25, 1e-4)
    i_gpu, i_ref, i_0 = ko.inertia(Z, Y), ko.inertia(Z, Yr), ko.inertia(Z, Y0)
    print(f"{cfg_name}: inertia seeds {i_0:.2f}, device {i_gpu:.2f} ({iters} it), oracle {i_ref:.2f} ({it_r} it)")
    assert np.isfinite(Y).all()
    assert i_gpu < i_0
    assert abs(i_gpu - i_ref) / i_ref < 5e-3


def test_harmonize_starts_from_the_kmeans_centres():
    cfg = make_config("C1", seed=6, n_cells=8_000)
    kw = dict(n_clusters=50, max_iter_harmony=2, max_iter_clustering=5, random_state=9)
    labels = pd.Categorical.from_codes(cfg["cats"], categories=["a", "b", "c"])
    Z = torch.as_tensor(cfg["Z"], device="cuda")
    Y0 = kmeans_centroids(Z, 50, 9)
    a = harmonize(Z, labels, None, precision="fp32", **kw)
    b = harmonize(Z, labels, None, init_centroids=Y0, precision="fp32", **kw)
    rel = (a - b).abs().max().item() / b.abs().max().item()
    assert rel < 1e-4


def test_kmeans_rejects_sizes_out_of_range():
    from rapids_singlecell_b200 import _lib

    lib = _lib.load()
    X = torch.zeros((10, 4), device="cuda")
    Y = torch.empty((20, 4), device="cuda")
    ws = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    st = lib.hb_kmeans_init(X.data_ptr(), 10, 4, 20, 5, 1e-4, 0, Y.data_ptr(), None, ws.data_ptr(), 1 << 20, None)
    assert st == _lib.HB_ERR_INVALID  # more clusters than cells


@pytest.mark.parametrize("n,d,K", [(1000, 5, 7), (2500, 128, 256), (129, 64, 3), (4100, 33, 129),
                                   (3000, 200, 100), (700, 256, 128), (5000, 129, 20)])
def test_odd_shapes(n, d, K):
    """Few and many PCs and clusters, a last tile of one cell, clusters just past a 64-block:
    the seeding bit for bit, and Lloyd within the oracle's inertia."""
    from rapids_singlecell_b200.synthetic import MixtureSpec, make_mixture

    Z, _, _ = make_mixture(MixtureSpec(n, d, 5, 2, "given", (0.6, 0.4), 0.5), 40 + d)
    X = torch.as_tensor(Z, device="cuda")
    Y0 = kmeans_centroids(X, K, 5, max_iter=0).cpu().numpy()
    assert np.array_equal(Y0, ko.seed_centres(Z, K, 5))
    Y = kmeans_centroids(X, K, 5).cpu().numpy()
    Yr, _ = ko.lloyd(Z, ko.seed_centres(Z, K, 5), 25, 1e-4)
    i_gpu, i_ref = ko.inertia(Z, Y), ko.inertia(Z, Yr)
    assert np.isfinite(Y).all() and i_gpu <= ko.inertia(Z, Y0)
    assert abs(i_gpu - i_ref) / max(i_ref, 1e-9) < 1e-2
