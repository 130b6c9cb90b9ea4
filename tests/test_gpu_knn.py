"""Exact kNN on the GPU through the C ABI against the float64 brute-force oracle.

The kernel ranks candidates with tensor-core (bf16 hi + lo) distances and re-ranks each query's
best candidates with exact float32 distances, so the bar is float32 rounding: the distances of
the k neighbours within 2e-5 relative (+1e-6 absolute) of float64, and every returned neighbour
within that margin of the true k-th distance (queries whose k-th and (k+1)-th distances tie
within it may hold either)."""

import numpy as np
import pytest
import torch

from oracle import knn_oracle as ko
from rapids_singlecell_b200 import neighbors as nb

pytestmark = pytest.mark.gpu


def _check(X, k, metric, queries=None):
    idx, dist = nb.knn_arrays(torch.as_tensor(X, device="cuda"), k, metric=metric,
                              queries=None if queries is None else torch.as_tensor(queries, device="cuda"))
    idx, dist = idx.cpu().numpy(), dist.cpu().numpy().astype(np.float64)
    ridx, rdist = ko.knn(X, k, metric, queries=queries)
    tol = 2e-5 * np.abs(rdist).max() + 1e-6
    assert np.abs(dist - rdist).max() <= tol
    # each returned neighbour is a true k-nearest one (up to the tolerance)
    Q = X if queries is None else queries
    fidx, fdist = ko.knn(X, min(k + 10, X.shape[0]), metric, queries=Q)
    kth = rdist[:, -1]
    sign = -1.0 if metric == "inner_product" else 1.0
    for qi in range(Q.shape[0]):
        got = set(idx[qi].tolist())
        assert len(got) == k
        ok = set(fidx[qi][sign * fdist[qi] <= sign * kth[qi] + tol].tolist())
        assert got <= ok, (qi, got - ok)
    return idx, dist


@pytest.mark.parametrize("metric", ["euclidean", "sqeuclidean", "cosine", "inner_product"])
@pytest.mark.parametrize("n,d,k", [(3000, 50, 15), (1000, 3, 5), (777, 100, 10), (129, 128, 24), (2500, 64, 30),
                                   (300, 20, 56), (64, 7, 1)])
def test_knn_matches_float64_brute_force(metric, n, d, k):
    X = np.random.default_rng(n + d).standard_normal((n, d)).astype(np.float32)
    idx, dist = _check(X, k, metric)
    if metric in ("euclidean", "sqeuclidean"):
        assert np.all(idx[:, 0] == np.arange(n)) and np.all(dist[:, 0] == 0)


def test_knn_on_a_clustered_pca_like_embedding():
    """Cells of a Gaussian mixture in 50 dimensions (nearby points, many near-ties)."""
    from rapids_singlecell_b200.synthetic import make_config

    Z = make_config("C1", seed=4, n_cells=6000)["Z"]
    _check(Z, 15, "euclidean")


def test_queries_other_than_the_data():
    rng = np.random.default_rng(2)
    X = rng.standard_normal((1500, 30)).astype(np.float32)
    Q = rng.standard_normal((333, 30)).astype(np.float32)
    _check(X, 12, "euclidean", queries=Q)


def test_pp_neighbors_surface():
    import pandas as pd

    from rapids_singlecell_b200 import pp
    from rapids_singlecell_b200.synthetic import make_config

    Z = make_config("C1", seed=5, n_cells=2000)["Z"]

    class AData:
        def __init__(self):
            self.X = np.zeros((2000, 60), np.float32)
            self.obsm = {"X_pca_harmony": Z}
            self.obsp, self.uns = {}, {}
            self.var = pd.DataFrame(index=range(60))

    a = AData()
    pp.neighbors(a, n_neighbors=10, use_rep="X_pca_harmony")
    D, C = a.obsp["distances"], a.obsp["connectivities"]
    assert D.shape == (2000, 2000) and D.nnz == 2000 * 10
    assert abs(C - C.T).max() < 1e-6 and C.max() <= 1.0 + 1e-6
    assert a.uns["neighbors"]["params"]["n_neighbors"] == 10
    for method in ("gauss", "jaccard"):
        pp.neighbors(a, n_neighbors=10, use_rep="X_pca_harmony", method=method, key_added=method)
        W = a.obsp[f"{method}_connectivities"]
        assert abs(W - W.T).max() < 1e-6
