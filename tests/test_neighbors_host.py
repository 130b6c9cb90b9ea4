"""Host-side graph arithmetic of ``pp.neighbors`` (no GPU): the connectivities built from kNN
arrays, run with CPU torch tensors, against dense NumPy restatements of the reference's formulas
(gauss, jaccard) and of the published UMAP fuzzy simplicial set; the distance matrix layout."""

import numpy as np
import pytest
import torch

from oracle import knn_oracle as ko
from rapids_singlecell_b200 import neighbors as nb


@pytest.fixture(scope="module")
def graph():
    X = np.random.default_rng(3).standard_normal((120, 6))
    idx, dist = ko.knn(X, 8)
    return torch.as_tensor(idx), torch.as_tensor(dist, dtype=torch.float32), 120


def test_gauss(graph):
    idx, dist, n = graph
    W = nb.connectivities_gauss(idx, dist.clone(), n).toarray()
    ref = ko.gauss_connectivities(idx.numpy(), dist.numpy(), n)
    np.testing.assert_allclose(W, ref, rtol=1e-5, atol=1e-7)


def test_jaccard(graph):
    idx, _, n = graph
    W = nb.connectivities_jaccard(idx, n, 8).toarray()
    np.testing.assert_allclose(W, ko.jaccard_connectivities(idx.numpy(), n, 8), rtol=1e-6, atol=1e-7)


def test_umap(graph):
    idx, dist, n = graph
    W = nb.connectivities_umap(idx, dist.clone(), n, 8).toarray()
    ref = ko.umap_connectivities(idx.numpy(), dist.numpy(), n, 8)
    np.testing.assert_allclose(W, ref, rtol=1e-4, atol=1e-6)
    assert np.allclose(W, W.T) and W.max() <= 1.0 + 1e-6 and np.all(np.diag(W) == 0)


def test_distance_matrix_and_self_distance(graph):
    idx, dist, n = graph
    d = nb.fix_self_distances(dist.clone() + 1e-3, "euclidean")
    assert bool((d[:, 0] == 0).all())
    D = nb.build_sparse_distances(idx, d, n)
    assert D.shape == (n, n) and D.nnz == n * 8
    np.testing.assert_array_equal(D.indptr, np.arange(0, n * 8 + 1, 8))
    ip = nb.fix_self_distances(dist.clone() + 1.0, "inner_product")
    assert bool((ip[:, 0] != 0).all())


def test_unsupported_metric_is_refused():
    with pytest.raises(NotImplementedError, match="not supported"):
        nb.knn_arrays(np.zeros((4, 2), np.float32), 2, metric="manhattan")
