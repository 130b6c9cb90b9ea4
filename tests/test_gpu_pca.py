"""PCA on the GPU through the C ABI: the Gram, covariance and projection kernels against the
float64 oracle, and against the reference's own kernels (the committed fixtures).

Bars: Gram entries and column sums within 2e-5 relative of float64; eigenvalues within 1e-4
relative (plus 1e-6 of the largest, the float32 accumulation floor) and the components / scores of the leading, well-separated components within 1e-4 of
the float64 oracle (signs aligned: an eigenvector's sign is arbitrary); within the reference's
float32 rounding (2e-3) of its fixtures.
"""

import ctypes
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import pca_oracle as po
from rapids_singlecell_b200 import _lib
from rapids_singlecell_b200.pca import pca_arrays
from tests._gpu import lib, ptr, stream

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _low_rank(n, g, rank=6, seed=0, noise=0.05):
    rng = np.random.default_rng(seed)
    F = rng.standard_normal((n, rank)) * np.linspace(3.0, 1.0, rank)
    L = rng.standard_normal((rank, g))
    return (F @ L + noise * rng.standard_normal((n, g)) + rng.uniform(0, 2, g)).astype(np.float32)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def _check_vs_oracle(res, X, n_comps, zero_center, top, tol=1e-4):
    r = po.pca(X, n_comps, zero_center=zero_center)
    # eigenvalues: float32 accumulation of the Gram leaves ~2e-7 of the largest eigenvalue
    np.testing.assert_allclose(res.variance.cpu().numpy()[:top], r.variance[:top], rtol=1e-4,
                               atol=1e-6 * r.variance[0])
    comps = res.components.double().cpu().numpy()
    s = po.align_signs(comps, r.components)
    assert np.abs(comps[:top] * s[:top, None] - r.components[:top]).max() < tol
    assert _rel(res.X_pca.double().cpu().numpy()[:, :top] * s[None, :top], r.X_pca[:, :top]) < tol


@pytest.mark.parametrize("n,g", [(5000, 300), (2000, 50), (700, 129), (130, 257), (20_000, 1000)])
def test_gram_and_column_sums(n, g):
    X = np.random.default_rng(n + g).random((n, g), dtype=np.float32) * 3
    Xt = torch.as_tensor(X, device="cuda")
    ws_bytes = lib().hb_pca_gram_workspace_bytes(n, g)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    G = torch.empty((g, g), dtype=torch.float64, device="cuda")
    cs = torch.empty(g, dtype=torch.float64, device="cuda")
    _lib.check(lib().hb_pca_gram(ptr(Xt), n, g, g, ptr(G), ptr(cs), ptr(ws), ws_bytes, stream()))
    X64 = X.astype(np.float64)
    ref = X64.T @ X64
    G = G.cpu().numpy()
    assert np.array_equal(G, G.T)
    assert np.abs(G - ref).max() / np.abs(ref).max() < 2e-5
    np.testing.assert_allclose(cs.cpu().numpy(), X64.sum(0), rtol=1e-9)


@pytest.mark.parametrize("n,g,k", [(4000, 200, 10), (1500, 64, 5), (777, 130, 7), (3000, 513, 20)])
@pytest.mark.parametrize("zero_center", [True, False])
def test_dense_pca_against_float64_oracle(n, g, k, zero_center):
    X = _low_rank(n, g, seed=g)
    res = pca_arrays(torch.as_tensor(X, device="cuda"), k, zero_center=zero_center)
    assert res.X_pca.shape == (n, k) and res.components.shape == (k, g)
    _check_vs_oracle(res, X, k, zero_center, top=5)


@pytest.mark.parametrize("name", ["pca_center", "pca_gram"])
def test_sparse_pca_against_the_reference_fixture_and_the_oracle(name):
    path = GOLDEN / f"ref_{name}.npz"
    if not path.exists():
        pytest.skip("fixture not generated")
    f = np.load(path)
    kw = json.loads(str(f["params"]))
    X = sp.csr_matrix((f["data"], f["indices"], f["indptr"]), shape=tuple(f["shape"]))
    res = pca_arrays(X, kw["n_comps"], zero_center=kw["zero_center"])
    _check_vs_oracle(res, X.toarray(), kw["n_comps"], kw["zero_center"], top=8)
    comps = res.components.double().cpu().numpy()
    s = po.align_signs(comps, f["components"])
    assert np.abs(comps[:8] * s[:8, None] - f["components"][:8]).max() < 2e-3
    assert _rel(res.X_pca.double().cpu().numpy()[:, :8] * s[None, :8], f["X_pca"][:, :8]) < 2e-3
    np.testing.assert_allclose(res.variance.cpu().numpy(), f["variance"], rtol=2e-4)


def test_torch_sparse_csr_input_equals_dense_input():
    X = _low_rank(1200, 90, seed=3)
    X[X < 1.0] = 0.0
    dense = pca_arrays(torch.as_tensor(X, device="cuda"), 6)
    csr = pca_arrays(torch.as_tensor(X, device="cuda").to_sparse_csr(), 6)
    assert torch.equal(dense.variance, csr.variance)
    assert torch.equal(dense.X_pca, csr.X_pca)


def test_sparse_input_with_an_unexpressed_gene_is_rejected():
    X = sp.random(500, 40, density=0.2, format="csr", random_state=1, dtype=np.float32)
    X = X[:, np.asarray((X != 0).sum(0)).ravel() > 0].tocsr()
    X = sp.hstack([X, sp.csr_matrix((500, 1), dtype=np.float32)]).tocsr()
    with pytest.raises(ValueError, match="genes with zero expression"):
        pca_arrays(X, 5)


def test_csr_column_index_out_of_range_is_reported():
    indptr = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    indices = torch.tensor([0, 7], dtype=torch.int32, device="cuda")
    data = torch.ones(2, dtype=torch.float32, device="cuda")
    out = torch.empty((2, 4), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib().hb_csr_to_dense(ptr(indptr), ptr(indices), ptr(data), 2, 4, ptr(out), 4, ptr(err), stream())
    assert st == _lib.HB_ERR_INVALID and b"column index" in lib().hb_last_error()


def test_pp_pca_surface_writes_obsm_varm_uns():
    import pandas as pd

    from rapids_singlecell_b200 import pp

    X = _low_rank(900, 60, seed=9)
    mask = np.ones(60, dtype=bool)
    mask[::7] = False

    class AData:
        def __init__(self):
            self.X = X
            self.obsm, self.varm, self.uns, self.layers = {}, {}, {}, {}
            self.var = pd.DataFrame({"highly_variable": mask})

    a = AData()
    pp.pca(a, n_comps=8)
    assert a.obsm["X_pca"].shape == (900, 8) and a.obsm["X_pca"].dtype == np.float32
    assert a.varm["PCs"].shape == (60, 8)
    assert np.all(a.varm["PCs"][~mask] == 0)  # genes outside the mask get zero loadings
    assert a.uns["pca"]["params"]["mask_var"] == "highly_variable"
    r = po.pca(X[:, mask], 8)
    np.testing.assert_allclose(a.uns["pca"]["variance"][:5], r.variance[:5], rtol=1e-5)
    pp.pca(a, n_comps=4, mask_var=None, key_added="pca_all")
    assert a.obsm["pca_all"].shape == (900, 4) and a.varm["pca_all"].shape == (60, 4)
