"""The NumPy PCA oracle against outputs of the reference itself, and the host-side logic of
``pp.pca`` (no GPU needed).

``tests/golden/ref_pca_*.npz`` were written by ``tests/golden/make_ref_golden.py`` on a B200 with
the reference's own covariance-PCA kernels (gram_csr_upper, copy_upper_to_lower, mean_var_minor,
cov_from_gram from the reference tree, built into ``oracle/_ref/libharmony_ref.so``) and
cuSOLVER's eigh in float32, as the reference runs for float32 sparse input.  The oracle computes
in float64, so the bars are the reference's float32 rounding.
"""

import json
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import pca_oracle as po

GOLDEN = Path(__file__).resolve().parent / "golden"
TOP = 8  # components with clear eigenvalue gaps (the input is a rank-8 factor model)


def _load(name):
    path = GOLDEN / f"ref_{name}.npz"
    if not path.exists():
        pytest.skip(f"fixture {path.name} not generated (tests/golden/make_ref_golden.py on a GPU)")
    f = np.load(path)
    X = sp.csr_matrix((f["data"], f["indices"], f["indptr"]), shape=tuple(f["shape"]))
    return f, X, json.loads(str(f["params"]))


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["pca_center", "pca_gram"])
def test_pca_oracle_matches_reference_outputs(name):
    f, X, kw = _load(name)
    r = po.pca(X.toarray(), kw["n_comps"], zero_center=kw["zero_center"])
    np.testing.assert_allclose(r.variance, f["variance"], rtol=2e-4)
    np.testing.assert_allclose(r.variance_ratio, f["variance_ratio"], rtol=2e-4)
    s = po.align_signs(r.components, f["components"])
    comps = r.components * s[:, None]
    assert np.abs(comps[:TOP] - f["components"][:TOP]).max() < 5e-4
    assert _rel((r.X_pca * s[None, :])[:, :TOP], f["X_pca"][:, :TOP]) < 2e-4
    if kw["zero_center"]:
        np.testing.assert_allclose(r.mean, f["mean"], rtol=1e-6)


def test_default_n_comps():
    assert po.default_n_comps(1000, 2000) == 50
    assert po.default_n_comps(30, 2000) == 29
    assert po.default_n_comps(1000, 40) == 39


def test_uncentred_covariance_is_the_plain_gram():
    X = np.random.default_rng(0).random((50, 7))
    cov, mean = po.covariance(X, zero_center=False)
    assert mean is None
    np.testing.assert_allclose(cov, X.T @ X)


def test_mask_var_resolution_mirrors_the_reference():
    import pandas as pd

    from rapids_singlecell_b200.pca import _empty, _resolve_mask_var

    class A:
        X = np.zeros((4, 3))
        var = pd.DataFrame({"highly_variable": [True, False, True]})

    assert _resolve_mask_var(A(), _empty, use_highly_variable=None)[0] == "highly_variable"
    p, m = _resolve_mask_var(A(), None, use_highly_variable=None)
    assert p is None and m is None
    p, m = _resolve_mask_var(A(), np.array([True, True, False]), use_highly_variable=None)
    assert p is None and m.tolist() == [True, True, False]
    with pytest.raises(ValueError, match="does not match"):
        _resolve_mask_var(A(), np.array([True, False]), use_highly_variable=None)
    with pytest.warns(FutureWarning), pytest.raises(ValueError, match="Cannot specify both"):
        _resolve_mask_var(A(), "highly_variable", use_highly_variable=True)
