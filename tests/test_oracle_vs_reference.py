"""The NumPy oracle against outputs of the reference itself (no GPU needed).

The fixtures ``tests/golden/ref_*.npz`` were written by ``tests/golden/make_ref_golden.py``,
which ran rapids_singlecell's own Harmony kernels (compiled from the reference tree into
``oracle/_ref/libharmony_ref.so``) in the launch sequence of its clustering loop and batched
correction, on a B200, with injected initial centroids.  Matching them pins the oracle --
and through it every engine parity test -- to the reference's arithmetic, iteration counts and
convergence decisions.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from oracle import harmony_oracle as ho

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ["h2_f64", "h2_f32", "h1_tau_f64", "k2_state_f64"]


def _load(name):
    path = GOLDEN / f"ref_{name}.npz"
    if not path.exists():
        pytest.skip(f"fixture {path.name} not generated (tests/golden/make_ref_golden.py on a GPU)")
    f = np.load(path)
    params = json.loads(str(f["params"]))
    return f, params


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _run_oracle(f, params):
    p = dict(params)
    dtype = np.dtype(p.pop("dtype"))
    K = p.pop("n_clusters")
    B = p.pop("n_batches")
    return ho.harmonize(f["Z"], f["cats"], B, f["Y0"], n_clusters=K, dtype=dtype, **p), dtype


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_outputs(name):
    f, params = _load(name)
    res, dtype = _run_oracle(f, params)
    # same loop decisions: outer iterations, k-means iterations per outer, convergence flag
    assert res.n_outer == int(f["n_outer"])
    assert [len(k) for k in res.kmeans_objectives] == f["kmeans_iters"].tolist()
    assert res.converged == bool(f["converged"])
    f64 = dtype == np.float64
    # float64: both sides round the same operations; float32: the reference accumulates its
    # objective sums in float32 (the oracle in float64) and sums in a different order
    tol_z, tol_obj = (1e-10, 1e-11) if f64 else (1e-4, 2e-5)
    assert _rel(res.Z_hat, f["Z_hat"]) < tol_z
    np.testing.assert_allclose(res.objectives_harmony, f["objectives"], rtol=tol_obj)
    km = np.concatenate([np.asarray(k, np.float64) for k in res.kmeans_objectives])
    np.testing.assert_allclose(km, f["kmeans_objectives"], rtol=tol_obj)


def test_oracle_state_matches_reference_after_two_iterations():
    """Component pin of the clustering loop: R, O and E after one outer iteration of two
    fixed k-means iterations (no early stop), float64."""
    f, params = _load("k2_state_f64")
    res, _ = _run_oracle(f, params)
    assert _rel(res.R, f["R"]) < 1e-11
    assert _rel(res.O, f["O"]) < 1e-11
    assert _rel(res.E, f["E"]) < 1e-11


def test_fixtures_cover_the_flavours():
    """The fixture set covers harmony2 and harmony1, both dtypes, an early stop of the k-means
    loop and a batch of fewer than ten cells."""
    seen = {}
    for name in CASES:
        f, params = _load(name)
        seen[name] = (params, f)
    assert seen["h1_tau_f64"][0]["stabilized_penalty"] is False
    assert np.bincount(seen["h1_tau_f64"][1]["cats"]).min() < 10
    iters = seen["h2_f64"][1]["kmeans_iters"]
    assert iters.min() < seen["h2_f64"][0]["max_iter_clustering"]  # the window-3 test stopped a loop
