"""Pin the CPU oracle against the analytical known-answer cases of the
reference's own tests (tests/test_harmony.py, tests/test_harmony_kernels.py)."""

import numpy as np
import pytest

from oracle import harmony_oracle as ho

SENT = ho.SUPPRESS_PENALTY


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_lambda_kb_pruning(dtype):
    # tests/test_harmony.py:342-382
    N_b = np.array([0, 100, 1, 50], dtype=dtype)
    O = np.array([[0, 0, 0], [30, 40, 30], [0, 0, 1], [20, 15, 15]], dtype=dtype)
    E = np.ones((4, 3), dtype=dtype) * 10
    r = ho.compute_lambda_kb(E, O, N_b, alpha=0.2, threshold=1e-5, ridge_lambda=1.0,
                             dynamic_lambda=True)
    assert np.all(r[0] == dtype(SENT))
    np.testing.assert_allclose(r[1], np.full(3, 0.2 * 10, dtype=dtype), rtol=1e-6)
    assert r[2, 0] == dtype(SENT) and r[2, 1] == dtype(SENT)
    np.testing.assert_allclose(r[2, 2], dtype(0.2 * 10), rtol=1e-6)
    np.testing.assert_allclose(r[3], np.full(3, 0.2 * 10, dtype=dtype), rtol=1e-6)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_lambda_kb_dynamic_false(dtype):
    # tests/test_harmony.py:385-402
    E = np.ones((3, 5), dtype=dtype)
    r = ho.compute_lambda_kb(E, np.ones_like(E), np.ones(3, dtype=dtype), alpha=0.5,
                             threshold=1e-5, ridge_lambda=1.0, dynamic_lambda=False)
    np.testing.assert_array_equal(r, np.full_like(E, 1.0))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_lambda_kb_fixed_ridge_zero(dtype):
    # tests/test_harmony.py:405-425
    E = np.array([[5.0, 0.0]], dtype=dtype)
    O = np.array([[10.0, 0.0]], dtype=dtype)
    r = ho.compute_lambda_kb(E, O, np.array([100.0], dtype=dtype), alpha=0.2, threshold=None,
                             ridge_lambda=0.0, dynamic_lambda=False)
    assert r[0, 0] == dtype(0.0)
    assert r[0, 1] == dtype(SENT)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_lambda_kb_zero_denom(dtype):
    # tests/test_harmony.py:428-450
    E = np.array([[0.0, 5.0]], dtype=dtype)
    O = np.array([[0.0, 10.0]], dtype=dtype)
    r = ho.compute_lambda_kb(E, O, np.array([100.0], dtype=dtype), alpha=0.2, threshold=None,
                             ridge_lambda=1.0, dynamic_lambda=True)
    assert r[0, 0] == dtype(SENT)
    np.testing.assert_allclose(r[0, 1], dtype(1.0), rtol=1e-6)


def _inv_reference_formula(O_col, lam_col, dtype):
    # tests/test_harmony_kernels.py:355-378 (formula restated)
    f = dtype(1) / (O_col + lam_col)
    P = -f * O_col
    c = O_col.sum() - (f * O_col * O_col).sum()
    ci = dtype(1) / c
    nb1 = len(O_col) + 1
    inv = np.empty((nb1, nb1), dtype=dtype)
    inv[0, 0] = ci
    inv[0, 1:] = ci * P
    inv[1:, 0] = P * ci
    inv[1:, 1:] = np.outer(P, P) * ci + np.diag(f)
    return inv


@pytest.mark.parametrize("n_batches", [5, 50, 200])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_arrowhead_inverse(n_batches, dtype):
    # tests/test_harmony_kernels.py:381-409: formula, sentinel included, and the
    # dense inverse of the aggregated matrix it replaces
    rng = np.random.default_rng(42)
    O = (rng.random((n_batches, 10)) * 100).astype(dtype)
    lam = (rng.random((n_batches, 10)) * 5 + 0.1).astype(dtype)
    lam[0, 0] = dtype(1e30)
    for k in range(3):
        got = ho.arrowhead_inverse(O[:, k], lam[:, k])
        exp = _inv_reference_formula(O[:, k], lam[:, k], dtype)
        atol = 1e-6 if dtype == np.float32 else 1e-12
        np.testing.assert_allclose(got, exp, atol=atol, rtol=1e-5)
        if dtype == np.float64:
            A = np.zeros((n_batches + 1, n_batches + 1))
            A[0, 0] = O[:, k].sum()
            A[0, 1:] = A[1:, 0] = O[:, k]
            A[1:, 1:] = np.diag(O[:, k] + lam[:, k])
            np.testing.assert_allclose(got @ A, np.eye(n_batches + 1), atol=1e-8)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_arrowhead_inverse_absent_batch(dtype):
    # tests/test_harmony_kernels.py:448-484
    rng = np.random.default_rng(99)
    O = (rng.random((5, 10)) * 100).astype(dtype)
    lam = (rng.random((5, 10)) * 2 + 0.1).astype(dtype)
    O[0, 0] = 0
    lam[0, 0] = dtype(1e30)
    O[3, 2] = 0
    lam[3, 2] = dtype(1e30)
    for k in (0, 2):
        inv = ho.arrowhead_inverse(O[:, k], lam[:, k])
        assert np.all(np.isfinite(inv))


@pytest.mark.parametrize("stabilized", [True, False])
def test_penalty_formula(stabilized):
    # tests/test_harmony_kernels.py:92-121,416-445 (absent batch: O=0 stays finite)
    rng = np.random.default_rng(123)
    E = rng.random((4, 10)) * 10
    O = rng.random((4, 10)) * 10
    O[0, 0] = 0
    th = rng.random(4) * 2 + 0.5
    pen = ho.penalty(E, O, th, stabilized)
    denom = (O + E + 1) if stabilized else (O + 1)
    np.testing.assert_allclose(pen, ((E + 1) / denom) ** th[:, None], rtol=1e-12)
    assert np.all(np.isfinite(pen))


def test_l2_normalize_zero_row():
    # tests/test_harmony_kernels.py:72-86
    X = np.zeros((3, 10))
    X[1] = 1.0
    Y = ho.l2_normalize(X)
    assert not np.isnan(Y).any()
    np.testing.assert_array_equal(Y[0], 0)
    np.testing.assert_allclose(np.linalg.norm(Y[1]), 1.0)


@pytest.mark.parametrize("stabilized", [True, False])
def test_objective_formula(stabilized):
    # tests/test_harmony_kernels.py:296-349
    rng = np.random.default_rng(42)
    R = rng.random((500, 20)) + 0.01
    S = rng.random((500, 20))
    O = rng.random((3, 20)) * 10 + 0.1
    E = rng.random((3, 20)) * 10 + 0.1
    th = rng.random(3) * 2
    got = ho.objective(R, S, O, E, th, 0.1, stabilized)
    km = np.sum(R * 2 * (1 - S))
    Rn = R / R.sum(1, keepdims=True)
    ent = 0.1 * np.sum(Rn * np.log(Rn + 1e-12))
    num = (O + E + 1) if stabilized else (O + 1)
    div = 0.1 * np.sum(th[:, None] * O * np.log(num / (E + 1)))
    np.testing.assert_allclose(got, km + ent + div, rtol=1e-10)


def test_scatter_add_integers():
    # tests/test_harmony.py:262-300 (integer-valued rows: exact)
    rng = np.random.default_rng(42)
    X = rng.integers(1, 10, size=(1000, 20)).astype(np.float32)
    cats = rng.integers(0, 3, size=1000)
    exp = np.zeros((3, 20), dtype=np.float32)
    for i in range(1000):
        exp[cats[i]] += X[i]
    np.testing.assert_array_equal(ho.scatter_rows_by_cat(X, cats, 3), exp)


def test_pcg_keys_bijective_and_reference_values():
    # keys are a bijection of the cell index (no ties), computed mod 2^32
    k = ho.pcg_keys(1 << 16, 12345)
    assert len(np.unique(k)) == 1 << 16
    # scalar restatement of kernels_clustering.cuh:106-117
    def pcg(i, seed):
        st = (i ^ seed) & 0xFFFFFFFF
        st = (st * 747796405 + 2891336453) & 0xFFFFFFFF
        w = (((st >> ((st >> 28) + 4)) ^ st) * 277803737) & 0xFFFFFFFF
        return (w >> 22) ^ w
    for i in (0, 1, 7, 999, 65535):
        assert int(k[i]) == pcg(i, 12345)


def test_block_permutation_stable():
    n = 5000
    idx = ho.block_permutation(n, 77)
    assert sorted(idx.tolist()) == list(range(n))
    keys = ho.pcg_keys(n, 77)
    assert np.all(np.diff(keys[idx].astype(np.int64)) > 0)


def test_correction_batched_matches_original():
    # the closed-form batched correction equals the dense-inverse one
    # (the reference's test_harmony_integrate_algos compares its methods)
    rng = np.random.default_rng(5)
    n, d, K, B = 600, 7, 5, 3
    X = rng.normal(size=(n, d))
    R = rng.random((n, K))
    R /= R.sum(1, keepdims=True)
    cats = rng.integers(0, B, n)
    O = ho.scatter_rows_by_cat(R, cats, B)
    E = (np.bincount(cats, minlength=B) / n)[:, None] * R.sum(0)[None, :]
    N_b = np.bincount(cats, minlength=B).astype(float)
    lam = ho.compute_lambda_kb(E, O, N_b, alpha=0.2, threshold=1e-5, ridge_lambda=1.0,
                               dynamic_lambda=True)
    a = ho.correction_batched(X, R, O, lam, cats, B)
    b = ho.correction_original(X, R, lam, cats, B)
    np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9)


def test_oracle_float32_tracks_float64():
    from rapids_singlecell_b200.synthetic import make_config
    cfg = make_config("C1", seed=3, n_cells=3000)
    kw = dict(n_clusters=30, max_iter_harmony=3, max_iter_clustering=6)
    r64 = ho.harmonize(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"][:30], dtype=np.float64, **kw)
    r32 = ho.harmonize(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"][:30], dtype=np.float32, **kw)
    err = np.abs(r32.Z_hat - r64.Z_hat).max() / np.abs(r64.Z_hat).max()
    assert err < 1e-4
