"""Kernel-level parity through the C ABI (mirrors the reference's
tests/test_harmony_kernels.py, with the oracle as the checker)."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import harmony_oracle as ho
from rapids_singlecell_b200 import _lib
from tests._gpu import dev, lib, ptr, rel_maxabs, stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,code", [(np.float32, _lib.HB_FP32), (np.float64, _lib.HB_FP64)])
@pytest.mark.parametrize("rows,cols", [(100, 50), (1, 20), (500, 3), (4097, 100)])
def test_l2_normalize(dtype, code, rows, cols):
    src = np.random.default_rng(42).standard_normal((rows, cols)).astype(dtype)
    s = dev(src)
    d = torch.empty_like(s)
    _lib.check(lib().hb_l2_normalize(ptr(s), ptr(d), rows, cols, code, stream()))
    torch.cuda.synchronize()
    atol = 1e-6 if dtype == np.float32 else 1e-12
    np.testing.assert_allclose(d.cpu().numpy(), ho.l2_normalize(src), atol=atol, rtol=1e-5)


def test_l2_normalize_zero_row():
    src = np.zeros((3, 10), dtype=np.float32)
    src[1] = 1
    s = dev(src)
    d = torch.empty_like(s)
    _lib.check(lib().hb_l2_normalize(ptr(s), ptr(d), 3, 10, _lib.HB_FP32, stream()))
    out = d.cpu().numpy()
    assert not np.isnan(out).any()
    np.testing.assert_array_equal(out[0], 0)
    np.testing.assert_array_equal(out[2], 0)


@pytest.mark.parametrize("n,bs", [(20_000, 1000), (1000, 50), (1003, 50), (777, 777), (100_000, 5000),
                                  (2_000_000, 100_000), (50, 1), (4099, 2048)])
@pytest.mark.parametrize("B", [0, 3, 32])
def test_block_lists_match_sorted_permutation(n, bs, B):
    seeds = [0, 12345, 1000003, 0xFFFFFFFF, 7, 99, 5, 31337, 42]
    cats = np.random.default_rng(n).integers(0, max(B, 1), n).astype(np.int32)
    ws_bytes = lib().hb_block_lists_workspace_bytes(n, bs, B)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    idx = torch.empty(len(seeds) * n, dtype=torch.int32, device="cuda")
    arr = (ctypes.c_uint32 * len(seeds))(*seeds)
    dcats = dev(cats)
    _lib.check(lib().hb_block_lists(n, bs, arr, len(seeds), ptr(dcats) if B else None, B, ptr(idx),
                                    ptr(ws), ws_bytes, stream()))
    got = idx.cpu().numpy().reshape(len(seeds), n)
    for c, s in enumerate(seeds):
        perm = ho.block_permutation(n, s)
        for j, p0 in enumerate(range(0, n, bs)):
            blk = perm[p0:p0 + bs]
            if B:  # within a block: ordered by (batch, cell)
                exp = blk[np.lexsort((blk, cats[blk]))]
            else:
                exp = np.sort(blk)
            np.testing.assert_array_equal(got[c, p0:p0 + bs], exp, err_msg=f"seed {s} block {j}")


@pytest.mark.parametrize("stabilized", [True, False])
@pytest.mark.parametrize("B,K", [(3, 20), (10, 100), (1, 5)])
def test_penalty(stabilized, B, K):
    rng = np.random.default_rng(123)
    E = rng.random((B, K)) * 10
    O = rng.random((B, K)) * 10
    O[0, 0] = 0
    th = rng.random(B) * 2 + 0.5
    pen = torch.empty((B, K), dtype=torch.float64, device="cuda")
    dE, dO, dth = dev(E), dev(O), dev(th)  # keep the inputs alive across the launch
    _lib.check(lib().hb_penalty(ptr(dE), ptr(dO), ptr(dth), ptr(pen), B, K, int(stabilized), stream()))
    np.testing.assert_allclose(pen.cpu().numpy(), ho.penalty(E, O, th, stabilized), rtol=1e-12)


def _lambda(E, O, Nb, **kw):
    B, K = E.shape
    out = torch.empty((B, K), dtype=torch.float64, device="cuda")
    thr = kw["threshold"]
    dE, dO, dNb = dev(E), dev(O), dev(Nb)
    _lib.check(lib().hb_lambda_kb(ptr(dE), ptr(dO), ptr(dNb), ptr(out), B, K, kw["alpha"],
                                  0.0 if thr is None else thr, int(thr is not None),
                                  kw["ridge_lambda"], int(kw["dynamic_lambda"]), stream()))
    return out.cpu().numpy()


def test_lambda_kb_known_answers():
    # tests/test_harmony.py:342-450
    N_b = np.array([0, 100, 1, 50], dtype=np.float64)
    O = np.array([[0, 0, 0], [30, 40, 30], [0, 0, 1], [20, 15, 15]], dtype=np.float64)
    E = np.ones((4, 3)) * 10
    r = _lambda(E, O, N_b, alpha=0.2, threshold=1e-5, ridge_lambda=1.0, dynamic_lambda=True)
    np.testing.assert_array_equal(r, ho.compute_lambda_kb(E, O, N_b, alpha=0.2, threshold=1e-5,
                                                          ridge_lambda=1.0, dynamic_lambda=True))
    assert np.all(r[0] == 1e30) and r[2, 0] == 1e30 and r[2, 1] == 1e30
    r = _lambda(np.array([[5.0, 0.0]]), np.array([[10.0, 0.0]]), np.array([100.0]), alpha=0.2,
                threshold=None, ridge_lambda=0.0, dynamic_lambda=False)
    assert r[0, 0] == 0.0 and r[0, 1] == 1e30
    r = _lambda(np.array([[0.0, 5.0]]), np.array([[0.0, 10.0]]), np.array([100.0]), alpha=0.2,
                threshold=None, ridge_lambda=1.0, dynamic_lambda=True)
    assert r[0, 0] == 1e30 and r[0, 1] == pytest.approx(1.0)


@pytest.mark.parametrize("B", [5, 50, 200])
def test_ridge_inverse(B):
    rng = np.random.default_rng(42)
    K = 10
    O = rng.random((B, K)) * 100
    lam = rng.random((B, K)) * 5 + 0.1
    lam[0, 0] = 1e30
    inv = torch.empty((K, B + 1, B + 1), dtype=torch.float64, device="cuda")
    dO, dlam = dev(O), dev(lam)
    _lib.check(lib().hb_ridge_inverse(ptr(dO), ptr(dlam), ptr(inv), B, K, stream()))
    got = inv.cpu().numpy()
    for k in range(K):
        np.testing.assert_allclose(got[k], ho.arrowhead_inverse(O[:, k], lam[:, k]), atol=1e-12,
                                   rtol=1e-10)
