"""Kernel-level checks of the 16-bit path's tensor-core kernels, each run alone through its C-ABI
entry point on seeded 16-bit inputs and compared with a float64 torch computation of the same op
on the same (already rounded) inputs:

* the cell-order centroid pass (k_tc_centroid_stream + its reduction): Y_norm and the per-key
  R sums (clustering.cu:272-281 and :321-332);
* the ridge moments (k_tc_moments + k_m_reduce, correction_batched.cu:55-100);
* the correction apply with its L2 renormalisation (k_tc_apply, kernels_outer.cuh:41-65).
"""

import ctypes

import numpy as np
import pytest
import torch

from rapids_singlecell_b200 import _lib

pytestmark = pytest.mark.gpu

DT = {"bf16": (torch.bfloat16, _lib.HB_BF16, 2.0 ** -8), "fp16": (torch.float16, _lib.HB_FP16, 2.0 ** -11)}


def _rows(n):
    return (n + 127) // 128 * 128 + 8


def _pad8(x):
    return (x + 7) // 8 * 8


def _call(fn, *args):
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(fn(*args, ctypes.c_void_p(st)))
    torch.cuda.synchronize()


def _ws(nbytes):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def _r16(rng, n, K, dt):
    """Positive rows summing to one, rounded to 16 bits, zero padded to [rows][ldr]."""
    R = rng.gamma(0.3, 1.0, (n, K)) + 1e-6
    R /= R.sum(1, keepdims=True)
    out = torch.zeros(_rows(n), _pad8(K), dtype=dt, device="cuda")
    out[:n, :K] = torch.as_tensor(R, device="cuda").to(dt)
    return out


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
@pytest.mark.parametrize("n,d,K,nkeys", [(5000, 50, 100, 180), (1000, 3, 7, 5), (20_000, 100, 200, 60),
                                         (777, 128, 256, 21)])
def test_centroid_pass(prec, n, d, K, nkeys):
    dt, code, ulp = DT[prec]
    rng = np.random.default_rng(n + d)
    lib = _lib.load()
    Z = rng.standard_normal((n, d))
    Z /= np.linalg.norm(Z, axis=1, keepdims=True)
    ldz, ldr, ldy = _pad8(d), _pad8(K), _pad8(d)
    Zn = torch.zeros(_rows(n), ldz, dtype=dt, device="cuda")
    Zn[:n, :d] = torch.as_tensor(Z, device="cuda").to(dt)
    R = _r16(rng, n, K, dt)
    ckey = torch.as_tensor(rng.integers(0, nkeys, n).astype(np.int32), device="cuda")
    Yn = torch.full((K, ldy), 7.0, dtype=dt, device="cuda")
    Osum = torch.zeros(nkeys, K, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws = _ws(lib.hb_tc_centroids_workspace_bytes(n, d, K, nkeys))
    _call(lib.hb_tc_centroids, Zn.data_ptr(), ldz, R.data_ptr(), ldr, n, d, K, ckey.data_ptr(), nkeys, code,
          Yn.data_ptr(), ldy, Osum.data_ptr(), ws.data_ptr(), ws.numel(), err.data_ptr())
    assert err.item() == 0
    Zf, Rf = Zn[:n, :d].double(), R[:n, :K].double()
    Y = Rf.T @ Zf
    Y = Y / Y.norm(dim=1, keepdim=True)
    # the kernel sums in float32 and rounds once to 16 bits: within one 16-bit step of the float64 value
    assert (Yn[:, :d].double() - Y).abs().max().item() <= ulp
    assert Yn[:, d:].double().abs().max().item() == 0.0 if ldy > d else True
    ref = torch.zeros(nkeys, K, dtype=torch.float64, device="cuda").index_add_(0, ckey.long(), Rf)
    assert (Osum - ref).abs().max().item() <= 1e-6 * ref.abs().max().item()


def _batches(rng, n, B):
    cats = rng.integers(0, B, n).astype(np.int32)
    if B > 2:
        cats[cats == 1] = 0  # an empty batch
    idx = np.argsort(cats, kind="stable").astype(np.int32)
    off = np.zeros(B + 1, dtype=np.int64)
    off[1:] = np.cumsum(np.bincount(cats, minlength=B))
    return cats, idx, off


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
@pytest.mark.parametrize("n,d,K,B", [(6000, 50, 100, 5), (1500, 3, 7, 1), (30_000, 100, 200, 12),
                                     (999, 256, 64, 3)])
def test_moments(prec, n, d, K, B):
    dt, code, _ = DT[prec]
    rng = np.random.default_rng(3 * n + d)
    lib = _lib.load()
    X = torch.as_tensor(rng.standard_normal((n, d)).astype(np.float32) * 3, device="cuda")
    R = _r16(rng, n, K, dt)
    cats, idx, off = _batches(rng, n, B)
    cidx = torch.as_tensor(idx, device="cuda")
    M = torch.full((K, B + 1, d), np.nan, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws = _ws(lib.hb_tc_moments_workspace_bytes(n, d, K, B))
    off_c = (ctypes.c_int64 * (B + 1))(*off.tolist())
    _call(lib.hb_tc_moments, X.data_ptr(), R.data_ptr(), _pad8(K), cidx.data_ptr(), off_c, n, d, K, B, code,
          M.data_ptr(), ws.data_ptr(), ws.numel(), err.data_ptr())
    assert err.item() == 0
    Xd, Rd = X.double(), R[:n, :K].double()
    ref = torch.zeros(K, B + 1, d, dtype=torch.float64, device="cuda")
    cat_t = torch.as_tensor(cats, device="cuda").long()
    for b in range(B):
        m = cat_t == b
        ref[:, b + 1] = Rd[m].T @ Xd[m]
    ref[:, 0] = Rd.T @ Xd
    # X enters as hi + lo 16-bit parts (>= 16 significant bits), float32 accumulation per tile
    assert (M - ref).abs().max().item() <= 5e-5 * ref.abs().max().item()


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
@pytest.mark.parametrize("n,d,K,B", [(6000, 50, 100, 5), (1500, 3, 7, 1), (30_000, 100, 200, 12),
                                     (999, 128, 64, 3)])
def test_apply(prec, n, d, K, B):
    dt, code, ulp = DT[prec]
    rng = np.random.default_rng(5 * n + d)
    lib = _lib.load()
    X = torch.as_tensor(rng.standard_normal((n, d)).astype(np.float32), device="cuda")
    R = _r16(rng, n, K, dt)
    W = torch.as_tensor((rng.standard_normal((B, K, d)) * 0.3).astype(np.float32), device="cuda")
    cats, idx, off = _batches(rng, n, B)
    cidx = torch.as_tensor(idx, device="cuda")
    ldz = _pad8(d)
    Zh = torch.full((n, d), np.nan, dtype=torch.float32, device="cuda")
    Zn = torch.zeros(_rows(n), ldz, dtype=dt, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws = _ws(lib.hb_tc_apply_workspace_bytes(n, B))
    off_c = (ctypes.c_int64 * (B + 1))(*off.tolist())
    _call(lib.hb_tc_apply, X.data_ptr(), R.data_ptr(), _pad8(K), W.data_ptr(), cidx.data_ptr(), off_c, n, d, K, B,
          code, Zh.data_ptr(), Zn.data_ptr(), ldz, ws.data_ptr(), ws.numel(), err.data_ptr())
    assert err.item() == 0
    cat_t = torch.as_tensor(cats, device="cuda").long()
    Rd = R[:n, :K].double()
    ref = X.double() - torch.einsum("nk,nkd->nd", Rd, W.double()[cat_t])
    # X, W as hi + lo parts, float32 accumulation: float32-level agreement
    assert (Zh.double() - ref).abs().max().item() <= 2e-5 * ref.abs().max().item()
    refn = ref / ref.norm(dim=1, keepdim=True)
    assert (Zn[:n, :d].double() - refn).abs().max().item() <= ulp
    if ldz > d:
        assert Zn[:n, d:].double().abs().max().item() == 0.0
