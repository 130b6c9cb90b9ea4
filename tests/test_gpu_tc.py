"""Tensor-core (tcgen05) path: the similarity tile against a plain PyTorch fp32
reference of the same op, and full 16-bit Harmony runs against the float64
oracle (error budget of the 16-bit path: 1e-3 relative max-abs on Z_hat)."""

import numpy as np
import pandas as pd
import pytest
import torch

from oracle import harmony_oracle as ho
from rapids_singlecell_b200 import _lib, harmonize
from rapids_singlecell_b200.synthetic import MixtureSpec, initial_centroids, make_config, make_mixture
from tests._gpu import dev, lib, ptr, rel_maxabs, stream

pytestmark = pytest.mark.gpu
HT = {"fp16": (torch.float16, _lib.HB_FP16), "bf16": (torch.bfloat16, _lib.HB_BF16)}


def _pad(t, ld):
    out = torch.zeros((t.shape[0], ld), dtype=t.dtype, device=t.device)
    out[:, : t.shape[1]] = t
    return out


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
@pytest.mark.parametrize("n,d,K", [(128, 64, 16), (300, 50, 100), (1000, 100, 200), (257, 3, 7),
                                   (5000, 128, 256), (129, 65, 129)])
def test_similarity_tile(prec, n, d, K):
    dt, code = HT[prec]
    g = torch.Generator(device="cuda").manual_seed(n + d + K)
    Z = torch.nn.functional.normalize(torch.randn(2 * n, d, device="cuda", generator=g), dim=1)
    Y = torch.nn.functional.normalize(torch.randn(K, d, device="cuda", generator=g), dim=1)
    ld = (d + 7) // 8 * 8
    Zh, Yh = _pad(Z.to(dt), ld), _pad(Y.to(dt), ld)
    idx = torch.randperm(2 * n, device="cuda", generator=g)[:n].to(torch.int32)
    S = torch.full((n, K), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib().hb_similarity(ptr(Zh), ld, ptr(Yh), ld, ptr(idx), n, d, K, code, ptr(S), ptr(err),
                                   stream()))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = Zh[idx.long(), :d].float() @ Yh[:, :d].float().T   # fp32 reference of the same op
    torch.testing.assert_close(S, ref, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_c1_small_16bit_vs_fp64_oracle(prec):
    cfg = make_config("C1", seed=1, n_cells=4000)
    Y0 = cfg["Y0"][:40]
    labels = pd.Categorical.from_codes(cfg["cats"], categories=["a", "b", "c"])
    kw = dict(n_clusters=40, max_iter_harmony=3, max_iter_clustering=8, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    out, info = harmonize(torch.as_tensor(cfg["Z"], device="cuda"), labels, None, init_centroids=Y0,
                          precision=prec, return_info=True, **kw)
    ref = ho.harmonize(cfg["Z"], cfg["cats"], 3, Y0, dtype=np.float64, **kw)
    err = rel_maxabs(out.cpu().numpy(), ref.Z_hat)
    print(f"{prec}: rel max-abs vs fp64 oracle = {err:.3e}; objectives {info.objectives_harmony} vs "
          f"{ref.objectives_harmony}")
    np.testing.assert_allclose(info.objectives_harmony, ref.objectives_harmony, rtol=5e-3)
    assert err < (1e-3 if prec == "fp16" else 5e-3)


@pytest.mark.parametrize("n,d,K,B", [(3001, 5, 17, 4), (6000, 100, 200, 12), (2000, 64, 129, 1)])
def test_16bit_odd_shapes_fp16(n, d, K, B):
    spec = MixtureSpec(n, d, 5, B, "dirichlet", (), 0.5, (0.8, 1.2))
    Z, cats, _ = make_mixture(spec, 21)
    Y0 = initial_centroids(Z, K, 22)
    labels = pd.Categorical.from_codes(cats, categories=[f"b{i}" for i in range(B)])
    kw = dict(n_clusters=K, max_iter_harmony=2, max_iter_clustering=4, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    out = harmonize(torch.as_tensor(Z, device="cuda"), labels, None, init_centroids=Y0,
                    precision="fp16", **kw)
    ref = ho.harmonize(Z, cats, B, Y0, dtype=np.float64, **kw)
    assert rel_maxabs(out.cpu().numpy(), ref.Z_hat) < 2e-3


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_many_blocks_times_batches(prec):
    """250 blocks x 48 batches exceeds the (block, batch) bucket limit of the
    partition, so the lists are ordered by cell index only inside each block."""
    n, d, K, B = 12000, 20, 30, 48
    spec = MixtureSpec(n, d, 4, B, "dirichlet", (), 0.5, (0.8, 1.2))
    Z, cats, _ = make_mixture(spec, 31)
    Y0 = initial_centroids(Z, K, 32)
    labels = pd.Categorical.from_codes(cats, categories=[f"b{i}" for i in range(B)])
    kw = dict(n_clusters=K, max_iter_harmony=2, max_iter_clustering=3, tol_harmony=-np.inf,
              tol_clustering=-np.inf, block_proportion=0.004)
    out = harmonize(torch.as_tensor(Z, device="cuda"), labels, None, init_centroids=Y0,
                    precision=prec, **kw)
    ref = ho.harmonize(Z, cats, B, Y0, dtype=np.float64, **kw)
    assert rel_maxabs(out.cpu().numpy(), ref.Z_hat) < (1e-4 if prec == "fp32" else 2e-3)


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_16bit_many_tiles_per_cta_vs_plain_fp32(prec):
    """150,000 cells: every CTA of the centroid pass and every thread group of the
    sweep handles several 128-cell tiles; checked against the plain fp32 path."""
    cfg = make_config("C2", seed=3, n_cells=150_000)
    kw = dict(n_clusters=100, max_iter_harmony=2, max_iter_clustering=4, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    labels = pd.Categorical.from_codes(cfg["cats"], categories=[f"b{i}" for i in range(cfg["n_batches"])])
    Z = torch.as_tensor(cfg["Z"], device="cuda")
    ref, ref_info = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="fp32", return_info=True, **kw)
    out, info = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision=prec, return_info=True, **kw)
    err = rel_maxabs(out.cpu().numpy(), ref.cpu().numpy())
    print(f"{prec} vs plain fp32: rel max-abs {err:.3e}; objectives {info.objectives_harmony} vs "
          f"{ref_info.objectives_harmony}")
    np.testing.assert_allclose(info.objectives_harmony, ref_info.objectives_harmony, rtol=5e-3)
    assert err < 5e-3


def test_bf16_wide_shapes_vs_plain_fp32():
    """The 2M-cell workload's shapes (100 PCs, K = 200, 32 Zipf-sized batches) on
    120,000 cells: the sweep runs one thread group per CTA with one A tile (two do
    not fit in shared memory next to the 32 x 200 tables) and the centroid pass
    runs in list order (660 (block, batch) keys); checked against plain fp32."""
    cfg = make_config("C3", seed=5, n_cells=120_000)
    kw = dict(n_clusters=200, max_iter_harmony=2, max_iter_clustering=4, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    labels = pd.Categorical.from_codes(cfg["cats"], categories=[f"b{i}" for i in range(cfg["n_batches"])])
    Z = torch.as_tensor(cfg["Z"], device="cuda")
    ref, ref_info = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="fp32", return_info=True, **kw)
    out, info = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="bf16", return_info=True, **kw)
    err = rel_maxabs(out.cpu().numpy(), ref.cpu().numpy())
    print(f"bf16 vs plain fp32 (C3 shapes): rel max-abs {err:.3e}; objectives "
          f"{info.objectives_harmony} vs {ref_info.objectives_harmony}")
    np.testing.assert_allclose(info.objectives_harmony, ref_info.objectives_harmony, rtol=5e-3)
    assert err < 5e-3


def _window_stop(objs, tol):
    """First k-means iteration count at which the reference's window-3 test holds
    (clustering.cu:380-387), or None."""
    for m in range(4, len(objs) + 1):
        o = objs[m - 2] + objs[m - 3] + objs[m - 4]
        nw = objs[m - 1] + objs[m - 2] + objs[m - 3]
        if (o - nw) < tol * abs(o):
            return m
    return None


def test_device_kmeans_stop_follows_the_window_rule():
    """With a finite tol_clustering the 16-bit path decides the k-means stop on the device
    (launches after it return at once); each outer iteration must stop exactly where the
    window-3 test first holds on its objectives, and the result must match the plain fp32
    path, which decides on the host."""
    cfg = make_config("C2", seed=8, n_cells=120_000)
    tol = 1e-3
    kw = dict(n_clusters=100, max_iter_harmony=3, max_iter_clustering=20, tol_harmony=-np.inf,
              tol_clustering=tol)
    labels = pd.Categorical.from_codes(cfg["cats"], categories=[f"b{i}" for i in range(cfg["n_batches"])])
    Z = torch.as_tensor(cfg["Z"], device="cuda")
    out, info = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="bf16", return_info=True, **kw)
    ref, ref_info = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="fp32", return_info=True, **kw)
    its = [len(k) for k in info.kmeans_objectives]
    print(f"k-means iterations bf16 {its}, fp32 {[len(k) for k in ref_info.kmeans_objectives]}")
    for outer, objs in enumerate(info.kmeans_objectives):
        m = _window_stop(objs, tol)
        assert m == len(objs) or (m is None and len(objs) == kw["max_iter_clustering"])
        assert info.objectives_harmony[outer + 1] == objs[-1]
    assert its == [len(k) for k in ref_info.kmeans_objectives]
    assert min(its) < kw["max_iter_clustering"]  # the stop was exercised
    assert rel_maxabs(out.cpu().numpy(), ref.cpu().numpy()) < 5e-3


def test_forced_sweep_forms_and_autotune(tmp_path):
    """Every sweep layout that ``hb_params.sweep_form`` can force gives the plain fp32 result on
    C2's shapes (150,000 cells), with and without a CTA cap; the autotuner picks one of them,
    stores it in its cache and ``harmonize(autotune=path)`` reproduces the plain result."""
    from rapids_singlecell_b200 import autotune as at

    cfg = make_config("C2", seed=4, n_cells=150_000)
    kw = dict(n_clusters=100, max_iter_harmony=2, max_iter_clustering=3, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    labels = pd.Categorical.from_codes(cfg["cats"], categories=[f"b{i}" for i in range(cfg["n_batches"])])
    Z = torch.as_tensor(cfg["Z"], device="cuda", dtype=torch.float32)
    ref = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="fp32", **kw).cpu().numpy()
    from rapids_singlecell_b200.harmony import HarmonyProblem
    Y0 = torch.as_tensor(cfg["Y0"], device="cuda", dtype=torch.float32)
    theta = np.full(cfg["n_batches"], 2.0)
    for form, cap in [(1, 0), (2, 0), (3, 0), (4, 0), (1, 74), (4, 111)]:
        prob = HarmonyProblem(Z, cfg["cats"].astype(np.int32), cfg["n_batches"], Y0, theta, precision="bf16",
                              sweep_form=form, max_sweep_ctas=cap, **kw)
        out, _ = prob.run()
        prob.close()
        err = rel_maxabs(out.cpu().numpy(), ref)
        print(f"sweep form {form}, cap {cap}: rel max-abs vs plain fp32 {err:.3e}")
        assert err < 5e-3
    path = str(tmp_path / "sweep.json")
    at._cache.clear()
    out = harmonize(Z, labels, None, init_centroids=cfg["Y0"], precision="bf16", autotune=path, **kw)
    key = at.shape_key(Z.device, "bf16", Z.shape[0], Z.shape[1], 100, cfg["n_batches"])
    choice = at.cached(key)
    print("autotune choice:", choice)
    assert (choice["sweep_form"], choice["max_sweep_ctas"]) in at.candidates(
        torch.cuda.get_device_properties(0).multi_processor_count)
    assert sum(v is not None for v in choice["timings"].values()) >= 4
    assert rel_maxabs(out.cpu().numpy(), ref) < 5e-3


@pytest.mark.parametrize("d,K,B,ok", [(128, 256, 8, True), (128, 256, 64, False), (50, 100, 160, True),
                                      (50, 100, 200, False)])
def test_plan_rejects_sweep_shapes_that_do_not_fit(d, K, B, ok):
    """The 16-bit plan asks the sweep's own layouts whether its tables, tiles and staged rows fit
    one CTA's shared memory, so a shape that would fail at the launch (B * K within the table
    bound, but 128 PCs with K = 256 and 64 batches, or 200 batches at K = 100) is refused when
    the plan is made; no kernel runs here."""
    import ctypes

    from rapids_singlecell_b200.harmony import make_params

    p = make_params(100_000, d, K, B, precision="bf16")
    plan = ctypes.c_void_p()
    st = lib().hb_plan_create(ctypes.byref(p), ctypes.byref(plan))
    if ok:
        assert st == _lib.HB_OK, lib().hb_last_error()
        lib().hb_plan_destroy(plan)
    else:
        assert st == _lib.HB_ERR_UNSUPPORTED
        assert b"shared" in lib().hb_last_error()
