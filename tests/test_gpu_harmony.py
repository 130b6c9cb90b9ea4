"""End-to-end parity of the plain FP32 / FP64 paths against the CPU oracle,
same seeded inputs and injected initial centroids."""

import numpy as np
import pandas as pd
import pytest
import torch

from oracle import harmony_oracle as ho
from rapids_singlecell_b200 import harmonize
from rapids_singlecell_b200.synthetic import MixtureSpec, initial_centroids, make_config, make_mixture
from tests._gpu import rel_maxabs

pytestmark = pytest.mark.gpu

# parity bars: relative max-abs error of Z_hat against the oracle of the same dtype
TOL = {"fp32": 1e-4, "fp64": 1e-9}
NP = {"fp32": np.float32, "fp64": np.float64}


def _run_both(Z, cats, B, Y0, prec, **kw):
    labels = pd.Categorical.from_codes(cats, categories=[f"b{i}" for i in range(B)])
    Zt = torch.as_tensor(Z.astype(NP[prec]), device="cuda")
    out, info = harmonize(Zt, labels, None, init_centroids=Y0, precision=prec, return_info=True, **kw)
    okw = {k: v for k, v in kw.items() if k not in ("correction_method", "colsum_algo")}
    ref = ho.harmonize(Z, cats, B, Y0, dtype=NP[prec], **okw)
    return out.cpu().numpy(), info, ref


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_c1_small_parity(prec):
    cfg = make_config("C1", seed=1, n_cells=4000)
    Y0 = cfg["Y0"][:40]
    out, info, ref = _run_both(cfg["Z"], cfg["cats"], cfg["n_batches"], Y0, prec, n_clusters=40,
                               max_iter_harmony=3, max_iter_clustering=8)
    assert info.n_outer == ref.n_outer
    assert [len(k) for k in info.kmeans_objectives] == [len(k) for k in ref.kmeans_objectives]
    np.testing.assert_allclose(info.objectives_harmony, ref.objectives_harmony, rtol=1e-5)
    assert rel_maxabs(out, ref.Z_hat) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_c1_full_default_tolerances(prec):
    cfg = make_config("C1", seed=0)
    out, info, ref = _run_both(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], prec,
                               n_clusters=100, max_iter_harmony=10, max_iter_clustering=20)
    assert info.converged == ref.converged and info.n_outer == ref.n_outer
    np.testing.assert_allclose(info.objectives_harmony, ref.objectives_harmony, rtol=1e-5)
    assert rel_maxabs(out, ref.Z_hat) < TOL[prec]


def test_harmony1_flavor_fixed_iterations():
    cfg = make_config("C1", seed=2, n_cells=3000)
    out, info, ref = _run_both(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"][:30], "fp32",
                               n_clusters=30, max_iter_harmony=4, max_iter_clustering=5,
                               tol_harmony=-np.inf, tol_clustering=-np.inf,
                               stabilized_penalty=False, dynamic_lambda=False, ridge_lambda=1.0)
    assert info.n_outer == 4
    assert rel_maxabs(out, ref.Z_hat) < TOL["fp32"]


@pytest.mark.parametrize("n,d,K,B,bp", [(1001, 3, 7, 1, 0.05), (997, 5, 17, 4, 0.07),
                                        (2500, 33, 65, 6, 0.1), (640, 64, 129, 2, 0.5),
                                        (5000, 100, 200, 12, 0.05)])
def test_odd_shapes(n, d, K, B, bp):
    spec = MixtureSpec(n, d, 5, B, "dirichlet", (), 0.5, (0.8, 1.2))
    Z, cats, _ = make_mixture(spec, 11)
    Y0 = initial_centroids(Z, K, 12)
    out, info, ref = _run_both(Z, cats, B, Y0, "fp32", n_clusters=K, max_iter_harmony=2,
                               max_iter_clustering=4, block_proportion=bp,
                               tol_harmony=-np.inf, tol_clustering=-np.inf)
    assert rel_maxabs(out, ref.Z_hat) < TOL["fp32"]


def test_theta_list_tau_and_empty_category():
    cfg = make_config("C1", seed=4, n_cells=3000)
    Z, cats = cfg["Z"], cfg["cats"]
    # a fourth, empty batch category: N_b = 0 is pruned
    labels = pd.Categorical.from_codes(cats, categories=["a", "b", "c", "unused"])
    Y0 = cfg["Y0"][:25]
    kw = dict(n_clusters=25, max_iter_harmony=2, max_iter_clustering=5, theta=[1.0, 2.0, 0.5, 3.0],
              tau=5)
    out = harmonize(torch.as_tensor(Z, device="cuda"), labels, None, init_centroids=Y0, **kw)
    ref = ho.harmonize(Z, cats, 4, Y0, dtype=np.float32, **kw)
    assert rel_maxabs(out.cpu().numpy(), ref.Z_hat) < TOL["fp32"]


def test_harmony_integrate_dropin_surface():
    from rapids_singlecell_b200.pp import harmony_integrate

    cfg = make_config("C1", seed=5, n_cells=2000)

    class AData:
        def __init__(self):
            self.obsm = {"X_pca": cfg["Z"].astype(np.float64)}
            self.obs = pd.DataFrame({"batch": [f"s{c}" for c in cfg["cats"]],
                                     "lane": [f"l{c % 2}" for c in cfg["cats"]]})

    a = AData()
    harmony_integrate(a, "batch", init_centroids=cfg["Y0"][:66].astype(np.float64), n_clusters=66)
    assert a.obsm["X_pca_harmony"].shape == a.obsm["X_pca"].shape
    assert a.obsm["X_pca_harmony"].dtype == np.float64
    ref = ho.harmonize(cfg["Z"].astype(np.float64), cfg["cats"], 3,
                       cfg["Y0"][:66].astype(np.float64), n_clusters=66)
    assert rel_maxabs(a.obsm["X_pca_harmony"], ref.Z_hat) < TOL["fp64"]
    # two keys joined with "," (6 combined batches), float32
    b = AData()
    harmony_integrate(b, ["batch", "lane"], dtype=np.float32, max_iter_harmony=2)
    assert np.isfinite(b.obsm["X_pca_harmony"]).all()
    with pytest.raises(ValueError, match="alpha must be a finite positive"):
        harmony_integrate(AData(), "batch", alpha=-1.0)
    c = AData()
    c.obsm["X_pca"][0, 0] = np.nan
    with pytest.raises(RuntimeError, match="NaN"):
        harmony_integrate(c, "batch")


def test_engine_cell_index_matches_caller_sorted():
    """cell_index=NULL (the engine sorts by batch) gives the result of the
    caller's stable argsort (up to the float64 atomic summation order of the
    observed counts, which differs from run to run)."""
    from rapids_singlecell_b200.harmony import HarmonyProblem

    spec = MixtureSpec(7000, 20, 4, 5, "dirichlet", (), 0.5, (0.8, 1.2))
    Z, cats, _ = make_mixture(spec, 41)
    Y0 = torch.as_tensor(initial_centroids(Z, 25, 42), device="cuda")
    X = torch.as_tensor(Z, device="cuda")
    kw = dict(precision="fp32", n_clusters=25, max_iter_harmony=2, max_iter_clustering=3,
              tol_harmony=-np.inf, tol_clustering=-np.inf)
    a = HarmonyProblem(X, cats, 5, Y0, np.full(5, 2.0), **kw)
    assert a.cell_index is None
    za = a.run()[0].clone()
    b = HarmonyProblem(X, cats, 5, Y0, np.full(5, 2.0), **kw)
    b.cell_index = torch.as_tensor(np.argsort(cats, kind="stable").astype(np.int32), device="cuda")
    zb = b.run()[0]
    assert rel_maxabs(za.cpu().numpy(), zb.cpu().numpy()) < 1e-5


def test_dlpack_device_input_runs_in_place():
    """An array of another library on the device (seen only through DLPack) is integrated
    without a copy to the host and gives the result of the equivalent torch tensor."""
    import torch

    class Exporter:
        def __init__(self, t):
            self._t = t

        def __dlpack__(self, *args, **kwargs):
            return self._t.__dlpack__(*args, **kwargs)

        def __dlpack_device__(self):
            return self._t.__dlpack_device__()

    cfg = make_config("C1", seed=12, n_cells=3000)
    Zt = torch.as_tensor(cfg["Z"], device="cuda")
    codes = torch.as_tensor(cfg["cats"].astype(np.int64), device="cuda")
    kw = dict(n_clusters=20, max_iter_harmony=2, max_iter_clustering=4, tol_harmony=-np.inf,
              tol_clustering=-np.inf, init_centroids=cfg["Y0"][:20], precision="fp32")
    a = harmonize(Exporter(Zt), Exporter(codes), None, **kw)
    b = harmonize(Zt, cfg["cats"].astype(np.int64), None, **kw)
    assert a.device.type == "cuda"
    assert (a - b).abs().max().item() <= 1e-5 * b.abs().max().item()


def test_device_labels_stay_on_the_device(monkeypatch):
    """Integer labels already on the GPU are coded, counted and sorted there: no host copy of
    the per-cell array (the reference keeps cats on the device, _utils/_multi_gpu.py:202-232).
    Arbitrary integer values (negative, gaps, unsorted) give the same result as the same labels
    on the host."""
    from rapids_singlecell_b200.harmony import _integer_codes

    cfg = make_config("C1", seed=13, n_cells=4000)
    values = np.array([40, -3, 7])[cfg["cats"]]  # categories sorted: -3, 7, 40
    dev_labels = torch.as_tensor(values, device="cuda")
    codes, nb = _integer_codes(dev_labels)
    assert nb == 3 and codes.is_cuda and codes.dtype == torch.int32
    host = pd.Series(values).astype("category").cat.codes.to_numpy()
    assert np.array_equal(codes.cpu().numpy(), host)
    kw = dict(n_clusters=25, max_iter_harmony=2, max_iter_clustering=4, tol_harmony=-np.inf,
              tol_clustering=-np.inf, init_centroids=cfg["Y0"][:25], precision="fp32")
    Zt = torch.as_tensor(cfg["Z"], device="cuda")
    b = harmonize(Zt, pd.Categorical(values), None, **kw)
    n = cfg["Z"].shape[0]
    real_cpu = torch.Tensor.cpu

    def guarded_cpu(self, *args, **kwargs):  # the per-cell label array must not come back
        assert not (self.is_cuda and self.dim() == 1 and self.numel() == n), "per-cell array copied to host"
        return real_cpu(self, *args, **kwargs)

    monkeypatch.setattr(torch.Tensor, "cpu", guarded_cpu)
    a = harmonize(Zt, dev_labels, None, **kw)
    monkeypatch.undo()
    assert (a - b).abs().max().item() <= 1e-5 * b.abs().max().item()


def test_device_labels_with_many_batches():
    """More than 4096 batches: the batch-sorted cell index is built with a device sort."""
    from rapids_singlecell_b200.harmony import HarmonyProblem

    n, B = 20_000, 4500  # two clusters keep the B x K tables of the plain path in shared memory
    rng = np.random.default_rng(3)
    Z = rng.standard_normal((n, 8)).astype(np.float32)
    cats = rng.integers(0, B, n).astype(np.int32)
    Y0 = torch.as_tensor(Z[:2], device="cuda")
    kw = dict(n_clusters=2, max_iter_harmony=1, max_iter_clustering=2, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    X = torch.as_tensor(Z, device="cuda")
    p_dev = HarmonyProblem(X, torch.as_tensor(cats, device="cuda"), B, Y0, np.full(B, 2.0), **kw)
    p_host = HarmonyProblem(X, cats, B, Y0, np.full(B, 2.0), **kw)
    assert torch.equal(p_dev.cell_index.cpu(),
                       torch.as_tensor(np.argsort(cats, kind="stable").astype(np.int32)))
    za = p_dev.run()[0].clone()
    zb = p_host.run()[0].clone()
    assert (za - zb).abs().max().item() <= 1e-5 * zb.abs().max().item()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_hundreds_of_batches_on_the_plain_paths(prec):
    """400 batches x K = 100 (atlas-sized donor counts) on the default float64 path and on fp32:
    the B x K penalty and count tables no longer fit in shared memory, so the block update runs
    with global tables and direct float64 atomics; parity with the oracle as for few batches."""
    spec = MixtureSpec(30_000, 20, 12, 400, "dirichlet", (), 0.5, (0.8, 1.2))
    Z, cats, _ = make_mixture(spec, 21)
    Y0 = initial_centroids(Z, 100, 22)
    out, info, ref = _run_both(Z, cats, 400, Y0, prec, n_clusters=100, max_iter_harmony=2,
                               max_iter_clustering=3, tol_harmony=-np.inf, tol_clustering=-np.inf)
    assert info.n_outer == 2
    assert rel_maxabs(out, ref.Z_hat) < TOL[prec]


def test_fp64_above_128_pcs():
    """The default float64 dtype with 200 PCs and the default tolerances: both loops stop where
    the oracle's stop, and Z_hat matches it to float64 rounding."""
    spec = MixtureSpec(3000, 200, 6, 3, "dirichlet", (), 0.5, (0.8, 1.2))
    Z, cats, _ = make_mixture(spec, 31)
    Y0 = initial_centroids(Z, 30, 32)
    out, info, ref = _run_both(Z, cats, 3, Y0, "fp64", n_clusters=30, max_iter_harmony=10,
                               max_iter_clustering=20)
    assert info.converged == ref.converged and info.n_outer == ref.n_outer
    assert [len(k) for k in info.kmeans_objectives] == [len(k) for k in ref.kmeans_objectives]
    np.testing.assert_allclose(info.objectives_harmony, ref.objectives_harmony, rtol=1e-9)
    assert rel_maxabs(out, ref.Z_hat) < TOL["fp64"]


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_device_stops_and_profiled_launches(prec):
    """The run enqueues its loops without waiting on the device: the k-means and outer stops are
    taken on the device and the launches after them return at once.  The iteration counts are
    the oracle's (same objectives), and the profile counts only the block updates that ran."""
    from rapids_singlecell_b200.harmony import HarmonyProblem

    cfg = make_config("C1", seed=5, n_cells=6000)
    B, K = cfg["n_batches"], 40
    Y0 = cfg["Y0"][:K]
    kw = dict(n_clusters=K, max_iter_harmony=8, max_iter_clustering=30, tol_harmony=1e-3,
              tol_clustering=1e-4)
    X = torch.as_tensor(cfg["Z"], device="cuda")
    prob = HarmonyProblem(X, cfg["cats"], B, torch.as_tensor(Y0, device="cuda"), np.full(B, 2.0),
                          precision=prec, **kw)
    _, info = prob.run(profile=True)
    prob.close()
    iters = [len(k) for k in info.kmeans_objectives]
    assert info.n_outer == len(iters) and info.n_outer < 8 and info.converged, (info.n_outer, iters)
    # the k-means loop stopped early in at least one outer iteration
    assert all(0 < i <= 30 for i in iters) and min(iters) < 30, iters
    nblk = -(-6000 // int(6000 * 0.05))
    per_iter = 1 if prec == "bf16" else nblk  # one persistent sweep, or one launch per block
    assert info.profile["block_launches"] == sum(iters) * per_iter
    if prec == "fp32":
        ref = ho.harmonize(cfg["Z"], cfg["cats"], B, Y0, dtype=np.float32,
                           **{k: v for k, v in kw.items()})
        assert iters == [len(k) for k in ref.kmeans_objectives]


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
@pytest.mark.parametrize("kw", [dict(max_iter_harmony=1, max_iter_clustering=5),
                                dict(max_iter_harmony=5, max_iter_clustering=10, tol_harmony=1e6),
                                dict(max_iter_harmony=4, max_iter_clustering=12, tol_clustering=1.0)],
                         ids=["one_outer", "converged_at_first_outer", "earliest_kmeans_stop"])
def test_loop_edges_of_the_device_run_control(prec, kw):
    """The edges of the device-side run control: a single outer iteration, a run that converges
    after its first outer iteration (the later ones enqueued, or not, and skipped on the device),
    and k-means loops that stop at the earliest point the window-3 rule allows (4 iterations)."""
    cfg = make_config("C1", seed=7, n_cells=3000)
    B = cfg["n_batches"]
    labels = pd.Categorical.from_codes(cfg["cats"], categories=[f"b{i}" for i in range(B)])
    Zt = torch.as_tensor(cfg["Z"], device="cuda")
    out, info = harmonize(Zt, labels, None, init_centroids=cfg["Y0"][:20], precision=prec, return_info=True,
                          n_clusters=20, **kw)
    ref = ho.harmonize(cfg["Z"], cfg["cats"], B, cfg["Y0"][:20], dtype=np.float32, n_clusters=20, **kw)
    assert info.n_outer == ref.n_outer and info.converged == ref.converged
    assert [len(k) for k in info.kmeans_objectives] == [len(k) for k in ref.kmeans_objectives]
    assert len(info.objectives_harmony) == ref.n_outer + 1
    assert rel_maxabs(out.cpu().numpy(), ref.Z_hat) < (TOL["fp32"] if prec == "fp32" else 1e-3)
