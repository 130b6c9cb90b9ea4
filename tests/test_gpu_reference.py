"""The engine against the reference itself, on the GPU.

``oracle/ref_harmony.py`` runs rapids_singlecell's Harmony with the reference's own CUDA
kernels (``oracle/_ref/libharmony_ref.so``, compiled from the reference tree by
``oracle/Makefile``): its clustering loop, objective, batched correction and helpers, in the
launch order of its nanobind modules.  Both sides get the same inputs and injected initial
centroids.  Bars (relative max-abs error of the corrected embedding):

* plain float32 / float64 paths against the reference in the same dtype: 1e-4 / 1e-9, and in
  float64 the same outer and k-means iteration counts under the default tolerances;
* the 16-bit tensor-core paths (bf16, fp16) against the reference in float64: 1e-3, at the
  benchmark configurations' full sizes (500k cells x 50 PCs and 2M cells x 100 PCs) for fixed
  iteration counts.
"""

import numpy as np
import pandas as pd
import pytest
import torch

from oracle import ref_harmony as rh
from rapids_singlecell_b200 import harmonize
from rapids_singlecell_b200.synthetic import make_config
from tests._gpu import rel_maxabs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not rh.available(), reason="reference shim not built (make -C oracle)")]

TOL_SAME = {"fp32": 1e-4, "fp64": 1e-9}
TOL_16 = 1e-3
NP = {"fp32": np.float32, "fp64": np.float64, "bf16": np.float32, "fp16": np.float32}


def _engine(Z, cats, B, Y0, prec, **kw):
    labels = pd.Categorical.from_codes(cats, categories=[f"b{i}" for i in range(B)])
    Zt = torch.as_tensor(np.ascontiguousarray(Z, dtype=NP[prec]), device="cuda")
    out, info = harmonize(Zt, labels, None, init_centroids=Y0, precision=prec, return_info=True, **kw)
    return out.cpu().numpy(), info


def test_c1_full_fp64_matches_reference_with_default_tolerances():
    """The drop-in call: 20k cells x 50 PCs, K = 100, default tolerances (both loops stop early):
    the same stop decisions, objectives and corrected embedding as the reference in float64."""
    cfg = make_config("C1", seed=0)
    kw = dict(n_clusters=100, max_iter_harmony=10, max_iter_clustering=20)
    out, info = _engine(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], "fp64", **kw)
    ref = rh.harmonize(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], dtype=np.float64, **kw)
    assert info.n_outer == ref.n_outer and info.converged == ref.converged
    assert [len(k) for k in info.kmeans_objectives] == [len(k) for k in ref.kmeans_objectives]
    np.testing.assert_allclose(info.objectives_harmony, ref.objectives_harmony, rtol=1e-9)
    assert rel_maxabs(out, ref.Z_hat) < TOL_SAME["fp64"]


def test_c1_full_fp32_matches_reference():
    """The float32 drop-in at fixed iteration counts (10 x 20).  The reference sums its float32
    objective with float32 atomics (kmeans_err_kernel, entropy_kernel): the value carries a few
    1e-4 of rounding that changes with the atomics' order from run to run, far above
    tol_clustering = 1e-5, so its own early-stop decisions are not repeatable in float32; the
    engine sums the objective in float64."""
    cfg = make_config("C1", seed=0)
    kw = dict(n_clusters=100, max_iter_harmony=10, max_iter_clustering=20, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    out, info = _engine(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], "fp32", **kw)
    ref = rh.harmonize(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], dtype=np.float32, **kw)
    np.testing.assert_allclose(info.objectives_harmony, ref.objectives_harmony, rtol=1e-3)
    assert rel_maxabs(out, ref.Z_hat) < TOL_SAME["fp32"]


def test_harmony1_flavour_matches_reference():
    cfg = make_config("C1", seed=2, n_cells=6000)
    kw = dict(n_clusters=40, max_iter_harmony=4, max_iter_clustering=6, stabilized_penalty=False,
              dynamic_lambda=False, ridge_lambda=1.0, theta=[1.0, 2.5, 0.5], tau=3)
    out, info = _engine(cfg["Z"], cfg["cats"], 3, cfg["Y0"][:40], "fp64", **kw)
    ref = rh.harmonize(cfg["Z"], cfg["cats"], 3, cfg["Y0"][:40], dtype=np.float64, **kw)
    assert info.n_outer == ref.n_outer
    assert rel_maxabs(out, ref.Z_hat) < TOL_SAME["fp64"]


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_c1_16bit_paths_within_1e3_of_reference_fp64(prec):
    cfg = make_config("C1", seed=0)
    kw = dict(n_clusters=100, max_iter_harmony=10, max_iter_clustering=20, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    out, _ = _engine(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], prec, **kw)
    ref = rh.harmonize(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], dtype=np.float64, **kw)
    assert rel_maxabs(out, ref.Z_hat) < TOL_16


@pytest.mark.parametrize("name,outer,inner", [("C2", 10, 20), ("C3", 3, 20)])
def test_full_size_configs_against_reference_fp64(name, outer, inner):
    """500k cells x 50 PCs (8 batches, K = 100; the full 10 x 20 iterations) and 2M cells x 100 PCs
    (32 batches, K = 200; 3 x 20 iterations): bf16 within 1e-3 and fp32 within 1e-4 of the
    reference's float64 run of the same iterations."""
    cfg = make_config(name, seed=0)
    kw = dict(n_clusters=cfg["n_clusters"], max_iter_harmony=outer, max_iter_clustering=inner,
              tol_harmony=-np.inf, tol_clustering=-np.inf)
    ref = rh.harmonize(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], dtype=np.float64, **kw)
    errs = {}
    for prec in ("bf16", "fp32"):
        out, _ = _engine(cfg["Z"], cfg["cats"], cfg["n_batches"], cfg["Y0"], prec, **kw)
        errs[prec] = rel_maxabs(out, ref.Z_hat)
        del out
        torch.cuda.empty_cache()
    print(f"{name}: rel max-abs vs reference fp64 {errs}")
    assert errs["bf16"] < TOL_16
    assert errs["fp32"] < 1e-4
