"""Batched / served problems: each result is the same alone and in the mix
(several problems of different shapes overlapping on the device), within the
run-to-run tolerance of the engine (float64 count atomics make the summation
order of the observed counts vary)."""

import numpy as np
import pytest

from rapids_singlecell_b200.batched import (HarmonyRequest, HarmonyServer, latency_summary, request_bytes,
                                            run_batched)
from rapids_singlecell_b200.synthetic import MixtureSpec, initial_centroids, make_mixture
from tests._gpu import rel_maxabs

pytestmark = pytest.mark.gpu


def _requests(prec):
    reqs = []
    for i, n in enumerate([3000, 12000, 7000, 20000, 5000, 9000]):
        B, d = 2 + i % 4, (30 if i % 2 else 50)
        K = min(100, n // 30)
        Z, cats, _ = make_mixture(MixtureSpec(n, d, 5, B, "dirichlet", (), 0.5, (0.8, 1.2)), 100 + i)
        Y0 = initial_centroids(Z, K, 200 + i)
        params = dict(n_clusters=K, max_iter_harmony=2, max_iter_clustering=5, tol_harmony=-np.inf,
                      tol_clustering=-np.inf)
        reqs.append(HarmonyRequest(Z, cats, B, Y0, np.full(B, 2.0), params, precision=prec, to_host=True))
    return reqs


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_results_alone_and_in_the_mix(prec):
    reqs = _requests(prec)
    alone = [run_batched([r], streams=1)[0] for r in reqs]
    mixed = run_batched(reqs, streams=4)
    tol = 1e-5 if prec == "fp32" else 2e-3
    for a, m in zip(alone, mixed):
        assert rel_maxabs(m.Z_hat.numpy(), a.Z_hat.numpy()) < tol
        np.testing.assert_allclose(m.info.objectives_harmony, a.info.objectives_harmony, rtol=1e-4)


def test_server_admits_by_budget():
    reqs = _requests("bf16")[:4]
    need = max(request_bytes(r) for r in reqs)
    with HarmonyServer(streams=4, hbm_budget_bytes=need) as srv:  # one request at a time fits
        res = [f.result() for f in [srv.submit(r) for r in reqs]]
        assert srv.in_use == 0 and srv.sms_in_use == 0
    assert all(np.isfinite(r.Z_hat.numpy()).all() for r in res)
    s = latency_summary(res)
    assert s["p99_ms"] >= s["p50_ms"] > 0
    with HarmonyServer(streams=1, hbm_budget_bytes=request_bytes(reqs[0]) // 2) as srv:
        with pytest.raises(MemoryError):
            srv.submit(reqs[0]).result()
