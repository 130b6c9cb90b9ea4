"""Bounded device waits: the persistent sweep's grid barrier gives up after its limit, the
run reports HB_ERR_TIMEOUT, and the GPU stays usable.

The plan's test hook ``test_unmet_arrivals = 1`` makes the barrier wait for one arrival more
than the grid makes -- a count that nothing reaches -- with the wait bounded at 1 ms.  Nothing
faults or hangs: every wait ends by its time bound (or at once once another CTA has given up),
the kernel finishes, and the host reads the error code."""

import time

import numpy as np
import pytest
import torch

from rapids_singlecell_b200 import _lib
from rapids_singlecell_b200.harmony import HarmonyProblem
from rapids_singlecell_b200.synthetic import make_config
from tests._gpu import rel_maxabs

pytestmark = pytest.mark.gpu


def _problem(cfg, **extra):
    kw = dict(n_clusters=50, max_iter_harmony=1, max_iter_clustering=2, tol_harmony=-np.inf,
              tol_clustering=-np.inf)
    return HarmonyProblem(torch.as_tensor(cfg["Z"], device="cuda"), cfg["cats"], cfg["n_batches"],
                          torch.as_tensor(cfg["Y0"][:50], device="cuda"), np.full(cfg["n_batches"], 2.0),
                          precision="bf16", **kw, **extra)


def test_sweep_barrier_wait_runs_out_and_the_gpu_stays_usable():
    cfg = make_config("C1", seed=3, n_cells=20_000)
    bad = _problem(cfg, sweep_wait_ns=1_000_000, test_unmet_arrivals=1)
    t0 = time.perf_counter()
    with pytest.raises(_lib.HarmonyLibError) as err:
        bad.run()
    elapsed = time.perf_counter() - t0
    bad.close()
    assert err.value.status == _lib.HB_ERR_TIMEOUT
    assert "timed out" in str(err.value)
    assert elapsed < 10.0  # 1 ms bound per wait; later waits give up at once
    # the same GPU, context and library run a normal problem afterwards
    good = _problem(cfg)
    z1 = good.run()[0].clone()
    z2 = good.run()[0].clone()
    good.close()
    assert bool(torch.isfinite(z1).all())
    assert rel_maxabs(z1.cpu().numpy(), z2.cpu().numpy()) < 1e-3
