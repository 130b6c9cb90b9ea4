"""Host-side parameter resolution mirrors the reference's validation
(tests/test_harmony.py:95-110 and _harmony/__init__.py:154-200); these raise
before any GPU work, so they run on CPU."""

import numpy as np
import pandas as pd
import pytest

from rapids_singlecell_b200.harmony import default_n_clusters, harmonize, theta_array


def _data(n=300):
    rng = np.random.default_rng(0)
    Z = rng.normal(size=(n, 10)).astype(np.float32)
    obs = pd.DataFrame({"batch": rng.integers(0, 3, n).astype(str), "b2": rng.integers(0, 2, n).astype(str)})
    return Z, obs


@pytest.mark.parametrize("bad_alpha", [-0.1, 0.0, float("inf"), float("nan")])
def test_bad_alpha(bad_alpha):
    Z, obs = _data()
    with pytest.raises(ValueError, match="alpha must be a finite positive"):
        harmonize(Z, obs, "batch", alpha=bad_alpha)


@pytest.mark.parametrize("bad_threshold", [-0.1, 1.5, 2.0])
def test_bad_prune_threshold(bad_threshold):
    Z, obs = _data()
    with pytest.raises(ValueError, match="batch_prune_threshold must be in"):
        harmonize(Z, obs, "batch", batch_prune_threshold=bad_threshold)


def test_bad_correction_method_and_iters():
    Z, obs = _data()
    with pytest.raises(ValueError, match="correction_method must be"):
        harmonize(Z, obs, "batch", correction_method="nope")
    with pytest.raises(ValueError, match="max_iter_harmony must be >= 1"):
        harmonize(Z, obs, "batch", max_iter_harmony=0)


def test_theta_size_mismatch():
    Z, obs = _data()
    with pytest.raises(ValueError, match="Theta array size"):
        harmonize(Z, obs, "batch", theta=[1.0, 2.0])
    np.testing.assert_array_equal(theta_array(2, 3), [2.0, 2.0, 2.0])


def test_default_n_clusters():
    assert default_n_clusters(20_000) == 100
    assert default_n_clusters(600) == 20
    assert default_n_clusters(10) == 2


def test_flavor_validation():
    from rapids_singlecell_b200.pp import harmony_integrate

    class A:
        obsm = {"X_pca": np.zeros((10, 3))}
        obs = pd.DataFrame({"batch": ["a"] * 10})

    with pytest.raises(ValueError, match="flavor must be"):
        harmony_integrate(A(), "batch", flavor="harmony3")
    with pytest.raises(ValueError, match="is not available in adata.obsm"):
        harmony_integrate(A(), "batch", basis="nope")


@pytest.mark.parametrize("labels", [np.array([5, 2, 2, 9, 5, 0], dtype=np.int64),
                                    np.array([3, 3, 3], dtype=np.int32),
                                    np.arange(1000, dtype=np.uint16)[::-1].copy()])
def test_integer_codes_match_pandas(labels):
    from rapids_singlecell_b200.harmony import _integer_codes, get_batch_codes

    codes, nb = _integer_codes(labels)
    ref = get_batch_codes(labels, None)
    assert nb == ref.cat.categories.size
    np.testing.assert_array_equal(codes, ref.cat.codes.values.astype(np.int32))


@pytest.mark.parametrize("labels", [np.array([-1, 2]), np.array(["a", "b"]), np.zeros((2, 2), int),
                                    np.array([1.0, 2.0])])
def test_integer_codes_declines(labels):
    from rapids_singlecell_b200.harmony import _integer_codes

    assert _integer_codes(labels) == (None, 0)


def test_request_bytes_counts_workspace_and_tensors():
    from rapids_singlecell_b200.batched import HarmonyRequest, request_bytes
    from rapids_singlecell_b200.harmony import HarmonyProblem, make_params

    params = dict(n_clusters=30, max_iter_harmony=2, max_iter_clustering=5)
    r = HarmonyRequest(np.zeros((1000, 50), np.float32), np.zeros(1000, np.int32), 3,
                       np.zeros((30, 50), np.float32), np.ones(3), params)
    ws = HarmonyProblem.workspace_bytes(make_params(1000, 50, 30, 3, precision="bf16",
                                                    max_iter_harmony=2, max_iter_clustering=5))
    assert request_bytes(r) == ws + 2 * 1000 * 50 * 4 + 30 * 50 * 4 + 1000 * 4


class _Exporter:
    """An array of another library: it exposes only the DLPack protocol."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, *args, **kwargs):
        return self._t.__dlpack__(*args, **kwargs)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


def test_dlpack_inputs_share_memory():
    import torch

    from rapids_singlecell_b200.harmony import _integer_codes, from_dlpack

    t = torch.arange(12, dtype=torch.float32).reshape(4, 3)
    z = from_dlpack(_Exporter(t))
    assert isinstance(z, torch.Tensor) and z.data_ptr() == t.data_ptr()
    codes, nb = _integer_codes(_Exporter(torch.tensor([5, 2, 5, 9], dtype=torch.int64)))
    assert nb == 3 and codes.tolist() == [1, 0, 1, 2]
    a = np.zeros(3)
    assert from_dlpack(a) is a and from_dlpack([1, 2]) == [1, 2]


def test_sweep_autotune_keys_and_cache(tmp_path):
    """The autotuner's host side: shape keys bucket the cell count by half octaves, the candidates
    cover every sweep layout, and choices round-trip through the JSON cache."""
    from rapids_singlecell_b200 import _lib
    from rapids_singlecell_b200 import autotune as at

    k1 = at.shape_key("cpu", "bf16", 500_000, 50, 100, 8)
    assert k1 == at.shape_key("cpu", "bf16", 520_000, 50, 100, 8)      # same half-octave bucket
    assert k1 != at.shape_key("cpu", "bf16", 800_000, 50, 100, 8)
    assert k1 != at.shape_key("cpu", "fp16", 500_000, 50, 100, 8)
    cands = at.candidates(148)
    assert {f for f, _ in cands} == set(_lib.SWEEP_FORMS) and {c for _, c in cands} == {0, 111, 74}
    path = str(tmp_path / "sweep.json")
    at.remember(k1, {"sweep_form": 2, "max_sweep_ctas": 74, "us_per_launch": 1.0, "timings": {}})
    at.save_cache(path)
    at._cache.clear()
    assert at.cached(k1) is None
    at.load_cache(path)
    assert at.cached(k1)["sweep_form"] == 2


def test_sweep_form_validation():
    import ctypes

    from rapids_singlecell_b200 import _lib
    from rapids_singlecell_b200.harmony import make_params

    lib = _lib.load()
    plan = ctypes.c_void_p()
    p = make_params(1000, 20, 10, 3, precision="bf16", sweep_form=5)
    assert lib.hb_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _lib.HB_ERR_INVALID
    p = make_params(1000, 20, 10, 3, precision="bf16", sweep_form=3)
    assert lib.hb_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _lib.HB_OK
    lib.hb_plan_destroy(plan)


def test_sweep_autotune_host_rules():
    """The tuner refuses the plain paths before touching a device, and its CTA caps stay valid on
    a GPU with few SMs (0 = every SM, otherwise at least one CTA)."""
    import numpy as np
    import pytest

    from rapids_singlecell_b200 import autotune as at

    with pytest.raises(ValueError):
        at.tune_sweep(np.zeros((10, 4), np.float32), np.zeros(10, np.int32), 1, None, np.ones(1),
                      precision="fp32", n_clusters=2)
    for sms in (1, 2, 3, 148):
        caps = {c for _, c in at.candidates(sms)}
        assert 0 in caps and all(c == 0 or 1 <= c <= sms for c in caps)


def test_sweep_autotune_bad_cache_file_is_ignored(tmp_path):
    import pytest

    from rapids_singlecell_b200 import autotune as at

    bad = tmp_path / "sweep.json"
    bad.write_text("{not json")
    at._cache.clear()
    with pytest.warns(RuntimeWarning):
        at.load_cache(str(bad))
    bad.write_text('{"k": 3}')
    with pytest.warns(RuntimeWarning):
        at.load_cache(str(bad))
    assert at._cache == {}
