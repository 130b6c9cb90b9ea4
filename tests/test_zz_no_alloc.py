"""hb_block_lists_static: block lists with the scratch in the library's fixed
device array (no workspace, no allocation in the call).  Its lists must equal
those of hb_block_lists with a caller workspace, on consecutive calls; sizes
beyond the fixed scratch are rejected before any device work.

Kept in its own file, collected last, so that it runs both alone in a fresh
process and after every other test."""

import ctypes

import numpy as np
import pytest

from rapids_singlecell_b200 import _lib


def _lib_or_skip():
    try:
        return _lib.load()
    except RuntimeError as e:  # library not built
        pytest.skip(str(e))


def test_static_block_lists_rejects_sizes_beyond_the_scratch():
    lib = _lib_or_skip()
    n, bs, B = 4_000_000, 40_000, 40  # 100 blocks x 40 batches: bucket counts far beyond 16 MiB
    assert lib.hb_block_lists_workspace_bytes(n, bs, B) > (16 << 20)
    seeds = (ctypes.c_uint32 * 1)(0)
    status = lib.hb_block_lists_static(n, bs, seeds, 1, ctypes.c_void_p(16), B, ctypes.c_void_p(16), None)
    assert status == _lib.HB_ERR_WORKSPACE
    assert b"static scratch" in lib.hb_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("n_seeds", [3, 9, 17])  # one, two and three chunks of eight k-means iterations
@pytest.mark.parametrize("B", [0, 5])
def test_static_block_lists_match_workspace_entry(B, n_seeds):
    import torch

    from tests._gpu import dev, lib, ptr, stream

    n, bs = 120_000, 6_000
    seeds = [3, 77, 1000003, 0xFFFFFFFF, 11, 12, 500, 501, 9, 1, 2, 4, 8, 16, 32, 64, 128][:n_seeds]
    cats = np.random.default_rng(9).integers(0, max(B, 1), n).astype(np.int32)
    dcats = dev(cats)
    arr = (ctypes.c_uint32 * len(seeds))(*seeds)
    ref = torch.full((len(seeds) * n,), -1, dtype=torch.int32, device="cuda")
    ws_bytes = lib().hb_block_lists_workspace_bytes(n, bs, B)
    assert ws_bytes <= (16 << 20)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    _lib.check(lib().hb_block_lists(n, bs, arr, len(seeds), ptr(dcats) if B else None, B, ptr(ref),
                                    ptr(ws), ws_bytes, stream()))
    for _ in range(2):  # two calls in a row: the fixed scratch is reused
        out = torch.full((len(seeds) * n,), -1, dtype=torch.int32, device="cuda")
        _lib.check(lib().hb_block_lists_static(n, bs, arr, len(seeds), ptr(dcats) if B else None, B,
                                               ptr(out), stream()))
        torch.cuda.synchronize()
        assert torch.equal(out, ref)


@pytest.mark.gpu
def test_static_block_lists_zero_iterations_is_a_no_op():
    """n_iters == 0 writes nothing and reports success, even right after a call that used
    the shared scratch."""
    import torch

    from tests._gpu import lib, ptr, stream

    n, bs = 50_000, 2_500
    seeds = (ctypes.c_uint32 * 2)(5, 6)
    out = torch.full((2 * n,), -1, dtype=torch.int32, device="cuda")
    _lib.check(lib().hb_block_lists_static(n, bs, seeds, 2, None, 0, ptr(out), stream()))
    untouched = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    assert lib().hb_block_lists_static(n, bs, seeds, 0, None, 0, ptr(untouched), stream()) == _lib.HB_OK
    torch.cuda.synchronize()
    assert bool((untouched == -7).all())
    # the workspace entry point agrees on both cases, and rejects a negative count
    assert lib().hb_block_lists(n, bs, seeds, 0, None, 0, ptr(untouched), None, 0, stream()) == _lib.HB_OK
    assert lib().hb_block_lists(n, bs, seeds, -1, None, 0, ptr(untouched), None, 0, stream()) == _lib.HB_ERR_INVALID
