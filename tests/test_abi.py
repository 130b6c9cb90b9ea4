"""The C-ABI library loads, exports every symbol include/harmony_b200.h declares,
and its ctypes structs match the header layout (no GPU needed)."""

import ctypes
import re
from pathlib import Path

import pytest

from rapids_singlecell_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "harmony_b200.h"


def _declared():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"HB_API\s+[\w\s\*]+?\b(hb_\w+)\s*\(", txt)))


def test_header_declares_expected_symbols():
    assert _declared() == sorted(_lib.EXPORTED)


def test_library_exports_all_declared_symbols():
    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name


def test_version_and_error_string():
    lib = _lib.load()
    assert b"sm_100a" in lib.hb_version()
    assert isinstance(lib.hb_last_error(), bytes)


def test_plan_validation_without_gpu():
    lib = _lib.load()
    p = _lib.HbParams()
    p.n_cells, p.n_pcs, p.n_clusters, p.n_batches = 1000, 20, 10, 3
    p.block_size, p.max_iter_harmony, p.max_iter_clustering = 0, 2, 3
    p.sigma = 0.1
    plan = ctypes.c_void_p()
    assert lib.hb_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _lib.HB_ERR_INVALID
    assert b"block_size" in lib.hb_last_error()
    p.block_size = 50
    p.n_clusters = 300
    assert lib.hb_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _lib.HB_ERR_UNSUPPORTED
    p.n_clusters = 10
    p.sweep_wait_ns = -1  # the grid-barrier wait bound must be in [0, 60 s]
    assert lib.hb_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _lib.HB_ERR_INVALID
    assert b"sweep_wait_ns" in lib.hb_last_error()
    p.sweep_wait_ns, p.test_unmet_arrivals = 0, 2  # the test hook takes 0 or 1
    assert lib.hb_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _lib.HB_ERR_INVALID
    assert b"test_unmet_arrivals" in lib.hb_last_error()


def test_struct_layout():
    # hb_params: 8+4*4+8+4*2+8*6+4*4+8 = 112 bytes, then the wait bound (8) and the test hook
    # (4, padded to 8)
    assert ctypes.sizeof(_lib.HbParams) == 128
    assert ctypes.sizeof(_lib.HbOutputs) == 6 * ctypes.sizeof(ctypes.c_void_p)
    assert ctypes.sizeof(_lib.HbProfile) == 56


def test_kmeans_init_validation_without_gpu():
    """hb_kmeans_init checks its arguments before touching the device."""
    lib = _lib.load()
    ws = lib.hb_kmeans_workspace_bytes(10_000, 50, 100)
    assert ws > 10_000 * 56 * 2  # at least the bf16 copy of the rows
    assert lib.hb_kmeans_workspace_bytes(0, 50, 100) == 0
    it = ctypes.c_int32(0)
    fake = ctypes.c_void_p(256)  # never dereferenced: every case fails before any device work
    def call(n, d, K, max_iter=25, tol=1e-4, ws_bytes=1 << 30):
        return lib.hb_kmeans_init(fake, n, d, K, max_iter, tol, 0, fake, ctypes.byref(it), fake, ws_bytes, None)
    assert call(100, 10, 200) == _lib.HB_ERR_INVALID        # more clusters than cells
    assert call(100, 10, 5, max_iter=-1) == _lib.HB_ERR_INVALID
    assert call(100, 10, 5, tol=float("nan")) == _lib.HB_ERR_INVALID
    assert call(1000, 257, 5) == _lib.HB_ERR_UNSUPPORTED    # more than 256 PCs
    assert call(1000, 129, 129) == _lib.HB_ERR_UNSUPPORTED  # more than 128 PCs and clusters
    assert call(1000, 10, 257) == _lib.HB_ERR_UNSUPPORTED   # more than 256 clusters
    assert call(1000, 10, 5, ws_bytes=16) == _lib.HB_ERR_WORKSPACE
    assert b"workspace" in lib.hb_last_error()
