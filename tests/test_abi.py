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


def test_struct_layout():
    # hb_params: 8+4*4+8+4*2+8*6+4*4+8 = 112 bytes
    assert ctypes.sizeof(_lib.HbParams) == 112
    assert ctypes.sizeof(_lib.HbOutputs) == 6 * ctypes.sizeof(ctypes.c_void_p)
    assert ctypes.sizeof(_lib.HbProfile) == 56
