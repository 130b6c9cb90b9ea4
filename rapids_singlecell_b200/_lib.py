"""ctypes binding of the engine's C ABI (include/harmony_b200.h).

The shared library is built in-tree (``rapids_singlecell_b200/_lib/``) by
``rapids_singlecell_b200.build.build()``.  There is no fallback: if the library
is missing every entry point raises.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_lib" / "libharmony_b200.so"

HB_OK = 0
HB_ERR_INVALID = 1
HB_ERR_WORKSPACE = 2
HB_ERR_TIMEOUT = 3
HB_ERR_CUDA = 4
HB_ERR_INTERNAL = 5
HB_ERR_UNSUPPORTED = 6

HB_FP32, HB_FP64, HB_BF16, HB_FP16 = 0, 1, 2, 3
HB_KNN_SQEUCLIDEAN, HB_KNN_EUCLIDEAN, HB_KNN_COSINE, HB_KNN_INNER_PRODUCT = 0, 1, 2, 3
# persistent-sweep layouts (hb_params.sweep_form): (thread groups, threads per row, A tiles)
SWEEP_FORMS = {1: (2, 2, 2), 2: (2, 2, 1), 3: (1, 4, 2), 4: (1, 4, 1)}
PRECISIONS = {"fp32": HB_FP32, "fp64": HB_FP64, "bf16": HB_BF16, "fp16": HB_FP16}

# every symbol include/harmony_b200.h declares
EXPORTED = (
    "hb_plan_create", "hb_plan_destroy", "hb_plan_workspace_bytes", "hb_harmonize",
    "hb_l2_normalize", "hb_block_lists_workspace_bytes", "hb_block_lists", "hb_block_lists_static",
    "hb_penalty",
    "hb_lambda_kb", "hb_ridge_inverse", "hb_similarity", "hb_tc_centroids_workspace_bytes", "hb_tc_centroids",
    "hb_tc_moments_workspace_bytes", "hb_tc_moments", "hb_tc_apply_workspace_bytes", "hb_tc_apply",
    "hb_kmeans_workspace_bytes", "hb_kmeans_init",
    "hb_pca_gram_workspace_bytes", "hb_pca_gram", "hb_pca_covariance", "hb_pca_project_workspace_bytes",
    "hb_pca_project", "hb_csr_to_dense", "hb_knn_workspace_bytes", "hb_knn",
    "hb_last_error", "hb_version",
)


class HbParams(ctypes.Structure):
    _fields_ = [
        ("n_cells", ctypes.c_int64),
        ("n_pcs", ctypes.c_int32),
        ("n_clusters", ctypes.c_int32),
        ("n_batches", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("block_size", ctypes.c_int64),
        ("max_iter_harmony", ctypes.c_int32),
        ("max_iter_clustering", ctypes.c_int32),
        ("tol_harmony", ctypes.c_double),
        ("tol_clustering", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("ridge_lambda", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("batch_prune_threshold", ctypes.c_double),
        ("prune", ctypes.c_int32),
        ("stabilized_penalty", ctypes.c_int32),
        ("dynamic_lambda", ctypes.c_int32),
        ("max_sweep_ctas", ctypes.c_int32),
        ("random_state", ctypes.c_uint64),
        ("sweep_wait_ns", ctypes.c_int64),
        ("test_unmet_arrivals", ctypes.c_int32),
        ("sweep_form", ctypes.c_int32),
    ]


class HbProfile(ctypes.Structure):
    _fields_ = [
        ("kernel_launches", ctypes.c_int64),
        ("block_launches", ctypes.c_int64),
        ("block_ms", ctypes.c_double),
        ("block_bytes", ctypes.c_double),
        ("centroid_launches", ctypes.c_int64),
        ("centroid_ms", ctypes.c_double),
        ("centroid_bytes", ctypes.c_double),
    ]


class HbOutputs(ctypes.Structure):
    _fields_ = [
        ("objectives", ctypes.POINTER(ctypes.c_double)),
        ("n_objectives", ctypes.POINTER(ctypes.c_int32)),
        ("kmeans_objectives", ctypes.POINTER(ctypes.c_double)),
        ("kmeans_iters", ctypes.POINTER(ctypes.c_int32)),
        ("converged", ctypes.POINTER(ctypes.c_int32)),
        ("profile", ctypes.POINTER(HbProfile)),
    ]


class HarmonyLibError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"harmony_b200 error {status}: {msg}")
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Load (once) the engine library; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"harmony_b200 CUDA library not found at {LIB_PATH}; build it with "
            "`python -c 'import rapids_singlecell_b200.build as b; b.build()'`"
        )
    lib = ctypes.CDLL(os.fspath(LIB_PATH))
    c_void_p, c_int, c_i32, c_i64, c_size = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int32,
                                             ctypes.c_int64, ctypes.c_size_t)
    P = ctypes.POINTER
    lib.hb_plan_create.argtypes = [P(HbParams), P(c_void_p)]
    lib.hb_plan_create.restype = c_int
    lib.hb_plan_destroy.argtypes = [c_void_p]
    lib.hb_plan_destroy.restype = None
    lib.hb_plan_workspace_bytes.argtypes = [c_void_p]
    lib.hb_plan_workspace_bytes.restype = c_size
    lib.hb_harmonize.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, P(c_i64),
                                 P(ctypes.c_double), c_void_p, c_void_p, c_size, c_void_p,
                                 P(HbOutputs), c_void_p]
    lib.hb_harmonize.restype = c_int
    lib.hb_l2_normalize.argtypes = [c_void_p, c_void_p, c_i64, c_i32, c_i32, c_void_p]
    lib.hb_l2_normalize.restype = c_int
    lib.hb_block_lists_workspace_bytes.argtypes = [c_i64, c_i64, c_i32]
    lib.hb_block_lists_workspace_bytes.restype = c_size
    lib.hb_block_lists.argtypes = [c_i64, c_i64, P(ctypes.c_uint32), c_i32, c_void_p, c_i32,
                                   c_void_p, c_void_p, c_size, c_void_p]
    lib.hb_block_lists.restype = c_int
    lib.hb_block_lists_static.argtypes = [c_i64, c_i64, P(ctypes.c_uint32), c_i32, c_void_p, c_i32,
                                          c_void_p, c_void_p]
    lib.hb_block_lists_static.restype = c_int
    lib.hb_penalty.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_i32, c_i32, c_i32, c_void_p]
    lib.hb_penalty.restype = c_int
    lib.hb_lambda_kb.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_i32, c_i32,
                                 ctypes.c_double, ctypes.c_double, c_i32, ctypes.c_double, c_i32,
                                 c_void_p]
    lib.hb_lambda_kb.restype = c_int
    lib.hb_ridge_inverse.argtypes = [c_void_p, c_void_p, c_void_p, c_i32, c_i32, c_void_p]
    lib.hb_ridge_inverse.restype = c_int
    lib.hb_similarity.argtypes = [c_void_p, c_i32, c_void_p, c_i32, c_void_p, c_i64, c_i32, c_i32,
                                  c_i32, c_void_p, c_void_p, c_void_p]
    lib.hb_similarity.restype = c_int
    lib.hb_tc_centroids_workspace_bytes.argtypes = [c_i64, c_i32, c_i32, c_i32]
    lib.hb_tc_centroids_workspace_bytes.restype = c_size
    lib.hb_tc_centroids.argtypes = [c_void_p, c_i32, c_void_p, c_i32, c_i64, c_i32, c_i32, c_void_p, c_i32, c_i32,
                                    c_void_p, c_i32, c_void_p, c_void_p, c_size, c_void_p, c_void_p]
    lib.hb_tc_centroids.restype = c_int
    lib.hb_tc_moments_workspace_bytes.argtypes = [c_i64, c_i32, c_i32, c_i32]
    lib.hb_tc_moments_workspace_bytes.restype = c_size
    lib.hb_tc_moments.argtypes = [c_void_p, c_void_p, c_i32, c_void_p, P(c_i64), c_i64, c_i32, c_i32, c_i32, c_i32,
                                  c_void_p, c_void_p, c_size, c_void_p, c_void_p]
    lib.hb_tc_moments.restype = c_int
    lib.hb_tc_apply_workspace_bytes.argtypes = [c_i64, c_i32]
    lib.hb_tc_apply_workspace_bytes.restype = c_size
    lib.hb_tc_apply.argtypes = [c_void_p, c_void_p, c_i32, c_void_p, c_void_p, P(c_i64), c_i64, c_i32, c_i32, c_i32,
                                c_i32, c_void_p, c_void_p, c_i32, c_void_p, c_size, c_void_p, c_void_p]
    lib.hb_tc_apply.restype = c_int
    lib.hb_kmeans_workspace_bytes.argtypes = [c_i64, c_i32, c_i32]
    lib.hb_kmeans_workspace_bytes.restype = c_size
    lib.hb_kmeans_init.argtypes = [c_void_p, c_i64, c_i32, c_i32, c_i32, ctypes.c_double, ctypes.c_uint64,
                                   c_void_p, P(c_i32), c_void_p, c_size, c_void_p]
    lib.hb_kmeans_init.restype = c_int
    lib.hb_pca_gram_workspace_bytes.argtypes = [c_i64, c_i32]
    lib.hb_pca_gram_workspace_bytes.restype = c_size
    lib.hb_pca_gram.argtypes = [c_void_p, c_i64, c_i32, c_i64, c_void_p, c_void_p, c_void_p, c_size, c_void_p]
    lib.hb_pca_gram.restype = c_int
    lib.hb_pca_covariance.argtypes = [c_void_p, c_void_p, c_i64, c_i32, c_i32, c_void_p, c_void_p, c_void_p]
    lib.hb_pca_covariance.restype = c_int
    lib.hb_pca_project_workspace_bytes.argtypes = [c_i32, c_i32]
    lib.hb_pca_project_workspace_bytes.restype = c_size
    lib.hb_pca_project.argtypes = [c_void_p, c_i64, c_i32, c_i64, c_void_p, c_i32, c_void_p, c_void_p,
                                   c_void_p, c_size, c_void_p]
    lib.hb_pca_project.restype = c_int
    lib.hb_csr_to_dense.argtypes = [c_void_p, c_void_p, c_void_p, c_i64, c_i32, c_void_p, c_i64, c_void_p,
                                    c_void_p]
    lib.hb_csr_to_dense.restype = c_int
    lib.hb_knn_workspace_bytes.argtypes = [c_i64, c_i64, c_i32, c_i32, c_i32]
    lib.hb_knn_workspace_bytes.restype = c_size
    lib.hb_knn.argtypes = [c_void_p, c_i64, c_void_p, c_i64, c_i32, c_i32, c_i32, c_void_p, c_void_p, c_void_p,
                           c_size, c_void_p]
    lib.hb_knn.restype = c_int
    lib.hb_last_error.argtypes = []
    lib.hb_last_error.restype = ctypes.c_char_p
    lib.hb_version.argtypes = []
    lib.hb_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != HB_OK:
        msg = load().hb_last_error().decode(errors="replace")
        if status == HB_ERR_INVALID:
            raise ValueError(msg)
        if status == HB_ERR_WORKSPACE:
            raise MemoryError(msg)
        raise HarmonyLibError(status, msg)
