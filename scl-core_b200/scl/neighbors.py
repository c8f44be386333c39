"""NumPy-level k-nearest neighbours through the drop-in C ABI (scl_neighbors.h):
the samples are the matrix's rows; the work runs on the GPU."""
from __future__ import annotations

import ctypes

import numpy as np

from .core.error import check_error
from .core.sparse import CsrMatrix


def compute_norms(mat: CsrMatrix) -> np.ndarray:
    lib = mat.lib
    out = np.zeros(mat.shape[0], dtype=mat.real_dtype)
    check_error(lib.scl_neighbors_compute_norms(mat.handle, out.ctypes.data_as(ctypes.POINTER(lib.real_type))),
                "compute_norms", lib)
    return out


def knn(mat: CsrMatrix, k: int, norms: np.ndarray = None):
    """(indices [n, k], distances [n, k]) of the k nearest other rows
    (scl_knn with the given squared norms, else scl_knn_simple)."""
    lib = mat.lib
    n = mat.shape[0]
    idx = np.zeros((n, int(k)), dtype=mat.index_dtype)
    dist = np.zeros((n, int(k)), dtype=mat.real_dtype)
    PI = idx.ctypes.data_as(ctypes.POINTER(lib.index_type))
    PD = dist.ctypes.data_as(ctypes.POINTER(lib.real_type))
    if norms is None:
        check_error(lib.scl_knn_simple(mat.handle, n, int(k), PI, PD), "knn_simple", lib)
    else:
        nr = np.ascontiguousarray(norms, dtype=mat.real_dtype)
        check_error(lib.scl_knn(mat.handle, nr.ctypes.data_as(ctypes.POINTER(lib.real_type)), n, int(k), PI, PD),
                    "knn", lib)
    return idx, dist


def set_kernel(kernel: int, mat_or_variant="f32_i32") -> int:
    """Choose the kernel scl_knn runs in one library variant (scl_gpu_knn_set_kernel):
    0 = automatic (default), 1 = every distance on CUDA cores (up to 128 features,
    k up to 64), 2 = tensor-core filter (any feature count and k). All return the
    same bits. Returns the previous choice."""
    from ._bindings._loader import get_library

    lib = mat_or_variant.lib if isinstance(mat_or_variant, CsrMatrix) else get_library(mat_or_variant)
    prev = ctypes.c_int(0)
    check_error(lib.scl_gpu_knn_set_kernel(int(kernel), ctypes.byref(prev)), "knn_set_kernel", lib)
    return prev.value
