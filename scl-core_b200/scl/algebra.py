"""NumPy-level sparse x dense product through the drop-in C ABI (scl_algebra.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from .core.error import check_error
from .core.sparse import CsrMatrix


def spmm(A: CsrMatrix, X: np.ndarray, Y: np.ndarray = None, alpha: float = 1.0, beta: float = 0.0) -> np.ndarray:
    """Y <- alpha A X + beta Y through scl_algebra_spmm (Y allocated when None); returns Y."""
    lib = A.lib
    X = np.ascontiguousarray(X, dtype=A.real_dtype)
    if Y is None:
        Y = np.zeros((A.shape[0] if A._is_csr else A.shape[1], X.shape[1]), dtype=A.real_dtype)
    if Y.dtype != A.real_dtype or not Y.flags["C_CONTIGUOUS"]:
        raise TypeError("Y must be a C-contiguous array of the matrix's value type")
    P = ctypes.POINTER(lib.real_type)
    check_error(lib.scl_algebra_spmm(A.handle, X.ctypes.data_as(P), X.shape[1], Y.ctypes.data_as(P), alpha, beta),
                "algebra_spmm", lib)
    return Y

