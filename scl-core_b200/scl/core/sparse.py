"""CSR handle wrapper (mirrors CsrMatrix of python/scl/core/sparse.py:277-459)."""
from __future__ import annotations

import ctypes
from enum import IntEnum
from typing import Tuple

import numpy as np

from .config import _infer_library
from .error import check_error


class BlockStrategy(IntEnum):
    CONTIGUOUS = 0
    SMALL = 1
    LARGE = 2
    ADAPTIVE = 3


class OwnershipMode(IntEnum):
    OWNED = 0
    WRAPPED = 1
    TRANSFERRED = 2


class CsrMatrix:
    """Owning wrapper of an ``scl_sparse_t`` CSR handle."""

    def __init__(self, handle: ctypes.c_void_p, lib, mode: OwnershipMode, data_refs=None, is_csr: bool = True):
        self._handle = handle
        self._lib = lib
        self._mode = mode
        self._refs = data_refs or []
        self._is_csr = is_csr

    # ---- properties ------------------------------------------------------
    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    @property
    def lib(self):
        return self._lib

    @property
    def real_dtype(self):
        return np.float64 if self._lib.real_type == ctypes.c_double else np.float32

    @property
    def index_dtype(self):
        return np.int64 if self._lib.index_type == ctypes.c_int64 else np.int32

    def _query(self, fn):
        out = self._lib.index_type()
        check_error(fn(self._handle, ctypes.byref(out)), fn.__name__, self._lib)
        return int(out.value)

    @property
    def shape(self) -> Tuple[int, int]:
        return self._query(self._lib.scl_sparse_rows), self._query(self._lib.scl_sparse_cols)

    @property
    def nnz(self) -> int:
        return self._query(self._lib.scl_sparse_nnz)

    @property
    def is_contiguous(self) -> bool:
        out = ctypes.c_int()
        check_error(self._lib.scl_sparse_is_contiguous(self._handle, ctypes.byref(out)), "is_contiguous", self._lib)
        return bool(out.value)

    # ---- factories ---------------------------------------------------------
    @classmethod
    def copy(cls, source, strategy: BlockStrategy = BlockStrategy.ADAPTIVE) -> "CsrMatrix":
        import scipy.sparse as sp

        if isinstance(source, np.ndarray):
            source = sp.csr_matrix(source)
        if source.format != "csr":
            source = source.tocsr()
        lib = _infer_library(data=source.data, indices=source.indices)
        return cls._create(source.indptr, source.indices, source.data, source.shape, lib, strategy, copy=True)

    from_scipy = copy

    @classmethod
    def wrap(cls, indptr, indices, data, shape) -> "CsrMatrix":
        """Zero-copy view: the arrays must stay alive (the wrapper keeps references)."""
        lib = _infer_library(data=data, indices=indices)
        return cls._create(indptr, indices, data, shape, lib, BlockStrategy.CONTIGUOUS, copy=False)

    @classmethod
    def _create(cls, indptr, indices, data, shape, lib, strategy, copy) -> "CsrMatrix":
        rows, cols = shape
        real = np.float64 if lib.real_type == ctypes.c_double else np.float32
        idx = np.int64 if lib.index_type == ctypes.c_int64 else np.int32
        data = np.ascontiguousarray(data, dtype=real)
        indptr = np.ascontiguousarray(indptr, dtype=idx)
        indices = np.ascontiguousarray(indices, dtype=idx)
        P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
        h = ctypes.c_void_p()
        if copy:
            check_error(lib.scl_sparse_create_with_strategy(ctypes.byref(h), rows, cols, len(data),
                                                            P(indptr, lib.index_type), P(indices, lib.index_type),
                                                            P(data, lib.real_type), 1, int(strategy)),
                        "create CSR matrix", lib)
            return cls(h, lib, OwnershipMode.OWNED)
        check_error(lib.scl_sparse_wrap(ctypes.byref(h), rows, cols, len(data), P(indptr, lib.index_type),
                                        P(indices, lib.index_type), P(data, lib.real_type), 1),
                    "wrap CSR matrix", lib)
        return cls(h, lib, OwnershipMode.WRAPPED, data_refs=[data, indptr, indices])

    def transpose(self) -> "CsrMatrix":
        """scl_sparse_transpose: same entries, primary and secondary swapped (a CSC handle)."""
        h = ctypes.c_void_p()
        check_error(self._lib.scl_sparse_transpose(self._handle, ctypes.byref(h)), "transpose", self._lib)
        return CsrMatrix(h, self._lib, OwnershipMode.OWNED, is_csr=not self._is_csr)

    # ---- export --------------------------------------------------------------
    def to_arrays(self):
        rows, cols = self.shape
        pdim = rows if self._is_csr else cols
        nnz = self.nnz
        indptr = np.empty(pdim + 1, self.index_dtype)
        indices = np.empty(max(nnz, 1), self.index_dtype)
        data = np.empty(max(nnz, 1), self.real_dtype)
        L = self._lib
        check_error(L.scl_sparse_export(self._handle, indptr.ctypes.data_as(ctypes.POINTER(L.index_type)),
                                        indices.ctypes.data_as(ctypes.POINTER(L.index_type)),
                                        data.ctypes.data_as(ctypes.POINTER(L.real_type))), "export", L)
        return indptr, indices[:nnz], data[:nnz]

    def to_scipy(self):
        import scipy.sparse as sp

        indptr, indices, data = self.to_arrays()
        if self._is_csr:
            return sp.csr_matrix((data, indices, indptr), shape=self.shape)
        return sp.csc_matrix((data, indices, indptr), shape=self.shape)

    # ---- lifecycle --------------------------------------------------------------
    def close(self):
        if self._handle is not None and self._handle.value:
            self._lib.scl_sparse_destroy(ctypes.byref(self._handle))
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __repr__(self):
        return f"<CsrMatrix shape={self.shape} nnz={self.nnz} variant={self._lib.variant}>"
