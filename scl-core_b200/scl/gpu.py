"""Device-resident graphs driven from torch tensors (scl_gpu.h).

torch supplies device memory and the current CUDA stream; every computation is
one of the library's own kernels, reached through the C ABI with raw pointers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .core.error import check_error
from ._bindings._loader import get_library

F32, F64, BF16, F16, I32, I64 = 0, 1, 2, 3, 4, 5


def _torch():
    import torch

    return torch


def dtype_code(t) -> int:
    torch = _torch()
    return {torch.float32: F32, torch.float64: F64, torch.bfloat16: BF16, torch.float16: F16, torch.int32: I32,
            torch.int64: I64}[t]


def torch_dtype(code: int):
    torch = _torch()
    return {F32: torch.float32, F64: torch.float64, BF16: torch.bfloat16, F16: torch.float16}[code]


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class GpuGraph:
    """A transition / affinity graph resident on the current CUDA device."""

    def __init__(self, handle: ctypes.c_void_p, lib):
        self._h = handle
        self._lib = lib
        self.storage = None

    @property
    def lib(self):
        return self._lib

    @property
    def handle(self):
        return self._h

    # ---- construction ---------------------------------------------------------
    @classmethod
    def from_knn(cls, knn_idx, knn_dist, variant: str = "f32_i32", stream=None) -> "GpuGraph":
        torch = _torch()
        lib = get_library(variant)
        idx = knn_idx.to(device="cuda", dtype=torch.int32).contiguous()
        dist = knn_dist.to(device="cuda", dtype=torch.float32).contiguous()
        n, k = idx.shape
        h = ctypes.c_void_p()
        check_error(lib.scl_gpu_graph_from_knn(ctypes.byref(h), n, k, _ptr(idx), _ptr(dist), _stream_ptr(stream)),
                    "graph_from_knn", lib)
        g = cls(h, lib)
        g.storage = F32
        return g

    @classmethod
    def from_csr(cls, indptr, indices, values, shape, variant: str = "f32_i32", stream=None) -> "GpuGraph":
        """From host NumPy arrays or CUDA tensors (values f32 or f64)."""
        lib = get_library(variant)
        n_rows, n_cols = shape
        h = ctypes.c_void_p()
        if isinstance(indptr, np.ndarray):
            indptr = np.ascontiguousarray(indptr)
            indices = np.ascontiguousarray(indices)
            values = np.ascontiguousarray(values)
            code = {np.dtype(np.int32): I32, np.dtype(np.int64): I64, np.dtype(np.float32): F32,
                    np.dtype(np.float64): F64}
            rc = lib.scl_gpu_graph_from_csr(ctypes.byref(h), n_rows, n_cols, values.size,
                                            ctypes.c_void_p(indptr.ctypes.data), code[indptr.dtype],
                                            ctypes.c_void_p(indices.ctypes.data), code[indices.dtype],
                                            ctypes.c_void_p(values.ctypes.data), code[values.dtype], 0,
                                            _stream_ptr(stream))
        else:
            indptr, indices, values = indptr.contiguous(), indices.contiguous(), values.contiguous()
            rc = lib.scl_gpu_graph_from_csr(ctypes.byref(h), n_rows, n_cols, values.numel(), _ptr(indptr),
                                            dtype_code(indptr.dtype), _ptr(indices), dtype_code(indices.dtype),
                                            _ptr(values), dtype_code(values.dtype), 1, _stream_ptr(stream))
        check_error(rc, "graph_from_csr", lib)
        g = cls(h, lib)
        g.storage = F32 if (values.dtype == np.float32 or str(values.dtype) == "torch.float32") else F64
        return g

    # ---- queries / transforms ------------------------------------------------------
    @property
    def shape(self):
        r, c, z = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check_error(self._lib.scl_gpu_graph_shape(self._h, ctypes.byref(r), ctypes.byref(c), ctypes.byref(z)),
                    "graph_shape", self._lib)
        return r.value, c.value, z.value

    def normalize(self, symmetric: bool = False, degree_mode: int = 0, stream=None) -> "GpuGraph":
        check_error(self._lib.scl_gpu_graph_normalize(self._h, int(symmetric), int(degree_mode), _stream_ptr(stream)),
                    "graph_normalize", self._lib)
        return self

    def set_storage(self, dtype, stream=None) -> "GpuGraph":
        code = dtype if isinstance(dtype, int) else dtype_code(dtype)
        check_error(self._lib.scl_gpu_graph_set_storage(self._h, code, _stream_ptr(stream)), "set_storage", self._lib)
        self.storage = code
        return self

    def reorder(self, mode: int = 1, stream=None) -> "GpuGraph":
        """Group rows by connected component for the diffusion (results unchanged)."""
        check_error(self._lib.scl_gpu_graph_reorder(self._h, int(mode), _stream_ptr(stream)), "reorder", self._lib)
        return self

    def set_plan(self, n_features: int, group: int, vec: int = 1, kind: int = 0, stage: int = 8) -> "GpuGraph":
        """Launch shape used by diffuse() at this width and storage dtype (group <= 0: default)."""
        check_error(self._lib.scl_gpu_graph_set_plan(self._h, int(n_features), int(group), int(vec), int(kind),
                                                     int(stage)), "set_plan", self._lib)
        return self

    def reorder_info(self):
        """(perm new->old as int32 array, component-labelling rounds)."""
        n = self.shape[0]
        perm = np.empty(n, np.int32)
        rounds = ctypes.c_int()
        check_error(self._lib.scl_gpu_graph_reorder_info(self._h, ctypes.c_void_p(perm.ctypes.data),
                                                         ctypes.byref(rounds), _stream_ptr()), "reorder_info",
                    self._lib)
        return perm, rounds.value

    def export(self, master_dtype=np.float32):
        """(indptr int64, indices int32, values) as host NumPy arrays."""
        n, _, nnz = self.shape
        indptr = np.empty(n + 1, np.int64)
        indices = np.empty(max(nnz, 1), np.int32)
        values = np.empty(max(nnz, 1), master_dtype)
        check_error(self._lib.scl_gpu_graph_export(self._h, ctypes.c_void_p(indptr.ctypes.data),
                                                   ctypes.c_void_p(indices.ctypes.data),
                                                   ctypes.c_void_p(values.ctypes.data), 0, _stream_ptr()),
                    "graph_export", self._lib)
        return indptr, indices[:nnz], values[:nnz]

    # ---- compute -----------------------------------------------------------------------
    def diffuse(self, X, n_steps: int, out=None, out_dtype=None, stream=None):
        """P^n_steps X for a CUDA tensor X (n x F); returns a new tensor unless `out` is given."""
        torch = _torch()
        X = X.contiguous()
        n, F = X.shape
        if out is None:
            od = out_dtype if out_dtype is not None else torch_dtype(self.storage)
            out = torch.empty((n, F), dtype=od, device=X.device)
        check_error(self._lib.scl_gpu_diffuse(self._h, _ptr(X), dtype_code(X.dtype), _ptr(out), dtype_code(out.dtype),
                                              F, int(n_steps), _stream_ptr(stream)), "diffuse", self._lib)
        return out

    def spmm(self, X, out, group: int = 0, vec: int = 1, kind: int = 0, stage: int = 8, stream=None):
        """One Y = P X in the original row order with an explicit launch shape (group <= 0: default)."""
        F = X.shape[1]
        check_error(self._lib.scl_gpu_spmm(self._h, _ptr(X), _ptr(out), dtype_code(out.dtype), F, int(group), int(vec),
                                           int(kind), int(stage), _stream_ptr(stream)), "spmm", self._lib)
        return out

    # ---- lifecycle -------------------------------------------------------------------------
    def close(self):
        if self._h is not None and self._h.value:
            self._lib.scl_gpu_graph_destroy(ctypes.byref(self._h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
