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
        """Reorder rows for the diffusion (results unchanged): 1 = connected components together, longest
        rows first inside each; 2 = longest rows first across the graph; 0 = off."""
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

    def autotune(self, n_features: int, reps: int = 3, stream=None) -> dict:
        """Pick the fastest bit-identical launch shape for this width and storage dtype."""
        k, st, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check_error(self._lib.scl_gpu_graph_autotune(self._h, int(n_features), int(reps), ctypes.byref(k),
                                                     ctypes.byref(st), ctypes.byref(ms), _stream_ptr(stream)),
                    "autotune", self._lib)
        return {"kind": k.value, "stage": st.value, "ms": ms.value}

    def spmm_status(self, stream=None):
        """(code, warp) of the bulk-copy SpMM's bounded waits in this graph's
        library since the last call (0 = none); synchronises and clears."""
        code, warp = ctypes.c_int(0), ctypes.c_int(0)
        check_error(self._lib.scl_gpu_spmm_status(ctypes.byref(code), ctypes.byref(warp), _stream_ptr(stream)),
                    "spmm_status", self._lib)
        return code.value, warp.value

    def inject_spmm_stall(self, warp: int, stream=None) -> "GpuGraph":
        """Test hook: global warp `warp` of later bulk-copy SpMM launches
        expects more bytes than it copies, so its first wait runs out (-1 = off)."""
        check_error(self._lib.scl_gpu_spmm_inject_stall(int(warp), _stream_ptr(stream)), "spmm_inject_stall",
                    self._lib)
        return self

    def gather_floor(self, n_features: int, dtype=None, reps: int = 5, stream=None) -> float:
        """Median ms of gathering one n_features-wide row per stored entry in
        diffusion order (the memory-system floor of one SpMM step)."""
        code = F32 if dtype is None else (dtype if isinstance(dtype, int) else dtype_code(dtype))
        ms = ctypes.c_double()
        check_error(self._lib.scl_gpu_graph_gather_floor(self._h, int(n_features), code, int(reps), ctypes.byref(ms),
                                                         _stream_ptr(stream)), "gather_floor", self._lib)
        return ms.value

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

    def set_weights(self, values, stream=None) -> "GpuGraph":
        """Replace the pre-normalisation weights (nnz entries in CSR order; host
        NumPy array or CUDA tensor, f32/f64). The graph is un-normalised after."""
        if isinstance(values, np.ndarray):
            values = np.ascontiguousarray(values)
            code = F32 if values.dtype == np.float32 else F64
            rc = self._lib.scl_gpu_graph_set_weights(self._h, ctypes.c_void_p(values.ctypes.data), code, 0,
                                                     _stream_ptr(stream))
        else:
            values = values.contiguous()
            rc = self._lib.scl_gpu_graph_set_weights(self._h, _ptr(values), dtype_code(values.dtype), 1,
                                                     _stream_ptr(stream))
        check_error(rc, "set_weights", self._lib)
        return self

    @staticmethod
    def checkpoint_slots(n_steps: int, every: int, keep_last: bool = True) -> int:
        """Blocks diffuse_checkpointed keeps: X_every, X_2every, ... and, with
        keep_last, the last segment's iterates after its checkpoint."""
        if n_steps <= 0 or every < 1:
            return 0
        nc = (n_steps - 1) // every
        return nc + ((n_steps - 1 - nc * every) if keep_last else 0)

    def diffuse_checkpointed(self, X0, n_steps: int, every: int, out=None, checkpoints=None, keep_last: bool = True,
                             stream=None):
        """(Y, checkpoints): Y = P^n_steps X0 keeping the iterates diffuse_backward needs."""
        torch = _torch()
        X0 = X0.contiguous()
        n, F = X0.shape
        Y = out if out is not None else torch.empty_like(X0)
        k = self.checkpoint_slots(n_steps, every, keep_last)
        if checkpoints is None:
            checkpoints = torch.empty((max(k, 0), n, F), dtype=X0.dtype, device=X0.device)
        cp = _ptr(checkpoints) if k > 0 else ctypes.c_void_p(0)
        check_error(self._lib.scl_gpu_diffuse_checkpointed(self._h, _ptr(X0), _ptr(Y), F, int(n_steps), int(every),
                                                           int(keep_last), cp, _stream_ptr(stream)),
                    "diffuse_checkpointed", self._lib)
        return Y, checkpoints

    def diffuse_backward(self, X0, checkpoints, dY, n_steps: int, every: int, need_dW: bool = True,
                         keep_last: bool = True, stream=None):
        """(dX0, dW or None) for the diffusion run by diffuse_checkpointed (same every / keep_last)."""
        torch = _torch()
        X0, dY = X0.contiguous(), dY.contiguous()
        n, F = X0.shape
        dX0 = torch.empty_like(X0)
        dW = torch.empty(self.shape[2], dtype=X0.dtype, device=X0.device) if need_dW else None
        k = self.checkpoint_slots(n_steps, every, keep_last)
        cp = _ptr(checkpoints) if k > 0 else ctypes.c_void_p(0)
        check_error(self._lib.scl_gpu_diffuse_backward(self._h, _ptr(X0), cp, _ptr(dY), F, int(n_steps), int(every),
                                                       int(keep_last), _ptr(dX0),
                                                       _ptr(dW) if dW is not None else ctypes.c_void_p(0),
                                                       _stream_ptr(stream)), "diffuse_backward", self._lib)
        return dX0, dW

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


def residual_fp64(X, X_ref, rel_floor: float = 1e-3, variant: str = "f32_i32", stream=None) -> dict:
    """FP64 error of a device block X (f32/f64/bf16/f16) against an FP64 device
    block X_ref of the same shape, reduced on the device (scl_gpu_residual_fp64).

    Returns rel_fro = ||X - X_ref|| / ||X_ref||, max_rel = max |x - r| /
    max(|r|, rel_floor), max_abs and ref_fro. Synchronises the stream."""
    torch = _torch()
    if X.shape != X_ref.shape or X_ref.dtype != torch.float64:
        raise ValueError("X_ref must be float64 with X's shape")
    X = X.contiguous()
    X_ref = X_ref.contiguous()
    n = X.shape[0]
    F = X.numel() // max(n, 1)
    lib = get_library(variant)
    out = (ctypes.c_double * 4)()
    check_error(lib.scl_gpu_residual_fp64(_ptr(X), dtype_code(X.dtype), _ptr(X_ref), int(n), int(F),
                                          float(rel_floor), out, _stream_ptr(stream)), "residual_fp64", lib)
    return {"rel_fro": out[0], "max_rel": out[1], "max_abs": out[2], "ref_fro": out[3]}


def warp_schedule(indptr, rows_per_group: int, n_warps: int, variant: str = "f32_i32"):
    """The per-warp schedule of row groups the SpMM plan kinds 9, 10, 12 and 14
    follow on a reordered graph (scl_gpu_warp_schedule; host only).

    Returns (offsets, groups): warp w's list is groups[offsets[w]:offsets[w + 1]]."""
    ip = np.ascontiguousarray(indptr, dtype=np.int64)
    n = ip.size - 1
    ng = (n + rows_per_group - 1) // rows_per_group
    out = np.empty(int(n_warps) + 1 + ng, np.int32)
    lib = get_library(variant)
    check_error(lib.scl_gpu_warp_schedule(ctypes.c_void_p(ip.ctypes.data), int(n), int(rows_per_group), int(n_warps),
                                          ctypes.c_void_p(out.ctypes.data), int(out.size)), "warp_schedule", lib)
    return out[: n_warps + 1].copy(), out[n_warps + 1:].copy()


class GpuBatch:
    """Many independent graphs diffused together in one persistent, CUDA-graph
    replayed launch (scl_gpu_batch_*). Blocks are the graphs' n_b x F blocks
    stacked row-wise; `row_offsets[b]` is graph b's first row."""

    def __init__(self, graphs, n_features: int, n_steps: int, stream=None):
        if not graphs:
            raise ValueError("a batch needs at least one graph")
        self._lib = graphs[0].lib
        self._graphs = list(graphs)  # keep the handles alive (the batch holds copies, not references)
        arr = (ctypes.c_void_p * len(graphs))(*[g.handle.value for g in graphs])
        h = ctypes.c_void_p()
        check_error(self._lib.scl_gpu_batch_create(ctypes.byref(h), len(graphs), ctypes.cast(arr, ctypes.c_void_p),
                                                   int(n_features), int(n_steps), _stream_ptr(stream)),
                    "batch_create", self._lib)
        self._h = h
        self.n_features, self.n_steps = int(n_features), int(n_steps)
        offs = np.empty(len(graphs) + 1, np.int64)
        nnz, tiles = ctypes.c_int64(), ctypes.c_int64()
        check_error(self._lib.scl_gpu_batch_layout(self._h, ctypes.c_void_p(offs.ctypes.data), ctypes.byref(nnz),
                                                   ctypes.byref(tiles)), "batch_layout", self._lib)
        self.row_offsets = offs
        self.nnz_total = nnz.value

    @property
    def n_rows(self) -> int:
        return int(self.row_offsets[-1])

    def schedule(self) -> dict:
        t, u, gr, lpr, ms = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check_error(self._lib.scl_gpu_batch_schedule(self._h, ctypes.byref(t), ctypes.byref(u), ctypes.byref(gr),
                                                     ctypes.byref(lpr), ctypes.byref(ms)), "batch_schedule", self._lib)
        offs = np.empty(len(self._graphs) + 1, np.int64)
        tiles = ctypes.c_int64()
        check_error(self._lib.scl_gpu_batch_layout(self._h, ctypes.c_void_p(offs.ctypes.data), None,
                                                   ctypes.byref(tiles)), "batch_layout", self._lib)
        return {"tile_nnz": t.value, "unroll": u.value, "grid": gr.value, "lanes_per_row": lpr.value,
                "tuned_ms": ms.value, "tiles_per_step": tiles.value}

    def set_schedule(self, tile_nnz: int, unroll: int = 8, blocks_per_sm: int = 0, stream=None) -> "GpuBatch":
        check_error(self._lib.scl_gpu_batch_set_schedule(self._h, int(tile_nnz), int(unroll), int(blocks_per_sm),
                                                         _stream_ptr(stream)), "batch_set_schedule", self._lib)
        return self

    def autotune(self, X0, Y, reps: int = 3, stream=None) -> dict:
        check_error(self._lib.scl_gpu_batch_autotune(self._h, _ptr(X0), _ptr(Y), int(reps), _stream_ptr(stream)),
                    "batch_autotune", self._lib)
        return self.schedule()

    def solve(self, X0, out=None, stream=None):
        torch = _torch()
        X0 = X0.contiguous()
        Y = out if out is not None else torch.empty_like(X0)
        check_error(self._lib.scl_gpu_batch_solve(self._h, _ptr(X0), _ptr(Y), _stream_ptr(stream)), "batch_solve",
                    self._lib)
        return Y

    def status(self, stream=None):
        """(code, item): synchronises the stream; 0 = every wait completed."""
        c, i = ctypes.c_int(), ctypes.c_int()
        check_error(self._lib.scl_gpu_batch_status(self._h, ctypes.byref(c), ctypes.byref(i), _stream_ptr(stream)),
                    "batch_status", self._lib)
        return c.value, i.value

    def inject_stall(self, graph: int) -> "GpuBatch":
        """Failure-path test hook: graph `graph`'s waits never complete (-1 = off)."""
        check_error(self._lib.scl_gpu_batch_inject_stall(self._h, int(graph)), "batch_inject_stall", self._lib)
        return self

    def close(self):
        if self._h is not None and self._h.value:
            self._lib.scl_gpu_batch_destroy(ctypes.byref(self._h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
