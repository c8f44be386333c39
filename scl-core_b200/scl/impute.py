"""NumPy-level imputation calls through the drop-in C ABI (scl_impute.h).

``diffusion`` and ``magic`` take the expression matrix and the cells graph as
``CsrMatrix`` handles and return a new dense ``n_cells x n_genes`` block, as a
caller of scl-core's ``scl_impute_diffusion`` / ``scl_impute_magic`` would get
it; the work runs on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .core.error import check_error
from .core.sparse import CsrMatrix


def _run(fn_name: str, matrix: CsrMatrix, graph: CsrMatrix, n_cells: int, n_genes: int, steps: int) -> np.ndarray:
    if matrix.lib is not graph.lib:
        raise TypeError("expression matrix and graph must use the same library variant")
    out = np.zeros((int(n_cells), int(n_genes)), dtype=matrix.real_dtype)
    P = ctypes.POINTER(matrix.lib.real_type)
    fn = getattr(matrix.lib, fn_name)
    check_error(fn(matrix.handle, graph.handle, int(n_cells), int(n_genes), int(steps), out.ctypes.data_as(P)),
                fn_name, matrix.lib)
    return out


def diffusion(matrix: CsrMatrix, transition: CsrMatrix, n_cells: int, n_genes: int, n_steps: int) -> np.ndarray:
    """T^n_steps X0 with X0 the dense form of ``matrix`` (scl_impute_diffusion)."""
    return _run("scl_impute_diffusion", matrix, transition, n_cells, n_genes, n_steps)


def magic(matrix: CsrMatrix, affinity: CsrMatrix, n_cells: int, n_genes: int, t: int) -> np.ndarray:
    """MAGIC: t steps over the row-normalised affinity (scl_impute_magic)."""
    return _run("scl_impute_magic", matrix, affinity, n_cells, n_genes, t)


def knn(matrix: CsrMatrix, knn_indices: np.ndarray, knn_distances: np.ndarray, n_cells: int, n_genes: int,
        bandwidth: float = 1.0, threshold: float = 0.0, weighted: bool = False) -> np.ndarray:
    """kNN imputation (scl_impute_knn, or scl_impute_knn_weighted, which scl-core
    runs with the same kernel): values not above `threshold` become the
    Gaussian-weighted mean of the neighbours that store the gene."""
    lib = matrix.lib
    idx = np.ascontiguousarray(knn_indices, dtype=matrix.index_dtype)
    dist = np.ascontiguousarray(knn_distances, dtype=matrix.real_dtype)
    out = np.zeros((int(n_cells), int(n_genes)), dtype=matrix.real_dtype)
    fn = lib.scl_impute_knn_weighted if weighted else lib.scl_impute_knn
    check_error(fn(matrix.handle, idx.ctypes.data_as(ctypes.POINTER(lib.index_type)),
                   dist.ctypes.data_as(ctypes.POINTER(lib.real_type)), int(n_cells), int(n_genes), idx.shape[1],
                   out.ctypes.data_as(ctypes.POINTER(lib.real_type)), bandwidth, threshold),
                "impute_knn", lib)
    return out
