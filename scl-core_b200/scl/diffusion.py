"""NumPy-level diffusion calls through the drop-in C ABI (scl_diffusion.h).

Each function takes a ``CsrMatrix`` and NumPy arrays in host memory, exactly as
a caller of scl-core's ``scl_diffusion_*`` functions would, and runs on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .core.error import check_error
from .core.sparse import CsrMatrix


def _as_real(mat: CsrMatrix, X: np.ndarray) -> np.ndarray:
    if X.dtype != mat.real_dtype or not X.flags["C_CONTIGUOUS"] or not X.flags["WRITEABLE"]:
        raise TypeError(f"X must be a writeable C-contiguous {np.dtype(mat.real_dtype).name} array")
    return X


def compute_transition_matrix(mat: CsrMatrix, symmetric: bool = False) -> None:
    """In-place row (or symmetric) normalisation of the handle's values."""
    check_error(mat.lib.scl_diffusion_compute_transition_matrix(mat.handle, int(bool(symmetric))),
                "compute_transition_matrix", mat.lib)


def diffuse_matrix(mat: CsrMatrix, X: np.ndarray, n_steps: int) -> np.ndarray:
    """X <- P^n_steps X in place (n x F row-major); returns X."""
    X = _as_real(mat, X)
    n, F = X.shape
    P = ctypes.POINTER(mat.lib.real_type)
    check_error(mat.lib.scl_diffusion_diffuse_matrix(mat.handle, X.ctypes.data_as(P), n, F, int(n_steps)),
                "diffuse_matrix", mat.lib)
    return X


def diffuse_vector(mat: CsrMatrix, x: np.ndarray, n_steps: int) -> np.ndarray:
    x = _as_real(mat, x)
    P = ctypes.POINTER(mat.lib.real_type)
    check_error(mat.lib.scl_diffusion_diffuse_vector(mat.handle, x.ctypes.data_as(P), x.shape[0], int(n_steps)),
                "diffuse_vector", mat.lib)
    return x


def magic_impute(mat: CsrMatrix, X: np.ndarray, t: int = 0) -> np.ndarray:
    X = _as_real(mat, X)
    n, F = X.shape
    P = ctypes.POINTER(mat.lib.real_type)
    check_error(mat.lib.scl_diffusion_magic_impute(mat.handle, X.ctypes.data_as(P), n, F, int(t)),
                "magic_impute", mat.lib)
    return X


def compute_dpt(mat: CsrMatrix, root: int, n_nodes: int = None, max_iter: int = 100, tol: float = 1e-6) -> np.ndarray:
    """Diffusion pseudotime from `root` in [0, 1] (scl_diffusion_compute_dpt)."""
    lib = mat.lib
    n = mat.shape[0] if n_nodes is None else int(n_nodes)
    out = np.zeros(n, dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_compute_dpt(mat.handle, int(root), out.ctypes.data_as(ctypes.POINTER(lib.real_type)),
                                              n, int(max_iter), tol), "compute_dpt", lib)
    return out


def compute_dpt_multi_root(mat: CsrMatrix, roots, n_nodes: int = None, max_iter: int = 100) -> np.ndarray:
    """Mean diffusion pseudotime over `roots` (scl_diffusion_compute_dpt_multi_root)."""
    lib = mat.lib
    n = mat.shape[0] if n_nodes is None else int(n_nodes)
    roots = np.ascontiguousarray(roots, dtype=mat.index_dtype)
    out = np.zeros(n, dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_compute_dpt_multi_root(
        mat.handle, roots.ctypes.data_as(ctypes.POINTER(lib.index_type)), roots.size,
        out.ctypes.data_as(ctypes.POINTER(lib.real_type)), n, int(max_iter)), "compute_dpt_multi_root", lib)
    return out


def diffusion_map_embedding(mat: CsrMatrix, n_components: int, n_iter: int = 50, n_nodes: int = None) -> np.ndarray:
    """n x n_components diffusion-map coordinates (scl_diffusion_diffusion_map_embedding)."""
    lib = mat.lib
    n = mat.shape[0] if n_nodes is None else int(n_nodes)
    out = np.zeros((n, int(n_components)), dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_diffusion_map_embedding(mat.handle, out.ctypes.data_as(ctypes.POINTER(lib.real_type)),
                                                          n, int(n_components), int(n_iter)),
                "diffusion_map_embedding", lib)
    return out


def diffusion_distance(mat: CsrMatrix, n_steps: int = 3) -> np.ndarray:
    """n x n pairwise diffusion distances (scl_diffusion_diffusion_distance)."""
    lib = mat.lib
    n = mat.shape[0]
    out = np.zeros((n, n), dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_diffusion_distance(mat.handle, out.ctypes.data_as(ctypes.POINTER(lib.real_type)), n,
                                                     int(n_steps)), "diffusion_distance", lib)
    return out


def random_walk_with_restart(mat: CsrMatrix, seeds, n_nodes: int = None, alpha: float = 0.85, max_iter: int = 100,
                             tol: float = 1e-6) -> np.ndarray:
    """Scores of the walk that restarts on `seeds` (scl_diffusion_random_walk_with_restart)."""
    lib = mat.lib
    n = mat.shape[0] if n_nodes is None else int(n_nodes)
    seeds = np.ascontiguousarray(seeds, dtype=mat.index_dtype)
    out = np.zeros(n, dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_random_walk_with_restart(
        mat.handle, seeds.ctypes.data_as(ctypes.POINTER(lib.index_type)), seeds.size,
        out.ctypes.data_as(ctypes.POINTER(lib.real_type)), n, alpha, int(max_iter), tol),
        "random_walk_with_restart", lib)
    return out


def personalized_pagerank(mat: CsrMatrix, seed: int, n_nodes: int = None, alpha: float = 0.85, max_iter: int = 100,
                          tol: float = 1e-6) -> np.ndarray:
    lib = mat.lib
    n = mat.shape[0] if n_nodes is None else int(n_nodes)
    out = np.zeros(n, dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_personalized_pagerank(mat.handle, int(seed),
                                                        out.ctypes.data_as(ctypes.POINTER(lib.real_type)), n, alpha,
                                                        int(max_iter), tol), "personalized_pagerank", lib)
    return out


def heat_kernel_signature(mat: CsrMatrix, n_nodes: int = None, t: float = 1.0, n_steps: int = 10) -> np.ndarray:
    lib = mat.lib
    n = mat.shape[0] if n_nodes is None else int(n_nodes)
    out = np.zeros(n, dtype=mat.real_dtype)
    check_error(lib.scl_diffusion_heat_kernel_signature(mat.handle, out.ctypes.data_as(ctypes.POINTER(lib.real_type)),
                                                        n, t, int(n_steps)), "heat_kernel_signature", lib)
    return out


def lazy_random_walk(mat: CsrMatrix, x: np.ndarray, n_steps: int, laziness: float = 0.5) -> np.ndarray:
    """x <- laziness x + (1 - laziness) P x, n_steps times, in place; returns x."""
    x = _as_real(mat, x)
    P = ctypes.POINTER(mat.lib.real_type)
    check_error(mat.lib.scl_diffusion_lazy_random_walk(mat.handle, x.ctypes.data_as(P), x.shape[0], int(n_steps),
                                                       laziness), "lazy_random_walk", mat.lib)
    return x


def set_degree_mode(mat_or_lib, mode: int) -> None:
    """0 = FP64 degrees (default), 1 = value-type degrees as scl-core computes them."""
    lib = getattr(mat_or_lib, "lib", mat_or_lib)
    check_error(lib.scl_diffusion_gpu_set_degree_mode(int(mode)), "set_degree_mode", lib)


def set_reorder(mat_or_lib, mode: int) -> None:
    """-1 = automatic (default), 0 = off, 1 = always; results are identical either way."""
    lib = getattr(mat_or_lib, "lib", mat_or_lib)
    check_error(lib.scl_diffusion_gpu_set_reorder(int(mode)), "set_reorder", lib)


def attach(mat: CsrMatrix) -> None:
    check_error(mat.lib.scl_diffusion_gpu_attach(mat.handle), "attach", mat.lib)


def detach(mat: CsrMatrix) -> None:
    check_error(mat.lib.scl_diffusion_gpu_detach(mat.handle), "detach", mat.lib)


def last_stats(lib) -> dict:
    ms, h2d, d2h = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    check_error(lib.scl_diffusion_gpu_last_stats(ctypes.byref(ms), ctypes.byref(h2d), ctypes.byref(d2h)),
                "last_stats", lib)
    return {"device_ms": ms.value, "h2d_bytes": h2d.value, "d2h_bytes": d2h.value}
