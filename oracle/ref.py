"""ORACLE — test infrastructure only.

ctypes front-end of scl-core's OWN diffusion implementation, compiled from the
reference sources (scl/binding/c_api/{diffusion,core/core,core/sparse,algebra,impute}.cpp)
into ``oracle/_ref/libscl_ref_<real>_<index>_<isa>.so`` by ``oracle/Makefile``.
It is driven exactly the way the reference's Python wrapper drives it
(python/scl/core/sparse.py:420-459): zero-copy ``scl_sparse_wrap`` of
contiguous CSR arrays, then the ``scl_diffusion_*`` entry points.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
REF_DIR = _HERE / "_ref"

_REAL = {"f32": (np.float32, ctypes.c_float), "f64": (np.float64, ctypes.c_double)}
_INDEX = {"i32": (np.int32, ctypes.c_int32), "i64": (np.int64, ctypes.c_int64)}


def host_isa() -> str:
    """'avx512' when the host has the x86-64-v4 feature set, else 'avx2'."""
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
        need = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}
        return "avx512" if need <= flags else "avx2"
    except OSError:
        return "avx2"


def available(variant: str = "f32_i32") -> bool:
    return (REF_DIR / f"libscl_ref_{variant}_{host_isa()}.so").exists()


class RefError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"scl error {code}: {msg}")
        self.code = code
        self.msg = msg


class RefLib:
    """One reference variant (e.g. 'f32_i32')."""

    def __init__(self, variant: str = "f32_i32", isa: str | None = None):
        real, index = variant.split("_")
        self.variant = variant
        self.real_dtype, self.c_real = _REAL[real]
        self.index_dtype, self.c_index = _INDEX[index]
        path = REF_DIR / f"libscl_ref_{variant}_{isa or host_isa()}.so"
        if not path.exists():
            raise RuntimeError(f"reference library missing: {path} (run `make -C oracle ref`)")
        self.path = path
        L = ctypes.CDLL(str(path))
        P = ctypes.c_void_p
        I = self.c_index
        L.scl_sparse_wrap.argtypes = [ctypes.POINTER(P), I, I, I, P, P, P, ctypes.c_int]
        L.scl_sparse_create_with_strategy.argtypes = [ctypes.POINTER(P), I, I, I, P, P, P, ctypes.c_int, ctypes.c_int]
        L.scl_sparse_destroy.argtypes = [ctypes.POINTER(P)]
        L.scl_sparse_transpose.argtypes = [P, ctypes.POINTER(P)]
        L.scl_sparse_export.argtypes = [P, P, P, P]
        L.scl_sparse_nnz.argtypes = [P, ctypes.POINTER(I)]
        L.scl_sparse_is_contiguous.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
        L.scl_diffusion_compute_transition_matrix.argtypes = [P, ctypes.c_int]
        L.scl_diffusion_diffuse_matrix.argtypes = [P, P, I, I, I]
        L.scl_diffusion_diffuse_vector.argtypes = [P, P, ctypes.c_size_t, I]
        L.scl_diffusion_magic_impute.argtypes = [P, P, I, I, I]
        L.scl_algebra_spmm.argtypes = [P, P, I, P, self.c_real, self.c_real]
        L.scl_impute_diffusion.argtypes = [P, P, I, I, I, P]
        R_ = self.c_real
        L.scl_diffusion_random_walk_with_restart.argtypes = [P, P, ctypes.c_size_t, P, ctypes.c_size_t, R_, I, R_]
        L.scl_diffusion_personalized_pagerank.argtypes = [P, I, P, ctypes.c_size_t, R_, I, R_]
        L.scl_diffusion_lazy_random_walk.argtypes = [P, P, ctypes.c_size_t, I, R_]
        L.scl_diffusion_heat_kernel_signature.argtypes = [P, P, ctypes.c_size_t, R_, I]
        L.scl_diffusion_compute_dpt.argtypes = [P, I, P, ctypes.c_size_t, I, R_]
        L.scl_knn.argtypes = [P, P, ctypes.c_size_t, ctypes.c_size_t, P, P]
        L.scl_diffusion_diffusion_map_embedding.argtypes = [P, P, I, I, I]
        L.scl_diffusion_diffusion_distance.argtypes = [P, P, ctypes.c_size_t, I]
        L.scl_neighbors_compute_norms.argtypes = [P, P]
        L.scl_diffusion_compute_dpt_multi_root.argtypes = [P, P, ctypes.c_size_t, P, ctypes.c_size_t, I]
        L.scl_impute_magic.argtypes = [P, P, I, I, I, P]
        L.scl_impute_knn.argtypes = [P, P, P, I, I, I, P, self.c_real, self.c_real]
        L.scl_get_last_error.restype = ctypes.c_char_p
        for fn in ("scl_sparse_wrap", "scl_sparse_create_with_strategy", "scl_sparse_destroy",
                   "scl_sparse_transpose", "scl_sparse_export", "scl_sparse_nnz", "scl_sparse_is_contiguous",
                   "scl_diffusion_compute_transition_matrix", "scl_diffusion_diffuse_matrix",
                   "scl_diffusion_diffuse_vector", "scl_diffusion_magic_impute", "scl_algebra_spmm",
                   "scl_impute_diffusion", "scl_impute_magic", "scl_impute_knn",
                   "scl_diffusion_random_walk_with_restart",
                   "scl_diffusion_personalized_pagerank", "scl_diffusion_lazy_random_walk",
                   "scl_diffusion_heat_kernel_signature", "scl_diffusion_compute_dpt",
                   "scl_diffusion_compute_dpt_multi_root", "scl_knn", "scl_neighbors_compute_norms",
                   "scl_diffusion_diffusion_map_embedding", "scl_diffusion_diffusion_distance"):
            getattr(L, fn).restype = ctypes.c_int32
        self.L = L

    # -- helpers --------------------------------------------------------
    def _check(self, code):
        if code != 0:
            raise RefError(code, self.L.scl_get_last_error().decode())

    def wrap(self, indptr, indices, data, shape, is_csr=True):
        """Zero-copy handle; returns (handle, keepalive arrays)."""
        indptr = np.ascontiguousarray(indptr, self.index_dtype)
        indices = np.ascontiguousarray(indices, self.index_dtype)
        data = np.ascontiguousarray(data, self.real_dtype)
        h = ctypes.c_void_p()
        self._check(self.L.scl_sparse_wrap(ctypes.byref(h), shape[0], shape[1], int(data.size),
                                           indptr.ctypes.data, indices.ctypes.data, data.ctypes.data,
                                           1 if is_csr else 0))
        return h, (indptr, indices, data)

    def destroy(self, h):
        self.L.scl_sparse_destroy(ctypes.byref(h))

    # -- the diffusion path ---------------------------------------------
    def transition(self, indptr, indices, data, n, symmetric=False):
        """Reference scl_diffusion_compute_transition_matrix on a wrapped copy."""
        data = np.array(data, dtype=self.real_dtype, copy=True)
        h, keep = self.wrap(indptr, indices, data, (n, n))
        try:
            self._check(self.L.scl_diffusion_compute_transition_matrix(h, 1 if symmetric else 0))
            return np.array(keep[2], copy=True)
        finally:
            self.destroy(h)

    def diffuse_matrix(self, indptr, indices, data, X, steps, n_nodes=None, is_csr=True):
        X = np.array(X, dtype=self.real_dtype, copy=True, order="C")
        n = X.shape[0] if n_nodes is None else n_nodes
        F = X.shape[1]
        h, keep = self.wrap(indptr, indices, data, (n, n), is_csr=is_csr)
        try:
            self._check(self.L.scl_diffusion_diffuse_matrix(h, X.ctypes.data, n, F, steps))
            return X
        finally:
            self.destroy(h)

    def diffuse_transpose(self, indptr, indices, data, X, steps):
        """P^T applied `steps` times: diffuse_matrix on scl_sparse_transpose(P)."""
        X = np.array(X, dtype=self.real_dtype, copy=True, order="C")
        n, F = X.shape
        h, keep = self.wrap(indptr, indices, data, (n, n))
        t = ctypes.c_void_p()
        try:
            self._check(self.L.scl_sparse_transpose(h, ctypes.byref(t)))
            self._check(self.L.scl_diffusion_diffuse_matrix(t, X.ctypes.data, n, F, steps))
            return X
        finally:
            self.destroy(t)
            self.destroy(h)

    def diffuse_vector(self, indptr, indices, data, x, steps):
        x = np.array(x, dtype=self.real_dtype, copy=True)
        n = x.shape[0]
        h, keep = self.wrap(indptr, indices, data, (n, n))
        try:
            self._check(self.L.scl_diffusion_diffuse_vector(h, x.ctypes.data, n, steps))
            return x
        finally:
            self.destroy(h)

    def magic_impute(self, indptr, indices, data, X, t):
        X = np.array(X, dtype=self.real_dtype, copy=True, order="C")
        n, F = X.shape
        h, keep = self.wrap(indptr, indices, data, (n, n))
        try:
            self._check(self.L.scl_diffusion_magic_impute(h, X.ctypes.data, n, F, t))
            return X
        finally:
            self.destroy(h)

    def spmm(self, indptr, indices, data, shape, X, alpha=1.0, beta=0.0):
        X = np.ascontiguousarray(X, self.real_dtype)
        Y = np.zeros((shape[0], X.shape[1]), self.real_dtype)
        h, keep = self.wrap(indptr, indices, data, shape)
        try:
            self._check(self.L.scl_algebra_spmm(h, X.ctypes.data, X.shape[1], Y.ctypes.data, alpha, beta))
            return Y
        finally:
            self.destroy(h)

    def impute_knn(self, x_csr, x_shape, x_is_csr, nbr, dist, n_cells, n_genes, bandwidth, threshold):
        hx, kx = self.wrap(*x_csr, x_shape, is_csr=x_is_csr)
        nbr = np.ascontiguousarray(nbr, self.index_dtype)
        dist = np.ascontiguousarray(dist, self.real_dtype)
        out = np.zeros((n_cells, n_genes), self.real_dtype)
        try:
            self._check(self.L.scl_impute_knn(hx, nbr.ctypes.data, dist.ctypes.data, n_cells, n_genes, nbr.shape[1],
                                              out.ctypes.data, bandwidth, threshold))
            return out
        finally:
            self.destroy(hx)

    def impute(self, kind, x_csr, x_shape, x_is_csr, t_csr, n_cells, n_genes, steps):
        """scl_impute_diffusion (kind 'diffusion') or scl_impute_magic on
        wrapped copies: x_csr / t_csr are (indptr, indices, data) triples."""
        hx, kx = self.wrap(*x_csr, x_shape, is_csr=x_is_csr)
        ht, kt = self.wrap(*t_csr, (n_cells, n_cells))
        out = np.zeros((n_cells, n_genes), self.real_dtype)
        fn = self.L.scl_impute_diffusion if kind == "diffusion" else self.L.scl_impute_magic
        try:
            self._check(fn(hx, ht, n_cells, n_genes, steps, out.ctypes.data))
            return out
        finally:
            self.destroy(ht)
            self.destroy(hx)

    def walk(self, kind, indptr, indices, data, n, out_len=None, **kw):
        """The vector walks on a wrapped n x n handle: kind 'rwr' (seeds, alpha,
        max_iter, tol), 'ppr' (seed, alpha, max_iter, tol), 'lazy' (x, steps,
        laziness) or 'hks' (t, steps). Returns the output vector."""
        h, keep = self.wrap(indptr, indices, data, (n, n))
        m = n if out_len is None else out_len
        try:
            if kind == "lazy":
                out = np.array(kw["x"], dtype=self.real_dtype, copy=True)
                self._check(self.L.scl_diffusion_lazy_random_walk(h, out.ctypes.data, out.size, kw["steps"],
                                                                  kw.get("laziness", 0.5)))
                return out
            out = np.full(m, -7.0, self.real_dtype)
            if kind == "dpt":
                self._check(self.L.scl_diffusion_compute_dpt(h, kw["root"], out.ctypes.data, m,
                                                             kw.get("max_iter", 100), kw.get("tol", 1e-6)))
            elif kind == "dpt_multi":
                roots = np.ascontiguousarray(kw["roots"], self.index_dtype)
                self._check(self.L.scl_diffusion_compute_dpt_multi_root(h, roots.ctypes.data, roots.size,
                                                                        out.ctypes.data, m, kw.get("max_iter", 100)))
            elif kind == "hks":
                self._check(self.L.scl_diffusion_heat_kernel_signature(h, out.ctypes.data, m, kw.get("t", 1.0),
                                                                       kw.get("steps", 10)))
            elif kind == "ppr":
                self._check(self.L.scl_diffusion_personalized_pagerank(h, kw["seed"], out.ctypes.data, m,
                                                                       kw.get("alpha", 0.85), kw.get("max_iter", 100),
                                                                       kw.get("tol", 1e-6)))
            else:
                seeds = np.ascontiguousarray(kw["seeds"], self.index_dtype)
                self._check(self.L.scl_diffusion_random_walk_with_restart(
                    h, seeds.ctypes.data, seeds.size, out.ctypes.data, m, kw.get("alpha", 0.85),
                    kw.get("max_iter", 100), kw.get("tol", 1e-6)))
            return out
        finally:
            self.destroy(h)

    def diffusion_map(self, indptr, indices, data, n, K, n_iter):
        h, keep = self.wrap(indptr, indices, data, (n, n))
        out = np.zeros((n, K), self.real_dtype)
        try:
            self._check(self.L.scl_diffusion_diffusion_map_embedding(h, out.ctypes.data, n, K, n_iter))
            return out
        finally:
            self.destroy(h)

    def diffusion_distance(self, indptr, indices, data, n, steps):
        h, keep = self.wrap(indptr, indices, data, (n, n))
        out = np.zeros((n, n), self.real_dtype)
        try:
            self._check(self.L.scl_diffusion_diffusion_distance(h, out.ctypes.data, n, steps))
            return out
        finally:
            self.destroy(h)

    def knn(self, indptr, indices, data, shape, k, norms=None):
        """scl_knn on a wrapped samples x features CSR (norms from
        scl_neighbors_compute_norms unless given): (indices, distances, norms)."""
        h, keep = self.wrap(indptr, indices, data, shape)
        n = shape[0]
        try:
            if norms is None:
                norms = np.zeros(n, self.real_dtype)
                self._check(self.L.scl_neighbors_compute_norms(h, norms.ctypes.data))
            norms = np.ascontiguousarray(norms, self.real_dtype)
            idx = np.zeros(n * k, self.index_dtype)
            dist = np.zeros(n * k, self.real_dtype)
            self._check(self.L.scl_knn(h, norms.ctypes.data, n, k, idx.ctypes.data, dist.ctypes.data))
            return idx.reshape(n, k), dist.reshape(n, k), norms
        finally:
            self.destroy(h)

    def create_transition_error(self, indptr, indices, data, n, strategy=3):
        """(code, message) of compute_transition_matrix on a block-allocated copy."""
        indptr = np.ascontiguousarray(indptr, self.index_dtype)
        indices = np.ascontiguousarray(indices, self.index_dtype)
        data = np.ascontiguousarray(data, self.real_dtype)
        h = ctypes.c_void_p()
        self._check(self.L.scl_sparse_create_with_strategy(ctypes.byref(h), n, n, int(data.size),
                                                           indptr.ctypes.data, indices.ctypes.data,
                                                           data.ctypes.data, 1, strategy))
        try:
            code = self.L.scl_diffusion_compute_transition_matrix(h, 0)
            return code, self.L.scl_get_last_error().decode()
        finally:
            self.destroy(h)
