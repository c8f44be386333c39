"""ORACLE — test infrastructure only.

NumPy front-end of the C restatement in ``diffusion_oracle.c`` (built into
``oracle/_build/liboracle_port.so`` by ``make -C oracle port``). All index
arrays are converted to int64; every function returns new arrays.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "liboracle_port.so"
_lib = None

F32, BF16, F16 = 0, 2, 3

_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int

_SIGS = {
    "oracle_row_sums_f32": ([_i64, _p, _p, _p], None),
    "oracle_row_sums_f64": ([_i64, _p, _p, _p], None),
    "oracle_transition_f32": ([_i64, _p, _p, _p, _int, _int], None),
    "oracle_transition_f64": ([_i64, _p, _p, _p, _int], None),
    "oracle_spmm_f32": ([_i64, _p, _p, _p, _p, _p, _i64], None),
    "oracle_spmm_f64": ([_i64, _p, _p, _p, _p, _p, _i64], None),
    "oracle_diffuse_matrix_f32": ([_i64, _p, _p, _p, _p, _i64, _i64], None),
    "oracle_diffuse_matrix_f64": ([_i64, _p, _p, _p, _p, _i64, _i64], None),
    "oracle_diffuse_lowp": ([_i64, _p, _p, _p, _p, _p, _i64, _i64, _int, _int], None),
    "oracle_diffuse_lowp_chains": ([_i64, _p, _p, _p, _p, _p, _i64, _i64, _int, _int, _int], None),
    "oracle_f32_to_bf16": ([ctypes.c_float], ctypes.c_uint16),
    "oracle_bf16_to_f32": ([ctypes.c_uint16], ctypes.c_float),
    "oracle_f32_to_f16": ([ctypes.c_float], ctypes.c_uint16),
    "oracle_f16_to_f32": ([ctypes.c_uint16], ctypes.c_float),
    "oracle_gauss_weights_f64": ([_i64, _i64, _p, _p, _p, _p], None),
    "oracle_gauss_weights_f32": ([_i64, _i64, _p, _p, _p, _p], None),
    "oracle_symmetrize_f64": ([_i64, _i64, _p, _p, _p, _p, _p], _i64),
    "oracle_symmetrize_f32": ([_i64, _i64, _p, _p, _p, _p, _p], _i64),
    "oracle_adjoint_f64": ([_i64, _p, _p, _p, _int, _p, _p, _i64, _i64, _p, _p], ctypes.c_double),
    "oracle_walk_linear_f32": ([_i64, _p, _p, _p, _p, _i64, ctypes.c_float, ctypes.c_float], None),
    "oracle_walk_linear_f64": ([_i64, _p, _p, _p, _p, _i64, ctypes.c_double, ctypes.c_double], None),
    "oracle_walk_restart_f32": ([_i64, _p, _p, _p, _p, _p, ctypes.c_float, _i64, ctypes.c_float], _i64),
    "oracle_walk_restart_f64": ([_i64, _p, _p, _p, _p, _p, ctypes.c_double, _i64, ctypes.c_double], _i64),
    "oracle_dpt_f32": ([_i64, _p, _p, _p, _i64, _i64, ctypes.c_float, _p], None),
    "oracle_dpt_f64": ([_i64, _p, _p, _p, _i64, _i64, ctypes.c_double, _p], None),
    "oracle_algebra_spmm_f32": ([_i64, _p, _p, _p, _p, _i64, _p, ctypes.c_float, ctypes.c_float], None),
    "oracle_algebra_spmm_f64": ([_i64, _p, _p, _p, _p, _i64, _p, ctypes.c_double, ctypes.c_double], None),
    "oracle_knn_dense_f32": ([_i64, _i64, _p, _p, _i64, _int, _p, _p], None),
    "oracle_knn_dense_f64": ([_i64, _i64, _p, _p, _i64, _int, _p, _p], None),
}


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(f"oracle port library missing: {_LIB_PATH} (run `make -C oracle port`)")
        _lib = ctypes.CDLL(str(_LIB_PATH))
        for name, (argt, rest) in _SIGS.items():
            fn = getattr(_lib, name)
            fn.argtypes = argt
            fn.restype = rest
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _csr(indptr, indices):
    return (np.ascontiguousarray(indptr, dtype=np.int64),
            np.ascontiguousarray(indices, dtype=np.int64))


def row_sums(indptr, values):
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    n = indptr.size - 1
    if values.dtype == np.float32:
        out = np.empty(n, np.float32)
        lib().oracle_row_sums_f32(n, _ptr(indptr), _ptr(values), _ptr(out))
    else:
        values = np.ascontiguousarray(values, dtype=np.float64)
        out = np.empty(n, np.float64)
        lib().oracle_row_sums_f64(n, _ptr(indptr), _ptr(values), _ptr(out))
    return out


def transition(indptr, indices, values, symmetric=False, degree_fp64=False):
    """Normalised copy of ``values`` (diffusion.hpp:492-603)."""
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    if values.dtype == np.float32:
        out = np.array(values, dtype=np.float32, copy=True)
        lib().oracle_transition_f32(n, _ptr(indptr), _ptr(indices), _ptr(out), int(symmetric), int(degree_fp64))
    else:
        out = np.array(values, dtype=np.float64, copy=True)
        lib().oracle_transition_f64(n, _ptr(indptr), _ptr(indices), _ptr(out), int(symmetric))
    return out


def spmm(indptr, indices, values, X):
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    X = np.ascontiguousarray(X)
    F = X.shape[1]
    Y = np.empty((n, F), X.dtype)
    if X.dtype == np.float32:
        v = np.ascontiguousarray(values, np.float32)
        lib().oracle_spmm_f32(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X), _ptr(Y), F)
    else:
        v = np.ascontiguousarray(values, np.float64)
        lib().oracle_spmm_f64(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X), _ptr(Y), F)
    return Y


def diffuse_matrix(indptr, indices, values, X, steps):
    """X_steps = P^steps X0 (diffusion.hpp:638-664); dtype follows X."""
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    X = np.array(X, copy=True, order="C")
    F = X.shape[1] if X.ndim == 2 else 1
    if X.dtype == np.float32:
        v = np.ascontiguousarray(values, np.float32)
        lib().oracle_diffuse_matrix_f32(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X), F, steps)
    else:
        v = np.ascontiguousarray(values, np.float64)
        lib().oracle_diffuse_matrix_f64(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X), F, steps)
    return X


def diffuse_lowp(indptr, indices, values_f32, X0_f32, steps, kind, final_f32=True):
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    v = np.ascontiguousarray(values_f32, np.float32)
    X0 = np.ascontiguousarray(X0_f32, np.float32)
    F = X0.shape[1]
    Y = np.empty((n, F), np.float32)
    lib().oracle_diffuse_lowp(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X0), _ptr(Y), F, steps,
                              int(kind), int(final_f32))
    return Y


def diffuse_lowp_chains(indptr, indices, values_f32, X0_f32, steps, kind, chains, final_f32=True):
    """16-bit storage diffusion with `chains` interleaved fma chains per row
    (oracle_diffuse_lowp_chains)."""
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    v = np.ascontiguousarray(values_f32, np.float32)
    X0 = np.ascontiguousarray(X0_f32, np.float32)
    F = X0.shape[1]
    Y = np.empty((n, F), np.float32)
    lib().oracle_diffuse_lowp_chains(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X0), _ptr(Y), F, steps,
                                     int(kind), int(final_f32), int(chains))
    return Y


def to_bf16_bits(x):
    f = lib().oracle_f32_to_bf16
    return np.array([f(float(v)) for v in np.asarray(x, np.float32).ravel()], np.uint16)


def to_f16_bits(x):
    f = lib().oracle_f32_to_f16
    return np.array([f(float(v)) for v in np.asarray(x, np.float32).ravel()], np.uint16)


def gauss_weights(knn_idx, knn_dist):
    """(sigma, w) for an n x k kNN list; FP64 when knn_dist is float64."""
    knn_idx = np.ascontiguousarray(knn_idx, np.int64)
    n, k = knn_idx.shape
    if knn_dist.dtype == np.float32:
        d = np.ascontiguousarray(knn_dist, np.float32)
        sigma = np.empty(n, np.float32)
        w = np.empty((n, k), np.float32)
        lib().oracle_gauss_weights_f32(n, k, _ptr(knn_idx), _ptr(d), _ptr(sigma), _ptr(w))
    else:
        d = np.ascontiguousarray(knn_dist, np.float64)
        sigma = np.empty(n, np.float64)
        w = np.empty((n, k), np.float64)
        lib().oracle_gauss_weights_f64(n, k, _ptr(knn_idx), _ptr(d), _ptr(sigma), _ptr(w))
    return sigma, w


def symmetrize(knn_idx, w):
    """CSR (indptr, indices, values) of (W + W^T)/2 over the kNN union."""
    knn_idx = np.ascontiguousarray(knn_idx, np.int64)
    n, k = knn_idx.shape
    if w.dtype == np.float32:
        fn, dt = lib().oracle_symmetrize_f32, np.float32
    else:
        fn, dt = lib().oracle_symmetrize_f64, np.float64
    w = np.ascontiguousarray(w, dt)
    nnz = fn(n, k, _ptr(knn_idx), _ptr(w), None, None, None)
    indptr = np.empty(n + 1, np.int64)
    indices = np.empty(max(nnz, 1), np.int64)
    values = np.empty(max(nnz, 1), dt)
    fn(n, k, _ptr(knn_idx), _ptr(w), _ptr(indptr), _ptr(indices), _ptr(values))
    return indptr, indices[:nnz], values[:nnz]


def adjoint(indptr, indices, W, X0, Y, steps, symmetric=False):
    """(loss, dL/dX0, dL/dW) in FP64 for L = sum((P^steps X0 - Y)^2)."""
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    W = np.ascontiguousarray(W, np.float64)
    X0 = np.ascontiguousarray(X0, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    F = X0.shape[1]
    dX0 = np.empty_like(X0)
    dW = np.empty_like(W)
    loss = lib().oracle_adjoint_f64(n, _ptr(indptr), _ptr(indices), _ptr(W), int(symmetric), _ptr(X0), _ptr(Y),
                                    F, steps, _ptr(dX0), _ptr(dW))
    return loss, dX0, dW


# ---- imputation (scl/kernel/impute.hpp:599-735) -------------------------------
def densify(indptr, indices, values, csr, n_cells, n_genes):
    """The dense block imputation starts from (impute.hpp:608-640, 680-697):
    zero, then every stored (cell, gene) with cell < n_cells and gene < n_genes
    in stored order, so a later duplicate overwrites an earlier one. A CSR
    matrix is cells x genes, a CSC one genes-major."""
    indptr = np.asarray(indptr, np.int64)
    ind = np.asarray(indices, np.int64)
    vals = np.asarray(values)
    n_prim = min(indptr.size - 1, n_cells if csr else n_genes)
    end = int(indptr[n_prim])
    prim = np.repeat(np.arange(n_prim, dtype=np.int64), np.diff(indptr[: n_prim + 1]))
    sec, v = ind[:end], vals[:end]
    c, g = (prim, sec) if csr else (sec, prim)
    ok = (c >= 0) & (c < n_cells) & (g >= 0) & (g < n_genes)
    pos, v = c[ok] * n_genes + g[ok], v[ok]
    out = np.zeros(n_cells * n_genes, vals.dtype)
    if pos.size:
        _, first_rev = np.unique(pos[::-1], return_index=True)  # last occurrence of each position
        keep = pos.size - 1 - first_rev
        out[pos[keep]] = v[keep]
    return out.reshape(n_cells, n_genes)


def impute_diffusion(x_csr, x_is_csr, t_csr, n_cells, n_genes, steps):
    """impute.hpp:599-661: densify, then `steps` SpMMs over the transition's
    rows (each output element the sequential fma chain)."""
    X = densify(*x_csr, x_is_csr, n_cells, n_genes)
    for _ in range(steps):
        X = spmm(t_csr[0], t_csr[1], np.asarray(t_csr[2], X.dtype), X)
    return X


def impute_magic(x_csr, x_is_csr, t_csr, n_cells, n_genes, steps):
    """impute.hpp:668-735: only a CSR matrix seeds the block; affinity rows are
    summed sequentially in the value precision, weighted a * (1 / sum), and a
    row whose sum is below 1e-12 keeps its previous values."""
    dt = np.asarray(t_csr[2]).dtype
    X = densify(*x_csr, True, n_cells, n_genes) if x_is_csr else np.zeros((n_cells, n_genes), dt)
    ip = np.asarray(t_csr[0], np.int64)
    a = np.ascontiguousarray(t_csr[2], dt)
    sums = row_sums(ip, a)
    copy = sums < dt.type(1e-12)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = (dt.type(1) / sums).astype(dt)
        w = (a * np.repeat(inv, np.diff(ip))).astype(dt)
    w[np.repeat(copy, np.diff(ip))] = 0
    for _ in range(steps):
        Y = spmm(ip, t_csr[1], w, X)
        Y[copy] = X[copy]
        X = Y
    return X


# ---- vector walks (scl/kernel/diffusion.hpp:833-900, 961-1007, 1157-1194) -----
def walk_linear(indptr, indices, values, x, steps, c_x, c_p):
    """x <- fma(c_x, x, c_p * (P x)), `steps` times (lazy random walk and the
    heat-kernel signature); dtype follows x."""
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    x = np.array(x, copy=True)
    v = np.ascontiguousarray(values, x.dtype)
    fn = lib().oracle_walk_linear_f32 if x.dtype == np.float32 else lib().oracle_walk_linear_f64
    fn(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(x), int(steps), float(c_x), float(c_p))
    return x


def restart_vector(seeds, n, dtype):
    """diffusion.hpp:852-870: 1 on every in-range seed, divided by the number
    of in-range seeds (repeats counted); None when there is none."""
    r = np.zeros(n, dtype)
    count = 0
    for s in seeds:
        if 0 <= int(s) < n:
            r[int(s)] = 1
            count += 1
    if count == 0:
        return None
    return (r * (dtype(1) / dtype(count))).astype(dtype)


def walk_restart(indptr, indices, values, seeds, n, alpha, max_iter, tol, dtype=np.float32):
    """Random walk with restart as scl-core runs it (scores start as the
    restart vector; buffers swap after each unconverged step). Returns
    (scores, steps taken)."""
    indptr, indices = _csr(indptr, indices)
    r = restart_vector(seeds, n, dtype)
    if r is None:
        return np.zeros(n, dtype), 0
    scores = r.copy()
    v = np.ascontiguousarray(values, dtype)
    fn = lib().oracle_walk_restart_f32 if dtype == np.float32 else lib().oracle_walk_restart_f64
    it = fn(n, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(r), _ptr(scores), float(alpha), int(max_iter), float(tol))
    return scores, int(it)


def dpt(indptr, indices, values, root, max_iter, tol, dtype=np.float32):
    """Diffusion pseudotime from one root (diffusion.hpp:670-772)."""
    indptr, indices = _csr(indptr, indices)
    n = indptr.size - 1
    v = np.ascontiguousarray(values, dtype)
    out = np.empty(n, dtype)
    fn = lib().oracle_dpt_f32 if dtype == np.float32 else lib().oracle_dpt_f64
    fn(n, _ptr(indptr), _ptr(indices), _ptr(v), int(root), int(max_iter), float(tol), _ptr(out))
    return out


def dpt_multi_root(indptr, indices, values, roots, max_iter, dtype=np.float32):
    """diffusion.hpp:774-830: the mean of the in-range roots' pseudotimes
    (each with tol 1e-6), summed in root order then scaled by 1 / count."""
    n = np.asarray(indptr).size - 1
    valid = [int(r) for r in roots if 0 <= int(r) < n]
    if not valid:
        return np.ones(n, dtype)
    s = np.zeros(n, dtype)
    for r in valid:
        s = (s + dpt(indptr, indices, values, r, max_iter, dtype(1e-6), dtype)).astype(dtype)
    return (s * (dtype(1) / dtype(len(valid)))).astype(dtype)


def algebra_spmm(indptr, indices, values, X, Y, alpha, beta):
    """Y' = alpha A X + beta Y as scl_algebra_spmm forms it (algebra.hpp:546-600)."""
    indptr, indices = _csr(indptr, indices)
    m = indptr.size - 1
    X = np.ascontiguousarray(X)
    Yo = np.array(Y, dtype=X.dtype, copy=True, order="C")
    v = np.ascontiguousarray(values, X.dtype)
    fn = lib().oracle_algebra_spmm_f32 if X.dtype == np.float32 else lib().oracle_algebra_spmm_f64
    fn(m, _ptr(indptr), _ptr(indices), _ptr(v), _ptr(X), X.shape[1], _ptr(Yo), float(alpha), float(beta))
    return Yo


def knn_dense(X, norms, k, contract=True):
    """Brute-force kNN of the rows of dense X with the given squared norms
    (neighbors.hpp:319-478): (indices int64 [n, k], distances [n, k])."""
    X = np.ascontiguousarray(X)
    n, d = X.shape
    nr = np.ascontiguousarray(norms, X.dtype)
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), X.dtype)
    fn = lib().oracle_knn_dense_f32 if X.dtype == np.float32 else lib().oracle_knn_dense_f64
    fn(n, d, _ptr(X), _ptr(nr), int(k), int(bool(contract)), _ptr(idx), _ptr(dist))
    return idx, dist
