"""C-ABI boundary checks that need no GPU: every declared symbol is exported by
every variant, argument validation returns scl-core's codes and messages, and
the sparse-handle layer behaves like the reference's (compared live against
oracle/_ref when present)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import scl
from oracle import ref
from scl._bindings._loader import find_library, get_library

ROOT = Path(__file__).resolve().parents[1]
VARIANTS = ["f32_i32", "f32_i64", "f64_i32", "f64_i64"]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        names |= set(re.findall(r"SCL_EXPORT\s+[\w\s\*]+?\b(scl_\w+)\s*\(", txt))
    return names


def test_headers_declare_the_reference_diffusion_abi():
    names = declared_symbols()
    for sym in ["scl_diffusion_compute_transition_matrix", "scl_diffusion_diffuse_matrix",
                "scl_diffusion_diffuse_vector", "scl_diffusion_magic_impute", "scl_sparse_create",
                "scl_sparse_wrap", "scl_sparse_destroy", "scl_sparse_transpose", "scl_get_last_error",
                "scl_gpu_diffuse", "scl_gpu_graph_from_knn"]:
        assert sym in names
    assert len(names) >= 50


@pytest.mark.parametrize("variant", VARIANTS)
def test_library_exports_every_declared_symbol(variant):
    path = find_library(variant)
    assert path is not None and path.exists()
    lib = ctypes.CDLL(str(path))
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert missing == []
    lib.scl_get_build_config.restype = ctypes.c_char_p
    real, idx = variant.split("_")
    cfg = lib.scl_get_build_config().decode()
    assert cfg.startswith({"f32": "float32", "f64": "float64"}[real] + "+" + {"i32": "int32", "i64": "int64"}[idx])




def test_null_and_dimension_errors_match_reference_codes():
    lib = get_library("f32_i32")
    P = ctypes.POINTER(ctypes.c_float)
    assert lib.scl_diffusion_diffuse_matrix(None, P(), 3, 2, 1) == 4
    assert lib.scl_get_last_error() == b"Transition matrix is null"
    m = scl.CsrMatrix.wrap(np.array([0, 2, 3, 6], np.int32), np.array([0, 2, 1, 0, 1, 2], np.int32),
                           np.array([1, 2, 3, 4, 5, 6], np.float32), (3, 3))
    assert lib.scl_diffusion_diffuse_matrix(m.handle, None, 3, 2, 1) == 4
    assert lib.scl_get_last_error() == b"Matrix X is null"
    X = np.zeros((3, 2), np.float32)
    for dims in [(0, 2, 1), (3, 0, 1), (3, 2, 0), (3, 2, -1)]:
        assert lib.scl_diffusion_diffuse_matrix(m.handle, X.ctypes.data_as(P), *dims) == 10
        assert lib.scl_get_last_error() == b"Dimensions must be positive"
    assert lib.scl_diffusion_diffuse_vector(m.handle, X.ctypes.data_as(P), 0, 1) == 10
    assert lib.scl_diffusion_magic_impute(m.handle, X.ctypes.data_as(P), 3, 0, 1) == 10
    assert lib.scl_diffusion_compute_transition_matrix(None, 0) == 4
    assert lib.scl_get_last_error() == b"Adjacency matrix is null"
    assert lib.scl_diffusion_compute_dpt(m.handle, 0, None, 3, 0, 0.0) == 4
    assert lib.scl_get_last_error() == b"Output pseudotime array is null"
    assert lib.scl_diffusion_compute_dpt(m.handle, 0, X.ctypes.data_as(P), 0, 0, 0.0) == 10
    assert lib.scl_diffusion_diffusion_distance(m.handle, X.ctypes.data_as(P), 9, 0) == 10
    assert lib.scl_impute_knn(m.handle, None, None, 3, 2, 1, X.ctypes.data_as(P), 1.0, 0.0) == 4
    assert lib.scl_get_last_error() == b"KNN indices array is null"
    lib.scl_clear_error()
    assert lib.scl_get_last_error() == b"No error" and lib.scl_get_last_error_code() == 0


def test_noalloc_argument_errors_before_any_launch():
    """scl_gpu_diffuse_noalloc rejects null and overlapping buffers on the host,
    before it touches the device (the addresses below are never dereferenced)."""
    lib = get_library("f32_i32")
    fn = lib.scl_gpu_diffuse_noalloc
    ip, ix, v, X, Y = (ctypes.c_void_p(a) for a in (0x10000, 0x20000, 0x30000, 0x100000, 0x200000))
    n, F = 100, 8  # one block is 3,200 bytes
    for pos, msg in [(0, b"Offset array pointer is null"), (1, b"Indices array pointer is null"),
                     (2, b"Data array pointer is null"), (3, b"Matrix X is null"), (4, b"Matrix Y is null")]:
        args = [ip, ix, v, X, Y]
        args[pos] = None
        assert fn(args[0], args[1], args[2], n, args[3], args[4], F, 2, None) == 4
        assert lib.scl_get_last_error() == msg
    for y_addr in (0x100000, 0x100000 + 3196, 0x100000 - 3196):  # same, tail overlap, head overlap
        assert fn(ip, ix, v, n, X, ctypes.c_void_p(y_addr), F, 2, None) == 10
        assert lib.scl_get_last_error() == b"X and Y must not overlap"
    assert fn(ip, ix, v, 0, X, Y, F, 2, None) == 10
    assert fn(ip, ix, v, 8388609, X, Y, 1, 2, None) == 10
    assert b"exceeds" in lib.scl_get_last_error()


def test_sparse_create_validation():
    lib = get_library("f64_i64")
    h = ctypes.c_void_p()
    PI = ctypes.POINTER(ctypes.c_int64)
    PD = ctypes.POINTER(ctypes.c_double)
    ip = np.array([0, 2, 1, 3])  # decreasing
    ix = np.array([0, 1, 2])
    d = np.ones(3)
    rc = lib.scl_sparse_create(ctypes.byref(h), 3, 3, 3, ip.ctypes.data_as(PI), ix.ctypes.data_as(PI),
                               d.ctypes.data_as(PD), 1)
    assert rc == 10 and lib.scl_get_last_error() == b"offsets must be non-decreasing"
    rc = lib.scl_sparse_create(ctypes.byref(h), 0, 3, 3, ip.ctypes.data_as(PI), ix.ctypes.data_as(PI),
                               d.ctypes.data_as(PD), 1)
    assert rc == 10 and lib.scl_get_last_error() == b"Matrix dimensions must be positive"
    assert lib.scl_sparse_destroy(None) == 0


def _dense_sparse(n, density, seed):
    rng = np.random.default_rng(seed)
    A = (rng.random((n, n)) < density) * rng.standard_normal((n, n))
    import scipy.sparse as sp

    S = sp.csr_matrix(A)
    S.sort_indices()
    return S


@pytest.mark.parametrize("n,density", [(50, 0.2), (3000, 0.01)])
def test_block_layout_and_export_like_reference(n, density):
    S = _dense_sparse(n, density, 3)
    for strategy in (scl.BlockStrategy.CONTIGUOUS, scl.BlockStrategy.ADAPTIVE, scl.BlockStrategy.SMALL):
        m = scl.CsrMatrix.copy(S, strategy=strategy)
        ip, ix, d = m.to_arrays()
        np.testing.assert_array_equal(ip, S.indptr)
        np.testing.assert_array_equal(ix, S.indices)
        np.testing.assert_array_equal(d, S.data)
        if ref.available("f64_i64"):
            R = ref.RefLib("f64_i64")
            h = ctypes.c_void_p()
            rip, rix = S.indptr.astype(np.int64), S.indices.astype(np.int64)
            R._check(R.L.scl_sparse_create_with_strategy(ctypes.byref(h), n, n, S.nnz, rip.ctypes.data,
                                                         rix.ctypes.data, S.data.ctypes.data, 1, int(strategy)))
            c = ctypes.c_int()
            R.L.scl_sparse_is_contiguous(h, ctypes.byref(c))
            R.destroy(h)
            assert bool(c.value) == m.is_contiguous


def test_non_contiguous_transition_error_matches_reference():
    S = _dense_sparse(3000, 0.01, 4)
    S.data = np.abs(S.data)
    m = scl.CsrMatrix.copy(S, strategy=scl.BlockStrategy.ADAPTIVE)
    assert not m.is_contiguous
    with pytest.raises(scl.SCLError) as e:
        scl.diffusion.compute_transition_matrix(m)
    assert e.value.code == 10
    assert "Matrix must be contiguous for transition matrix computation" in str(e.value)
    if ref.available("f64_i64"):
        code, msg = ref.RefLib("f64_i64").create_transition_error(S.indptr, S.indices, S.data, 3000)
        assert (code, msg) == (10, "Matrix must be contiguous for transition matrix computation")


def test_transpose_matches_reference():
    S = _dense_sparse(200, 0.05, 5)
    m = scl.CsrMatrix.copy(S, strategy=scl.BlockStrategy.CONTIGUOUS)
    t = m.transpose()
    ip, ix, d = t.to_arrays()
    T = S.T.tocsr()
    T.sort_indices()
    np.testing.assert_array_equal(ip, T.indptr)
    np.testing.assert_array_equal(ix, T.indices)
    np.testing.assert_array_equal(d, T.data)


def test_no_gpu_fails_loudly(cuda_available):
    if cuda_available:
        pytest.skip("a GPU is present")
    m = scl.CsrMatrix.wrap(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32),
                           np.array([1, 1], np.float32), (2, 2))
    X = np.ones((2, 4), np.float32)
    with pytest.raises(scl.SCLError) as e:
        scl.diffusion.diffuse_matrix(m, X, 2)
    assert e.value.code == 41
