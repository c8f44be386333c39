"""Diffusion map embedding through the drop-in C ABI on the GPU against
scl-core's own scl_diffusion_diffusion_map_embedding (compiled from the
reference sources and shipped with the tests). The GPU reduces the
Gram-Schmidt dot products in FP64 blocks where the reference sums
sequentially in the value type, and its starting cosines come from CUDA's
cos/sin, so the two agree to a tolerance, not bit for bit; both outputs are
orthonormal. Against scl-core's FP64 build the FP32 GPU result is within 1e-5
of the largest entry, and no further from it than scl-core's own FP32 build."""
import numpy as np
import pytest
import scipy.sparse as sp

import scl
from oracle import ref

pytestmark = pytest.mark.gpu


def _graph(n, dt, idt, seed):
    rng = np.random.default_rng(seed)
    pts = np.concatenate([rng.standard_normal((n // 2, 5)), rng.standard_normal((n - n // 2, 5)) + 4.0])
    d2 = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    W = np.exp(-d2 / 4.0) * (d2 < 9.0)
    np.fill_diagonal(W, 0.0)
    P = sp.csr_matrix(W / W.sum(1, keepdims=True)).astype(dt)
    P.sort_indices()
    m = scl.CsrMatrix.wrap(P.indptr.astype(idt), P.indices.astype(idt), P.data, P.shape)
    return m, P


@pytest.mark.parametrize("dt,idt,tol", [(np.float32, np.int32, 1e-6), (np.float64, np.int64, 1e-8)])
@pytest.mark.parametrize("n,K,n_iter", [(200, 3, 10), (400, 6, 50), (300, 1, 0)])
def test_diffusion_map_matches_reference(dt, idt, tol, n, K, n_iter):
    variant = "f32_i32" if dt == np.float32 else "f64_i64"
    m, P = _graph(n, dt, idt, seed=n + K)
    got = scl.diffusion.diffusion_map_embedding(m, K, n_iter)
    G = got.astype(np.float64)
    np.testing.assert_allclose(G.T @ G, np.eye(K), atol=50 * tol)
    if not ref.available(variant):
        pytest.skip("reference library not shipped with the tests")
    want = ref.RefLib(variant).diffusion_map(P.indptr, P.indices, P.data, n, K, n_iter)
    np.testing.assert_allclose(got, want, atol=tol, rtol=0)
    if dt == np.float32 and ref.available("f64_i64"):
        # whose error: both FP32 results against scl-core's FP64 build of the same P
        want64 = ref.RefLib("f64_i64").diffusion_map(P.indptr.astype(np.int64), P.indices.astype(np.int64),
                                                     P.data.astype(np.float64), n, K, n_iter)
        err_gpu = np.abs(got - want64).max()
        err_ref32 = np.abs(want - want64).max()
        assert err_gpu <= 1e-5 * np.abs(want64).max()
        assert err_gpu <= 2.0 * err_ref32 + 1e-7


def test_diffusion_map_errors():
    m, _ = _graph(20, np.float32, np.int32, 1)
    out = np.zeros((20, 2), np.float32)
    import ctypes

    lib = m.lib
    P = out.ctypes.data_as(ctypes.POINTER(lib.real_type))
    assert lib.scl_diffusion_diffusion_map_embedding(None, P, 20, 2, 5) == 4
    assert lib.scl_diffusion_diffusion_map_embedding(m.handle, None, 20, 2, 5) == 4
    assert lib.scl_diffusion_diffusion_map_embedding(m.handle, P, 0, 2, 5) == 10
    assert lib.scl_diffusion_diffusion_map_embedding(m.handle, P, 20, 0, 5) == 10
    assert lib.scl_diffusion_diffusion_map_embedding(m.handle, P, 19, 2, 5) == 11


@pytest.mark.parametrize("dt,idt", [(np.float32, np.int32), (np.float64, np.int64)])
def test_diffusion_distance_small_graph_bit_exact_with_reference(dt, idt):
    """n <= 1000: the reference diffuses the identity with spmm_block (the
    library's SpMM gives the same bits) and sums the rounded squares of row
    differences in order. In FP64 the GPU output equals it bit for bit; in FP32
    0.05 % of the entries of this graph differ by one ulp, which a sequential
    multiply-add restatement in NumPy reproduces as well (the reference's own
    compiled loop rounds a few of those sums differently)."""
    variant = "f32_i32" if dt == np.float32 else "f64_i64"
    m, P = _graph(300, dt, idt, seed=4)
    got = scl.diffusion.diffusion_distance(m, 3)
    assert np.all(np.diag(got) == 0) and np.array_equal(got, got.T)
    if not ref.available(variant):
        pytest.skip("reference library not shipped with the tests")
    want = ref.RefLib(variant).diffusion_distance(P.indptr, P.indices, P.data, 300, 3)
    if dt == np.float64:
        np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    else:
        np.testing.assert_array_max_ulp(got, want, maxulp=1)
        assert np.mean(got == want) > 0.99


def test_diffusion_distance_large_graph_compares_columns():
    """n > 1000: the reference's row-by-row branch diffuses unit vectors, so it
    compares columns of P^t; checked against an FP64 restatement."""
    m, P = _graph(1100, np.float64, np.int64, seed=5)
    got = scl.diffusion.diffusion_distance(m, 2)
    Z = np.eye(1100)
    for _ in range(2):
        Z = P @ Z
    C = Z.T  # column i of P^t as row i
    sq = (C * C).sum(1)
    want = np.sqrt(np.maximum(sq[:, None] + sq[None, :] - 2 * C @ C.T, 0))
    np.testing.assert_allclose(got, want, atol=1e-7)
