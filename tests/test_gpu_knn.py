"""Brute-force kNN through the drop-in C ABI on the GPU (scl_knn,
scl_knn_simple, scl_neighbors_compute_norms) against the restatement, which
test_knn_oracle.py pins to scl-core's own scl_knn bit for bit: indices and
distances equal, in the same order, ties included."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import scl
from oracle import port, ref

pytestmark = pytest.mark.gpu


def _matrix(n, d, dt, idt, dens=1.0, seed=0, quantised=False):
    rng = np.random.default_rng(seed)
    X = sp.random(n, d, density=dens, random_state=seed, format="csr", dtype=np.float64)
    X.data = rng.standard_normal(X.nnz)
    if quantised:
        X.data = np.round(X.data)
    X = X.astype(dt)
    X.sort_indices()
    m = scl.CsrMatrix.wrap(X.indptr.astype(idt), X.indices.astype(idt), X.data, X.shape)
    return m, X


@pytest.fixture(params=[1, 2], ids=["cuda_cores", "tensor_cores"])
def knn_kernel(request):
    """Runs a test once per kNN kernel (scl_gpu_knn_set_kernel) in every library variant."""
    prev = {v: scl.neighbors.set_kernel(request.param, v) for v in ("f32_i32", "f64_i64")}
    yield request.param
    for v, k in prev.items():
        scl.neighbors.set_kernel(k, v)


@pytest.mark.parametrize("dt,idt", [(np.float32, np.int32), (np.float64, np.int64)])
@pytest.mark.parametrize("n,d,k,dens,quant", [(1, 3, 4, 1.0, False), (12, 5, 15, 1.0, False),
                                              (300, 20, 10, 1.0, False), (700, 50, 30, 1.0, False),
                                              (400, 60, 12, 0.3, False), (500, 8, 6, 1.0, True),
                                              (2000, 128, 64, 1.0, False), (129, 1, 3, 1.0, True),
                                              (3000, 33, 40, 1.0, True)])
def test_knn_bit_exact(knn_kernel, dt, idt, n, d, k, dens, quant):
    m, X = _matrix(n, d, dt, idt, dens, seed=n + d, quantised=quant)
    Xd = X.toarray()
    norms = np.einsum("ij,ij->i", Xd.astype(np.float64), Xd.astype(np.float64)).astype(dt)
    gi, gd = scl.neighbors.knn(m, k, norms)
    oi, od = port.knn_dense(Xd, norms, k)
    np.testing.assert_array_equal(gd.view(np.uint8), od.view(np.uint8))
    np.testing.assert_array_equal(gi.astype(np.int64), oi)
    # scl_knn_simple and scl_neighbors_compute_norms: the device's norms, then the same search
    gn = scl.neighbors.compute_norms(m)
    si, sd = scl.neighbors.knn(m, k)
    oi2, od2 = port.knn_dense(Xd, gn, k)
    np.testing.assert_array_equal(sd.view(np.uint8), od2.view(np.uint8))
    np.testing.assert_array_equal(si.astype(np.int64), oi2)
    np.testing.assert_allclose(gn, norms, rtol=1e-5 if dt == np.float32 else 1e-13)


def test_knn_equals_the_reference_with_its_norms(knn_kernel):
    if not ref.available("f32_i32"):
        pytest.skip("reference library not shipped with the tests")
    R = ref.RefLib("f32_i32")
    m, X = _matrix(600, 30, np.float32, np.int32, seed=3, quantised=True)
    ri, rd, norms = R.knn(X.indptr, X.indices, X.data, X.shape, 15)
    gi, gd = scl.neighbors.knn(m, 15, norms)
    np.testing.assert_array_equal(gd.view(np.uint8), rd.view(np.uint8))
    np.testing.assert_array_equal(gi, ri)


def test_knn_errors():
    m, X = _matrix(10, 4, np.float32, np.int32)
    lib = m.lib
    idx = np.zeros(30, np.int32)
    dist = np.zeros(30, np.float32)
    nr = np.ones(10, np.float32)
    PI = idx.ctypes.data_as(ctypes.POINTER(lib.index_type))
    PD = dist.ctypes.data_as(ctypes.POINTER(lib.real_type))
    PN = nr.ctypes.data_as(ctypes.POINTER(lib.real_type))
    assert lib.scl_knn(None, PN, 10, 3, PI, PD) == 4
    assert lib.scl_knn(m.handle, None, 10, 3, PI, PD) == 4
    assert lib.scl_knn(m.handle, PN, 0, 3, PI, PD) == 10
    assert lib.scl_knn(m.handle, PN, 9, 3, PI, PD) == 11  # n_samples must be the row count
    # the CUDA-core kernel is limited to k <= 64 and 128 features; the automatic choice is not
    wide, _ = _matrix(10, 129, np.float32, np.int32)
    prev = scl.neighbors.set_kernel(1, m)
    try:
        assert lib.scl_knn(m.handle, PN, 10, 65, PI, PD) == 10
        assert lib.scl_knn_simple(wide.handle, 10, 3, PI, PD) == 10
    finally:
        scl.neighbors.set_kernel(prev, m)
    big = np.zeros(10 * 65, np.int32), np.zeros(10 * 65, np.float32)
    assert lib.scl_knn(m.handle, PN, 10, 65, big[0].ctypes.data_as(ctypes.POINTER(lib.index_type)),
                       big[1].ctypes.data_as(ctypes.POINTER(lib.real_type))) == 0
    assert lib.scl_knn_simple(wide.handle, 10, 3, PI, PD) == 0
    assert lib.scl_gpu_knn_set_kernel(3, None) == 10
    assert lib.scl_neighbors_compute_norms(None, PN) == 4


def _dense_case(n, d, dt, seed, dens=1.0, scale=1.0, dup=0):
    rng = np.random.default_rng(seed)
    Xd = rng.standard_normal((n, d)) * scale
    if dens < 1.0:
        Xd *= rng.random((n, d)) < dens
    if dup:  # repeated rows: exact distance ties and zero distances
        Xd[n - dup:] = Xd[:dup]
    Xd = Xd.astype(dt)
    X = sp.csr_matrix(Xd)
    X.sort_indices()
    idt = np.int32 if dt == np.float32 else np.int64
    m = scl.CsrMatrix.wrap(X.indptr.astype(idt), X.indices.astype(idt), X.data.astype(dt), X.shape)
    norms = np.einsum("ij,ij->i", Xd.astype(np.float64), Xd.astype(np.float64)).astype(dt)
    return m, Xd, norms


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("n,d,k,dens,scale,dup", [
    (1000, 300, 20, 1.0, 1.0, 0),       # more than 128 features
    (700, 1500, 15, 0.05, 3.0, 0),      # raw-expression-like width and sparsity
    (600, 40, 100, 1.0, 1.0, 0),        # k above 64
    (300, 17, 250, 1.0, 1.0, 0),        # k close to n
    (40, 9, 64, 1.0, 1.0, 0),           # k >= n: unfilled slots (-1, inf)
    (777, 64, 30, 1.0, 1.0, 200),       # duplicated rows: ties and zero distances
    (513, 62, 30, 1.0, 1e12, 0),        # large magnitudes (norms near 1e26)
    (900, 50, 30, 1.0, 1e-9, 0),        # tiny magnitudes
    (257, 1, 5, 1.0, 1.0, 100),         # one feature, many ties
])
def test_knn_any_width_and_k(dt, n, d, k, dens, scale, dup):
    """The tensor-core filter at sizes the CUDA-core kernel does not take (and
    at sizes it does), against the restatement, bit for bit."""
    variant = "f32_i32" if dt == np.float32 else "f64_i64"
    prev = scl.neighbors.set_kernel(2, variant)
    try:
        _any_width_case(dt, n, d, k, dens, scale, dup)
    finally:
        scl.neighbors.set_kernel(prev, variant)


def _any_width_case(dt, n, d, k, dens, scale, dup):
    m, Xd, norms = _dense_case(n, d, dt, seed=n + d + k, dens=dens, scale=scale, dup=dup)
    gi, gd = scl.neighbors.knn(m, k, norms)
    oi, od = port.knn_dense(Xd, norms, k)
    np.testing.assert_array_equal(gd.view(np.uint8), od.view(np.uint8))
    np.testing.assert_array_equal(gi.astype(np.int64), oi)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_knn_kernels_agree(dt):
    """Tensor-core filter and CUDA-core kernel: the same bits, including with
    norms that are not the rows' own (the filter's bound does not assume them)."""
    m, Xd, norms = _dense_case(3000, 50, dt, seed=5, dup=300)
    rng = np.random.default_rng(9)
    odd = (norms * rng.uniform(0.5, 2.0, norms.shape)).astype(dt)
    for nr in (norms, odd):
        prev = scl.neighbors.set_kernel(2, m)
        try:
            a = scl.neighbors.knn(m, 30, nr)
            scl.neighbors.set_kernel(1, m)
            b = scl.neighbors.knn(m, 30, nr)
        finally:
            scl.neighbors.set_kernel(prev, m)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1].view(np.uint8), b[1].view(np.uint8))


def test_knn_non_finite_values_replay_every_candidate():
    """A non-finite sample switches the filter off; the result is still the
    restatement's."""
    m0, Xd, norms = _dense_case(400, 12, np.float32, seed=2)
    Xd[7, 3] = np.inf
    norms[7] = np.inf
    X = sp.csr_matrix(Xd)
    X.sort_indices()
    m = scl.CsrMatrix.wrap(X.indptr.astype(np.int32), X.indices.astype(np.int32), X.data, X.shape)
    prev = scl.neighbors.set_kernel(2, m)
    try:
        gi, gd = scl.neighbors.knn(m, 10, norms)
    finally:
        scl.neighbors.set_kernel(prev, m)
    oi, od = port.knn_dense(Xd, norms, 10)
    np.testing.assert_array_equal(gd.view(np.uint8), od.view(np.uint8))
    np.testing.assert_array_equal(gi.astype(np.int64), oi)


def test_knn_kernels_agree_on_a_large_mixture():
    """100,000 cells of the benchmark's 50-D mixture, k = 30: the tensor-core
    filter and the exact CUDA-core kernel return the same neighbours and
    distances, bit for bit (the restatement is too slow at this size)."""
    pts = scl.synthetic.mixture(100_000, seed=5).astype(np.float32)
    n, d = pts.shape
    ip = np.arange(0, (n + 1) * d, d, dtype=np.int64).astype(np.int32)
    m = scl.CsrMatrix.wrap(ip, np.tile(np.arange(d, dtype=np.int32), n), pts.reshape(-1), (n, d))
    norms = scl.neighbors.compute_norms(m)
    prev = scl.neighbors.set_kernel(2, m)
    try:
        a = scl.neighbors.knn(m, 30, norms)
        scl.neighbors.set_kernel(1, m)
        b = scl.neighbors.knn(m, 30, norms)
    finally:
        scl.neighbors.set_kernel(prev, m)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_knn_tensor_wait_runs_out_without_fault():
    """The tensor-core kernel's bounded waits: a host-set hook keeps one CTA's
    first accumulator from ever being signalled. Its epilogue gives up after
    2 s, the CTA drains and frees its tensor memory, scl_knn returns
    SCL_ERROR_CONVERGENCE, and the library keeps working afterwards."""
    m, Xd, norms = _dense_case(3000, 20, np.float32, seed=1)
    lib = m.lib
    k = 10
    idx = np.zeros(3000 * k, np.int32)
    dist = np.zeros(3000 * k, np.float32)
    nr = np.ascontiguousarray(norms, np.float32)
    prev = scl.neighbors.set_kernel(2, m)
    try:
        assert lib.scl_gpu_knn_inject_stall(3, None) == 0
        rc = lib.scl_knn(m.handle, nr.ctypes.data_as(ctypes.POINTER(lib.real_type)), 3000, k,
                         idx.ctypes.data_as(ctypes.POINTER(lib.index_type)),
                         dist.ctypes.data_as(ctypes.POINTER(lib.real_type)))
        assert rc == 54  # SCL_ERROR_CONVERGENCE
        assert lib.scl_gpu_knn_inject_stall(-1, None) == 0
        gi, gd = scl.neighbors.knn(m, k, norms)
    finally:
        lib.scl_gpu_knn_inject_stall(-1, None)
        scl.neighbors.set_kernel(prev, m)
    oi, od = port.knn_dense(Xd, norms, k)
    np.testing.assert_array_equal(gd.view(np.uint8), od.view(np.uint8))
    np.testing.assert_array_equal(gi.astype(np.int64), oi)
