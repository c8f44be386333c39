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


@pytest.mark.parametrize("dt,idt", [(np.float32, np.int32), (np.float64, np.int64)])
@pytest.mark.parametrize("n,d,k,dens,quant", [(1, 3, 4, 1.0, False), (12, 5, 15, 1.0, False),
                                              (300, 20, 10, 1.0, False), (700, 50, 30, 1.0, False),
                                              (400, 60, 12, 0.3, False), (500, 8, 6, 1.0, True),
                                              (2000, 128, 64, 1.0, False), (129, 1, 3, 1.0, True),
                                              (3000, 33, 40, 1.0, True)])
def test_knn_bit_exact(dt, idt, n, d, k, dens, quant):
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


def test_knn_equals_the_reference_with_its_norms():
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
    assert lib.scl_knn(m.handle, PN, 10, 65, PI, PD) == 10  # this build: k <= 64
    wide, _ = _matrix(10, 129, np.float32, np.int32)
    assert lib.scl_knn_simple(wide.handle, 10, 3, PI, PD) == 10  # this build: <= 128 features
    assert lib.scl_neighbors_compute_norms(None, PN) == 4
