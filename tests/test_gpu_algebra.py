"""scl_algebra_spmm through the drop-in C ABI on the GPU against the
restatement (bit for bit), which test_algebra_oracle.py pins to scl-core."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import scl
from oracle import port

pytestmark = pytest.mark.gpu

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)


@pytest.mark.parametrize("dt,idt", [(np.float32, np.int32), (np.float64, np.int64)])
@pytest.mark.parametrize("m,kdim,K", [(1, 1, 1), (50, 40, 7), (3000, 2000, 64), (700, 900, 129)])
def test_algebra_spmm_bit_exact(dt, idt, m, kdim, K):
    rng = np.random.default_rng(m + K)
    A = sp.random(m, kdim, density=min(1.0, 20.0 / kdim), random_state=3, format="csr", dtype=np.float64).astype(dt)
    A.sort_indices()
    A.data[::5] = 0
    M = scl.CsrMatrix.wrap(A.indptr.astype(idt), A.indices.astype(idt), A.data, A.shape)
    X = rng.standard_normal((kdim, K)).astype(dt)
    for alpha, beta in ((1.0, 0.0), (0.5, 2.0), (2.0, 1.0), (0.0, 3.0), (-1.5, 0.25)):
        Y0 = rng.standard_normal((m, K)).astype(dt)
        got = scl.algebra.spmm(M, X, Y0.copy(), alpha, beta)
        np.testing.assert_array_equal(bits(got), bits(port.algebra_spmm(A.indptr, A.indices, A.data, X, Y0,
                                                                         dt(alpha), dt(beta))))


def test_algebra_spmm_errors():
    A = sp.random(4, 3, density=0.5, random_state=1, format="csr", dtype=np.float32)
    M = scl.CsrMatrix.wrap(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, A.shape)
    lib = M.lib
    X = np.zeros((3, 2), np.float32)
    Y = np.zeros((4, 2), np.float32)
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(lib.real_type))
    assert lib.scl_algebra_spmm(None, P(X), 2, P(Y), 1.0, 0.0) == 4
    assert lib.scl_algebra_spmm(M.handle, None, 2, P(Y), 1.0, 0.0) == 4
    assert lib.scl_algebra_spmm(M.handle, P(X), 2, None, 1.0, 0.0) == 4
    assert lib.scl_algebra_spmm(M.handle, P(X), 0, P(Y), 1.0, 0.0) == 10
