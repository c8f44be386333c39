"""Imputation through the drop-in C ABI (scl_impute_diffusion,
scl_impute_magic) on the GPU against the oracle restatement, which
test_impute_oracle.py pins to scl-core's own implementation bit for bit."""
import numpy as np
import pytest
import scipy.sparse as sp

import scl
from oracle import port, ref

pytestmark = pytest.mark.gpu

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)
VARIANTS = [(np.float32, np.int32), (np.float64, np.int64)]


def _wrap(csr, shape, idt):
    ip, ind, val = csr
    return scl.CsrMatrix.wrap(np.asarray(ip, idt), np.asarray(ind, idt), val, shape)


def _expr(rng, n_cells, n_genes, dt, density=0.3):
    X = sp.random(n_cells, n_genes, density=density, random_state=int(rng.integers(1 << 30)), format="csr",
                  dtype=np.float64).astype(dt)
    X.sort_indices()
    return (X.indptr.astype(np.int64), X.indices.astype(np.int64), X.data), X.shape


def _graph(rng, n, dt, density=0.2, empty=()):
    T = sp.random(n, n, density=density, random_state=int(rng.integers(1 << 30)), format="lil",
                  dtype=np.float64)
    for r in empty:
        T[r, :] = 0
    T = T.tocsr().astype(dt)
    T.sort_indices()
    return T.indptr.astype(np.int64), T.indices.astype(np.int64), T.data


@pytest.mark.parametrize("dt,idt", VARIANTS)
@pytest.mark.parametrize("kind", ["diffusion", "magic"])
@pytest.mark.parametrize("n_cells,n_genes", [(1, 1), (3, 3), (200, 1), (500, 64), (700, 333), (2000, 96)])
def test_impute_bit_exact(dt, idt, kind, n_cells, n_genes):
    rng = np.random.default_rng(n_cells * 7 + n_genes)
    x, shape = _expr(rng, n_cells, n_genes, dt)
    t = _graph(rng, n_cells, dt, density=min(1.0, 12.0 / n_cells), empty=(0,) if n_cells > 5 else ())
    fn = scl.impute.diffusion if kind == "diffusion" else scl.impute.magic
    ora = port.impute_diffusion if kind == "diffusion" else port.impute_magic
    M = _wrap(x, shape, idt)
    G = _wrap(t, (n_cells, n_cells), idt)
    for steps in (1, 4):
        got = fn(M, G, n_cells, n_genes, steps)
        np.testing.assert_array_equal(bits(got), bits(ora(x, True, t, n_cells, n_genes, steps).astype(dt)))


def test_reference_fixtures_and_reference_outputs():
    """The 3x3 inputs of the reference's own test_impute.cpp; when the
    reference library travels with the tests, its outputs too."""
    x = (np.array([0, 2, 3, 5]), np.array([0, 1, 0, 1, 2]), np.array([1.0, 2.0, 3.0, 4.0, 5.0]))
    cases = (("diffusion", (np.array([0, 2, 4, 6]), np.array([0, 1, 0, 2, 1, 2]), np.full(6, 0.5))),
             ("magic", (np.array([0, 2, 4, 6]), np.array([0, 1, 0, 2, 1, 2]),
                        np.array([0.8, 0.2, 0.7, 0.3, 0.6, 0.4]))))
    R = ref.RefLib("f64_i64") if ref.available("f64_i64") else None
    for kind, t in cases:
        fn = scl.impute.diffusion if kind == "diffusion" else scl.impute.magic
        got = fn(_wrap(x, (3, 3), np.int64), _wrap(t, (3, 3), np.int64), 3, 3, 2)
        ora = (port.impute_diffusion if kind == "diffusion" else port.impute_magic)(x, True, t, 3, 3, 2)
        np.testing.assert_array_equal(bits(got), bits(ora))
        if R is not None:
            np.testing.assert_array_equal(bits(got), bits(R.impute(kind, x, (3, 3), True, t, 3, 3, 2)))


@pytest.mark.parametrize("kind", ["diffusion", "magic"])
def test_csc_expression_duplicates_and_entries_outside_the_block(kind):
    rng = np.random.default_rng(9)
    n_cells, n_genes = 300, 40
    t = _graph(rng, n_cells, np.float32, density=0.05, empty=(3, 4))
    fn = scl.impute.diffusion if kind == "diffusion" else scl.impute.magic
    ora = port.impute_diffusion if kind == "diffusion" else port.impute_magic
    G = _wrap(t, (n_cells, n_cells), np.int32)
    # CSR with extra rows and columns beyond the block and duplicated positions
    X = sp.random(n_cells + 5, n_genes + 7, density=0.3, random_state=4, format="csr", dtype=np.float32)
    X.sort_indices()
    ip, ind, val = X.indptr.astype(np.int64), X.indices.astype(np.int64), X.data
    rows = [(list(ind[ip[r]:ip[r + 1]]), list(val[ip[r]:ip[r + 1]])) for r in range(X.shape[0])]
    for r, (ri, rv) in enumerate(rows):
        if ri and r % 3 == 0:
            ri.extend([ri[0]] * 40)  # a position repeated across chunks; the last value wins
            rv.extend(rng.standard_normal(40).astype(np.float32))
    ip2 = np.concatenate([[0], np.cumsum([len(ri) for ri, _ in rows])])
    ind2 = np.concatenate([np.array(ri, np.int64) for ri, _ in rows])
    val2 = np.concatenate([np.array(rv, np.float32) for _, rv in rows])
    x = (ip2, ind2, val2)
    got = fn(_wrap(x, X.shape, np.int32), G, n_cells, n_genes, 3)
    np.testing.assert_array_equal(bits(got), bits(ora(x, True, t, n_cells, n_genes, 3)))
    # the same entries as a genes-major (CSC) handle
    M = sp.random(n_genes, n_cells, density=0.3, random_state=5, format="csr", dtype=np.float32)
    M.sort_indices()
    xc = (M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data)
    # the cells x genes matrix as a CSC handle: its primary (gene-major) arrays are xc
    import ctypes

    lib = G.lib
    arrs = [np.ascontiguousarray(xc[0], np.int32), np.ascontiguousarray(xc[1], np.int32),
            np.ascontiguousarray(xc[2], np.float32)]
    h = ctypes.c_void_p()
    ptr = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    assert lib.scl_sparse_wrap(ctypes.byref(h), n_cells, n_genes, arrs[2].size, ptr(arrs[0], lib.index_type),
                               ptr(arrs[1], lib.index_type), ptr(arrs[2], lib.real_type), 0) == 0
    csc = scl.CsrMatrix(h, lib, scl.core.sparse.OwnershipMode.WRAPPED, data_refs=arrs, is_csr=False)
    got_c = fn(csc, G, n_cells, n_genes, 2)
    want_c = ora(xc, False, t, n_cells, n_genes, 2)
    np.testing.assert_array_equal(bits(got_c), bits(want_c))


def test_errors_follow_the_reference_convention():
    x = (np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, 2.0], np.float32))
    t = (np.array([0, 1, 2]), np.array([1, 0]), np.array([1.0, 1.0], np.float32))
    M, G = _wrap(x, (2, 2), np.int32), _wrap(t, (2, 2), np.int32)
    lib = M.lib
    out = np.zeros((2, 2), np.float32)
    import ctypes

    P = out.ctypes.data_as(ctypes.POINTER(lib.real_type))
    assert lib.scl_impute_diffusion(None, G.handle, 2, 2, 1, P) == 4
    assert lib.scl_impute_magic(M.handle, None, 2, 2, 1, P) == 4
    assert lib.scl_impute_magic(M.handle, G.handle, 2, 2, 1, None) == 4
    assert lib.scl_impute_diffusion(M.handle, G.handle, 0, 2, 1, P) == 10
    assert lib.scl_impute_magic(M.handle, G.handle, 2, 2, 0, P) == 10
    assert lib.scl_impute_diffusion(M.handle, G.handle, 3, 2, 1, P) == 11  # graph has 2 cells
    assert lib.scl_impute_knn(M.handle, None, None, 2, 2, 1, P, 1.0, 0.0) == 4


@pytest.mark.parametrize("dt,idt,rtol", [(np.float32, np.int32, 2e-6), (np.float64, np.int64, 1e-14)])
@pytest.mark.parametrize("csr", [True, False])
def test_knn_impute_matches_reference(dt, idt, rtol, csr):
    """scl_impute_knn (and scl_impute_knn_weighted, the same kernel in
    scl-core) against scl-core's own build: the positions imputed are the
    same and the values agree to rounding (the Gaussian weights come from
    CUDA's exp, the reference's from the C library's)."""
    if not ref.available("f32_i32" if dt == np.float32 else "f64_i64"):
        pytest.skip("reference library not shipped with the tests")
    R = ref.RefLib("f32_i32" if dt == np.float32 else "f64_i64")
    rng = np.random.default_rng(13)
    n_cells, n_genes, K = 400, 60, 8
    X = sp.random(n_cells, n_genes, density=0.3, random_state=3, format="csr", dtype=np.float64).astype(dt)
    X.sort_indices()
    X.data[::11] = 0  # stored zeros still count as expressed
    nbr = rng.integers(0, n_cells, size=(n_cells, K)).astype(np.int64)
    nbr[::17, 0] = n_cells + 3  # out-of-range neighbours are ignored
    dist = rng.random((n_cells, K)).astype(dt)
    if csr:
        x = (X.indptr.astype(np.int64), X.indices.astype(np.int64), X.data)
        shape = X.shape
        M = _wrap(x, shape, idt)
    else:
        C = X.tocsc()
        C.sort_indices()
        x = (C.indptr.astype(np.int64), C.indices.astype(np.int64), C.data)
        shape = X.shape
        import ctypes

        lib = scl.get_library("f32_i32" if dt == np.float32 else "f64_i64")
        arrs = [np.ascontiguousarray(x[0], idt), np.ascontiguousarray(x[1], idt), np.ascontiguousarray(x[2], dt)]
        h = ctypes.c_void_p()
        ptr = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
        assert lib.scl_sparse_wrap(ctypes.byref(h), n_cells, n_genes, arrs[2].size, ptr(arrs[0], lib.index_type),
                                   ptr(arrs[1], lib.index_type), ptr(arrs[2], lib.real_type), 0) == 0
        M = scl.CsrMatrix(h, lib, scl.core.sparse.OwnershipMode.WRAPPED, data_refs=arrs, is_csr=False)
    for bw, thr in ((1.0, 0.0), (0.3, 0.05)):
        want = R.impute_knn(x, shape, csr, nbr, dist, n_cells, n_genes, bw, thr)
        for weighted in (False, True):
            got = scl.impute.knn(M, nbr, dist, n_cells, n_genes, bw, thr, weighted=weighted)
            np.testing.assert_array_equal(got == 0, want == 0)
            np.testing.assert_allclose(got, want, rtol=rtol, atol=0)
