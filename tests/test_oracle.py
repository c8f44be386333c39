"""The oracle (C restatement) pinned against scl-core itself: its known-answer
tests, golden vectors produced by its compiled code, and live runs of
oracle/_ref when present. CPU only."""
import numpy as np
import pytest

from oracle import port, ref

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)


# ---- known-answer tests from the reference's own test suite -------------------
def test_kat_spmm_tiny_3x3(golden):
    # tests/c_api/src/test_algebra.cpp:281-307 on tests/c_api/include/data.hpp:350-363
    ip, ix = np.array([0, 2, 3, 6]), np.array([0, 2, 1, 0, 1, 2])
    d = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    X = np.array([[1.0, 2.0], [3.0, 4.0], [5.0, 6.0]])
    Y = port.spmm(ip, ix, d, X)
    np.testing.assert_array_equal(Y, [[11, 14], [9, 12], [49, 64]])
    np.testing.assert_array_equal(Y, golden["kat_spmm"])
    # one diffusion step is one SpMM (diffusion.hpp:638-664)
    np.testing.assert_array_equal(port.diffuse_matrix(ip, ix, d, X, 1), Y)
    np.testing.assert_array_equal(port.diffuse_matrix(ip, ix, d.astype(np.float32), X.astype(np.float32), 1), Y)


def test_kat_spmv_tiny_3x3():
    # tests/c_api/src/test_algebra.cpp:73-108: A x = [7, 6, 32]
    ip, ix = np.array([0, 2, 3, 6]), np.array([0, 2, 1, 0, 1, 2])
    d = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    y = port.diffuse_matrix(ip, ix, d, np.array([[1.0], [2.0], [3.0]]), 1)[:, 0]
    np.testing.assert_array_equal(y, [7, 6, 32])


def test_kat_gaussian_at_zero_distance():
    # tests/c_api/src/test_kernel.cpp:369-386: K(0) = 1 for the Gaussian kernel
    _, w = port.gauss_weights(np.array([[1, 2]]), np.array([[0.0, 1.0]]))
    assert w[0, 0] == 1.0
    _, w32 = port.gauss_weights(np.array([[1, 2]]), np.array([[0.0, 1.0]], np.float32))
    assert w32[0, 0] == 1.0


# ---- golden vectors generated by the reference build --------------------------
@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("sym", [False, True])
def test_transition_matches_golden(golden, tag, sym):
    g = golden
    P = port.transition(g["indptr"], g["indices"], g[f"W_{tag}"], symmetric=sym, degree_fp64=False)
    np.testing.assert_array_equal(bits(P), bits(g[f"P_{'sym' if sym else 'row'}_{tag}"]))


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_diffuse_matches_golden(golden, tag):
    g = golden
    X = port.diffuse_matrix(g["indptr"], g["indices"], g[f"P_row_{tag}"], g[f"X0_{tag}"], int(g["T"]))
    np.testing.assert_array_equal(bits(X), bits(g[f"XT_{tag}"]))


def test_transpose_diffuse_matches_golden(golden):
    import scipy.sparse as sp

    g = golden
    n = int(g["n"])
    PT = sp.csr_matrix((g["P_row_f32"].astype(np.float64), g["indices"], g["indptr"]), shape=(n, n)).T.tocsr()
    PT.sort_indices()
    X = port.diffuse_matrix(PT.indptr, PT.indices, PT.data.astype(np.float32), g["X0_f32"], 2)
    np.testing.assert_array_equal(bits(X), bits(g["XT_csc_f32"]))


def test_diffuse_vector_golden_within_tolerance(golden):
    # scl-core's SpMV (diffusion.hpp:169-221) lets GCC's vectoriser fuse some
    # products and not others, so only a tolerance is meaningful here.
    g = golden
    x = port.diffuse_matrix(g["indptr"], g["indices"], g["P_row_f32"], g["X0_f32"][:, :1], 3)[:, 0]
    np.testing.assert_allclose(x, g["xv_f32"], rtol=1e-5, atol=1e-7)


def test_symmetrize_matches_scipy(golden):
    import scipy.sparse as sp

    g = golden
    n, k = int(g["n"]), int(g["k"])
    _, w = port.gauss_weights(g["knn_idx"], g["knn_dist"])
    W = sp.csr_matrix((w.ravel(), (np.repeat(np.arange(n), k), g["knn_idx"].ravel())), shape=(n, n))
    S = ((W + W.T) * 0.5).tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(S.indptr, g["indptr"])
    np.testing.assert_array_equal(S.indices, g["indices"])
    np.testing.assert_allclose(S.data, g["W_f64"], rtol=1e-15)


def test_symmetrize_edge_cases():
    # padded lists (-1), self loops and duplicate neighbours
    idx = np.array([[1, -1, 1], [0, 2, -1], [2, 0, 1], [-1, -1, -1]])
    w = np.array([[0.5, 9.0, 0.25], [1.0, 2.0, 9.0], [4.0, 3.0, 8.0], [9.0, 9.0, 9.0]])
    ip, ind, val = port.symmetrize(idx, w)
    dense = np.zeros((4, 4))
    for i in range(4):
        for m in range(3):
            if idx[i, m] >= 0:
                dense[i, idx[i, m]] += w[i, m]
    S = 0.5 * (dense + dense.T)
    np.testing.assert_array_equal(ip, np.concatenate([[0], np.cumsum((S != 0).sum(1))]))
    np.testing.assert_array_equal(ip, [0, 2, 4, 7, 7])
    got = np.zeros((4, 4))
    for i in range(4):
        got[i, ind[ip[i]:ip[i + 1]]] = val[ip[i]:ip[i + 1]]
    np.testing.assert_allclose(got, S, rtol=1e-15)


def test_lowp_conversions_are_rne():
    import torch

    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(2000).astype(np.float32) * 10 ** rng.uniform(-6, 4, 2000),
                        np.array([0.0, -0.0, 65504.0, 65520.0, 1e-8, 6.1e-5, 3e-7], np.float32)]).astype(np.float32)
    np.testing.assert_array_equal(port.to_f16_bits(x), x.astype(np.float16).view(np.uint16))
    tb = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    np.testing.assert_array_equal(port.to_bf16_bits(x), tb)


def test_adjoint_matches_finite_differences():
    rng = np.random.default_rng(1)
    n, F, T = 30, 3, 3
    A = (rng.random((n, n)) < 0.2).astype(float)
    A = np.maximum(A, A.T)
    np.fill_diagonal(A, 0)
    A[0, :] = 0
    A[:, 0] = 0
    A[0, 1] = A[1, 0] = 1
    import scipy.sparse as sp

    S = sp.csr_matrix(A * rng.uniform(0.1, 1.0, (n, n)))
    S.sort_indices()
    X0, Y = rng.standard_normal((n, F)), rng.standard_normal((n, F))
    for sym in (False, True):
        L, dX, dW = port.adjoint(S.indptr, S.indices, S.data, X0, Y, T, symmetric=sym)
        eps = 1e-6
        for q in range(0, S.nnz, max(1, S.nnz // 12)):
            Wp, Wm = S.data.copy(), S.data.copy()
            Wp[q] += eps
            Wm[q] -= eps
            lp = port.adjoint(S.indptr, S.indices, Wp, X0, Y, T, symmetric=sym)[0]
            lm = port.adjoint(S.indptr, S.indices, Wm, X0, Y, T, symmetric=sym)[0]
            assert abs((lp - lm) / (2 * eps) - dW[q]) < 1e-6 * max(1.0, abs(dW[q]))
        for (i, c) in [(0, 0), (3, 1), (n - 1, 2)]:
            Xp, Xm = X0.copy(), X0.copy()
            Xp[i, c] += eps
            Xm[i, c] -= eps
            lp = port.adjoint(S.indptr, S.indices, S.data, Xp, Y, T, symmetric=sym)[0]
            lm = port.adjoint(S.indptr, S.indices, S.data, Xm, Y, T, symmetric=sym)[0]
            assert abs((lp - lm) / (2 * eps) - dX[i, c]) < 1e-6 * max(1.0, abs(dX[i, c]))


# ---- live reference runs (oracle/_ref built from the reference sources) --------
needs_ref = pytest.mark.skipif(not ref.available("f32_i32"), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("variant", ["f32_i32", "f64_i64", "f32_i64", "f64_i32"])
def test_port_bit_exact_vs_reference(graph_3k, variant):
    _, _, ip, ind, W = graph_3k
    R = ref.RefLib(variant)
    n = ip.size - 1
    Wt = W.astype(R.real_dtype)
    for sym in (False, True):
        Pr = R.transition(ip, ind, Wt, n, symmetric=sym)
        Pp = port.transition(ip, ind, Wt, symmetric=sym, degree_fp64=False)
        np.testing.assert_array_equal(bits(Pr), bits(Pp))
    X0 = np.random.default_rng(2).standard_normal((n, 24)).astype(R.real_dtype)
    np.testing.assert_array_equal(bits(R.diffuse_matrix(ip, ind, Pr, X0, 5)),
                                  bits(port.diffuse_matrix(ip, ind, Pr, X0, 5)))


@needs_ref
def test_reference_rejects_non_contiguous_transition(graph_3k):
    _, _, ip, ind, W = graph_3k
    code, msg = ref.RefLib("f32_i32").create_transition_error(ip, ind, W.astype(np.float32), ip.size - 1)
    assert code == 10 and msg == "Matrix must be contiguous for transition matrix computation"
