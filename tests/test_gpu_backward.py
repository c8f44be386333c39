"""Backward pass of the diffusion (scl_gpu_diffuse_checkpointed / scl_gpu_diffuse_backward
and the torch.autograd wrapper) against the FP64 adjoint restatement
(oracle_adjoint_f64) and central finite differences in FP64.

Tolerances: FP32 gradients vs the FP64 adjoint within 2e-5 relative Frobenius
error and 2e-4 of the largest entry per entry; FP64 gradients within 1e-11
relative; finite differences (eps = 1e-3, FP64 forward) within 1e-4 relative
to max(|analytic|, 1e-3 * max|gradient|)."""
import numpy as np
import pytest

import scl
from oracle import port

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev_graph(ip, ind, W, n, dtype, symmetric):
    variant = "f32_i32" if dtype == np.float32 else "f64_i64"
    g = scl.gpu.GpuGraph.from_csr(ip.astype(np.int64), ind.astype(np.int32), W.astype(dtype), (n, n), variant=variant)
    g.normalize(symmetric=symmetric)
    return g


def _loss_grads_gpu(g, X0, Yt, T, every, keep_last=True):
    X0d = torch.from_numpy(X0).cuda()
    Yd = torch.from_numpy(Yt).cuda()
    XT, ck = g.diffuse_checkpointed(X0d, T, every, keep_last=keep_last)
    assert ck.shape[0] == g.checkpoint_slots(T, every, keep_last)
    dY = 2.0 * (XT - Yd)
    dX, dW = g.diffuse_backward(X0d, ck, dY, T, every, keep_last=keep_last)
    return XT, dX.cpu().numpy(), dW.cpu().numpy()


def _rel_fro(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _max_rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("F", [32, 64, 128, 5, 100])
@pytest.mark.parametrize("symmetric", [False, True])
def test_fp32_backward_matches_fp64_adjoint(graph_3k, F, symmetric):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    T, every = 8, 4
    rng = np.random.default_rng(F + 7 * symmetric)
    X0 = rng.standard_normal((n, F)).astype(np.float32)
    Yt = rng.standard_normal((n, F)).astype(np.float32)
    W32 = W.astype(np.float32)
    g = _dev_graph(ip, ind, W32, n, np.float32, symmetric)
    try:
        _, dX, dW = _loss_grads_gpu(g, X0, Yt, T, every)
    finally:
        g.close()
    _, dX64, dW64 = port.adjoint(ip, ind, W32.astype(np.float64), X0.astype(np.float64), Yt.astype(np.float64), T,
                                 symmetric=symmetric)
    assert _rel_fro(dX, dX64) < 2e-5 and _max_rel(dX, dX64) < 2e-4
    assert _rel_fro(dW, dW64) < 2e-5 and _max_rel(dW, dW64) < 2e-4


@pytest.mark.parametrize("keep_last", [True, False])
@pytest.mark.parametrize("every", [1, 3, 4, 8, 11])
def test_checkpoint_interval_does_not_change_results(graph_3k, every, keep_last):
    """The forward is bit-identical for every checkpoint interval. Gradients
    agree to rounding: on a structurally symmetric graph a recomputed iterate
    may come from the fused backward pass, whose 4 interleaved chains round
    differently from the forward's sequential chain."""
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    rng = np.random.default_rng(3)
    X0 = rng.standard_normal((n, 32)).astype(np.float32)
    Yt = rng.standard_normal((n, 32)).astype(np.float32)
    g = _dev_graph(ip, ind, W, n, np.float32, False)
    try:
        XT, dX, dW = _loss_grads_gpu(g, X0, Yt, 8, every, keep_last)
        XT1, dX1, dW1 = _loss_grads_gpu(g, X0, Yt, 8, 1)
        # forward with checkpoints = the plain diffusion, bit for bit
        Yp = g.diffuse(torch.from_numpy(X0).cuda(), 8)
    finally:
        g.close()
    assert torch.equal(XT, XT1) and torch.equal(XT, Yp)
    assert _rel_fro(dX, dX1) < 1e-6 and _max_rel(dX, dX1) < 1e-5
    assert _rel_fro(dW, dW1) < 1e-6 and _max_rel(dW, dW1) < 1e-5


@pytest.mark.parametrize("symmetric", [False, True])
def test_fp64_backward_is_tight(graph_3k, symmetric):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    rng = np.random.default_rng(11)
    X0 = rng.standard_normal((n, 24))
    Yt = rng.standard_normal((n, 24))
    g = _dev_graph(ip, ind, W, n, np.float64, symmetric)
    try:
        _, dX, dW = _loss_grads_gpu(g, X0, Yt, 6, 4)
    finally:
        g.close()
    _, dX64, dW64 = port.adjoint(ip, ind, W, X0, Yt, 6, symmetric=symmetric)
    assert _rel_fro(dX, dX64) < 1e-11 and _rel_fro(dW, dW64) < 1e-11


def test_zero_degree_rows_get_zero_weight_gradient():
    # node 0 isolated by zero weights; node 5 has no entries at all
    import scipy.sparse as sp

    rng = np.random.default_rng(5)
    n = 40
    A = (rng.random((n, n)) < 0.2).astype(float)
    A = np.maximum(A, A.T)
    np.fill_diagonal(A, 0)
    A[5, :] = 0
    A[:, 5] = 0
    S = sp.csr_matrix(A * rng.uniform(0.1, 1.0, (n, n)))
    S.sort_indices()
    S.data[S.indptr[0]:S.indptr[1]] = 0.0
    X0, Yt = rng.standard_normal((n, 7)), rng.standard_normal((n, 7))
    for sym in (False, True):
        g = _dev_graph(S.indptr, S.indices, S.data, n, np.float64, sym)
        try:
            _, dX, dW = _loss_grads_gpu(g, X0, Yt, 5, 2)
        finally:
            g.close()
        _, dX64, dW64 = port.adjoint(S.indptr, S.indices, S.data, X0, Yt, 5, symmetric=sym)
        assert np.all(dW[S.indptr[0]:S.indptr[1]] == 0.0)
        assert _rel_fro(dX, dX64) < 1e-11 and _rel_fro(dW, dW64) < 1e-11


def _fd_check(ip, ind, W, n, X0, Yt, T, symmetric, dX, dW, n_entries, seed):
    """Central differences (eps = 1e-3) of L = sum((P^T X0 - Y)^2) with the FP64
    device forward, at n_entries random entries of X0 and of W. The difference
    L(+) - L(-) is formed elementwise as sum((X+ - X-) * (X+ + X- - 2Y)), so no
    large sums are subtracted."""
    g = _dev_graph(ip, ind, W, n, np.float64, symmetric)
    Wd = torch.from_numpy(W.astype(np.float64)).cuda()
    X0d = torch.from_numpy(X0.astype(np.float64)).cuda()
    Yd = torch.from_numpy(Yt.astype(np.float64)).cuda()
    eps = 1e-3
    rng = np.random.default_rng(seed)

    def out_w(Wv):
        g.set_weights(Wv)
        g.normalize(symmetric=symmetric)
        return g.diffuse(X0d, T)

    def dl(Xp, Xm):
        return float(((Xp - Xm) * (Xp + Xm - 2.0 * Yd)).sum()) / (2 * eps)

    try:
        qs = rng.choice(W.size, n_entries, replace=False)
        fd_w = []
        for q in qs:
            Wp, Wm = Wd.clone(), Wd.clone()
            Wp[q] += eps
            Wm[q] -= eps
            fd_w.append(dl(out_w(Wp), out_w(Wm)))
        out_w(Wd)  # restore P
        cells = rng.choice(X0.size, n_entries, replace=False)
        fd_x = []
        for c in cells:
            i, f = divmod(int(c), X0.shape[1])
            Xp, Xm = X0d.clone(), X0d.clone()
            Xp[i, f] += eps
            Xm[i, f] -= eps
            fd_x.append(dl(g.diffuse(Xp, T), g.diffuse(Xm, T)))
    finally:
        g.close()
    an_w, an_x = dW[qs], dX.reshape(-1)[cells]
    sw = 1e-3 * np.abs(dW).max()
    sx = 1e-3 * np.abs(dX).max()
    err_w = np.abs(np.array(fd_w) - an_w) / np.maximum(np.abs(an_w), sw)
    err_x = np.abs(np.array(fd_x) - an_x) / np.maximum(np.abs(an_x), sx)
    return float(err_w.max()), float(err_x.max())


@pytest.mark.parametrize("symmetric", [False, True])
def test_finite_differences_256_entries(graph_3k, symmetric):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    rng = np.random.default_rng(21)
    X0 = rng.standard_normal((n, 32)).astype(np.float32)
    Yt = rng.standard_normal((n, 32)).astype(np.float32)
    W32 = W.astype(np.float32)
    g = _dev_graph(ip, ind, W32, n, np.float32, symmetric)
    try:
        _, dX, dW = _loss_grads_gpu(g, X0, Yt, 8, 4)
    finally:
        g.close()
    ew, ex = _fd_check(ip, ind, W32.astype(np.float64), n, X0, Yt, 8, symmetric, dX.astype(np.float64),
                       dW.astype(np.float64), 128, seed=4)
    assert ew < 1e-4 and ex < 1e-4, (ew, ex)


def test_autograd_function_matches_direct_calls(graph_3k):
    import scl.autograd

    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    rng = np.random.default_rng(8)
    X0 = torch.from_numpy(rng.standard_normal((n, 32)).astype(np.float32)).cuda().requires_grad_(True)
    Yt = torch.from_numpy(rng.standard_normal((n, 32)).astype(np.float32)).cuda()
    w = torch.from_numpy(W.astype(np.float32)).cuda().requires_grad_(True)
    g = scl.gpu.GpuGraph.from_csr(ip.astype(np.int64), ind.astype(np.int32), W.astype(np.float32), (n, n))
    try:
        XT = scl.autograd.diffuse(g, X0, 8, weights=w, symmetric=False, every=4)
        loss = ((XT - Yt) ** 2).sum()
        loss.backward()
        # direct
        g.set_weights(w.detach())
        g.normalize(symmetric=False)
        XT2, ck = g.diffuse_checkpointed(X0.detach(), 8, 4)
        dX2, dW2 = g.diffuse_backward(X0.detach(), ck, 2.0 * (XT2 - Yt), 8, 4)
    finally:
        g.close()
    assert torch.equal(XT.detach(), XT2)
    assert torch.allclose(X0.grad, dX2, rtol=0, atol=0)
    assert torch.allclose(w.grad, dW2, rtol=0, atol=0)


def test_autograd_gradcheck_fp64():
    import scipy.sparse as sp

    import scl.autograd

    rng = np.random.default_rng(2)
    n = 30
    A = (rng.random((n, n)) < 0.25).astype(float)
    A = np.maximum(A, A.T)
    np.fill_diagonal(A, 0)
    S = sp.csr_matrix(A * rng.uniform(0.2, 1.0, (n, n)))
    S.sort_indices()
    g = scl.gpu.GpuGraph.from_csr(S.indptr.astype(np.int64), S.indices.astype(np.int32), S.data, (n, n),
                                  variant="f64_i64")
    try:
        X0 = torch.from_numpy(rng.standard_normal((n, 3))).cuda().requires_grad_(True)
        w = torch.from_numpy(S.data.copy()).cuda().requires_grad_(True)
        for sym in (False, True):
            f = lambda x, ww: scl.autograd.diffuse(g, x, 4, weights=ww, symmetric=sym, every=2)
            assert torch.autograd.gradcheck(f, (X0, w), eps=1e-6, atol=1e-7, rtol=1e-5)
    finally:
        g.close()


def test_backward_argument_errors(graph_3k):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    g = _dev_graph(ip, ind, W, n, np.float32, False)
    try:
        X0 = torch.zeros((n, 8), device="cuda")
        with pytest.raises(scl.SCLError):
            g.diffuse_checkpointed(X0, 8, 0)
        g.set_storage(torch.bfloat16)
        with pytest.raises(scl.SCLError):
            g.diffuse_checkpointed(X0, 8, 4)
    finally:
        g.close()


def test_differentiation_configuration_full_size():
    """The differentiation configuration at full size: 200,000 cells, k=30,
    X0 200,000 x 32 FP32, 8 steps, L = sum((X_8 - Y)^2), checkpoint every 4.
    dL/dX0 and dL/dW against the FP64 adjoint restatement and against central
    finite differences (eps = 1e-3, FP64 device forward) on 256 random entries
    (128 of W, 128 of X0)."""
    n, k, F, T, every = 200_000, 30, 32, 8, 4
    pts = scl.synthetic.mixture(n, seed=0)
    ki, kd = scl.synthetic.knn_device(pts, k, block=4096)
    g = scl.gpu.GpuGraph.from_knn(ki, kd)
    del ki, kd
    ip, ind, W32 = g.export()
    g.normalize(symmetric=False)
    rng = np.random.default_rng(12)
    X0 = rng.standard_normal((n, F)).astype(np.float32)
    Yt = rng.standard_normal((n, F)).astype(np.float32)
    try:
        _, dX, dW = _loss_grads_gpu(g, X0, Yt, T, every)
    finally:
        g.close()
    torch.cuda.empty_cache()
    _, dX64, dW64 = port.adjoint(ip, ind, W32.astype(np.float64), X0.astype(np.float64), Yt.astype(np.float64), T)
    assert _rel_fro(dX, dX64) < 2e-5 and _max_rel(dX, dX64) < 2e-4
    assert _rel_fro(dW, dW64) < 2e-5 and _max_rel(dW, dW64) < 2e-4
    ew, ex = _fd_check(ip, ind, W32.astype(np.float64), n, X0, Yt, T, False, dX.astype(np.float64),
                       dW.astype(np.float64), 128, seed=9)
    assert ew < 1e-4 and ex < 1e-4, (ew, ex)
