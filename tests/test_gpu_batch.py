"""Batched diffusion (scl_gpu_batch_*): many uneven graphs in one persistent,
CUDA-graph-replayed launch. Every graph's result must be bit-identical to
diffusing that graph alone (scl_gpu_diffuse) and to the oracle's sequential
fma chain, for every schedule the autotuner can pick."""
import numpy as np
import pytest

import scl
from oracle import port

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
bits = lambda a: np.ascontiguousarray(a).view(np.uint8)


def _graphs(sizes, k=10, seed=0):
    out = []
    for b, n in enumerate(sizes):
        pts = scl.synthetic.mixture(n, seed=seed + b)
        ki, kd = scl.synthetic.knn_exact(pts, min(k, n - 1))
        g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd.astype(np.float32)))
        g.normalize(symmetric=False)
        out.append(g)
    return out


@pytest.fixture(scope="module")
def small_batch():
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(40), np.log(3000), 12)).astype(int).tolist()
    gs = _graphs(sizes)
    yield gs
    for g in gs:
        g.close()


def _stack(graphs, F, seed):
    rng = np.random.default_rng(seed)
    blocks = [rng.standard_normal((g.shape[0], F)).astype(np.float32) for g in graphs]
    return blocks, torch.from_numpy(np.concatenate(blocks)).cuda()


@pytest.mark.parametrize("F,T", [(16, 8), (5, 3), (64, 2), (1, 1), (33, 4)])
def test_batch_bit_identical_to_single_graphs(small_batch, F, T):
    blocks, X0 = _stack(small_batch, F, seed=F)
    b = scl.gpu.GpuBatch(small_batch, F, T)
    try:
        Y = b.solve(X0)
        assert b.status() == (0, 0)
        Yh = Y.cpu().numpy()
        for gi, g in enumerate(small_batch):
            r0, r1 = b.row_offsets[gi], b.row_offsets[gi + 1]
            Ys = g.diffuse(torch.from_numpy(blocks[gi]).cuda(), T).cpu().numpy()
            np.testing.assert_array_equal(bits(Yh[r0:r1]), bits(Ys))
            if gi < 3:
                ip, ind, P = g.export()
                np.testing.assert_array_equal(bits(Yh[r0:r1]), bits(port.diffuse_matrix(ip, ind, P, blocks[gi], T)))
    finally:
        b.close()


@pytest.mark.parametrize("tile,unroll,bps", [(1, 4, 1), (64, 8, 2), (4096, 8, 0), (1 << 20, 4, 0)])
def test_every_schedule_gives_the_same_bits(small_batch, tile, unroll, bps):
    blocks, X0 = _stack(small_batch, 16, seed=1)
    b = scl.gpu.GpuBatch(small_batch, 16, 8)
    try:
        ref = b.solve(X0).clone()
        b.set_schedule(tile, unroll, bps)
        Y = b.solve(X0)
        assert b.status() == (0, 0)
        assert torch.equal(Y, ref)
    finally:
        b.close()


def test_graph_replay_with_new_buffers_and_autotune(small_batch):
    blocks, X0 = _stack(small_batch, 16, seed=2)
    _, X1 = _stack(small_batch, 16, seed=5)
    b = scl.gpu.GpuBatch(small_batch, 16, 8)
    try:
        ref0 = b.solve(X0).clone()
        ref1 = b.solve(X1).clone()
        Ya = torch.empty_like(X0)
        for _ in range(3):  # replays of the captured graph, pointers swapped each time
            b.solve(X0, out=Ya)
            assert torch.equal(Ya, ref0)
            Yb = b.solve(X1)
            assert torch.equal(Yb, ref1)
        sched = b.autotune(X0, torch.empty_like(X0), reps=2)
        assert sched["tile_nnz"] > 0 and sched["grid"] > 0 and sched["tuned_ms"] > 0
        assert torch.equal(b.solve(X0), ref0)
        assert b.status() == (0, 0)
    finally:
        b.close()


def test_single_graph_batch_and_empty_rows():
    import scipy.sparse as sp

    rng = np.random.default_rng(4)
    n = 500
    A = sp.random(n, n, density=0.02, random_state=4, format="csr")
    A.data[:] = rng.uniform(0.1, 1.0, A.nnz)
    A = A.tolil()
    A[7, :] = 0  # an empty row
    A = A.tocsr()
    A.eliminate_zeros()
    A.sort_indices()
    g = scl.gpu.GpuGraph.from_csr(A.indptr.astype(np.int64), A.indices.astype(np.int32),
                                  A.data.astype(np.float32), (n, n))
    g.normalize()
    X0 = rng.standard_normal((n, 16)).astype(np.float32)
    b = scl.gpu.GpuBatch([g], 16, 5)
    try:
        Y = b.solve(torch.from_numpy(X0).cuda()).cpu().numpy()
        ip, ind, P = g.export()
        np.testing.assert_array_equal(bits(Y), bits(port.diffuse_matrix(ip, ind, P, X0, 5)))
        assert np.all(Y[7] == 0)
    finally:
        b.close()
        g.close()


def test_wait_that_never_completes_reports_an_error(small_batch):
    """A host-made failure: graph 0's waits are given a target no tile reaches,
    so they run into their time limit; the launch must return, the status must
    say so, and the context must stay usable."""
    blocks, X0 = _stack(small_batch, 16, seed=6)
    b = scl.gpu.GpuBatch(small_batch, 16, 4)
    try:
        ref = b.solve(X0).clone()
        assert b.status() == (0, 0)
        b.inject_stall(0)
        b.solve(X0)
        code, item = b.status()
        assert code == 54 and item >= 0  # SCL_ERROR_CONVERGENCE
        b.inject_stall(-1)
        assert torch.equal(b.solve(X0), ref)
        assert b.status() == (0, 0)
    finally:
        b.close()


def test_batch_rejects_bad_inputs(small_batch):
    with pytest.raises(scl.SCLError):
        scl.gpu.GpuBatch(small_batch, 0, 8)
    g = small_batch[0]
    g.set_storage(torch.bfloat16)
    try:
        with pytest.raises(scl.SCLError):
            scl.gpu.GpuBatch([g], 16, 8)
    finally:
        g.set_storage(torch.float32)
