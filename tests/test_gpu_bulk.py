"""Gather kernels for FP32/FP64 beside the default row kernel.

Plan kind 11: the X rows of a chunk's entries are copied into a per-warp
shared-memory ring by tensor gathers (four rows per copy). Plan kind 12: 16-byte
lanes, so one warp advances 1, 2 or 4 rows together. Both must give the same
bits as the oracle's sequential fma chain (scl-core's spmm_block order) for
FP32 and FP64, every stage, every row pitch, on a reordered graph and on
skewed and tiny graphs; kind 11's bounded wait must report a wait that runs
out."""
import numpy as np
import pytest

import scl
from oracle import port

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
bits = lambda a: np.ascontiguousarray(a).view(np.uint8)

STAGES = (2, 3, 4, 6)


def _graph(graph_3k, variant="f32_i32", dtype=np.float32):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    if dtype == np.float64:
        P = port.transition(ip, ind, W.astype(np.float64), False, True)
    else:
        P = port.transition(ip, ind, W.astype(np.float32), False, True)
    idx = ind.astype(np.int64 if variant.endswith("i64") else np.int32)
    return scl.gpu.GpuGraph.from_csr(ip, idx, P, (n, n), variant=variant), ip, ind, P


@pytest.mark.parametrize("F,vec", [(32, 1), (64, 2), (128, 4)])
def test_fp32_every_ring_depth_is_exact(graph_3k, F, vec):
    g, ip, ind, P = _graph(graph_3k)
    try:
        X0 = np.random.default_rng(F).standard_normal((ip.size - 1, F)).astype(np.float32)
        ref = port.spmm(ip, ind, P, X0)
        Xd = torch.from_numpy(X0).cuda()
        for st in STAGES:
            Y = torch.full_like(Xd, float("nan"))
            g.spmm(Xd, Y, group=32, vec=vec, kind=11, stage=st)
            np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
        assert g.spmm_status() == (0, 0)
    finally:
        g.close()


@pytest.mark.parametrize("F,vec", [(32, 1), (64, 2)])
def test_fp64_every_ring_depth_is_exact(graph_3k, F, vec):
    g, ip, ind, P = _graph(graph_3k, "f64_i64", np.float64)
    try:
        X0 = np.random.default_rng(F + 1).standard_normal((ip.size - 1, F))
        ref = port.spmm(ip, ind, P, X0)
        Xd = torch.from_numpy(X0).cuda()
        for st in STAGES:
            Y = torch.full_like(Xd, float("nan"))
            g.spmm(Xd, Y, group=32, vec=vec, kind=11, stage=st)
            np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
        assert g.spmm_status() == (0, 0)
    finally:
        g.close()


def test_diffusion_with_bulk_plan_on_reordered_graph(graph_3k):
    """A reordered graph writes output rows through the row map; the T-step
    diffusion with the kind-11 plan equals the oracle's chain bit for bit."""
    g, ip, ind, P = _graph(graph_3k)
    try:
        g.reorder(1)
        X0 = np.random.default_rng(9).standard_normal((ip.size - 1, 64)).astype(np.float32)
        ref = port.diffuse_matrix(ip, ind, P, X0, 5)
        for st in STAGES:
            g.set_plan(64, 32, 2, 11, st)
            Y = g.diffuse(torch.from_numpy(X0).cuda(), 5)
            np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
        assert g.spmm_status() == (0, 0)
    finally:
        g.close()


def test_skewed_rows_and_tiny_graphs():
    """Empty rows (also runs of them and a trailing one), a hub row spanning
    many chunks, graphs with fewer rows than warps in one block and row counts
    that are not a multiple of the rows a warp advances together."""
    rng = np.random.default_rng(17)
    for n in (1, 2, 3, 5, 2001):
        rows = []
        for i in range(n):
            if n > 5 and (i % 9 == 0 or 100 <= i < 140 or i == n - 1):
                rows.append(np.array([], np.int64))
            elif n > 5 and i == 7:
                rows.append(np.sort(rng.choice(n, 1500, replace=False)))
            else:
                rows.append(np.sort(rng.choice(n, int(rng.integers(1, 70)), replace=True)))
        ip = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.int64)
        ind = np.concatenate(rows).astype(np.int64)
        vals = rng.random(ind.size).astype(np.float32)
        P = port.transition(ip, ind, vals, False, True)
        g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
        try:
            for F, vec in ((32, 1), (64, 2), (128, 4)):
                X0 = rng.standard_normal((n, F)).astype(np.float32)
                ref = port.spmm(ip, ind, P, X0)
                Xd = torch.from_numpy(X0).cuda()
                for st in STAGES:
                    Y = torch.full_like(Xd, float("nan"))
                    g.spmm(Xd, Y, group=32, vec=vec, kind=11, stage=st)
                    np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
                for st in (4, 8, 16):
                    Y = torch.full_like(Xd, float("nan"))
                    g.spmm(Xd, Y, group=F // 4, vec=4, kind=12, stage=st)
                    np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
            assert g.spmm_status() == (0, 0)
        finally:
            g.close()


def test_bad_plans_are_rejected(graph_3k):
    g, ip, ind, P = _graph(graph_3k)
    try:
        Xd = torch.zeros((ip.size - 1, 64), device="cuda")
        Y = torch.empty_like(Xd)
        for group, vec, stage in ((32, 2, 5), (16, 4, 3), (32, 1, 3)):
            with pytest.raises(scl.SCLError):
                g.spmm(Xd, Y, group=group, vec=vec, kind=11, stage=stage)
        with pytest.raises(scl.SCLError):  # 48 columns: a 192-byte row has no bulk form
            X48 = torch.zeros((ip.size - 1, 48), device="cuda")
            g.spmm(X48, torch.empty_like(X48), group=32, vec=1, kind=11, stage=3)
        with pytest.raises(scl.SCLError):
            g.set_plan(64, 32, 2, 11, 5)
        g.set_storage(torch.bfloat16)
        with pytest.raises(scl.SCLError):
            g.set_plan(64, 32, 2, 11, 3)
    finally:
        g.close()


def test_wait_that_never_completes_reports_an_error(graph_3k):
    """A host-made failure: one warp expects 16 bytes more than it copies, so
    its first bounded wait (2 s) runs out. The launch must return, the status
    must name the warp, the context must stay usable, and the next launch
    without the hook must give the exact result again."""
    g, ip, ind, P = _graph(graph_3k)
    try:
        X0 = np.random.default_rng(3).standard_normal((ip.size - 1, 64)).astype(np.float32)
        ref = port.spmm(ip, ind, P, X0)
        Xd = torch.from_numpy(X0).cuda()
        Y = torch.empty_like(Xd)
        g.inject_spmm_stall(3)
        try:
            g.spmm(Xd, Y, group=32, vec=2, kind=11, stage=3)
            code, warp = g.spmm_status()
        finally:
            g.inject_spmm_stall(-1)
        assert code == 54 and warp == 3  # SCL_ERROR_CONVERGENCE
        assert g.spmm_status() == (0, 0)  # read once, then cleared
        g.spmm(Xd, Y, group=32, vec=2, kind=11, stage=3)
        np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
        assert g.spmm_status() == (0, 0)
    finally:
        g.close()


@pytest.mark.parametrize("F", [32, 64, 128])
def test_multirow_fp32_and_fp64(graph_3k, F):
    for variant, dt in (("f32_i32", np.float32), ("f64_i64", np.float64)):
        if dt == np.float64 and F == 128:
            continue  # a 1 KiB row has no 16-byte-lane form
        g, ip, ind, P = _graph(graph_3k, variant, dt)
        try:
            X0 = np.random.default_rng(F).standard_normal((ip.size - 1, F)).astype(dt)
            ref = port.spmm(ip, ind, P, X0)
            Xd = torch.from_numpy(X0).cuda()
            lanes = F * X0.itemsize // 16
            for st in (4, 8, 16):
                Y = torch.full_like(Xd, float("nan"))
                g.spmm(Xd, Y, group=lanes, vec=16 // X0.itemsize, kind=12, stage=st)
                np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
        finally:
            g.close()


def test_diffusion_with_multirow_plan_on_reordered_graph(graph_3k):
    g, ip, ind, P = _graph(graph_3k)
    try:
        g.reorder(1)
        for F in (32, 64):
            X0 = np.random.default_rng(F + 9).standard_normal((ip.size - 1, F)).astype(np.float32)
            ref = port.diffuse_matrix(ip, ind, P, X0, 5)
            for st in (4, 8, 16):
                g.set_plan(F, F // 4, 4, 12, st)
                Y = g.diffuse(torch.from_numpy(X0).cuda(), 5)
                np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref))
        with pytest.raises(scl.SCLError):
            g.set_plan(64, 16, 4, 12, 5)
        with pytest.raises(scl.SCLError):
            g.set_plan(64, 32, 2, 12, 8)
    finally:
        g.close()
