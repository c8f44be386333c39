"""Grouped-row SpMM (plan kind 13) on the reordered structure.

C = 32 / (row bytes / 16) rows share a warp, their (index, value) pairs stored
in 32-slot blocks; every output element is still the sequential fma chain over
its row's entries in stored order (scl/kernel/diffusion.hpp:227-278), so FP32
results equal the oracle's restatement of scl-core's diffuse_matrix bit for
bit, and 16-bit storage equals the oracle's one-chain 16-bit restatement."""
import numpy as np
import pytest

import scl
from oracle import port

pytestmark = pytest.mark.gpu

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)


def _skewed_graph(seed=11, n=3000):
    """Empty rows, a hub row of 2500 entries, self loops, duplicate columns,
    rows of every length from 1 to 41 (groups mix lengths at component edges)."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        if i % 7 == 0:
            rows.append(np.array([], np.int64))
        elif i == 5:
            rows.append(np.sort(rng.choice(n, 2500, replace=False)))
        else:
            rows.append(np.sort(np.concatenate([[i], rng.choice(n, rng.integers(1, 40), replace=True)])))
    ip = np.concatenate([[0], np.cumsum([r.size for r in rows])])
    ind = np.concatenate(rows).astype(np.int64)
    vals = rng.random(ind.size).astype(np.float32)
    P = port.transition(ip, ind, vals, False, True)
    return ip, ind, P, n


def _mixture_graph(n=4000, k=12, seed=8):
    import torch

    pts = scl.synthetic.mixture(n, seed=seed)
    ki, kd = scl.synthetic.knn_exact(pts, k)
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd.astype(np.float32)))
    g.normalize()
    return g


def _shapes(F, elem):
    C = 32 // (F * elem // 16)
    return [u for u in (4, 8, 16) if not (u == 16 and C == 4)]


@pytest.mark.parametrize("F", [32, 64, 128])
def test_grouped_fp32_matches_oracle(F):
    import torch

    ip, ind, P, n = _skewed_graph()
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    try:
        g.reorder(1)
        X0 = np.random.default_rng(F).standard_normal((n, F)).astype(np.float32)
        want = port.diffuse_matrix(ip, ind, P, X0, 3)
        Xd = torch.from_numpy(X0).cuda()
        for u in _shapes(F, 4):
            g.set_plan(F, 32, 4, 13, u)
            Y = g.diffuse(Xd, 3)
            np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(want), err_msg=f"F={F} U={u}")
            X1 = Xd.clone()
            g.diffuse(X1, 3, out=X1)  # in place
            np.testing.assert_array_equal(bits(X1.cpu().numpy()), bits(want))
        g.set_plan(F, 0)
    finally:
        g.close()


@pytest.mark.parametrize("storage,F", [("bf16", 64), ("bf16", 128), ("f16", 64), ("f16", 128)])
def test_grouped_lowp_matches_one_chain_oracle(storage, F):
    import torch

    ip, ind, P, n = _skewed_graph(seed=12)
    tdt = torch.bfloat16 if storage == "bf16" else torch.float16
    kind_code = port.BF16 if storage == "bf16" else port.F16
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    try:
        g.reorder(1)
        g.set_storage(tdt)
        X0 = np.random.default_rng(F + 1).standard_normal((n, F)).astype(np.float32)
        Xd = torch.from_numpy(X0).cuda().to(tdt)
        for u in _shapes(F, 2):
            g.set_plan(F, 32, 8, 13, u)
            Y32 = g.diffuse(Xd, 3, out_dtype=torch.float32).cpu().numpy()
            np.testing.assert_array_equal(bits(Y32), bits(port.diffuse_lowp(ip, ind, P, X0, 3, kind_code, True)))
            Y16 = g.diffuse(Xd, 2, out_dtype=tdt).float().cpu().numpy()
            np.testing.assert_array_equal(bits(Y16), bits(port.diffuse_lowp(ip, ind, P, X0, 2, kind_code, False)))
    finally:
        g.close()


def test_grouped_on_mixture_graph_and_autotune():
    """Components of the mixture graph, rows longest-first inside each; the
    autotuner may pick kind 13 and the bits stay those of the oracle."""
    import torch

    g = _mixture_graph()
    try:
        ip, ind, P = g.export()
        n = ip.size - 1
        g.reorder(1)
        perm, _ = g.reorder_info()
        lens = np.diff(ip)[perm]
        from scipy.sparse.csgraph import connected_components
        import scipy.sparse as sp

        _, lab = connected_components(sp.csr_matrix((P, ind, ip), shape=(n, n)), directed=False)
        lab = lab[perm]
        same = lab[1:] == lab[:-1]
        assert np.all(lens[1:][same] <= lens[:-1][same]), "rows are not longest-first inside a component"
        X0 = np.random.default_rng(3).standard_normal((n, 64)).astype(np.float32)
        want = port.diffuse_matrix(ip, ind, P, X0, 4)
        Xd = torch.from_numpy(X0).cuda()
        for u in (4, 8, 16):
            g.set_plan(64, 32, 4, 13, u)
            np.testing.assert_array_equal(bits(g.diffuse(Xd, 4).cpu().numpy()), bits(want))
        res = g.autotune(64, reps=2)
        assert res["kind"] in (4, 7, 11, 12, 13)
        np.testing.assert_array_equal(bits(g.diffuse(Xd, 4).cpu().numpy()), bits(want))
        # values changed after the layout was built: the grouped slots follow them
        g.normalize(symmetric=True)
        ip2, ind2, P2 = g.export()
        g.set_plan(64, 32, 4, 13, 8)
        np.testing.assert_array_equal(bits(g.diffuse(Xd, 2).cpu().numpy()),
                                      bits(port.diffuse_matrix(ip2, ind2, P2, X0, 2)))
    finally:
        g.close()


def test_grouped_plan_needs_reordering():
    import torch

    ip, ind, P, n = _skewed_graph()
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    try:
        g.set_plan(64, 32, 4, 13, 8)
        X = torch.zeros((n, 64), device="cuda")
        with pytest.raises(scl.SCLError) as e:
            g.diffuse(X, 1)
        assert e.value.code == 10
        with pytest.raises(scl.SCLError):
            g.set_plan(64, 32, 4, 13, 5)  # batch must be 4, 8 or 16
        with pytest.raises(scl.SCLError):
            g.set_plan(32, 32, 4, 13, 16)  # 128-byte rows: 8-entry blocks
    finally:
        g.close()
