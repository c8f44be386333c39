"""SpMM plans that follow a per-warp schedule of row groups (kinds 9, 10, 12,
14) on a reordered graph with long rows: three components of 12,000 rows, each
with two rows of about 600 entries (over eight times the mean, so the schedule
deals them first) and enough rows that every warp's list holds several groups.
The diffusion must return the oracle's bits for every plan."""
import numpy as np
import pytest
import scipy.sparse as sp

import scl
from oracle import port

pytestmark = pytest.mark.gpu

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)


def hub_graph(n_comp=3, size=12000, k=12, hubs=2, hub_deg=600, seed=5):
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for c in range(n_comp):
        base = c * size
        rows.append(base + np.repeat(np.arange(size), k))
        cols.append(base + rng.integers(0, size, size * k))
        for h in rng.choice(size, hubs, replace=False):
            rows.append(np.full(hub_deg, base + h))
            cols.append(base + rng.choice(size, hub_deg, replace=False))
    n = n_comp * size
    r, c = np.concatenate(rows), np.concatenate(cols)
    A = sp.csr_matrix((np.ones(r.size, np.float32), (r, c)), shape=(n, n))
    A = ((A + A.T) > 0).astype(np.float32).tocsr()
    A.sort_indices()
    ip = A.indptr.astype(np.int64)
    lens = np.diff(ip)
    vals = (rng.random(A.nnz) + 0.01).astype(np.float32)
    rs = np.add.reduceat(vals, ip[:-1]) if A.nnz else vals
    vals = (vals / np.repeat(rs, lens)).astype(np.float32)  # rows sum to about 1
    assert lens.max() > 8 * (A.nnz // n + 1)
    return ip, A.indices.astype(np.int32), vals, n


@pytest.mark.parametrize("F,group", [(32, 8), (64, 16), (128, 32)])
def test_scheduled_multirow_plans_are_exact(F, group):
    import torch

    ip, ind, P, n = hub_graph()
    X0 = np.random.default_rng(F).standard_normal((n, F)).astype(np.float32)
    want = port.diffuse_matrix(ip, ind, P, X0, 2)
    g = scl.gpu.GpuGraph.from_csr(ip, ind, P, (n, n))
    try:
        g.reorder(1)
        Xd = torch.from_numpy(X0).cuda()
        for stage in (4, 8, 16):
            g.set_plan(F, group, 4, 12, stage)
            Y = g.diffuse(Xd, 2).cpu().numpy()
            np.testing.assert_array_equal(bits(Y), bits(want))
    finally:
        g.close()


@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_scheduled_split_chain_plans_are_exact(storage):
    import torch

    ip, ind, P, n = hub_graph(seed=9)
    F, group = 64, 8
    chains = 32 // group
    tdt = torch.bfloat16 if storage == "bf16" else torch.float16
    code = port.BF16 if storage == "bf16" else port.F16
    X0 = np.random.default_rng(3).standard_normal((n, F)).astype(np.float32)
    want = port.diffuse_lowp_chains(ip, ind, P, X0, 2, code, chains)
    g = scl.gpu.GpuGraph.from_csr(ip, ind, P, (n, n))
    try:
        g.set_storage(tdt)
        g.reorder(1)
        Xd = torch.from_numpy(X0).cuda().to(tdt)
        shapes = [(9, 0), (9, 1), (10, 0), (14, 4), (14, 8), (14, 16)]
        if storage == "bf16":
            shapes.append((10, 1))
        for kind, stage in shapes:
            g.set_plan(F, group, 8, kind, stage)
            Y = g.diffuse(Xd, 2, out_dtype=torch.float32).cpu().numpy()
            np.testing.assert_array_equal(bits(Y), bits(want))
    finally:
        g.close()
