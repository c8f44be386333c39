"""GPU parity through the C ABI (libscl_<variant>.so) against scl-core's own
results (golden vectors, oracle/_ref) and the C restatement (oracle.port).

Bars: structure and column indices bit-exact; FP32/FP64 diffusion bit-exact on
the same P and X (same fma sequence as scl-core's axpy_simd); FP64-degree
transition matrices within 2 ulp of scl-core's native-precision ones and
bit-exact against the restatement of that FP64 contract; end-to-end chains
within 1e-5 relative per entry (absolute floor 1e-7 for near-zero entries)."""
import numpy as np
import pytest

import scl
from oracle import port, ref

pytestmark = pytest.mark.gpu

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)
RTOL_F32, ATOL_F32 = 1e-5, 1e-7


def wrap(ip, ind, vals, n, index_dtype=np.int32):
    return scl.CsrMatrix.wrap(np.asarray(ip, index_dtype), np.asarray(ind, index_dtype), vals, (n, n))


def test_kat_tiny_3x3():
    for rd, idt in ((np.float32, np.int32), (np.float64, np.int64)):
        m = wrap([0, 2, 3, 6], [0, 2, 1, 0, 1, 2], np.array([1, 2, 3, 4, 5, 6], rd), 3, idt)
        X = np.array([[1, 2], [3, 4], [5, 6]], rd)
        scl.diffusion.diffuse_matrix(m, X, 1)
        np.testing.assert_array_equal(X, [[11, 14], [9, 12], [49, 64]])
        x = np.array([1, 2, 3], rd)
        scl.diffusion.diffuse_vector(m, x, 1)
        np.testing.assert_array_equal(x, [7, 6, 32])


@pytest.mark.parametrize("tag,idt", [("f32", np.int32), ("f64", np.int64)])
@pytest.mark.parametrize("sym", [False, True])
def test_transition_native_mode_bit_exact_with_golden(golden, tag, idt, sym):
    g = golden
    n = int(g["n"])
    vals = g[f"W_{tag}"].copy()
    m = wrap(g["indptr"], g["indices"], vals, n, idt)
    scl.diffusion.set_degree_mode(m, 1)
    try:
        scl.diffusion.compute_transition_matrix(m, symmetric=sym)
    finally:
        scl.diffusion.set_degree_mode(m, 0)
    np.testing.assert_array_equal(bits(vals), bits(g[f"P_{'sym' if sym else 'row'}_{tag}"]))


@pytest.mark.parametrize("sym", [False, True])
def test_transition_fp64_degrees(golden, sym):
    g = golden
    n = int(g["n"])
    key = f"P_{'sym' if sym else 'row'}"
    # f64 build: FP64 degrees are scl-core's own arithmetic -> bit-exact
    v64 = g["W_f64"].copy()
    scl.diffusion.compute_transition_matrix(wrap(g["indptr"], g["indices"], v64, n, np.int64), symmetric=sym)
    np.testing.assert_array_equal(bits(v64), bits(g[f"{key}_f64"]))
    # f32 build: FP64 degrees differ from scl-core's float sums by rounding only
    v32 = g["W_f32"].copy()
    scl.diffusion.compute_transition_matrix(wrap(g["indptr"], g["indices"], v32, n), symmetric=sym)
    np.testing.assert_array_equal(bits(v32), bits(port.transition(g["indptr"], g["indices"], g["W_f32"], sym, True)))
    np.testing.assert_allclose(v32, g[f"{key}_f32"], rtol=5e-7, atol=0)  # <= 4 ulp


@pytest.mark.parametrize("tag,idt", [("f32", np.int32), ("f64", np.int64), ("f32", np.int64), ("f64", np.int32)])
def test_diffuse_matrix_bit_exact_with_golden(golden, tag, idt):
    g = golden
    n = int(g["n"])
    m = wrap(g["indptr"], g["indices"], g[f"P_row_{tag}"].copy(), n, idt)
    X = g[f"X0_{tag}"].copy()
    scl.diffusion.diffuse_matrix(m, X, int(g["T"]))
    np.testing.assert_array_equal(bits(X), bits(g[f"XT_{tag}"]))


def test_csc_handle_applies_transpose(golden):
    g = golden
    n = int(g["n"])
    m = wrap(g["indptr"], g["indices"], g["P_row_f32"].copy(), n)
    t = m.transpose()
    X = g["X0_f32"].copy()
    scl.diffusion.diffuse_matrix(t, X, 2)
    np.testing.assert_array_equal(bits(X), bits(g["XT_csc_f32"]))


def test_diffuse_vector_within_tolerance(golden):
    g = golden
    n = int(g["n"])
    m = wrap(g["indptr"], g["indices"], g["P_row_f32"].copy(), n)
    x = g["X0_f32"][:, 0].copy()
    scl.diffusion.diffuse_vector(m, x, 3)
    np.testing.assert_allclose(x, g["xv_f32"], rtol=RTOL_F32, atol=ATOL_F32)
    # and bit-exact against the sequential-fma restatement
    xp = port.diffuse_matrix(g["indptr"], g["indices"], g["P_row_f32"], g["X0_f32"][:, :1], 3)[:, 0]
    np.testing.assert_array_equal(bits(x), bits(xp))


def test_magic_impute_default_steps(golden):
    g = golden
    n = int(g["n"])
    m = wrap(g["indptr"], g["indices"], g["P_row_f32"].copy(), n)
    X = g["X0_f32"].copy()
    scl.diffusion.magic_impute(m, X, 0)
    np.testing.assert_array_equal(bits(X), bits(port.diffuse_matrix(g["indptr"], g["indices"], g["P_row_f32"],
                                                                   g["X0_f32"], 3)))


def test_config1_chain_20k(graph_20k):
    """20,000 cells, k=15, 32 features, 8 steps: the CPU-runnable configuration."""
    _, _, ip, ind, W = graph_20k
    n = ip.size - 1
    W32 = W.astype(np.float32)
    X0 = scl.synthetic.features(n, 32, seed=1)
    # (a) transition on the GPU (FP64 degrees) == FP64-degree restatement, bit for bit
    P_gpu = W32.copy()
    m = wrap(ip, ind, P_gpu, n)
    scl.diffusion.compute_transition_matrix(m)
    np.testing.assert_array_equal(bits(P_gpu), bits(port.transition(ip, ind, W32, False, True)))
    # (b) diffusion on the same P == restatement == scl-core, bit for bit
    X = X0.copy()
    scl.diffusion.diffuse_matrix(m, X, 8)
    Xp = port.diffuse_matrix(ip, ind, P_gpu, X0, 8)
    np.testing.assert_array_equal(bits(X), bits(Xp))
    if ref.available("f32_i32"):
        R = ref.RefLib("f32_i32")
        np.testing.assert_array_equal(bits(X), bits(R.diffuse_matrix(ip, ind, P_gpu, X0, 8)))
        # (c) the whole chain vs scl-core's own chain (native-precision degrees)
        P_ref = R.transition(ip, ind, W32, n)
        X_ref = R.diffuse_matrix(ip, ind, P_ref, X0, 8)
        np.testing.assert_allclose(X, X_ref, rtol=RTOL_F32, atol=ATOL_F32)
    # FP64 oracle: error of the FP32 GPU chain
    P64 = port.transition(ip, ind, W, False)
    X64 = port.diffuse_matrix(ip, ind, P64, X0.astype(np.float64), 8)
    assert np.max(np.abs(X - X64)) < 1e-5


@pytest.mark.parametrize("F", [1, 2, 3, 5, 8, 16, 32, 33, 64, 96, 128, 200])
@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_feature_widths_bit_exact(graph_3k, F, tag):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    dt = np.float32 if tag == "f32" else np.float64
    P = port.transition(ip, ind, W.astype(dt), False, False)
    X0 = np.random.default_rng(F).standard_normal((n, F)).astype(dt)
    X = X0.copy()
    scl.diffusion.diffuse_matrix(wrap(ip, ind, P.copy(), n, np.int32 if tag == "f32" else np.int64), X, 3)
    np.testing.assert_array_equal(bits(X), bits(port.diffuse_matrix(ip, ind, P, X0, 3)))


def test_block_allocated_handle(graph_3k):
    """ADAPTIVE-created (non-contiguous) handles diffuse like contiguous ones and
    reject compute_transition_matrix exactly as scl-core does."""
    import scipy.sparse as sp

    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    P = port.transition(ip, ind, W.astype(np.float32), False, False)
    S = sp.csr_matrix((P, ind, ip), shape=(n, n))
    m = scl.CsrMatrix.copy(S, strategy=scl.BlockStrategy.ADAPTIVE)
    assert not m.is_contiguous
    X0 = np.random.default_rng(0).standard_normal((n, 16)).astype(np.float32)
    X = X0.copy()
    scl.diffusion.diffuse_matrix(m, X, 4)
    np.testing.assert_array_equal(bits(X), bits(port.diffuse_matrix(ip, ind, P, X0, 4)))
    with pytest.raises(scl.SCLError) as e:
        scl.diffusion.compute_transition_matrix(m)
    assert e.value.code == 10


def test_skewed_and_empty_rows():
    """Empty rows, a hub row of 2500 entries, self loops, duplicate columns."""
    rng = np.random.default_rng(11)
    n = 3000
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
    for sym in (False, True):
        v = vals.copy()
        scl.diffusion.compute_transition_matrix(wrap(ip, ind, v, n), symmetric=sym)
        np.testing.assert_array_equal(bits(v), bits(port.transition(ip, ind, vals, sym, True)))
    P = port.transition(ip, ind, vals, False, True)
    for F in (4, 64):
        X0 = rng.standard_normal((n, F)).astype(np.float32)
        X = X0.copy()
        scl.diffusion.diffuse_matrix(wrap(ip, ind, P.copy(), n), X, 3)
        np.testing.assert_array_equal(bits(X), bits(port.diffuse_matrix(ip, ind, P, X0, 3)))
    # the fixed-pitch kernels on the same rows (runs of empty rows inside a
    # row block, a hub row spanning many batches)
    import torch

    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    try:
        for F, vec in ((32, 1), (64, 2), (128, 4)):
            X0 = rng.standard_normal((n, F)).astype(np.float32)
            ref1 = port.spmm(ip, ind, P, X0)
            Xd = torch.from_numpy(X0).cuda()
            for kind, stage in ((4, 8), (4, 32), (7, 8), (7, 16), (7, 32), (11, 2), (11, 3), (11, 6)):
                Y = torch.empty_like(Xd)
                g.spmm(Xd, Y, group=32, vec=vec, kind=kind, stage=stage)
                np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref1))
            for stage in (4, 8, 16):  # multi-row kernel: F/4 lanes per row, 32/(F/4) rows per warp
                Y = torch.empty_like(Xd)
                g.spmm(Xd, Y, group=F // 4, vec=4, kind=12, stage=stage)
                np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref1))
        # 16-bit storage kernels (interleaved chains) on the same rows
        g.set_storage(torch.bfloat16)
        for F, group in ((64, 8), (128, 16)):
            X0 = rng.standard_normal((n, F)).astype(np.float32)
            Xd = torch.from_numpy(X0).cuda().to(torch.bfloat16)
            ref1 = port.diffuse_lowp_chains(ip, ind, P, Xd.float().cpu().numpy(), 1, port.BF16, 32 // group, True)
            for kind, stage in ((5, 4), (6, 4), (9, 0), (9, 1), (10, 0), (10, 1)):
                Y = torch.empty((n, F), dtype=torch.float32, device="cuda")
                g.spmm(Xd, Y, group=group, vec=8, kind=kind, stage=stage)
                np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref1))
    finally:
        g.close()


def test_index_out_of_range_is_reported():
    m = wrap([0, 1, 2], [1, 5], np.ones(2, np.float32), 2)
    X = np.ones((2, 4), np.float32)
    with pytest.raises(scl.SCLError) as e:
        scl.diffusion.diffuse_matrix(m, X, 1)
    assert e.value.code == 14


def test_attach_keeps_graph_resident(graph_3k):
    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    P = port.transition(ip, ind, W.astype(np.float32), False, False)
    m = wrap(ip, ind, P.copy(), n)
    X0 = np.random.default_rng(3).standard_normal((n, 32)).astype(np.float32)
    X1 = X0.copy()
    scl.diffusion.diffuse_matrix(m, X1, 2)
    s1 = scl.diffusion.last_stats(m.lib)
    scl.diffusion.attach(m)
    X2 = X0.copy()
    scl.diffusion.diffuse_matrix(m, X2, 2)
    s2 = scl.diffusion.last_stats(m.lib)
    scl.diffusion.detach(m)
    np.testing.assert_array_equal(X1, X2)
    assert s2["h2d_bytes"] < s1["h2d_bytes"] and s2["device_ms"] > 0


# ---- device-resident graphs (scl_gpu.h) ------------------------------------------
def test_graph_build_from_knn_matches_oracle(graph_3k):
    import torch

    ki, kd, _, _, _ = graph_3k
    kd32 = kd.astype(np.float32)
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd32))
    ip, ind, val = g.export()
    _, w32 = port.gauss_weights(ki, kd32)
    oip, oind, oval = port.symmetrize(ki, w32)
    np.testing.assert_array_equal(ip, oip)
    np.testing.assert_array_equal(ind, oind)
    np.testing.assert_allclose(val, oval, rtol=4e-7, atol=0)


def test_graph_build_edge_cases():
    import torch

    idx = np.array([[1, -1, 1], [0, 2, -1], [2, 0, 1], [-1, -1, -1]], np.int32)
    dist = np.array([[0.5, 9.0, 0.25], [1.0, 2.0, 9.0], [4.0, 3.0, 8.0], [9.0, 9.0, 9.0]], np.float32)
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(idx), torch.from_numpy(dist))
    ip, ind, val = g.export()
    _, w = port.gauss_weights(idx.astype(np.int64), dist)
    oip, oind, oval = port.symmetrize(idx.astype(np.int64), w)
    np.testing.assert_array_equal(ip, oip)
    np.testing.assert_array_equal(ind, oind)
    np.testing.assert_allclose(val, oval, rtol=4e-7)


@pytest.mark.parametrize("kind", ["bf16", "f16"])
def test_low_precision_storage_bit_exact(graph_3k, kind):
    import torch

    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    P = port.transition(ip, ind, W.astype(np.float32), False, True)
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    tdt = torch.bfloat16 if kind == "bf16" else torch.float16
    g.set_storage(tdt)
    X0 = np.random.default_rng(9).standard_normal((n, 64)).astype(np.float32)
    Xd = torch.from_numpy(X0).cuda()
    # 64 16-bit columns = 128-byte rows: the split-chain kernel with 4 interleaved chains
    for final_f32 in (True, False):
        Y = g.diffuse(Xd, 4, out_dtype=torch.float32 if final_f32 else tdt).float().cpu().numpy()
        Yo = port.diffuse_lowp_chains(ip, ind, P, X0, 4, port.BF16 if kind == "bf16" else port.F16, 4, final_f32)
        np.testing.assert_array_equal(bits(Y), bits(Yo))
    # a width the sequential kernels handle (48 columns = 96-byte rows)
    X1 = np.random.default_rng(10).standard_normal((n, 48)).astype(np.float32)
    Y1 = g.diffuse(torch.from_numpy(X1).cuda(), 3, out_dtype=torch.float32).cpu().numpy()
    Yo1 = port.diffuse_lowp(ip, ind, P, X1, 3, port.BF16 if kind == "bf16" else port.F16, True)
    np.testing.assert_array_equal(bits(Y1), bits(Yo1))


@pytest.mark.parametrize("group", [1, 2, 4, 8, 16, 32])
def test_every_launch_shape_is_exact(graph_3k, group):
    import torch

    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    P = port.transition(ip, ind, W.astype(np.float32), False, True)
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    X0 = np.random.default_rng(4).standard_normal((n, 64)).astype(np.float32)
    Xd = torch.from_numpy(X0).cuda()
    ref1 = port.spmm(ip, ind, P, X0)
    shapes = [(1, 0, 8), (4, 0, 8)] + ([(4, 1, s) for s in (4, 8, 16)] if group >= 4 else [])
    if group == 16:
        shapes += [(4, 12, 4), (4, 12, 8), (4, 12, 16)]  # two rows per warp, 16-byte lanes
    if group == 32:
        shapes.append((2, 0, 8))  # whole warp per row, 8-byte lane chunks
        shapes += [(2, 2, 8), (2, 2, 16), (2, 3, 16), (2, 3, 32), (1, 3, 16)]  # row-block streams
        shapes += [(2, 4, 8), (2, 4, 16), (2, 4, 32)]  # fixed-pitch warp-per-row
        shapes += [(2, 7, 8), (2, 7, 16), (2, 7, 32)]  # flat entry stream over row blocks
        shapes += [(2, 11, 2), (2, 11, 3), (2, 11, 4), (2, 11, 6)]  # bulk-copy gathers into a ring
    for vec, kind, stage in shapes:
        Y = torch.empty_like(Xd)
        g.spmm(Xd, Y, group=group, vec=vec, kind=kind, stage=stage)
        np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref1))


# ---- locality reordering: a permutation of rows that must not change any bit ----
def _components_graph(n_comp=6, size=700, k=12, seed=21):
    """Disjoint mixture components interleaved in random row order."""
    from scl import synthetic

    rng = np.random.default_rng(seed)
    parts = []
    for c in range(n_comp):
        pts = synthetic.mixture(size, seed=seed + c, n_comp=1) + 100.0 * c
        ki, kd = synthetic.knn_exact(pts, k)
        parts.append((ki + c * size, kd))
    ki = np.concatenate([p[0] for p in parts])
    kd = np.concatenate([p[1] for p in parts])
    n = ki.shape[0]
    shuffle = rng.permutation(n)          # new id of old row
    inv = np.argsort(shuffle)
    ki = shuffle[ki[inv]]
    kd = kd[inv]
    return ki, kd


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_reordered_device_graph_is_bit_identical(storage):
    import torch

    ki, kd = _components_graph()
    n = ki.shape[0]
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd.astype(np.float32)))
    g.normalize()
    if storage == "bf16":
        g.set_storage(torch.bfloat16)
    X0 = torch.from_numpy(np.random.default_rng(0).standard_normal((n, 64)).astype(np.float32)).cuda()
    Y_plain = g.diffuse(X0, 5, out_dtype=torch.float32).cpu().numpy()
    g.reorder(1)
    perm, rounds = g.reorder_info()
    assert sorted(perm.tolist()) == list(range(n)) and rounds >= 1
    # rows of one component are contiguous after reordering
    from scipy.sparse.csgraph import connected_components
    import scipy.sparse as sp

    ip, ind, val = g.export()
    nc, lab = connected_components(sp.csr_matrix((val, ind, ip), shape=(n, n)), directed=False)
    assert nc == 6
    assert (np.diff(lab[perm]) != 0).sum() == nc - 1
    Y_re = g.diffuse(X0, 5, out_dtype=torch.float32).cpu().numpy()
    np.testing.assert_array_equal(bits(Y_re), bits(Y_plain))
    # in place
    X1 = X0.clone() if storage == "f32" else X0.to(torch.bfloat16)
    if storage == "f32":
        g.diffuse(X1, 5, out=X1)
        np.testing.assert_array_equal(bits(X1.cpu().numpy()), bits(Y_plain))


def test_reordered_drop_in_is_bit_identical():
    import torch

    ki, kd = _components_graph(seed=33)
    n = ki.shape[0]
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd.astype(np.float32)))
    g.normalize()
    ip, ind, P = g.export()
    X0 = np.random.default_rng(1).standard_normal((n, 32)).astype(np.float32)
    want = port.diffuse_matrix(ip, ind, P, X0, 6)
    m = wrap(ip, ind, P.copy(), n)
    for mode in (0, 1, -1):
        scl.diffusion.set_reorder(m, mode)
        X = X0.copy()
        scl.diffusion.diffuse_matrix(m, X, 6)
        np.testing.assert_array_equal(bits(X), bits(want))
        scl.diffusion.attach(m)
        X = X0.copy()
        scl.diffusion.diffuse_matrix(m, X, 6)
        scl.diffusion.detach(m)
        np.testing.assert_array_equal(bits(X), bits(want))
    scl.diffusion.set_reorder(m, -1)


# ---- split-chain kernel (16-bit storage, 16-byte lanes) ------------------------------
@pytest.mark.parametrize("storage,F", [("bf16", 64), ("bf16", 128), ("f16", 64), ("f16", 128)])
def test_split_chain_shapes_are_exact(graph_3k, storage, F):
    """Every split-chain launch shape (one 16-byte chunk per lane, 32/group
    entries per load feeding as many interleaved fma chains; batches of gathers;
    plain or mixed-precision fma) gives the bits of the oracle's chain
    restatement."""
    import torch

    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    P = port.transition(ip, ind, W.astype(np.float32), False, True)
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    tdt = torch.bfloat16 if storage == "bf16" else torch.float16
    kind_code = port.BF16 if storage == "bf16" else port.F16
    try:
        g.set_storage(tdt)
        X0 = np.random.default_rng(F).standard_normal((n, F)).astype(np.float32)
        Xd = torch.from_numpy(X0).cuda().to(tdt)
        group = F * 2 // 16
        chains = 32 // group
        ref1 = port.diffuse_lowp_chains(ip, ind, P, Xd.float().cpu().numpy(), 1, kind_code, chains, True)
        stages = (2, 4, 8) if group == 8 else (4, 8, 16)
        shapes = [(k, st) for k in (5, 6) for st in stages] + [(9, 0), (9, 1), (10, 0)]
        shapes += [(14, st) for st in (4, 8, 16)]  # rows in lockstep, 32/group rows per warp
        if storage == "bf16":
            shapes.append((10, 1))  # packed f32x2 fma
        ref1_lowp = port.diffuse_lowp_chains(ip, ind, P, Xd.float().cpu().numpy(), 1, kind_code, chains, False)
        for kind, stage in shapes:
            Y = torch.empty((n, F), dtype=torch.float32, device="cuda")
            g.spmm(Xd, Y, group=group, vec=8, kind=kind, stage=stage)
            np.testing.assert_array_equal(bits(Y.cpu().numpy()), bits(ref1))
            Yl = torch.empty((n, F), dtype=tdt, device="cuda")  # 16-bit output, rounded once
            g.spmm(Xd, Yl, group=group, vec=8, kind=kind, stage=stage)
            np.testing.assert_array_equal(bits(Yl.float().cpu().numpy()), bits(ref1_lowp))
        Yd = g.diffuse(Xd, 3, out_dtype=torch.float32).cpu().numpy()
        np.testing.assert_array_equal(bits(Yd), bits(port.diffuse_lowp_chains(ip, ind, P, X0, 3, kind_code, chains)))
    finally:
        g.close()


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_autotune_keeps_the_bits(graph_3k, storage):
    """The autotuner only picks among launch shapes of the default kernel's
    family, so diffusion results are bit-identical before and after it."""
    import torch

    _, _, ip, ind, W = graph_3k
    n = ip.size - 1
    P = port.transition(ip, ind, W.astype(np.float32), False, True)
    g = scl.gpu.GpuGraph.from_csr(ip, ind.astype(np.int32), P, (n, n))
    try:
        g.reorder(1)
        if storage == "bf16":
            g.set_storage(torch.bfloat16)
        X0 = torch.from_numpy(np.random.default_rng(2).standard_normal((n, 64)).astype(np.float32)).cuda()
        before = g.diffuse(X0, 4, out_dtype=torch.float32)
        res = g.autotune(64, reps=2)
        assert res["ms"] > 0 and res["kind"] in (4, 5, 6, 7, 9, 10, 11, 12, 13)
        after = g.diffuse(X0, 4, out_dtype=torch.float32)
        assert torch.equal(before, after)
        assert g.gather_floor(64, reps=2) > 0
    finally:
        g.close()
