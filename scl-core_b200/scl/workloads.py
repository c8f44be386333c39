"""Synthetic diffusion workloads on the device (benchmark and profiling cases).

    python -m scl.workloads spmm --cells 200000 --k 30 --features 64 --steps 3 [--storage bf16] [--no-reorder]
    python -m scl.workloads backward --cells 200000 --k 30 --features 32 --steps 8 --every 4

builds the seeded mixture graph on the current GPU (kNN with torch as an input
generator, then this library's weights / symmetrisation / normalisation /
reordering) and runs `steps` diffusion steps through scl_gpu_diffuse (spmm),
or a checkpointed forward plus the backward pass of L = sum((X_T - Y)^2)
through scl_gpu_diffuse_checkpointed / scl_gpu_diffuse_backward (backward) —
the cases the ncu captures under profiles/ were taken on.
"""
from __future__ import annotations

import argparse
import time


def build_graph(n_cells: int, k: int, device="cuda", seed: int = 0, reorder: bool = True, stream=None):
    """(GpuGraph, knn_idx, knn_dist, timings dict) for the seeded mixture."""
    import torch

    from . import synthetic
    from .gpu import GpuGraph

    t0 = time.time()
    pts = synthetic.mixture(n_cells, seed=seed)
    ki, kd = synthetic.knn_device(pts, k, device=device, block=2048)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # the kNN blocks' distance tiles (GBs) are not needed any more
    t_knn = time.time() - t0
    s = stream if stream is not None else torch.cuda.current_stream()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(s)
    g = GpuGraph.from_knn(ki, kd, stream=s)
    g.normalize(symmetric=False, stream=s)
    e1.record(s)
    if reorder:
        g.reorder(1, stream=s)
    e2.record(s)
    e2.synchronize()
    return g, ki, kd, {"knn_s": t_knn, "build_ms": e0.elapsed_time(e1), "reorder_ms": e1.elapsed_time(e2)}


def _main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["spmm", "backward", "knn", "ppr", "dpt"])
    ap.add_argument("--every", type=int, default=4)
    ap.add_argument("--cells", type=int, default=200_000)
    ap.add_argument("--k", type=int, default=30)
    ap.add_argument("--features", type=int, default=64)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16"])
    ap.add_argument("--no-reorder", action="store_true")
    ap.add_argument("--plan", default="", help="group,vec,kind,stage launch shape for diffuse (default: built-in)")
    a = ap.parse_args()
    if a.case == "knn":  # brute-force kNN of the mixture through scl_knn (host buffers)
        import numpy as np

        from . import neighbors, synthetic
        from .core.sparse import CsrMatrix

        pts = synthetic.mixture(a.cells, seed=21).astype(np.float32)[:, : a.features]
        pts = np.ascontiguousarray(pts)
        n, d = pts.shape
        m = CsrMatrix.wrap(np.arange(0, (n + 1) * d, d, dtype=np.int32), np.tile(np.arange(d, dtype=np.int32), n),
                           pts.reshape(-1), (n, d))
        norms = neighbors.compute_norms(m)
        for _ in range(max(a.steps, 1)):
            idx, dist = neighbors.knn(m, a.k, norms)
        print(f"cells={n} features={d} k={a.k} checksum={float(dist[np.isfinite(dist)].sum()):.6e}")
        return
    if a.case == "ppr":  # personalized PageRank from cell 0 on the row-normalised graph
        from . import diffusion
        from .core.sparse import CsrMatrix

        g, _, _, tm = build_graph(a.cells, a.k, reorder=False)
        ip, ind, P = g.export()
        m = CsrMatrix.wrap(ip.astype("int32"), ind.astype("int32"), P, (a.cells, a.cells))
        for _ in range(max(a.steps, 1)):
            pr = diffusion.personalized_pagerank(m, 0)
        print(f"cells={a.cells} nnz={ind.size} checksum={float(pr.sum()):.6e}")
        return
    if a.case == "dpt":  # diffusion pseudotime from cell 0 on the row-normalised graph (max 100 steps, tol 1e-6)
        from . import diffusion
        from .core.sparse import CsrMatrix

        g, _, _, tm = build_graph(a.cells, a.k, reorder=False)
        ip, ind, P = g.export()
        m = CsrMatrix.wrap(ip.astype("int32"), ind.astype("int32"), P, (a.cells, a.cells))
        for _ in range(max(a.steps, 1)):
            pt = diffusion.compute_dpt(m, 0)
        print(f"cells={a.cells} nnz={ind.size} checksum={float(pt.sum()):.6e}")
        return
    if a.case == "backward":
        g, _, _, tm = build_graph(a.cells, a.k, reorder=False)
        gen = torch.Generator(device="cuda").manual_seed(7)
        X0 = torch.randn((a.cells, a.features), device="cuda", generator=gen)
        Yt = torch.randn((a.cells, a.features), device="cuda", generator=gen)
        XT, ck = g.diffuse_checkpointed(X0, a.steps, a.every)
        dX, dW = g.diffuse_backward(X0, ck, 2.0 * (XT - Yt), a.steps, a.every)
        torch.cuda.synchronize()
        n, _, nnz = g.shape
        print(f"cells={n} nnz={nnz} features={a.features} steps={a.steps} every={a.every} "
              f"loss={float(((XT - Yt) ** 2).sum()):.6e} |dX|={float(dX.norm()):.6e} |dW|={float(dW.norm()):.6e}")
        return
    g, _, _, tm = build_graph(a.cells, a.k, reorder=not a.no_reorder)
    if a.storage != "f32":
        g.set_storage(torch.bfloat16 if a.storage == "bf16" else torch.float16)
    if a.plan:
        grp, vec, kind, stage = (int(x) for x in a.plan.split(","))
        g.set_plan(a.features, grp, vec, kind, stage)
    X = torch.randn((a.cells, a.features), device="cuda")
    if a.storage != "f32":
        X = X.to(torch.bfloat16 if a.storage == "bf16" else torch.float16)
    Y = g.diffuse(X, a.steps)
    torch.cuda.synchronize()
    n, _, nnz = g.shape
    print(f"cells={n} nnz={nnz} features={a.features} steps={a.steps} storage={a.storage} "
          f"reorder={not a.no_reorder} build_ms={tm['build_ms']:.2f} reorder_ms={tm['reorder_ms']:.2f} "
          f"checksum={float(Y.float().sum()):.6e}")


if __name__ == "__main__":
    _main()
