"""Seeded synthetic inputs for the diffusion workloads.

Cells are drawn from a 10-component Gaussian mixture in 50-D: component means
~ N(0, 4 I) (std 2), unit-variance isotropic noise, labels uniform. The kNN
graph is built by brute force (self excluded, neighbours in ascending distance,
Euclidean distances) in the same list format as scl-core's kNN
(scl/kernel/neighbors.hpp:319-478): row i holds k (index, distance) pairs.

Two kNN builders:
  * ``knn_exact``  — FP64 NumPy, ties broken by (distance, index); used for the
                     parity cases, where both sides must read identical lists.
  * ``knn_device`` — FP32 torch on a CUDA device: the kNN lists of the
                     benchmark's reference arm, which runs scl-core's own CPU
                     code and loads none of this library (an input generator,
                     not a measured step).
"""
from __future__ import annotations

import numpy as np


def mixture(n: int, dim: int = 50, n_comp: int = 10, seed: int = 0) -> np.ndarray:
    """n x dim float64 points from the seeded mixture."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, 2.0, size=(n_comp, dim))
    labels = rng.integers(0, n_comp, size=n)
    return means[labels] + rng.normal(0.0, 1.0, size=(n, dim))


def features(n: int, F: int, seed: int = 1, dtype=np.float32) -> np.ndarray:
    """n x F N(0, 1) feature block."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, F)).astype(dtype)


def knn_exact(points: np.ndarray, k: int, block: int = 1024):
    """Exact FP64 kNN: (indices int64 n x k, distances float64 n x k).

    d^2 = |a|^2 + |b|^2 - 2 a.b clamped at 0 (as neighbors.hpp:416-417), self
    excluded, ascending by (d^2, j)."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n = pts.shape[0]
    if k >= n:
        raise ValueError("k must be < n")
    norms = np.einsum("ij,ij->i", pts, pts)
    out_i = np.empty((n, k), np.int64)
    out_d = np.empty((n, k), np.float64)
    cols = np.arange(n)
    for s in range(0, n, block):
        e = min(n, s + block)
        d2 = norms[s:e, None] + norms[None, :] - 2.0 * (pts[s:e] @ pts.T)
        np.maximum(d2, 0.0, out=d2)
        d2[np.arange(e - s), np.arange(s, e)] = np.inf
        part = np.argpartition(d2, k, axis=1)[:, : k + 1]
        for r in range(e - s):
            cand = part[r]
            dv = d2[r, cand]
            order = np.lexsort((cols[cand], dv))[:k]
            out_i[s + r] = cand[order]
            out_d[s + r] = np.sqrt(dv[order])
    return out_i, out_d


def knn_device(points, k: int, device="cuda", block: int = 4096):
    """FP32 kNN on a CUDA device with torch: (indices int32, distances float32) tensors."""
    import torch

    pts = torch.as_tensor(np.ascontiguousarray(points, dtype=np.float32), device=device)
    n = pts.shape[0]
    norms = (pts * pts).sum(1)
    out_i = torch.empty((n, k), dtype=torch.int32, device=device)
    out_d = torch.empty((n, k), dtype=torch.float32, device=device)
    for s in range(0, n, block):
        e = min(n, s + block)
        d2 = norms[s:e, None] + norms[None, :] - 2.0 * (pts[s:e] @ pts.T)
        d2.clamp_(min=0.0)
        d2[torch.arange(e - s, device=device), torch.arange(s, e, device=device)] = float("inf")
        vals, idx = torch.topk(d2, k, dim=1, largest=False, sorted=True)
        out_i[s:e] = idx.to(torch.int32)
        out_d[s:e] = vals.sqrt()
    return out_i, out_d
