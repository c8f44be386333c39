"""Differentiable graph diffusion for PyTorch.

    Y = scl.autograd.diffuse(graph, X0, n_steps, weights=w, symmetric=False, every=4)

computes Y = P^n_steps X0 with P = normalise(W) on a device graph and, in
backward, dL/dX0 and dL/dW through the library's own kernels
(scl_gpu_diffuse_checkpointed / scl_gpu_diffuse_backward): the forward keeps
every `every`-th iterate (and, by default, the last segment's iterates), the
backward recomputes the rest of each segment from its checkpoint and runs one
fused transpose-SpMM + SDDMM kernel per step.

`weights` (optional) is a CUDA tensor of the graph's nnz pre-normalisation
weights in its CSR order; when given, the forward loads it into the graph and
normalises, so gradients flow to it. Without it the graph's current values are
used as P and only X0 receives a gradient.

No scl-core counterpart: scl-core computes no gradients. The forward is
scl_diffusion_compute_transition_matrix + scl_diffusion_diffuse_matrix
(scl/kernel/diffusion.hpp:492-603, 638-664).
"""
from __future__ import annotations

import torch

from .gpu import GpuGraph


class DiffusionFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, X0, weights, graph: GpuGraph, n_steps: int, every: int, symmetric: bool, keep_last: bool):
        if weights is not None:
            graph.set_weights(weights.detach())
            graph.normalize(symmetric=symmetric)
        X0c = X0.detach().contiguous()
        Y, ckpt = graph.diffuse_checkpointed(X0c, n_steps, every, keep_last=keep_last)
        ctx.graph = graph
        ctx.n_steps, ctx.every, ctx.keep_last = n_steps, every, keep_last
        ctx.has_weights = weights is not None
        ctx.save_for_backward(X0c, ckpt)
        return Y

    @staticmethod
    def backward(ctx, dY):
        X0, ckpt = ctx.saved_tensors
        need_w = ctx.has_weights and ctx.needs_input_grad[1]
        dX0, dW = ctx.graph.diffuse_backward(X0, ckpt, dY.contiguous(), ctx.n_steps, ctx.every, need_dW=need_w,
                                             keep_last=ctx.keep_last)
        return (dX0 if ctx.needs_input_grad[0] else None), (dW if need_w else None), None, None, None, None, None


def diffuse(graph: GpuGraph, X0, n_steps: int, weights=None, symmetric: bool = False, every: int = 4,
            keep_last: bool = True):
    """Differentiable P^n_steps X0 (f32 or f64 CUDA tensors, graph in the same dtype).

    Memory: (n_steps - 1) // every checkpoint blocks, plus the last segment's
    iterates when keep_last (saving their recomputation in backward)."""
    if every < 1:
        raise ValueError("every must be >= 1")
    return DiffusionFunction.apply(X0, weights, graph, int(n_steps), int(every), bool(symmetric), bool(keep_last))
