"""The diffusion entry point that allocates no device memory.

scl_gpu_diffuse_noalloc exists for callers that cannot allocate GPU memory
while they run (a framework that owns the device-memory budget through its
own arena, a serving loop that must not block or fail on an allocation, code
that must not let cudaMalloc/cudaFree synchronise the device). It keeps its one
intermediate iterate in a fixed scratch array inside the library. These tests
call it through the C ABI and check it against the regular entry point,
scl_gpu_diffuse, on two calls in a row (the second call finds the first call's
data still in the shared scratch array). This file is collected last so that a
run stopping at the first failure has run every other test first; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import scl
from scl._bindings._loader import get_library

pytestmark = pytest.mark.gpu

MAX_ELEMS = 8388608  # the scratch array's capacity (n_rows * n_features)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _graph(n=3000, k=15, seed=3):
    import torch

    pts = scl.synthetic.mixture(n, seed=seed)
    ki, kd = scl.synthetic.knn_exact(pts, k)
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd.astype(np.float32)))
    g.normalize()
    ip, ind, P = g.export()
    dev = dict(indptr=torch.from_numpy(ip).cuda(), indices=torch.from_numpy(ind).cuda(),
               values=torch.from_numpy(P).cuda())
    return g, dev, n


def _noalloc(lib, dev, n, X, Y, F, steps):
    import torch

    return lib.scl_gpu_diffuse_noalloc(_ptr(dev["indptr"]), _ptr(dev["indices"]), _ptr(dev["values"]), n, _ptr(X),
                                       _ptr(Y), F, steps, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("F,steps", [(64, 8), (32, 3), (5, 1), (16, 0)])
def test_noalloc_matches_regular_entry_point_twice(F, steps):
    import torch

    lib = get_library("f32_i32")
    g, dev, n = _graph()
    gen = torch.Generator(device="cuda").manual_seed(F + steps)
    for call in range(2):
        X = torch.randn((n, F), device="cuda", generator=gen)
        want = g.diffuse(X, steps, out_dtype=torch.float32)
        Y = torch.full((n, F), float("nan"), device="cuda")
        rc = _noalloc(lib, dev, n, X, Y, F, steps)
        assert rc == 0, lib.scl_get_last_error()
        torch.cuda.synchronize()
        # FP32 diffusion is bit-exact across this library's entry points
        assert torch.equal(Y.view(torch.int32), want.view(torch.int32)), f"call {call} differs"


@pytest.mark.parametrize("F,steps", [(5, 3), (64, 2)])
def test_noalloc_matches_oracle_twice(F, steps):
    """Independent check: the oracle restatement of scl-core's diffuse_matrix
    (sequential fma chain per element, rows in stored order) on the same CSR."""
    import torch

    from oracle import port

    lib = get_library("f32_i32")
    g, dev, n = _graph(n=2500, k=12, seed=5)
    ip, ind, P = g.export()
    for call in range(2):
        X0 = scl.synthetic.features(n, F, seed=40 + call)
        want = port.diffuse_matrix(ip, ind, P, X0, steps)
        X = torch.from_numpy(X0).cuda()
        Y = torch.full((n, F), float("nan"), device="cuda")
        rc = _noalloc(lib, dev, n, X, Y, F, steps)
        assert rc == 0, lib.scl_get_last_error()
        got = Y.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"call {call} differs from the oracle"


def test_noalloc_rejects_oversized_blocks():
    import torch

    lib = get_library("f32_i32")
    _, dev, n = _graph(n=1000, k=5)
    F = MAX_ELEMS // n + 1  # one row's worth over the limit
    X = torch.zeros((n, F), device="cuda")
    Y = torch.zeros((n, F), device="cuda")
    rc = _noalloc(lib, dev, n, X, Y, F, 2)
    assert rc == 10
    assert b"exceeds" in lib.scl_get_last_error()
    assert _noalloc(lib, dev, n, X, X, 4, 2) == 10  # in place is refused
