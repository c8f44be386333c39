"""FP64 residual check on the device (scl_gpu_residual_fp64).

The reduction must give the same errors as an FP64 NumPy computation over the
same two blocks (sums to rounding of the order, maxima exactly), for every
storage dtype, and be bit-stable across runs. The end-to-end case checks a
16-bit diffusion against the oracle's FP64 restatement of scl-core's
diffuse_matrix (scl/kernel/diffusion.hpp:638-664) on the same graph."""
import numpy as np
import pytest

import scl
from oracle import port

pytestmark = pytest.mark.gpu


def _numpy_errors(x, r, floor):
    x = x.astype(np.float64)
    d = x - r
    return {"rel_fro": np.sqrt((d * d).sum()) / np.sqrt((r * r).sum()),
            "max_rel": float((np.abs(d) / np.maximum(np.abs(r), floor)).max()),
            "max_abs": float(np.abs(d).max()), "ref_fro": float(np.sqrt((r * r).sum()))}


@pytest.mark.parametrize("dtype", ["float32", "float64", "bfloat16", "float16"])
@pytest.mark.parametrize("shape", [(1, 1), (37, 5), (20000, 64)])
def test_residual_matches_numpy(dtype, shape):
    import torch

    gen = np.random.default_rng([len(dtype), *shape])
    R = gen.standard_normal(shape)
    Xd = (torch.from_numpy(R) + 1e-3 * torch.from_numpy(gen.standard_normal(shape))).to(getattr(torch, dtype))
    x_host = Xd.float().numpy() if dtype in ("bfloat16", "float16") else Xd.numpy()
    want = _numpy_errors(x_host, R, 1e-3)
    got = scl.gpu.residual_fp64(Xd.cuda(), torch.from_numpy(R).cuda(), rel_floor=1e-3)
    assert got["max_abs"] == want["max_abs"]
    assert got["max_rel"] == want["max_rel"]
    assert got["rel_fro"] == pytest.approx(want["rel_fro"], rel=1e-12)
    assert got["ref_fro"] == pytest.approx(want["ref_fro"], rel=1e-12)
    again = scl.gpu.residual_fp64(Xd.cuda(), torch.from_numpy(R).cuda(), rel_floor=1e-3)
    assert again == got  # fixed reduction order


def test_residual_zero_reference_and_identity():
    import torch

    z = torch.zeros((100, 3), dtype=torch.float64, device="cuda")
    assert scl.gpu.residual_fp64(z.float(), z)["rel_fro"] == 0.0
    x = torch.randn((100, 3), dtype=torch.float64, device="cuda")
    r = scl.gpu.residual_fp64(x, x)
    assert r["rel_fro"] == 0.0 and r["max_abs"] == 0.0


@pytest.mark.parametrize("storage", ["bfloat16", "float16"])
def test_lowp_diffusion_error_vs_fp64_oracle(storage):
    """16-bit storage / FP32 accumulation against the FP64 oracle diffusion of
    the same weights: the device residual equals NumPy's over the same blocks."""
    import torch

    n, k, F, T = 3000, 15, 16, 8
    pts = scl.synthetic.mixture(n, seed=4)
    ki, kd = scl.synthetic.knn_exact(pts, k)
    g = scl.gpu.GpuGraph.from_knn(torch.from_numpy(ki.astype(np.int32)), torch.from_numpy(kd.astype(np.float32)))
    ip, ind, W = g.export()
    g.normalize()
    P64 = port.transition(ip, ind, W.astype(np.float64))
    X0 = scl.synthetic.features(n, F, seed=9)
    Y64 = port.diffuse_matrix(ip, ind, P64, X0.astype(np.float64), T)
    g.set_storage(getattr(torch, storage))
    Yl = g.diffuse(torch.from_numpy(X0).cuda().to(getattr(torch, storage)), T, out_dtype=torch.float32)
    got = scl.gpu.residual_fp64(Yl, torch.from_numpy(Y64).cuda(), rel_floor=1e-3)
    want = _numpy_errors(Yl.cpu().numpy(), Y64, 1e-3)
    assert got["max_abs"] == want["max_abs"] and got["max_rel"] == want["max_rel"]
    assert got["rel_fro"] == pytest.approx(want["rel_fro"], rel=1e-12)
    # 16-bit iterates: 8 (bf16) or 11 (f16) mantissa bits per stored step
    assert got["rel_fro"] < (2e-2 if storage == "bfloat16" else 3e-3)
    g.close()
