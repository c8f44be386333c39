"""Test configuration.

Markers:
  gpu — needs a CUDA device (B200); everything else runs on CPU.

The product libraries (scl-core_b200/scl/libs) and the oracle port
(oracle/_build) are built on first use if missing; the reference build
(oracle/_ref) is used when present and those tests skip otherwise.
"""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "scl-core_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU")


def _ensure_built():
    libs = ROOT / "scl-core_b200" / "scl" / "libs"
    if not all((libs / f"libscl_{v}.so").exists() for v in ("f32_i32", "f32_i64", "f64_i32", "f64_i64")):
        sys.path.insert(0, str(ROOT / "scl-core_b200"))
        import build as _b  # scl-core_b200/build.py

        _b.build()
    if not (ROOT / "oracle" / "_build" / "liboracle_port.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "port"], check=True, capture_output=True)


_ensure_built()

GOLDEN = ROOT / "tests" / "golden" / "diffusion_small.npz"


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def mixture_graph(n, k, seed=0):
    """(knn_idx, knn_dist, indptr, indices, W f64) for a seeded mixture graph."""
    from oracle import port
    from scl import synthetic

    pts = synthetic.mixture(n, seed=seed)
    ki, kd = synthetic.knn_exact(pts, k)
    _, w = port.gauss_weights(ki, kd)
    ip, ind, W = port.symmetrize(ki, w)
    return ki, kd, ip, ind, W


@pytest.fixture(scope="session")
def graph_20k():
    """The 20,000-cell, k=15 graph of the CPU-runnable diffusion configuration."""
    return mixture_graph(20000, 15, seed=0)


@pytest.fixture(scope="session")
def graph_3k():
    return mixture_graph(3000, 15, seed=5)
