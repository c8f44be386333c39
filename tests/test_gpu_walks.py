"""Vector walks through the drop-in C ABI on the GPU (random walk with
restart, personalized PageRank, heat-kernel signature, lazy random walk)
against the restatement (oracle/port.py) bit for bit; the restatement is
checked against scl-core's own build in test_walks_oracle.py."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import scl
from oracle import port

pytestmark = pytest.mark.gpu

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)
VARIANTS = [(np.float32, np.int32), (np.float64, np.int64)]


def _graph(n, dt, idt, seed=3, density=0.03, empty=()):
    T = sp.random(n, n, density=min(1.0, density), random_state=seed, format="lil", dtype=np.float64)
    for r in empty:
        T[r, :] = 0
    T = T.tocsr()
    rs = np.asarray(T.sum(1)).ravel()
    T = (sp.diags(np.where(rs > 0, 1.0 / np.maximum(rs, 1e-300), 0.0)) @ T).tocsr().astype(dt)
    T.sort_indices()
    m = scl.CsrMatrix.wrap(T.indptr.astype(idt), T.indices.astype(idt), T.data, (n, n))
    return m, (T.indptr, T.indices, T.data)


@pytest.mark.parametrize("dt,idt", VARIANTS)
@pytest.mark.parametrize("n", [1, 7, 300, 1500, 20000])
def test_lazy_walk_and_heat_kernel_bit_exact(dt, idt, n):
    m, (ip, ind, v) = _graph(n, dt, idt, density=12.0 / n, empty=(0,) if n > 5 else ())
    x0 = np.random.default_rng(n).random(n).astype(dt)
    for lazy, steps in ((0.3, 5), (0.0, 2), (1.0, 3)):
        x = x0.copy()
        scl.diffusion.lazy_random_walk(m, x, steps, lazy)
        eff = dt(0.5) if lazy == 0.0 else dt(lazy)  # 0 means the default 0.5
        np.testing.assert_array_equal(bits(x), bits(port.walk_linear(ip, ind, v, x0, steps, eff, dt(1) - eff)))
    for t, steps in ((1.0, 10), (2.5, 4), (0.5, 0)):
        s = scl.diffusion.heat_kernel_signature(m, t=t, n_steps=steps)
        k = 10 if steps == 0 else steps
        d = dt(t) / dt(k)
        np.testing.assert_array_equal(bits(s), bits(port.walk_linear(ip, ind, v, np.ones(n, dt), k, dt(1) - d, d)))


@pytest.mark.parametrize("dt,idt", VARIANTS)
@pytest.mark.parametrize("n", [5, 500, 1500, 20000])
def test_restart_walk_and_pagerank_bit_exact(dt, idt, n):
    m, (ip, ind, v) = _graph(n, dt, idt, seed=5, density=10.0 / n)
    for seeds in ([0, 3, 3, n + 4, -1], [n - 1]):
        for max_iter in (1, 2, 3, 100):
            got = scl.diffusion.random_walk_with_restart(m, seeds, alpha=0.7, max_iter=max_iter, tol=1e-6)
            want, _ = port.walk_restart(ip, ind, v, seeds, n, dt(0.7), max_iter, dt(1e-6), dt)
            np.testing.assert_array_equal(bits(got), bits(want))
    got = scl.diffusion.personalized_pagerank(m, n // 2)
    want, _ = port.walk_restart(ip, ind, v, [n // 2], n, dt(0.85), 100, dt(1e-6), dt)
    np.testing.assert_array_equal(bits(got), bits(want))
    # defaults: alpha 0 -> 0.85, max_iter 0 -> 100, tol 0 -> 1e-6
    got0 = scl.diffusion.random_walk_with_restart(m, [1 % n], alpha=0.0, max_iter=0, tol=0.0)
    want0, _ = port.walk_restart(ip, ind, v, [1 % n], n, dt(0.85), 100, dt(1e-6), dt)
    np.testing.assert_array_equal(bits(got0), bits(want0))
    # no seed in range: zero scores
    assert not scl.diffusion.random_walk_with_restart(m, [-3, n], alpha=0.5).any()


def test_longer_output_buffers_keep_their_tail_and_errors_follow_the_reference():
    n = 50
    m, (ip, ind, v) = _graph(n, np.float32, np.int32, density=0.1)
    lib = m.lib
    P = lambda a: a.ctypes.data_as(ctypes.POINTER(lib.real_type))
    out = np.full(n + 5, -3.0, np.float32)
    assert lib.scl_diffusion_heat_kernel_signature(m.handle, P(out), n + 5, 1.0, 3) == 0
    assert (out[n:] == -3.0).all()
    seeds = np.array([1, 2], np.int32)
    sp_ = seeds.ctypes.data_as(ctypes.POINTER(lib.index_type))
    assert lib.scl_diffusion_random_walk_with_restart(m.handle, sp_, 2, P(out), n + 5, 0.5, 10, 1e-6) == 0
    assert (out[n:] == -3.0).all()
    # the reference's argument checks and codes
    assert lib.scl_diffusion_random_walk_with_restart(None, sp_, 2, P(out), n, 0.5, 10, 1e-6) == 4
    assert lib.scl_diffusion_random_walk_with_restart(m.handle, None, 2, P(out), n, 0.5, 10, 1e-6) == 4
    assert lib.scl_diffusion_random_walk_with_restart(m.handle, sp_, 0, P(out), n, 0.5, 10, 1e-6) == 10
    assert lib.scl_diffusion_random_walk_with_restart(m.handle, sp_, 2, P(out), n, 1.5, 10, 1e-6) == 10
    assert lib.scl_diffusion_random_walk_with_restart(m.handle, sp_, 2, P(out), n - 1, 0.5, 10, 1e-6) == 11
    assert lib.scl_diffusion_personalized_pagerank(m.handle, 0, P(out), 0, 0.5, 10, 1e-6) == 10
    assert lib.scl_diffusion_heat_kernel_signature(m.handle, P(out), n, 0.0, 3) == 10
    assert lib.scl_diffusion_lazy_random_walk(m.handle, P(out), n, 0, 0.5) == 10
    assert lib.scl_diffusion_lazy_random_walk(m.handle, P(out), n, 2, -0.1) == 10
    assert lib.scl_diffusion_lazy_random_walk(m.handle, P(out), n - 1, 2, 0.5) == 11


@pytest.mark.parametrize("dt,idt", VARIANTS)
def test_pseudotime_long_rows_bit_exact(dt, idt):
    """Rows far longer than one staging round of the DPT step (and 32-row
    groups holding many rounds), next to empty rows."""
    n = 3000
    m, (ip, ind, v) = _graph(n, dt, idt, seed=12, density=0.4, empty=(5, 6, 2999))
    for root, max_iter, tol in ((0, 30, 1e-6), (1700, 100, 1e-3)):
        got = scl.diffusion.compute_dpt(m, root, max_iter=max_iter, tol=tol)
        np.testing.assert_array_equal(bits(got), bits(port.dpt(ip, ind, v, root, max_iter, dt(tol), dt)))


@pytest.mark.parametrize("dt,idt", VARIANTS)
@pytest.mark.parametrize("n", [3, 400, 20000])
def test_pseudotime_bit_exact(dt, idt, n):
    m, (ip, ind, v) = _graph(n, dt, idt, seed=8, density=10.0 / n)
    for root, max_iter, tol in ((0, 100, 1e-6), (n - 1, 3, 1e-6), (n // 2, 100, 1e-2), (1 % n, 0, 0.0)):
        got = scl.diffusion.compute_dpt(m, root, max_iter=max_iter, tol=tol)
        mi = 100 if max_iter == 0 else max_iter
        t = dt(1e-6) if tol == 0.0 else dt(tol)
        np.testing.assert_array_equal(bits(got), bits(port.dpt(ip, ind, v, root, mi, t, dt)))
    got = scl.diffusion.compute_dpt_multi_root(m, [0, n // 3, -2, n + 5, 0], max_iter=40)
    np.testing.assert_array_equal(bits(got), bits(port.dpt_multi_root(ip, ind, v, [0, n // 3, -2, n + 5, 0], 40, dt)))
    assert (scl.diffusion.compute_dpt_multi_root(m, [-1, n]) == 1).all()
    lib = m.lib
    out = np.zeros(n, dt)
    P = out.ctypes.data_as(ctypes.POINTER(lib.real_type))
    assert lib.scl_diffusion_compute_dpt(m.handle, n, P, n, 10, 1e-6) == 10  # root out of range
    assert lib.scl_diffusion_compute_dpt(m.handle, 0, P, n - 1, 10, 1e-6) == (11 if n > 1 else 10)
    assert lib.scl_diffusion_compute_dpt(None, 0, P, n, 10, 1e-6) == 4
