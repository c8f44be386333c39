"""The vector-walk restatement (oracle/port.py: walk_linear, walk_restart)
against scl-core's own random walk with restart, personalized PageRank,
heat-kernel signature and lazy random walk compiled from the reference
sources. scl-core's SpMV rounding depends on its compiler's contraction of
`sum += v * x`, so agreement is to a few ulps (tolerances below), while the
restart walk's buffer semantics (the caller's array after max_iter unconverged
steps) and its step count must match exactly."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import port, ref

TOL = {np.float32: dict(rtol=2e-6, atol=1e-9), np.float64: dict(rtol=1e-14, atol=1e-18)}


def _ref(variant):
    if not ref.available(variant):
        pytest.skip("reference library not built (make -C oracle ref)")
    return ref.RefLib(variant)


def _walk_graph(n, dt, seed=3, density=0.03):
    T = sp.random(n, n, density=density, random_state=seed, format="csr", dtype=np.float64)
    rs = np.asarray(T.sum(1)).ravel()
    T = (sp.diags(np.where(rs > 0, 1.0 / np.maximum(rs, 1e-300), 0.0)) @ T).tocsr().astype(dt)
    T.sort_indices()
    return T.indptr, T.indices, T.data


@pytest.mark.parametrize("variant,dt", [("f32_i32", np.float32), ("f64_i64", np.float64)])
def test_linear_walks_match_reference(variant, dt):
    R = _ref(variant)
    for n in (40, 500):  # below and above the reference's parallel threshold
        ip, ind, v = _walk_graph(n, dt)
        x0 = np.random.default_rng(n).random(n).astype(dt)
        for lazy, steps in ((0.3, 5), (0.5, 1), (1.0, 3)):
            want = R.walk("lazy", ip, ind, v, n, x=x0, steps=steps, laziness=lazy)
            got = port.walk_linear(ip, ind, v, x0, steps, dt(lazy), dt(1) - dt(lazy))
            np.testing.assert_allclose(got, want, **TOL[dt])
        for t, steps in ((1.0, 10), (2.5, 4)):
            want = R.walk("hks", ip, ind, v, n, t=t, steps=steps)
            d = dt(t) / dt(steps)
            got = port.walk_linear(ip, ind, v, np.ones(n, dt), steps, dt(1) - d, d)
            np.testing.assert_allclose(got, want, **TOL[dt])


@pytest.mark.parametrize("variant,dt", [("f32_i32", np.float32), ("f64_i64", np.float64)])
def test_restart_walk_matches_reference(variant, dt):
    R = _ref(variant)
    n = 500
    ip, ind, v = _walk_graph(n, dt, seed=4)
    for seeds in ([3, 7, 7, 900, -1], [0], [499, 250]):
        for max_iter in (1, 2, 3, 100):
            want = R.walk("rwr", ip, ind, v, n, seeds=seeds, alpha=0.7, max_iter=max_iter, tol=1e-6)
            got, _ = port.walk_restart(ip, ind, v, seeds, n, dt(0.7), max_iter, dt(1e-6), dt)
            np.testing.assert_allclose(got, want, **TOL[dt])
    want = R.walk("ppr", ip, ind, v, n, seed=11, alpha=0.85, max_iter=100, tol=1e-6)
    got, _ = port.walk_restart(ip, ind, v, [11], n, dt(0.85), 100, dt(1e-6), dt)
    np.testing.assert_allclose(got, want, **TOL[dt])
    # no seed in range: zero scores
    assert not R.walk("rwr", ip, ind, v, n, seeds=[-5, n], alpha=0.5, max_iter=10, tol=1e-6).any()
    assert port.walk_restart(ip, ind, v, [-5, n], n, dt(0.5), 10, dt(1e-6), dt)[0].sum() == 0


@pytest.mark.parametrize("variant,dt", [("f32_i32", np.float32), ("f64_i64", np.float64)])
def test_pseudotime_matches_reference(variant, dt):
    """Diffusion pseudotime: on these graphs the restatement equals the
    reference bit for bit (single-root and multi-root, converged and capped)."""
    R = _ref(variant)
    n = 400
    ip, ind, v = _walk_graph(n, dt)
    for root, max_iter, tol in ((0, 100, 1e-6), (5, 3, 1e-6), (17, 100, 1e-2)):
        want = R.walk("dpt", ip, ind, v, n, root=root, max_iter=max_iter, tol=tol)
        got = port.dpt(ip, ind, v, root, max_iter, dt(tol), dt)
        np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    want = R.walk("dpt_multi", ip, ind, v, n, roots=[1, 9, -3, 500], max_iter=50)
    got = port.dpt_multi_root(ip, ind, v, [1, 9, -3, 500], 50, dt)
    np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
    assert (R.walk("dpt_multi", ip, ind, v, n, roots=[-1, n], max_iter=5) == 1).all()
