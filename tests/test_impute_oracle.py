"""The imputation restatement (oracle/port.py: densify, impute_diffusion,
impute_magic) against scl-core's own scl_impute_diffusion / scl_impute_magic
compiled from the reference sources (oracle/_ref), bit for bit: CSR and CSC
expression matrices, duplicates, entries outside the block, zero-sum affinity
rows, both precisions."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import port, ref

bits = lambda a: np.ascontiguousarray(a).view(np.uint8)


def _reference(variant):
    if not ref.available(variant):
        pytest.skip("reference library not built (make -C oracle ref)")
    return ref.RefLib(variant)


def _case(rng, n_cells, n_genes, dt, extra_rows=0, extra_cols=0, dups=False, zero_rows=()):
    X = sp.random(n_cells + extra_rows, n_genes + extra_cols, density=0.3, random_state=rng.integers(1 << 30),
                  format="csr", dtype=np.float64).astype(dt)
    X.sort_indices()
    ip, ind, val = X.indptr.astype(np.int64), X.indices.astype(np.int64), X.data
    if dups:  # repeat the first entry of every other row at its end with another value
        rows_ip, rows_ind, rows_val = [0], [], []
        for r in range(X.shape[0]):
            a, b = ip[r], ip[r + 1]
            ri, rv = list(ind[a:b]), list(val[a:b])
            if b > a and r % 2 == 0:
                ri.append(ri[0])
                rv.append(dt(rng.standard_normal()))
            rows_ind += ri
            rows_val += rv
            rows_ip.append(len(rows_ind))
        ip, ind, val = np.array(rows_ip), np.array(rows_ind, np.int64), np.array(rows_val, dt)
    T = sp.random(n_cells, n_cells, density=0.2, random_state=rng.integers(1 << 30), format="csr",
                  dtype=np.float64).astype(dt)
    T = T.tolil()
    for r in zero_rows:
        T[r, :] = 0
    T = T.tocsr()
    T.sort_indices()  # zeroed rows are empty: their sum (0) is below 1e-12
    return (ip, ind, val), X.shape, (T.indptr.astype(np.int64), T.indices.astype(np.int64), T.data.copy())


@pytest.mark.parametrize("variant,dt", [("f32_i32", np.float32), ("f64_i64", np.float64)])
@pytest.mark.parametrize("kind", ["diffusion", "magic"])
def test_impute_restatement_matches_reference(variant, dt, kind):
    R = _reference(variant)
    rng = np.random.default_rng(5)
    f = port.impute_diffusion if kind == "diffusion" else port.impute_magic
    for n_cells, n_genes, kw in ((30, 40, {}), (17, 5, {"dups": True}), (40, 33, {"extra_rows": 3, "extra_cols": 4}),
                                 (25, 64, {"zero_rows": (0, 7)}), (1, 1, {})):
        x, shape, t = _case(rng, n_cells, n_genes, dt, **kw)
        for steps in (1, 3):
            want = R.impute(kind, x, shape, True, t, n_cells, n_genes, steps)
            got = f(x, True, t, n_cells, n_genes, steps).astype(dt)
            np.testing.assert_array_equal(bits(got), bits(want))


@pytest.mark.parametrize("kind", ["diffusion", "magic"])
def test_impute_restatement_csc_expression_matches_reference(kind):
    """A CSC expression handle is genes-major; MAGIC leaves X0 zero for it."""
    R = _reference("f32_i32")
    rng = np.random.default_rng(6)
    n_cells, n_genes = 20, 12
    M = sp.random(n_genes, n_cells, density=0.3, random_state=3, format="csr", dtype=np.float64).astype(np.float32)
    M.sort_indices()
    x = (M.indptr.astype(np.int64), M.indices.astype(np.int64), M.data)
    _, _, t = _case(rng, n_cells, n_genes, np.float32)
    want = R.impute(kind, x, (n_cells, n_genes), False, t, n_cells, n_genes, 2)
    f = port.impute_diffusion if kind == "diffusion" else port.impute_magic
    np.testing.assert_array_equal(bits(f(x, False, t, n_cells, n_genes, 2)), bits(want))
    if kind == "magic":
        assert not want.any()


def test_reference_fixtures_from_its_own_tests():
    """The 3x3 inputs of the reference's tests/c_api/src/test_impute.cpp
    (diffusion_impute_basic, magic_impute_basic), outputs from the reference."""
    R = _reference("f64_i64")
    x = (np.array([0, 2, 3, 5]), np.array([0, 1, 0, 1, 2]), np.array([1.0, 2.0, 3.0, 4.0, 5.0]))
    t_diff = (np.array([0, 2, 4, 6]), np.array([0, 1, 0, 2, 1, 2]), np.full(6, 0.5))
    t_magic = (np.array([0, 2, 4, 6]), np.array([0, 1, 0, 2, 1, 2]), np.array([0.8, 0.2, 0.7, 0.3, 0.6, 0.4]))
    for kind, t, f in (("diffusion", t_diff, port.impute_diffusion), ("magic", t_magic, port.impute_magic)):
        want = R.impute(kind, x, (3, 3), True, t, 3, 3, 2)
        np.testing.assert_array_equal(bits(f(x, True, t, 3, 3, 2)), bits(want))
        assert np.isfinite(want).all()
