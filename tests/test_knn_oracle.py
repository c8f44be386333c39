"""The brute-force kNN restatement (oracle/port.py: knn_dense) against
scl-core's own scl_knn / scl_neighbors_compute_norms compiled from the
reference sources: with the reference's norms the neighbour indices and
distances are equal bit for bit and in the same order, ties included (the
restatement replays the reference's heap and its final heap sort)."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import port, ref


@pytest.mark.parametrize("variant,dt", [("f32_i32", np.float32), ("f64_i64", np.float64)])
def test_knn_restatement_matches_reference(variant, dt):
    if not ref.available(variant):
        pytest.skip("reference library not built (make -C oracle ref)")
    R = ref.RefLib(variant)
    rng = np.random.default_rng(7)
    cases = [(300, 20, 10, 1.0, False), (500, 50, 15, 1.0, False), (400, 60, 12, 0.3, False),
             (12, 5, 15, 1.0, False), (200, 8, 6, 1.0, True)]
    for n, d, k, dens, quantised in cases:
        X = sp.random(n, d, density=dens, random_state=int(rng.integers(1 << 30)), format="csr", dtype=np.float64)
        X.data = rng.standard_normal(X.nnz)
        if quantised:  # many exact ties in distance
            X.data = np.round(X.data)
        X = X.astype(dt)
        X.sort_indices()
        ri, rd, norms = R.knn(X.indptr, X.indices, X.data, X.shape, k)
        oi, od = port.knn_dense(X.toarray(), norms, k)
        np.testing.assert_array_equal(od.view(np.uint8), rd.view(np.uint8))
        np.testing.assert_array_equal(oi, ri.astype(np.int64))
