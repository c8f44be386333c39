"""The general SpMM restatement (oracle/port.py: algebra_spmm) against
scl-core's own scl_algebra_spmm compiled from the reference sources, bit for
bit: every beta branch (0, 1, other), alpha 0, zero-valued entries, widths
inside and across the reference's 64-column blocks, both precisions."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import port, ref


@pytest.mark.parametrize("variant,dt", [("f32_i32", np.float32), ("f64_i64", np.float64)])
def test_algebra_spmm_restatement_matches_reference(variant, dt):
    if not ref.available(variant):
        pytest.skip("reference library not built (make -C oracle ref)")
    R = ref.RefLib(variant)
    for m, kdim, K in ((50, 40, 7), (300, 200, 64), (300, 300, 100), (1, 1, 1)):
        A = sp.random(m, kdim, density=0.1 if m > 1 else 1.0, random_state=2, format="csr",
                      dtype=np.float64).astype(dt)
        A.sort_indices()
        A.data[::7] = 0  # explicit zeros are skipped by the reference's axpy
        X = np.random.default_rng(1).standard_normal((kdim, K)).astype(dt)
        for alpha, beta in ((1.0, 0.0), (0.5, 2.0), (2.0, 1.0), (0.0, 3.0), (-1.5, 0.25)):
            Y0 = np.random.default_rng(2).standard_normal((m, K)).astype(dt)
            h, keep = R.wrap(A.indptr, A.indices, A.data, A.shape)
            want = Y0.copy()
            try:
                R._check(R.L.scl_algebra_spmm(h, X.ctypes.data, K, want.ctypes.data, alpha, beta))
            finally:
                R.destroy(h)
            got = port.algebra_spmm(A.indptr, A.indices, A.data, X, Y0, dt(alpha), dt(beta))
            np.testing.assert_array_equal(got.view(np.uint8), want.view(np.uint8))
