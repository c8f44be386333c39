"""Regenerate the golden fixtures in this directory from scl-core itself.

    make -C oracle ref && python tests/golden/make_golden.py

Inputs: a seeded 600-cell mixture (scl.synthetic), its exact k=10 kNN lists and
the (W + W^T)/2 Gaussian affinity built by the oracle restatement (scl-core has
no scalable function for that step). Every OUTPUT array below is produced by the
reference's own compiled code (oracle/_ref, scl/binding/c_api/diffusion.cpp and
friends) through its C ABI:
  P_{row,sym}_{f32,f64}     scl_diffusion_compute_transition_matrix
  XT_{f32,f64}              scl_diffusion_diffuse_matrix, 4 steps, 8 columns
  XT_csc_f32                diffuse_matrix on scl_sparse_transpose(P) (= P^T), 2 steps
  xv_f32                    scl_diffusion_diffuse_vector, 3 steps
  kat_spmm                  scl_algebra_spmm on the 3x3 fixture of
                            tests/c_api/include/data.hpp:350-363
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "scl-core_b200"))

from oracle import port, ref  # noqa: E402
from scl import synthetic  # noqa: E402


def main():
    n, k, F, T = 600, 10, 8, 4
    pts = synthetic.mixture(n, seed=7)
    knn_i, knn_d = synthetic.knn_exact(pts, k)
    _, w = port.gauss_weights(knn_i, knn_d)
    ip, ind, W = port.symmetrize(knn_i, w)
    r32, r64 = ref.RefLib("f32_i32"), ref.RefLib("f64_i64")
    out = dict(n=n, k=k, F=F, T=T, knn_idx=knn_i.astype(np.int32), knn_dist=knn_d, indptr=ip, indices=ind,
               W_f64=W, W_f32=W.astype(np.float32))
    for tag, R in (("f32", r32), ("f64", r64)):
        Wt = W.astype(R.real_dtype)
        out[f"P_row_{tag}"] = R.transition(ip, ind, Wt, n, symmetric=False)
        out[f"P_sym_{tag}"] = R.transition(ip, ind, Wt, n, symmetric=True)
        X0 = synthetic.features(n, F, seed=3, dtype=R.real_dtype)
        out[f"X0_{tag}"] = X0
        out[f"XT_{tag}"] = R.diffuse_matrix(ip, ind, out[f"P_row_{tag}"], X0, T)
    out["XT_csc_f32"] = r32.diffuse_transpose(ip, ind, out["P_row_f32"], out["X0_f32"], 2)
    out["xv_f32"] = r32.diffuse_vector(ip, ind, out["P_row_f32"], out["X0_f32"][:, 0].copy(), 3)
    kat_ip = np.array([0, 2, 3, 6])
    kat_ix = np.array([0, 2, 1, 0, 1, 2])
    kat_d = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    out["kat_spmm"] = r64.spmm(kat_ip, kat_ix, kat_d, (3, 3), np.array([[1.0, 2], [3, 4], [5, 6]]))
    dst = Path(__file__).resolve().parent / "diffusion_small.npz"
    np.savez_compressed(dst, **out)
    print("wrote", dst, dst.stat().st_size, "bytes; nnz =", ind.size)


if __name__ == "__main__":
    main()
