/*
 * ORACLE — test infrastructure only. Nothing in the product libraries links,
 * loads or calls this code; it is the CPU checker that the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark compare against.
 *
 * Plain-C restatement of scl-core's graph-diffusion path:
 *   - row sums / transition-matrix normalisation
 *       scl/kernel/diffusion.hpp:452-484 (compute_row_sums_parallel)
 *       scl/kernel/diffusion.hpp:492-603 (compute_transition_matrix)
 *   - SpMM power iteration
 *       scl/kernel/diffusion.hpp:227-278 (spmm_block), 100-134 (axpy_simd),
 *       scl/kernel/diffusion.hpp:638-664 (diffuse_matrix),
 *       scl/kernel/diffusion.hpp:169-221, 609-632 (spmv_parallel, diffuse_vector)
 *   - Gaussian kNN affinity + (W+W^T)/2 union (no single reference function:
 *       scl/kernel/kernel.hpp:403-453 local_bandwidth, scl/kernel/impute.hpp:156-159
 *       distance_to_weight, scl/kernel/neighbors.hpp:319-478 kNN list format)
 *   - vector walks: lazy random walk, heat-kernel signature, random walk with
 *       restart, diffusion pseudotime (scl/kernel/diffusion.hpp:670-831,
 *       833-900, 961-1007, 1157-1194)
 *   - BF16/FP16 storage variants and the FP64 adjoint (new in this project).
 *
 * Arithmetic contract: every multiply-add that the reference performs through
 * Highway MulAdd (or a contracted `y += a*x`) is an explicit fma()/fmaf() here,
 * performed in the same order (row by row, nonzeros in stored order). The file
 * is compiled with -ffp-contract=off so nothing else is fused.
 *
 * Indices are int64 throughout; callers convert.
 */
#ifndef SCL_DIFFUSION_ORACLE_H
#define SCL_DIFFUSION_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Storage kinds for the low-precision restatement. */
enum { ORACLE_F32 = 0, ORACLE_BF16 = 2, ORACLE_F16 = 3 };

/* ---- normalisation --------------------------------------------------- */
/* Sequential per-row sums in the value type (diffusion.hpp:452-484). */
void oracle_row_sums_f32(int64_t n, const int64_t* indptr, const float* values, float* out);
void oracle_row_sums_f64(int64_t n, const int64_t* indptr, const double* values, double* out);

/* In-place transition normalisation (diffusion.hpp:492-603).
 * degree_fp64 = 0: sums and scale factors in the value type, exactly as the
 *                  reference (f32 build: float sums, 1.0f/d, v *= inv).
 * degree_fp64 = 1: sequential FP64 row sums, FP64 scale factors, one rounding
 *                  of v*scale to the value type (the GPU build's contract). */
void oracle_transition_f32(int64_t n, const int64_t* indptr, const int64_t* indices,
                           float* values, int symmetric, int degree_fp64);
void oracle_transition_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                           double* values, int symmetric);

/* ---- power iteration ------------------------------------------------- */
/* One Y = P·X over n primary rows (spmm_block): sequential fma per output. */
void oracle_spmm_f32(int64_t n, const int64_t* indptr, const int64_t* indices,
                     const float* values, const float* X, float* Y, int64_t F);
void oracle_spmm_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                     const double* values, const double* X, double* Y, int64_t F);
/* X <- P^T_steps X in place (diffuse_matrix). */
void oracle_diffuse_matrix_f32(int64_t n, const int64_t* indptr, const int64_t* indices,
                               const float* values, float* X, int64_t F, int64_t steps);
void oracle_diffuse_matrix_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                               const double* values, double* X, int64_t F, int64_t steps);

/* Low-precision storage: values and X stored as `kind` (bf16/f16 bit patterns
 * in uint16, or f32), FP32 accumulation by sequential fmaf, each intermediate
 * iterate rounded (RNE) to `kind`; the final iterate is written as FP32 to
 * Y_out when final_f32 != 0, else rounded to `kind` and widened. X0 is given
 * as FP32 and rounded to `kind` first. */
void oracle_diffuse_lowp(int64_t n, const int64_t* indptr, const int64_t* indices,
                         const float* values_f32, const float* X0_f32, float* Y_out,
                         int64_t F, int64_t steps, int kind, int final_f32);
/* Same with Q interleaved fma chains per row summed pairwise (the entry order
 * of the B200 kernel for 16-bit storage). */
void oracle_diffuse_lowp_chains(int64_t n, const int64_t* indptr, const int64_t* indices,
                                const float* values_f32, const float* X0_f32, float* Y_out,
                                int64_t F, int64_t steps, int kind, int final_f32, int chains);

/* RNE conversions used above, exposed for tests. */
uint16_t oracle_f32_to_bf16(float x);
float oracle_bf16_to_f32(uint16_t h);
uint16_t oracle_f32_to_f16(float x);
float oracle_f16_to_f32(uint16_t h);

/* ---- graph build ----------------------------------------------------- */
/* sigma_i = max(max_{m<k, idx>=0} dist[i,m], 1e-10) (kernel.hpp:403-453,
 * 1.0 when a row has no neighbour); w = exp(-(d/sigma_i)^2). FP64. */
void oracle_gauss_weights_f64(int64_t n, int64_t k, const int64_t* knn_idx,
                              const double* knn_dist, double* sigma, double* w);
/* FP32 form: q = d / sigma_i (float), w = expf(-(q*q)). */
void oracle_gauss_weights_f32(int64_t n, int64_t k, const int64_t* knn_idx,
                              const float* knn_dist, float* sigma, float* w);

/* Union symmetrisation S = (W + W^T)/2 of the kNN graph (W[i, idx[i,m]] =
 * w[i,m], entries with idx < 0 skipped). Rows sorted by column, one entry per
 * distinct (i, j). Value = 0.5 * (sum of W[i,j] entries + sum of W[j,i]
 * entries). Returns nnz; writes the arrays only when they are non-NULL
 * (indptr has n+1 entries). */
int64_t oracle_symmetrize_f64(int64_t n, int64_t k, const int64_t* knn_idx, const double* w,
                              int64_t* indptr, int64_t* indices, double* values);
int64_t oracle_symmetrize_f32(int64_t n, int64_t k, const int64_t* knn_idx, const float* w,
                              int64_t* indptr, int64_t* indices, float* values);

/* ---- FP64 adjoint ---------------------------------------------------- */
/* Loss L = sum((X_T - Y)^2) for X_{s+1} = P X_s, P = normalise(W) (row or
 * symmetric). Returns L; writes dL/dX0 (n*F) and dL/dW on W's stored entries
 * (nnz), propagated through the normalisation with W's structure fixed. */
double oracle_adjoint_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                          const double* W, int symmetric, const double* X0, const double* Y,
                          int64_t F, int64_t steps, double* dX0, double* dW);

/* ---- vector walks (diffusion.hpp:833-900, 961-1007, 1157-1194) ------ */
void oracle_walk_linear_f32(int64_t n, const int64_t* indptr, const int64_t* indices, const float* values, float* x,
                            int64_t steps, float cx, float cp);
void oracle_walk_linear_f64(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values, double* x,
                            int64_t steps, double cx, double cp);
int64_t oracle_walk_restart_f32(int64_t n, const int64_t* indptr, const int64_t* indices, const float* values,
                                const float* r, float* scores, float alpha, int64_t max_iter, float tol);
int64_t oracle_walk_restart_f64(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values,
                                const double* r, double* scores, double alpha, int64_t max_iter, double tol);

/* ---- diffusion pseudotime (diffusion.hpp:670-772) --------------------- */
void oracle_dpt_f32(int64_t n, const int64_t* indptr, const int64_t* indices, const float* values, int64_t root,
                    int64_t max_iter, float tol, float* out);
void oracle_dpt_f64(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values, int64_t root,
                    int64_t max_iter, double tol, double* out);

/* ---- general SpMM, Y = alpha A X + beta Y (algebra.hpp:546-600) ------- */
void oracle_algebra_spmm_f32(int64_t m, const int64_t* indptr, const int64_t* indices, const float* values,
                             const float* X, int64_t K, float* Y, float alpha, float beta);
void oracle_algebra_spmm_f64(int64_t m, const int64_t* indptr, const int64_t* indices, const double* values,
                             const double* X, int64_t K, double* Y, double alpha, double beta);

/* ---- brute-force kNN on a dense block (neighbors.hpp:319-478) --------- */
void oracle_knn_dense_f32(int64_t n, int64_t d, const float* X, const float* norms, int64_t k, int contract,
                          int64_t* out_idx, float* out_dist);
void oracle_knn_dense_f64(int64_t n, int64_t d, const double* X, const double* norms, int64_t k, int contract,
                          int64_t* out_idx, double* out_dist);

#ifdef __cplusplus
}
#endif
#endif
