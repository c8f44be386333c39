/*
 * scl_impute.h — drop-in imputation C ABI (diffusion and MAGIC), executed on a
 * B200 GPU.
 *
 * Replaces scl/binding/c_api/impute/impute.h:15-58 of scl-core (implementation
 * in scl/binding/c_api/impute.cpp:93-157 and scl/kernel/impute.hpp:599-735).
 * Signatures, argument meaning and error codes are the reference's. Host
 * pointers in, host pointers out: each call uploads the handles' arrays, builds
 * the dense block and diffuses it on the device, and writes X_imputed back,
 * synchronously. There is no CPU fallback: without a usable CUDA device every
 * entry point returns SCL_ERROR_FEATURE_UNAVAILABLE.
 */
#ifndef SCL_B200_IMPUTE_H
#define SCL_B200_IMPUTE_H

#include "scl_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* impute.h:15-25 (impute.cpp:19-52, impute.hpp:400-510): X_imputed is the
 * dense block (later duplicates winning), then every value not above
 * `threshold` becomes the mean of the listed neighbours (knn_indices, n_cells
 * x k_neighbors; out-of-range ones skipped) that store the gene (their first
 * stored value; a stored zero counts), weighted by
 * exp(-(d / (bandwidth + 1e-12))^2), when the weight sum exceeds 1e-12 and the
 * mean exceeds 1e-10. The weights use CUDA's exp, so values agree with the
 * reference to rounding. */
SCL_EXPORT scl_error_t scl_impute_knn(scl_sparse_t matrix, const scl_index_t* knn_indices,
                                      const scl_real_t* knn_distances, scl_index_t n_cells, scl_index_t n_genes,
                                      scl_index_t k_neighbors, scl_real_t* X_imputed, scl_real_t bandwidth,
                                      scl_real_t threshold);

/* impute.h:28-38: the same computation (scl-core's impute.cpp:54-87 runs the
 * same kernel for it). */
SCL_EXPORT scl_error_t scl_impute_knn_weighted(scl_sparse_t matrix, const scl_index_t* knn_indices,
                                               const scl_real_t* knn_distances, scl_index_t n_cells,
                                               scl_index_t n_genes, scl_index_t k_neighbors, scl_real_t* X_imputed,
                                               scl_real_t bandwidth, scl_real_t threshold);

/* impute.h:41-48 (impute.cpp:93-122, impute.hpp:599-661). X_imputed (n_cells x
 * n_genes, row-major) <- T^n_steps X0, where X0 is `matrix` made dense (zero,
 * then every stored entry with cell < n_cells and gene < n_genes; a CSR handle
 * is cells x genes, a CSC handle genes-major) and T is `transition_matrix`
 * over its primary dimension (a CSC handle applies the transpose). Here the
 * transition's primary dimension must equal n_cells and its column indices
 * must address cells (else SCL_ERROR_DIMENSION_MISMATCH; the reference reads
 * out of bounds). Each output element is the sequential fma chain over the
 * transition row's entries. */
SCL_EXPORT scl_error_t scl_impute_diffusion(scl_sparse_t matrix, scl_sparse_t transition_matrix, scl_index_t n_cells,
                                            scl_index_t n_genes, scl_index_t n_steps, scl_real_t* X_imputed);

/* impute.h:51-58 (impute.cpp:128-157, impute.hpp:668-735). As
 * scl_impute_diffusion with the affinity rows normalised on the fly: a
 * sequential row sum s_i in scl_real_t, weights a_ij * (1 / s_i), and rows with
 * s_i < 1e-12 keep their previous row. As in the reference, only a CSR
 * `matrix` seeds X0 (a CSC one leaves it zero). */
SCL_EXPORT scl_error_t scl_impute_magic(scl_sparse_t matrix, scl_sparse_t affinity_matrix, scl_index_t n_cells,
                                        scl_index_t n_genes, scl_index_t t, scl_real_t* X_imputed);

#ifdef __cplusplus
}
#endif

#endif /* SCL_B200_IMPUTE_H */
