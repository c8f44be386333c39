/*
 * scl_neighbors.h — k-nearest neighbours of scl-core's neighbors C ABI,
 * executed on a B200 GPU: the graph-building step before the transition
 * matrix.
 *
 * Replaces scl/binding/c_api/neighbors/neighbors.h:18-41 (implementation in
 * scl/binding/c_api/neighbors.cpp and scl/kernel/neighbors.hpp:302-478).
 * Signatures, argument meaning and error codes are the reference's. The
 * samples are the handle's primary rows and the features its secondary
 * dimension; host pointers in and out, synchronously. On the device the
 * samples are made dense, so this build takes at most 128 features and k <= 64
 * (SCL_ERROR_INVALID_ARGUMENT otherwise). There is no CPU fallback.
 */
#ifndef SCL_B200_NEIGHBORS_H
#define SCL_B200_NEIGHBORS_H

#include "scl_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* neighbors.h:18-22: squared norm of every sample, as a sequential fma chain
 * over its stored values (the reference sums in SIMD lanes, so the two agree
 * to a few ulps). */
SCL_EXPORT scl_error_t scl_neighbors_compute_norms(scl_sparse_t matrix, scl_real_t* norms_sq);

/* neighbors.h:25-32: for every sample i the k nearest other samples by
 * dist_sq = norm_i + norm_j - 2 <x_i, x_j> (the caller's norms; the dot an fma
 * chain over the features in order; negative values clamped to 0), ties kept
 * in favour of the smaller index; out_distances = sqrt(dist_sq) ascending,
 * slots beyond the n - 1 candidates (inf, -1). n_samples must equal the
 * handle's primary dimension. With the reference's norms the result equals
 * the reference's (the reference also skips candidates by a Cauchy-Schwarz
 * bound, which can differ only when that bound rounds above the distance). */
SCL_EXPORT scl_error_t scl_knn(scl_sparse_t matrix, const scl_real_t* norms_sq, scl_size_t n_samples, scl_size_t k,
                               scl_index_t* out_indices, scl_real_t* out_distances);

/* neighbors.h:35-41: scl_knn with the norms of scl_neighbors_compute_norms. */
SCL_EXPORT scl_error_t scl_knn_simple(scl_sparse_t matrix, scl_size_t n_samples, scl_size_t k,
                                      scl_index_t* out_indices, scl_real_t* out_distances);

#ifdef __cplusplus
}
#endif

#endif /* SCL_B200_NEIGHBORS_H */
