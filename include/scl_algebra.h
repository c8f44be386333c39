/*
 * scl_algebra.h — scl_algebra_spmm of scl-core's algebra C ABI, executed on a
 * B200 GPU.
 *
 * Replaces scl/binding/c_api/algebra.h:121-140 (implementation in
 * scl/binding/c_api/algebra.cpp:164-192 and scl/kernel/algebra.hpp:546-600).
 * Signature, argument meaning and error codes are the reference's. Host
 * pointers in and out: each call uploads A, X and (when beta != 0) Y, computes
 * on the device and writes Y back, synchronously. The other entry points of
 * scl-core's algebra.h are not part of this build.
 */
#ifndef SCL_B200_ALGEBRA_H
#define SCL_B200_ALGEBRA_H

#include "scl_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Y (primary_dim x n_cols, row-major) <- alpha A X + beta Y with X
 * secondary_dim x n_cols: Y is scaled first (beta 0: zero, beta 1: kept), then,
 * unless alpha is 0, each stored entry in order adds fma(a * alpha, x_row, y)
 * (entries with a * alpha == 0 are skipped), as the reference's axpy does.
 * A CSC handle multiplies by its primary (column) view, as in the reference. */
SCL_EXPORT scl_error_t scl_algebra_spmm(scl_sparse_t A, const scl_real_t* X, scl_index_t n_cols, scl_real_t* Y,
                                        scl_real_t alpha, scl_real_t beta);

#ifdef __cplusplus
}
#endif

#endif /* SCL_B200_ALGEBRA_H */
