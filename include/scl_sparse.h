/*
 * scl_sparse.h — sparse-handle C ABI (the subset the diffusion path uses).
 *
 * Replaces scl/binding/c_api/core/sparse.h:54-297 of scl-core. Same signatures,
 * ownership rules and error codes:
 *   - create*      deep-copies into block-allocated storage (the block layout
 *                  follows scl/core/sparse.hpp:67-113,1761-1830, so a large
 *                  ADAPTIVE matrix is non-contiguous exactly as in scl-core);
 *   - wrap         is zero-copy: the caller keeps indptr/indices/data alive;
 *   - wrap_and_own takes data and indices (allocated with new[]); indptr stays
 *                  with the caller (sparse.cpp:235-336);
 *   - destroy(&h)  frees and nulls the handle; NULL is accepted.
 */
#ifndef SCL_B200_SPARSE_H
#define SCL_B200_SPARSE_H

#include "scl_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sparse.h:54-70 */
typedef enum {
  SCL_BLOCK_STRATEGY_CONTIGUOUS = 0,
  SCL_BLOCK_STRATEGY_SMALL = 1,
  SCL_BLOCK_STRATEGY_LARGE = 2,
  SCL_BLOCK_STRATEGY_ADAPTIVE = 3
} scl_block_strategy_t;

/* sparse.h:76-84 */
typedef struct {
  scl_index_t data_block_count;
  scl_index_t index_block_count;
  scl_size_t data_bytes;
  scl_size_t index_bytes;
  scl_size_t metadata_bytes;
  scl_bool_t is_contiguous;
  scl_bool_t is_traditional_format;
} scl_sparse_layout_info_t;

/* sparse.h:103-112 */
SCL_EXPORT scl_error_t scl_sparse_create(scl_sparse_t* out, scl_index_t rows, scl_index_t cols, scl_index_t nnz,
                                         const scl_index_t* indptr, const scl_index_t* indices,
                                         const scl_real_t* data, scl_bool_t is_csr);
/* sparse.h:126-136 */
SCL_EXPORT scl_error_t scl_sparse_create_with_strategy(scl_sparse_t* out, scl_index_t rows, scl_index_t cols,
                                                       scl_index_t nnz, const scl_index_t* indptr,
                                                       const scl_index_t* indices, const scl_real_t* data,
                                                       scl_bool_t is_csr, scl_block_strategy_t strategy);
/* sparse.h:150-159 */
SCL_EXPORT scl_error_t scl_sparse_wrap(scl_sparse_t* out, scl_index_t rows, scl_index_t cols, scl_index_t nnz,
                                       scl_index_t* indptr, scl_index_t* indices, scl_real_t* data,
                                       scl_bool_t is_csr);
/* sparse.h:173-182 */
SCL_EXPORT scl_error_t scl_sparse_wrap_and_own(scl_sparse_t* out, scl_index_t rows, scl_index_t cols,
                                               scl_index_t nnz, scl_index_t* indptr, scl_index_t* indices,
                                               scl_real_t* data, scl_bool_t is_csr);
/* sparse.h:190 */
SCL_EXPORT scl_error_t scl_sparse_clone(scl_sparse_t src, scl_sparse_t* out);
/* sparse.h:196 */
SCL_EXPORT scl_error_t scl_sparse_destroy(scl_sparse_t* matrix);

/* sparse.h:202-229 — property queries */
SCL_EXPORT scl_error_t scl_sparse_rows(scl_sparse_t matrix, scl_index_t* out);
SCL_EXPORT scl_error_t scl_sparse_cols(scl_sparse_t matrix, scl_index_t* out);
SCL_EXPORT scl_error_t scl_sparse_nnz(scl_sparse_t matrix, scl_index_t* out);
SCL_EXPORT scl_error_t scl_sparse_is_csr(scl_sparse_t matrix, scl_bool_t* out);
SCL_EXPORT scl_error_t scl_sparse_is_csc(scl_sparse_t matrix, scl_bool_t* out);
SCL_EXPORT scl_error_t scl_sparse_is_valid(scl_sparse_t matrix, scl_bool_t* out);
SCL_EXPORT scl_error_t scl_sparse_is_contiguous(scl_sparse_t matrix, scl_bool_t* out);
SCL_EXPORT scl_error_t scl_sparse_layout_info(scl_sparse_t matrix, scl_sparse_layout_info_t* info);

/* sparse.h:246-251 — export to traditional CSR/CSC (caller allocates) */
SCL_EXPORT scl_error_t scl_sparse_export(scl_sparse_t matrix, scl_index_t* indptr, scl_index_t* indices,
                                         scl_real_t* data);
/* sparse.h:262-294 — zero-copy views of internal arrays */
SCL_EXPORT scl_error_t scl_sparse_get_lengths(scl_sparse_t matrix, const scl_index_t** lengths,
                                              scl_size_t* lengths_size);
SCL_EXPORT scl_error_t scl_sparse_get_indices(scl_sparse_t matrix, const scl_index_t** indices,
                                              scl_size_t* indices_size);
SCL_EXPORT scl_error_t scl_sparse_get_data(scl_sparse_t matrix, const scl_real_t** data, scl_size_t* data_size);

/* sparse.h:305 — CSR <-> CSC (same entries, primary and secondary swapped) */
SCL_EXPORT scl_error_t scl_sparse_transpose(scl_sparse_t src, scl_sparse_t* out);
/* sparse.h:313 */
SCL_EXPORT scl_error_t scl_sparse_to_contiguous(scl_sparse_t src, scl_sparse_t* out);

#ifdef __cplusplus
}
#endif
#endif /* SCL_B200_SPARSE_H */
