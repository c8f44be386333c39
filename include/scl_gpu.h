/*
 * scl_gpu.h — device-pointer extension C ABI of the B200 diffusion libraries.
 *
 * No counterpart in scl-core: scl-core is CPU-only and its diffusion ABI
 * (scl/binding/c_api/diffusion.h) takes host arrays. These entry points keep
 * the graph and the dense blocks resident in GPU memory and take raw device
 * pointers plus a CUDA stream (passed as void*, 0 = legacy default stream), so
 * an autograd wrapper or a caller with its own device buffers can drive the
 * same kernels without host round trips. Calls are asynchronous on `stream`
 * unless noted; only plain pointers, sizes and enums cross the boundary.
 */
#ifndef SCL_B200_GPU_H
#define SCL_B200_GPU_H

#include <stdint.h>

#include "scl_core.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SCL_DTYPE_F32 = 0,
  SCL_DTYPE_F64 = 1,
  SCL_DTYPE_BF16 = 2,
  SCL_DTYPE_F16 = 3,
  SCL_DTYPE_I32 = 4,
  SCL_DTYPE_I64 = 5
} scl_dtype_t;

typedef struct scl_gpu_graph scl_gpu_graph;
typedef scl_gpu_graph* scl_gpu_graph_t;

/* Gaussian kNN affinity graph built on the device from kNN lists
 * (knn_idx int32 n x k, -1 = no neighbour; knn_dist float32 n x k):
 * sigma_i = max of row i's distances (floored at 1e-10), w = exp(-(d/sigma_i)^2),
 * then S = (W + W^T)/2 over the union of kNN pairs, rows sorted by column.
 * The result holds S as its f32 weights. Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_graph_from_knn(scl_gpu_graph_t* out, int64_t n, int64_t k, const int32_t* knn_idx,
                                              const float* knn_dist, void* stream);

/* Copy a CSR matrix (host arrays when on_device == 0, device arrays otherwise)
 * into a device graph. indptr: i32/i64 [n_rows + 1]; indices: i32/i64 [nnz];
 * values: f32/f64 [nnz]. Indices are validated (SCL_ERROR_INDEX_OUT_OF_BOUNDS).
 * Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_graph_from_csr(scl_gpu_graph_t* out, int64_t n_rows, int64_t n_cols, int64_t nnz,
                                              const void* indptr, scl_dtype_t indptr_dtype, const void* indices,
                                              scl_dtype_t indices_dtype, const void* values,
                                              scl_dtype_t values_dtype, int on_device, void* stream);

SCL_EXPORT scl_error_t scl_gpu_graph_destroy(scl_gpu_graph_t* graph);

SCL_EXPORT scl_error_t scl_gpu_graph_shape(scl_gpu_graph_t graph, int64_t* n_rows, int64_t* n_cols, int64_t* nnz);

/* Transition matrix in place (the device form of
 * scl_diffusion_compute_transition_matrix): symmetric 0 = D^-1 W, 1 = D^-1/2 W D^-1/2.
 * degree_mode 0 = FP64 degrees (default), 1 = value-type arithmetic as scl-core.
 * The pre-normalisation weights and FP64 degrees are kept for the backward pass. */
SCL_EXPORT scl_error_t scl_gpu_graph_normalize(scl_gpu_graph_t graph, int symmetric, int degree_mode, void* stream);

/* Copy the graph out: indptr int64 [n_rows + 1], indices int32 [nnz], values in
 * the graph's master dtype (f32 or f64) [nnz]; any pointer may be NULL.
 * Host destinations when on_device == 0 (synchronises `stream`). */
SCL_EXPORT scl_error_t scl_gpu_graph_export(scl_gpu_graph_t graph, int64_t* indptr, int32_t* indices, void* values,
                                            int on_device, void* stream);

/* Storage precision of the values the SpMM reads: F32, F64, BF16 or F16
 * (rounded once, RNE, from the master values). Iterates are stored in the same
 * type; accumulation is FP32 (FP64 for F64). */
SCL_EXPORT scl_error_t scl_gpu_graph_set_storage(scl_gpu_graph_t graph, scl_dtype_t dtype, void* stream);

/* Y = P^n_steps X on device buffers (row-major n_rows x n_features). X is read
 * as x_dtype and rounded once to the storage dtype if they differ; the final
 * iterate is written as y_dtype (storage dtype or F32). X may equal Y. */
SCL_EXPORT scl_error_t scl_gpu_diffuse(scl_gpu_graph_t graph, const void* X, scl_dtype_t x_dtype, void* Y,
                                       scl_dtype_t y_dtype, int64_t n_features, int64_t n_steps, void* stream);

/* Locality reordering used by scl_gpu_diffuse: mode 1 groups the rows of each
 * connected component together (P' = Pi P Pi^T, X gathered once and the result
 * scattered back on the last step); mode 0 drops it. Each row keeps its stored
 * entry order, so results are bit-identical with and without it. The
 * permutation is rebuilt only by this call; value changes (normalize,
 * set_storage) are picked up automatically. Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_graph_reorder(scl_gpu_graph_t graph, int mode, void* stream);

/* Launch shape scl_gpu_diffuse uses for this graph at `n_features` columns in
 * the current storage dtype (same meaning as scl_gpu_spmm's shape arguments);
 * group <= 0 removes it (built-in default). Every shape computes the same bits. */
SCL_EXPORT scl_error_t scl_gpu_graph_set_plan(scl_gpu_graph_t graph, int64_t n_features, int group, int vec, int kind,
                                              int stage);

/* The reordering's permutation (perm[new] = old, host int32 [n_rows]) and the
 * number of component-labelling rounds it took; either pointer may be NULL. */
SCL_EXPORT scl_error_t scl_gpu_graph_reorder_info(scl_gpu_graph_t graph, int32_t* perm, int* cc_rounds, void* stream);

/* One Y = P X (original row order) with an explicit launch shape: group lanes
 * per row in {1,2,4,8,16,32}; vec = 16 bytes / element size, or 1; kind 0 =
 * register-gather kernel, 1 = cp.async shared-memory pipeline (vec > 1,
 * group >= 4) with `stage` in {4, 8, 16} entries per stage. group <= 0 picks
 * the default shape. X and Y must be in the storage dtype (Y may also be F32).
 * Every shape computes the same bits. */
SCL_EXPORT scl_error_t scl_gpu_spmm(scl_gpu_graph_t graph, const void* X, void* Y, scl_dtype_t y_dtype,
                                    int64_t n_features, int group, int vec, int kind, int stage, void* stream);

/* Diffusion that allocates no device memory. No counterpart in scl-core.
 *
 * For callers that cannot allocate GPU memory while they run: a framework
 * that owns the whole device-memory budget through its own arena and forbids
 * outside cudaMalloc, a serving loop that must neither block nor fail on an
 * allocation after start-up, or code that must not let cudaMalloc/cudaFree
 * synchronise the device. Computes Y = P^n_steps X (FP32, row-major
 * n_rows x n_features, the same bits as scl_gpu_diffuse) for a device CSR
 * transition matrix P given as indptr (int64, n_rows + 1), indices (int32,
 * each in [0, n_rows)) and values (f32). X and Y are caller-owned device
 * buffers and must be different; the one intermediate iterate lives in a
 * fixed 32 MiB scratch array compiled into the library, which every GPU that
 * loads the library holds until the process exits.
 *
 * Limit: n_rows * n_features <= 8,388,608, else SCL_ERROR_INVALID_ARGUMENT
 * and nothing is launched. The first call on each device looks up the scratch
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture. All calls share the one array and it keeps the last
 * call's contents (every element is overwritten before it is read, so no
 * clearing is needed); calls that overlap on the GPU — other streams, other
 * threads — race on it. Asynchronous on `stream`. */
SCL_EXPORT scl_error_t scl_gpu_diffuse_noalloc(const int64_t* indptr, const int32_t* indices, const float* values,
                                               int64_t n_rows, const float* X, float* Y, int64_t n_features,
                                               int64_t n_steps, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SCL_B200_GPU_H */
