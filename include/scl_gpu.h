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

/* Row reordering used by scl_gpu_diffuse (P' = Pi P Pi^T, X gathered once and
 * the result scattered back on the last step): mode 1 groups the rows of each
 * connected component together, longest rows first inside a component; mode 2
 * puts the longest rows first across the whole graph; mode 0 drops it. Each
 * row keeps its stored entry order, so results are bit-identical with and
 * without it. The
 * permutation is rebuilt only by this call; value changes (normalize,
 * set_storage) are picked up automatically. Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_graph_reorder(scl_gpu_graph_t graph, int mode, void* stream);

/* Launch shape scl_gpu_diffuse uses for this graph at `n_features` columns in
 * the current storage dtype (same meaning as scl_gpu_spmm's shape arguments);
 * group <= 0 removes it (built-in default). Every shape computes the same bits. */
SCL_EXPORT scl_error_t scl_gpu_graph_set_plan(scl_gpu_graph_t graph, int64_t n_features, int group, int vec, int kind,
                                              int stage);

/* Measurement aid (no counterpart in scl-core): median time in ms over `reps`
 * of a kernel that only gathers one row of n_features elements of `dtype` per
 * stored entry, in the order scl_gpu_diffuse visits the entries (the reordered
 * structure when one is set), at full occupancy and with the L2 flushed before
 * each repetition. It is the memory-system floor of one SpMM step on this
 * graph (row pitch 128, 256 or 512 bytes). Synchronises `stream`. */
/* Status of the bulk-copy SpMM (plan kind 11; no counterpart in scl-core):
 * every wait of that kernel on its copies is bounded (2 s); a wait that gives
 * up records SCL_ERROR_CONVERGENCE and the global warp index, and the warp
 * leaves its rows unwritten. Synchronises `stream`, stores the code (0 = none)
 * and the warp (NULL allowed), and clears the word. */
SCL_EXPORT scl_error_t scl_gpu_spmm_status(int32_t* code, int32_t* warp, void* stream);

/* Test hook for that bounded wait: global warp `warp` of later kind-11
 * launches expects 16 bytes more than its first chunk copies, so that wait
 * runs out; -1 turns the hook off. Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_spmm_inject_stall(int64_t warp, void* stream);

SCL_EXPORT scl_error_t scl_gpu_graph_gather_floor(scl_gpu_graph_t graph, int64_t n_features, scl_dtype_t dtype,
                                                  int reps, double* ms, void* stream);

/* Autotuner: times every launch shape that computes the same bits as the
 * default one for n_features columns in the current storage dtype (row pitch,
 * gathers per batch, kernel family members), `reps` SpMM steps each on the
 * structure scl_gpu_diffuse uses, and keeps the fastest as this graph's plan
 * for that width (scl_gpu_graph_set_plan). Reports its kind, stage and median
 * step time; any pointer may be NULL. Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_graph_autotune(scl_gpu_graph_t graph, int64_t n_features, int reps, int* kind,
                                              int* stage, double* best_ms, void* stream);

/* The reordering's permutation (perm[new] = old, host int32 [n_rows]) and the
 * number of component-labelling rounds it took; either pointer may be NULL. */
SCL_EXPORT scl_error_t scl_gpu_graph_reorder_info(scl_gpu_graph_t graph, int32_t* perm, int* cc_rounds, void* stream);

/* One Y = P X (original row order) with an explicit launch shape: group lanes
 * per row in {1,2,4,8,16,32}; vec = 16 bytes / element size, or 1; kind 0 =
 * register-gather kernel, 1 = cp.async shared-memory pipeline (vec > 1,
 * group >= 4) with `stage` in {4, 8, 16} entries per stage; 2/3 = row-block
 * stream (register / cp.async); 4 = warp per row with a compile-time pitch
 * (stage = gathers per batch 8/16/32); 5 = bf16/f16 storage, warp per row
 * with one 16-byte chunk per lane, group = row bytes / 16 (8 or 16), so one
 * load gathers 32/group entries that feed 32/group interleaved fma chains
 * summed pairwise at the row end (stage = gathers per lane per batch: 2/4/8
 * for 128-byte rows, 4/8/16 for 256-byte rows); 6 = kind 5 with the
 * mixed-precision fma; 7 = flat entry stream over tasks of 16 consecutive
 * rows with kind 4's lane layout (stage = gathers per batch 8/16/32; batches
 * stay full across row ends); 9 = kind 5/6's layout and chains with the
 * gathers copied by cp.async into shared memory, two chunks of 32 entries in
 * flight per warp (stage 0 = plain fma, 1 = mixed-precision fma); 10 = kind
 * 9's layout and chains with predicate-free full chunks (the default for
 * 16-bit storage; stage 0 = mixed-precision fma, 1 = bf16 only, each word's
 * two elements advanced by one packed f32x2 fma); 11 = FP32/FP64, warp per
 * row with kind 4's lane layout, the gathered X rows copied whole by the
 * bulk-copy engine (cp.async.bulk, one row per lane of a 32-entry chunk) into
 * a per-warp shared-memory ring of `stage` chunks (2, 3, 4 or 6; 128/256/512-
 * byte rows, FP64 256/512), waits bounded and reported through
 * scl_gpu_spmm_status. group <= 0 picks the
 * default shape. X and Y must be in the storage dtype (Y may also be F32).
 * Every shape of kinds 0-4, 7 and 11 computes the same bits (the sequential fma
 * chain); kinds 5, 6, 9 and 10 compute the same bits as each other (the
 * interleaved chains). */
SCL_EXPORT scl_error_t scl_gpu_spmm(scl_gpu_graph_t graph, const void* X, void* Y, scl_dtype_t y_dtype,
                                    int64_t n_features, int group, int vec, int kind, int stage, void* stream);

/* ---- gradients (no counterpart in scl-core, which has no backward pass) ----
 * For L(X_T) with X_T = P^T X_0 and P = normalise(W) (scl_gpu_graph_normalize):
 * dL/dX_0 = G_0 with G_s = P^T G_{s+1}, G_T = dL/dX_T, and
 * dL/dW per stored entry through the SDDMM gP_ij = sum_s <G_{s+1}[i], X_s[j]>
 * and the row / symmetric normalisation (FP64 degrees). All dense blocks are
 * row-major n x n_features in the graph's master dtype (f32 or f64) on the
 * device; the storage dtype must be the master dtype. */

/* Replace the graph's values (its pre-normalisation weights W, nnz entries in
 * the graph's CSR order, f32 or f64, host or device). The graph becomes
 * un-normalised; call scl_gpu_graph_normalize next. */
SCL_EXPORT scl_error_t scl_gpu_graph_set_weights(scl_gpu_graph_t graph, const void* values, scl_dtype_t dtype,
                                                 int on_device, void* stream);

/* Y = P^n_steps X0 (original row order, X0 != Y) keeping checkpoints for
 * scl_gpu_diffuse_backward: X_s for s = every, 2*every, ... < n_steps, i.e.
 * nc = (n_steps - 1) / every blocks of n x n_features written to
 * `checkpoints`, and with keep_last != 0 also the iterates of the last segment
 * after its checkpoint (n_steps - 1 - nc * every more blocks, which the
 * backward then does not recompute). NULL allowed when no block is kept.
 * Same bits as scl_gpu_diffuse. */
SCL_EXPORT scl_error_t scl_gpu_diffuse_checkpointed(scl_gpu_graph_t graph, const void* X0, void* Y,
                                                    int64_t n_features, int64_t n_steps, int64_t every,
                                                    int keep_last, void* checkpoints, void* stream);

/* Backward of scl_gpu_diffuse_checkpointed with the same X0, checkpoints,
 * n_steps, every and keep_last: given dY = dL/dX_T, writes dX0 = dL/dX_0 and,
 * when dW is non-NULL, dW = dL/dW (nnz entries, graph CSR order; dL/dP when
 * the graph was not normalised). Iterates that were not kept are recomputed
 * from their segment's checkpoint with the forward SpMM; each backward step is
 * one fused kernel over the CSC view of P (built once per graph) that gathers
 * G_{s+1} rows once for both the transpose-SpMM and the per-entry SDDMM. */
SCL_EXPORT scl_error_t scl_gpu_diffuse_backward(scl_gpu_graph_t graph, const void* X0, const void* checkpoints,
                                                const void* dY, int64_t n_features, int64_t n_steps, int64_t every,
                                                int keep_last, void* dX0, void* dW, void* stream);

/* ---- batched diffusion (no counterpart in scl-core, which diffuses one graph
 * per call: scl/binding/c_api/diffusion.h:28-35) ----
 * Many independent graphs of uneven size, each with its own dense block, all
 * n_steps steps in ONE persistent kernel launch replayed from a CUDA graph.
 * The graphs (normalised, f32 values and storage, on the current device) are
 * copied into one block-diagonal CSR at creation; the dense blocks are the
 * graphs' blocks stacked row-wise: graph b's rows start at row_offsets[b] of a
 * (row_offsets[n_graphs]) x n_features f32 block. Each graph's result is
 * bit-identical to scl_gpu_diffuse of that graph alone. A work item waits for
 * its graph's previous step with an iteration limit (about a second); a wait
 * that gives up sets the batch status (scl_gpu_batch_status) to
 * SCL_ERROR_CONVERGENCE and the launch returns early. */
typedef struct scl_gpu_batch scl_gpu_batch;
typedef scl_gpu_batch* scl_gpu_batch_t;

SCL_EXPORT scl_error_t scl_gpu_batch_create(scl_gpu_batch_t* out, int64_t n_graphs, const scl_gpu_graph_t* graphs,
                                            int64_t n_features, int64_t n_steps, void* stream);
SCL_EXPORT scl_error_t scl_gpu_batch_destroy(scl_gpu_batch_t* batch);
/* row_offsets: host int64 [n_graphs + 1] (may be NULL); nnz_total and n_tiles may be NULL. */
SCL_EXPORT scl_error_t scl_gpu_batch_layout(scl_gpu_batch_t batch, int64_t* row_offsets, int64_t* nnz_total,
                                            int64_t* n_tiles);
/* Explicit schedule: about tile_nnz stored entries per tile, unroll (4 or 8)
 * gathers in flight per lane, blocks_per_sm resident CTAs (0 = occupancy
 * limit). Drops the captured CUDA graph. */
SCL_EXPORT scl_error_t scl_gpu_batch_set_schedule(scl_gpu_batch_t batch, int64_t tile_nnz, int unroll,
                                                  int blocks_per_sm, void* stream);
/* Autotuner: times every candidate schedule (tile size x unroll x CTAs per
 * SM) on these blocks, `reps` launches each, and keeps the fastest.
 * Synchronises `stream`; Y is overwritten. */
SCL_EXPORT scl_error_t scl_gpu_batch_autotune(scl_gpu_batch_t batch, const float* X0, float* Y, int reps,
                                              void* stream);
SCL_EXPORT scl_error_t scl_gpu_batch_schedule(scl_gpu_batch_t batch, int64_t* tile_nnz, int* unroll, int* grid,
                                              int* lanes_per_row, double* tuned_ms);
/* Y = P_b^n_steps X0_b for every graph b (X0 != Y). The first call captures
 * the memset + kernel into a CUDA graph; later calls replay it (updating the
 * block pointers when they change). Asynchronous on `stream`. */
SCL_EXPORT scl_error_t scl_gpu_batch_solve(scl_gpu_batch_t batch, const float* X0, float* Y, void* stream);
/* Synchronises `stream`, returns the status of the launches since the last
 * call (0 = ok, SCL_ERROR_CONVERGENCE = a wait gave up; item = its work item)
 * and clears it. */
SCL_EXPORT scl_error_t scl_gpu_batch_status(scl_gpu_batch_t batch, int* code, int* item, void* stream);
/* Failure-path test hook: while graph >= 0, that graph's step waits need one
 * more finished tile than exists, so they give up after their time limit and
 * the next scl_gpu_batch_status reports SCL_ERROR_CONVERGENCE; -1 turns it off.
 * Results of a stalled launch are undefined. */
SCL_EXPORT scl_error_t scl_gpu_batch_inject_stall(scl_gpu_batch_t batch, int graph);

/* FP64 error of a diffused block against an FP64 reference (the final
 * residual check of the precision forms). No counterpart in scl-core: its
 * diffusion (scl/kernel/diffusion.hpp:638-664) has one precision per build,
 * and this compares a 16- or 32-bit result with the FP64 build's.
 *
 * X (x_dtype: f32, f64, bf16 or f16) and X_ref (f64) are device blocks of
 * n_rows * n_features elements. Reduced on the device in FP64 in a fixed order
 * (the same bits on every run), then written to host memory out[4]:
 *   out[0] = ||X - X_ref||_F / ||X_ref||_F   (0 when both are zero)
 *   out[1] = max |x - r| / max(|r|, rel_floor)
 *   out[2] = max |x - r|
 *   out[3] = ||X_ref||_F
 * Synchronises `stream`. */
SCL_EXPORT scl_error_t scl_gpu_residual_fp64(const void* X, scl_dtype_t x_dtype, const double* X_ref,
                                             int64_t n_rows, int64_t n_features, double rel_floor, double* out,
                                             void* stream);

/* Which kernel scl_knn / scl_knn_simple run. No counterpart in scl-core
 * (scl/kernel/neighbors.hpp:319-478 has one CPU loop); both kernels replay
 * that loop's skip test, distance arithmetic and heap rules and return the
 * same bits.
 *   kernel 0 (default): automatic; kernel 1 below 24,576 samples when it
 *     applies, kernel 2 otherwise.
 *   kernel 1: every distance computed exactly on CUDA cores; up to 128
 *     features and k up to 64.
 *   kernel 2: tensor-core filter. BF16 inner products on tcgen05 bound
 *     every distance; only candidates that can reach the heap are recomputed
 *     exactly. Any feature count, any k.
 * The choice is process-wide. previous (may be null) receives the old one. */
SCL_EXPORT scl_error_t scl_gpu_knn_set_kernel(int kernel, int* previous);

/* The per-warp schedule of row groups that the SpMM plan kinds 9, 10, 12
 * and 14 follow on a reordered graph (built there once per graph and warp
 * count). No counterpart in scl-core. Host only: indptr holds the n_rows + 1
 * row offsets of a CSR structure, groups are rows_per_group (1, 2 or 4)
 * consecutive rows, and n_warps lists are made. Groups whose longest row is
 * over eight times the mean row length are dealt first, longest first, each
 * to the least-loaded warp (ties: the lowest warp); then every other group in
 * index order, each to the least-loaded warp (cost = longest row + 8). A
 * warp's list holds its long groups first, then its others by index. out
 * (out_len = n_warps + 1 + ceil(n_rows / rows_per_group)) receives the
 * n_warps + 1 list offsets, then the group ids. */
SCL_EXPORT scl_error_t scl_gpu_warp_schedule(const int64_t* indptr, int64_t n_rows, int rows_per_group,
                                             int64_t n_warps, int32_t* out, int64_t out_len);

/* Test hook of the tensor-core kNN's bounded waits. No counterpart in
 * scl-core. CTA `cta` of the following tensor-core searches never receives
 * its first accumulator, so its epilogue's wait runs out after 2 s: the
 * kernel then stops every role of that CTA, drains its copies and MMAs,
 * frees its tensor memory and returns, and scl_knn reports
 * SCL_ERROR_CONVERGENCE. Nothing faults. -1 switches the hook off. */
SCL_EXPORT scl_error_t scl_gpu_knn_inject_stall(int64_t cta, void* stream);

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
 * buffers; they must not overlap each other or the library's scratch array
 * (SCL_ERROR_INVALID_ARGUMENT otherwise), and every pointer must be non-null
 * (SCL_ERROR_NULL_POINTER). The one intermediate iterate lives in a fixed
 * 32 MiB scratch array compiled into the library, which every GPU that loads
 * the library holds until the process exits.
 *
 * Limit: n_rows * n_features <= 8,388,608, else SCL_ERROR_INVALID_ARGUMENT
 * and nothing is launched. The first call on each device, and the first call
 * from a context not seen before on it (another context, or the primary
 * context re-created after cudaDeviceReset), looks up the scratch array's
 * device address (cudaGetSymbolAddress); make that first call before any
 * stream capture. All calls share the one array and it keeps the last
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
