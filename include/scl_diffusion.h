/*
 * scl_diffusion.h — drop-in diffusion C ABI, executed on a B200 GPU.
 *
 * Replaces scl/binding/c_api/diffusion.h:15-122 of scl-core (implementation in
 * scl/binding/c_api/diffusion.cpp). Signatures, argument meaning, in-place
 * semantics and error codes are the reference's; the arithmetic runs as CUDA
 * kernels on the current device. Host pointers in, host pointers out: each
 * call uploads the handle's arrays and the dense block, runs on the device and
 * writes the result back in place, synchronously.
 *
 * There is no CPU fallback: without a usable CUDA device every entry point
 * returns SCL_ERROR_FEATURE_UNAVAILABLE.
 */
#ifndef SCL_B200_DIFFUSION_H
#define SCL_B200_DIFFUSION_H

#include "scl_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* diffusion.h:15-18 (diffusion.cpp:36-62). Normalises the handle's values in
 * place: row (D^-1 A) when symmetric == 0, D^-1/2 A D^-1/2 otherwise; rows with
 * degree <= 1e-15 become zero. The handle must be contiguous, else
 * SCL_ERROR_INVALID_ARGUMENT "Matrix must be contiguous for transition matrix
 * computation" (as the reference). Degrees are reduced in FP64 on the device
 * (see scl_diffusion_gpu_set_degree_mode for the reference's native-precision
 * arithmetic). */
SCL_EXPORT scl_error_t scl_diffusion_compute_transition_matrix(scl_sparse_t adjacency, int symmetric);

/* diffusion.h:21-26 (diffusion.cpp:68-88). x <- P^n_steps x over the handle's
 * primary dimension; n_nodes must be >= that dimension. */
SCL_EXPORT scl_error_t scl_diffusion_diffuse_vector(scl_sparse_t transition, scl_real_t* x, scl_size_t n_nodes,
                                                    scl_index_t n_steps);

/* diffusion.h:29-35 (diffusion.cpp:94-116). X (n_nodes x n_features, row-major)
 * <- P^n_steps X in place. A CSR handle applies P, a CSC handle applies P^T
 * (its primary dimension is the column), exactly as in the reference. Here
 * n_nodes must equal the primary dimension. */
SCL_EXPORT scl_error_t scl_diffusion_diffuse_matrix(scl_sparse_t transition, scl_real_t* X, scl_index_t n_nodes,
                                                    scl_index_t n_features, scl_index_t n_steps);

/* diffusion.h:99-105 (diffusion.cpp:318-341). diffuse_matrix with t == 0
 * meaning 3 steps. */
SCL_EXPORT scl_error_t scl_diffusion_magic_impute(scl_sparse_t transition, scl_real_t* X, scl_index_t n_nodes,
                                                  scl_index_t n_features, scl_index_t t);

/* Vector walks (diffusion.h:58-96, 119; diffusion.cpp:179-248, 285-312,
 * 375-399): scl_diffusion_random_walk_with_restart,
 * scl_diffusion_personalized_pagerank, scl_diffusion_heat_kernel_signature and
 * scl_diffusion_lazy_random_walk keep the reference's arguments, defaults
 * (alpha 0 -> 0.85, tol 0 -> 1e-6, max_iter 0 -> 100, HKS steps 0 -> 10,
 * laziness 0 -> 0.5), checks and the restart walk's buffer swap (after an
 * unconverged last step the caller's array holds the previous iterate, as in
 * the reference). Each step is one kernel: (P x)_i as 32 lane fma chains
 * (entries l, l+32, ...) combined by a fixed xor butterfly, then
 * y = fma(c_x, x, c_p (P x)) (lazy, HKS) or y = fma(alpha, (P x),
 * (1 - alpha) r) (restart); the restart walk's L1 change is summed in FP64 in
 * a fixed block order and tested against tol on the device, the host reading
 * the result once per eight queued steps.
 * scl-core's own SpMV rounding depends on its compiler's contraction, so these
 * agree with it to a few ulps rather than bit for bit. The walk's size is the
 * handle's primary dimension; n_nodes must be at least that
 * (SCL_ERROR_DIMENSION_MISMATCH otherwise).
 *
 * Diffusion pseudotime (diffusion.h:38-55; diffusion.cpp:122-172;
 * diffusion.hpp:670-831): scl_diffusion_compute_dpt walks from one root
 * (max_iter 0 -> 100, tol 0 -> 1e-6; a root outside the graph is
 * SCL_ERROR_INVALID_ARGUMENT), accumulating hitting times and visit
 * probabilities until the largest unvisited probability is below tol, then
 * scales the visited rows' (> 0.5) mean hitting times to [0, 1] (others 1);
 * scl_diffusion_compute_dpt_multi_root averages that over the in-range roots
 * (none: all ones), each walked with the default tolerance.
 *
 * Diffusion map embedding (diffusion.h:79-84; diffusion.hpp:366-446,
 * 901-955): the reference's cosine start, modified Gram-Schmidt with its
 * re-orthogonalisation rule, then n_iter (0 -> 50) rounds of Q <- P Q and
 * Gram-Schmidt; the dot products are FP64 block sums and the start uses
 * CUDA's cos/sin, so the result agrees with the reference to a tolerance.
 * n_nodes must be at least the primary dimension.
 *
 * Diffusion distance (diffusion.h:108-113; diffusion.hpp:1024-1130): the n x n
 * pairwise L2 distances (row stride n) between the rows of P^n_steps for
 * n <= 1000 and between its columns for n > 1000, the reference's two
 * branches; each pair sums its rounded squares in order. At most 46,340
 * nodes. */
SCL_EXPORT scl_error_t scl_diffusion_compute_dpt(scl_sparse_t transition, scl_index_t root_cell,
                                                 scl_real_t* pseudotime, scl_size_t n_nodes, scl_index_t max_iter,
                                                 scl_real_t tol);
SCL_EXPORT scl_error_t scl_diffusion_compute_dpt_multi_root(scl_sparse_t transition, const scl_index_t* root_cells,
                                                            scl_size_t n_roots, scl_real_t* pseudotime,
                                                            scl_size_t n_nodes, scl_index_t max_iter);
SCL_EXPORT scl_error_t scl_diffusion_random_walk_with_restart(scl_sparse_t transition, const scl_index_t* seed_nodes,
                                                              scl_size_t n_seeds, scl_real_t* scores,
                                                              scl_size_t n_nodes, scl_real_t alpha,
                                                              scl_index_t max_iter, scl_real_t tol);
SCL_EXPORT scl_error_t scl_diffusion_personalized_pagerank(scl_sparse_t transition, scl_index_t seed_node,
                                                           scl_real_t* scores, scl_size_t n_nodes, scl_real_t alpha,
                                                           scl_index_t max_iter, scl_real_t tol);
SCL_EXPORT scl_error_t scl_diffusion_diffusion_map_embedding(scl_sparse_t transition, scl_real_t* embedding,
                                                             scl_index_t n_nodes, scl_index_t n_components,
                                                             scl_index_t n_iter);
SCL_EXPORT scl_error_t scl_diffusion_heat_kernel_signature(scl_sparse_t transition, scl_real_t* signature,
                                                           scl_size_t n_nodes, scl_real_t t, scl_index_t n_steps);
SCL_EXPORT scl_error_t scl_diffusion_diffusion_distance(scl_sparse_t transition, scl_real_t* distances,
                                                        scl_size_t n_nodes, scl_index_t n_steps);
SCL_EXPORT scl_error_t scl_diffusion_lazy_random_walk(scl_sparse_t transition, scl_real_t* x, scl_size_t n_nodes,
                                                      scl_index_t n_steps, scl_real_t laziness);

/* ---- additions (no counterpart in scl-core) --------------------------------
 * Degree arithmetic for scl_diffusion_compute_transition_matrix on this thread:
 * 0 = FP64 degrees and scales, one rounding of v * scale (default);
 * 1 = degrees, 1/d and 1/sqrt(d) in scl_real_t, as scl-core computes them
 *     (bit-identical to the reference build of the same precision). */
SCL_EXPORT scl_error_t scl_diffusion_gpu_set_degree_mode(int mode);

/* Locality reordering of diffuse_matrix on this thread: -1 = automatic (when
 * the dense block is at least 32 MiB and n_steps >= 2; default), 0 = off,
 * 1 = always. Results are bit-identical either way: rows of each connected
 * component are grouped for cache locality and every row keeps its stored
 * entry order. */
SCL_EXPORT scl_error_t scl_diffusion_gpu_set_reorder(int mode);

/* Keep a device copy of the handle's arrays between calls. Later diffusion
 * calls on the handle skip the upload of the graph; the caller promises not to
 * modify the wrapped arrays except through this library until detach. */
SCL_EXPORT scl_error_t scl_diffusion_gpu_attach(scl_sparse_t handle);
SCL_EXPORT scl_error_t scl_diffusion_gpu_detach(scl_sparse_t handle);

/* Device time (ms, CUDA events around the kernels) and host<->device bytes of
 * the last scl_diffusion_* call on this thread. */
SCL_EXPORT scl_error_t scl_diffusion_gpu_last_stats(double* device_ms, double* h2d_bytes, double* d2h_bytes);

#ifdef __cplusplus
}
#endif
#endif /* SCL_B200_DIFFUSION_H */
