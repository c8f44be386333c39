// Internal C++ interface of the B200 diffusion engine.
//
// Everything here is host-callable C++ implemented in the .cu files; the C ABI
// layers (c_api_*.cpp) are the only callers. No torch types anywhere: device
// memory comes from a per-device stream-ordered pool owned by the engine, or
// from the caller as raw device pointers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace sclgpu {

// Error codes mirror scl/binding/c_api/core/core.h:128-166.
enum : int32_t {
  kOk = 0,
  kErrUnknown = 1,
  kErrInternal = 2,
  kErrOutOfMemory = 3,
  kErrNullPointer = 4,
  kErrInvalidArgument = 10,
  kErrDimensionMismatch = 11,
  kErrIndexOutOfBounds = 14,
  kErrTypeMismatch = 21,
  kErrNotImplemented = 40,
  kErrFeatureUnavailable = 41,
  kErrConvergence = 54,
};

struct Error : std::runtime_error {
  int32_t code;
  Error(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);

#define SCL_CUDA(call)                                                      \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) ::sclgpu::throw_cuda(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define SCL_REQUIRE(cond, code, msg)                 \
  do {                                               \
    if (!(cond)) throw ::sclgpu::Error((code), (msg)); \
  } while (0)

// Storage / element types accepted by the engine.
enum DType : int32_t { kF32 = 0, kF64 = 1, kBF16 = 2, kF16 = 3, kI32 = 4, kI64 = 5 };
size_t dtype_size(DType t);
bool is_float_dtype(DType t);

// ---------------------------------------------------------------------------
// Per-device runtime: one library stream and one stream-ordered memory pool.
// ---------------------------------------------------------------------------
int current_device();                 // throws kErrFeatureUnavailable without a GPU
cudaStream_t library_stream(int dev);  // non-blocking stream owned by the engine
cudaStream_t library_copy_stream(int dev);  // second engine stream, for copies overlapped with work
void* dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);
int sm_count(int dev);

// RAII device buffer from the engine pool (freed on the given stream).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(size_t b, cudaStream_t st) : bytes(b), s(st) { p = b ? dev_alloc(b, st) : nullptr; }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes), s(o.s) { o.p = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { reset(); p = o.p; bytes = o.bytes; s = o.s; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() { if (p) dev_free(p, s); p = nullptr; bytes = 0; }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// Device CSR graph (primary-major: rows of a CSR handle, columns of a CSC one).
// Row offsets are int64 (indptr), column indices int32, values in `vtype`.
// ---------------------------------------------------------------------------
// Non-owning view of a device CSR (structure + one value array).
struct CsrView {
  int64_t n_rows = 0;
  int64_t n_cols = 0;
  int64_t nnz = 0;
  const int64_t* indptr = nullptr;
  const int32_t* indices = nullptr;
  const void* values = nullptr;
  DType vtype = kF32;
};

struct DeviceCSR {
  int64_t n_rows = 0;   // primary dimension
  int64_t n_cols = 0;   // secondary dimension
  int64_t nnz = 0;
  DevBuf indptr;        // int64[n_rows + 1]
  DevBuf indices;       // int32[nnz]
  DevBuf values;        // vtype[nnz]
  DType vtype = kF32;
  CsrView view() const {
    CsrView v;
    v.n_rows = n_rows; v.n_cols = n_cols; v.nnz = nnz;
    v.indptr = indptr.as<int64_t>(); v.indices = indices.as<int32_t>();
    v.values = values.p; v.vtype = vtype;
    return v;
  }
};

// Status word written by kernels that validate inputs or wait with a bound.
// Layout: [0] = error code (0 ok), [1] = first offending index (low 32 bits).
struct DevStatus {
  DevBuf buf;
  explicit DevStatus(cudaStream_t s);
  void check(cudaStream_t s, const char* what);  // syncs s, throws on error
  int32_t* ptr() const { return buf.as<int32_t>(); }
};

// ---- conversions / validation --------------------------------------------
// Convert an index array of type `src` (kI32/kI64) on the device to int32 or int64.
void convert_indices(const void* src, DType src_t, int32_t* dst, int64_t count, cudaStream_t s);
void convert_offsets(const void* src, DType src_t, int64_t* dst, int64_t count, cudaStream_t s);
void convert_values(const void* src, DType src_t, void* dst, DType dst_t, int64_t count, cudaStream_t s);
// Checks 0 <= indices < n_cols, indptr[0] == 0, indptr non-decreasing, indptr[n] == nnz.
void validate_csr(const DeviceCSR& g, int32_t* status, cudaStream_t s);

// ---- SpMM / power iteration ------------------------------------------------
struct Reordered;
struct SpmmArgs {
  const int64_t* indptr;
  const int32_t* indices;
  const void* values;
  DType vtype;
  int64_t n_rows;
  int64_t F;
  const void* X;   // n_cols x F, row-major
  DType xtype;
  void* Y;         // n_rows x F, row-major
  DType ytype;
  const int32_t* row_map = nullptr;  // optional: output row r is written to Y[row_map[r]]
  // optional: the reordered graph whose structure indptr/indices are; the
  // kernels that take a per-warp schedule of rows (plan kinds 9, 10, 12, 14)
  // look theirs up in it (warp_schedule_for)
  const Reordered* reo = nullptr;
};
// Launch shape of the SpMM kernel: `group` lanes own one output row and each
// lane owns `vec` contiguous columns (16 bytes of X) per pass; vec == 1 is the
// scalar fallback for rows whose pitch is not a multiple of 16 bytes.
// kind 0 = register-gather kernel, kind 1 = cp.async shared-memory pipeline
// (16-byte lane chunks only) with `stage` entries per pipeline stage (4/8/16).
constexpr int kSpmmThreads = 256;
struct SpmmPlan {
  int group = 32;
  int vec = 1;
  int kind = 0;
  int stage = 8;
};
SpmmPlan default_spmm_plan(int64_t F, DType xtype, const void* X, const void* Y, DType ytype);
// Launch shapes that compute the same bits as the default one for this width
// and dtype (the default first): the autotuner's search space.
std::vector<SpmmPlan> candidate_plans(int64_t F, DType xtype, const void* X, const void* Y, DType ytype);

// One Y = P X. Each output element is the sequential fma chain over the row's
// nonzeros in stored order (FP32 accumulation, FP64 when values/X are f64).
void spmm(const SpmmArgs& a, cudaStream_t s);
void spmm_with_plan(const SpmmArgs& a, const SpmmPlan& plan, cudaStream_t s);
// Plan kind 11: row gathers by bulk copies into a per-warp shared-memory ring
// of `ns` stages (2, 3, 4 or 6); FP32/FP64 rows of 128/256/512 bytes (FP64:
// 256/512), same bits as kinds 0-4. Its bounded waits report through
// spmm_bulk_status (error code, 0 if none; the warp that gave up), which
// synchronises `s` and clears the word.
bool spmm_bulk_fits(int64_t F, DType t, const void* X, const void* Y);
void spmm_bulk(const SpmmArgs& a, int ns, cudaStream_t s);
int32_t spmm_bulk_status(cudaStream_t s, int32_t* warp);
void spmm_bulk_inject_stall(int64_t warp, cudaStream_t s);

// Y = P^steps X0. Intermediate iterates are stored as `mtype` (which must equal
// the graph's value dtype) in pool buffers; the last step writes Y in `ytype`.
// X0 may equal Y (in place). `plan` overrides the default launch shape.
void diffuse(const CsrView& g, const void* X0, DType xtype, void* Y, DType ytype, DType mtype, int64_t F,
             int64_t steps, cudaStream_t s, const SpmmPlan* plan = nullptr);

// ---- grouped-row layout (plan kind 13, spmm_grouped.cu) ------------------------------
// The rows of a structure taken C at a time (C = 32 lanes / (row bytes / 16)),
// each group's entries stored as blocks of 32 slots: slot s of block b holds
// entry b*(32/C) + s%(32/C) of row gC + s/(32/C), padding past a row's end.
struct Grouped {
  int C = 0;
  int64_t n_groups = 0, n_blocks = 0;
  DevBuf lens;   // int32[n]          row lengths
  DevBuf boff;   // int64[n_groups+1] first block of each group
  DevBuf gidx;   // int32[n_blocks*32] column ids (0 in padding)
  DevBuf gmap;   // int32[n_blocks*32] entry position in the source structure, -1 = padding
  DevBuf gval;   // vtype[n_blocks*32] values (0 in padding)
  DType vtype = kF32;
  uint64_t values_version = 0;  // source values version the slots were filled from
};
// Rows per group for this row pitch (0 when the pitch is not 128/256/512 bytes).
int grouped_rows_per_warp(int64_t F, DType xtype);
bool grouped_fits(int64_t F, DType xtype, const void* X, const void* Y, DType ytype);
void build_grouped(const CsrView& r, int C, Grouped& gr, cudaStream_t s);
void grouped_values(const void* vals, DType t, uint64_t version, Grouped& gr, cudaStream_t s);
// One Y = P X (a.X, a.Y, a.row_map, a.n_rows, a.F, dtypes) on the grouped layout with
// U gathers in flight per lane (4, 8 or 16); same bits as the sequential-chain kernels.
void spmm_grouped(const Grouped& gr, const SpmmArgs& a, int U, cudaStream_t s);

// ---- locality reordering ------------------------------------------------------
// Rows grouped by connected component, longest rows first inside a component
// (stable among equal lengths); entries of each row keep their original order,
// so diffusion results are bit-identical.
struct Reordered {
  int64_t n = 0, nnz = 0;
  int cc_rounds = 0;
  DevBuf perm;     // int32[n]   new row -> old row
  DevBuf iperm;    // int32[n]   old row -> new row
  DevBuf indptr;   // int64[n+1] permuted structure
  DevBuf indices;  // int32[nnz] renamed column ids
  DevBuf emap;     // int32[nnz] new entry -> old entry
  DevBuf values;   // vtype[nnz] values gathered through emap
  DType vtype = kF32;
  bool values_ok = false;
  uint64_t values_version = 0;  // bumped whenever `values` is rewritten
  // grouped layouts of the permuted structure for C = 1, 2, 4 rows per warp (built on first use)
  mutable std::unique_ptr<Grouped> grouped[3];
  // per-warp schedules of groups of R rows over nw warps (built on first use)
  struct Schedule {
    int R = 0;
    int64_t nw = 0;
    DevBuf list;
  };
  mutable std::vector<Schedule> schedules;
};
// Static schedule of the groups of R consecutive rows over nw warps, built on
// the host from the row lengths: groups whose longest row is over eight times
// the mean row length are dealt first, longest first, each to the least-loaded
// warp; then every other group in index order to the least-loaded warp (cost
// = longest row + 8). Each warp's list starts with its long groups. Layout:
// int32[nw + 1] list offsets, then int32[groups] group ids.
DevBuf warp_schedule(const int64_t* indptr, int64_t n, int R, int64_t nw, cudaStream_t s);
// The same schedule from host row offsets ip[0..n] (the host part of warp_schedule).
std::vector<int32_t> warp_schedule_host(const int64_t* ip, int64_t n, int R, int64_t nw);
// r's schedule for (R, nw), built and kept on first use; nullptr while s is
// capturing a CUDA graph (the build reads the row lengths on the host).
const int32_t* warp_schedule_for(const Reordered& r, int R, int64_t nw, cudaStream_t s);
// The grouped layout for C rows per warp with current values (built or refreshed on demand).
const Grouped& reordered_grouped(const Reordered& r, int C, cudaStream_t s);
// One SpMM step on the permuted structure with `plan` (kind 13 runs on the grouped layout).
void spmm_reordered(const Reordered& r, SpmmArgs a, const SpmmPlan& plan, cudaStream_t s);
// mode 1: connected components together, longest rows first inside each; mode 2: longest rows
// first across the whole graph (no component labelling).
void build_reorder(const CsrView& g, Reordered& r, cudaStream_t s, int mode = 1);
void reorder_values(const void* vals, DType t, Reordered& r, cudaStream_t s);
// Y = P^steps X0 through the permuted structure: X0 is gathered into permuted
// order once, the last step scatters rows back (Y may equal X0).
void diffuse_reordered(const Reordered& r, const void* X0, DType xtype, void* Y, DType ytype, int64_t F,
                       int64_t steps, cudaStream_t s, const SpmmPlan* plan = nullptr);

// ---- transition build -------------------------------------------------------
// degrees[i] = sequential FP64 sum of row i's values.
void row_degrees_fp64(const DeviceCSR& g, double* degrees, cudaStream_t s);
// In-place normalisation of g.values (f32 or f64): row (D^-1 W) or symmetric
// (D^-1/2 W D^-1/2); zero scale where d <= 1e-15. degree_mode 0 = FP64 degrees
// (one rounding of v*scale), 1 = degrees and scales in the value type exactly
// as scl-core computes them.
void normalize(DeviceCSR& g, int symmetric, int degree_mode, double* degrees_out, cudaStream_t s);

// Gaussian kNN weights: sigma_i = max(valid dists, 1e-10); w = expf(-(d/sigma)^2).
void gauss_weights(const int32_t* knn_idx, const float* knn_dist, int64_t n, int64_t k, float* sigma,
                   float* w, cudaStream_t s);
// (W + W^T)/2 over the union of kNN pairs -> fresh DeviceCSR (f32 values).
void symmetrize_knn(const int32_t* knn_idx, const float* w, int64_t n, int64_t k, DeviceCSR& out,
                    cudaStream_t s);

// ---- sorting / scans (building blocks) ----------------------------------------
// Stable LSD radix sort of 64-bit keys with a 32-bit payload, sorting on the
// low `key_bits` bits. Results in keys_out/vals_out; inputs are clobbered.
void radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_out, uint32_t* vals_out, int64_t count,
                      int key_bits, cudaStream_t s);
// Exclusive prefix sum over int64 (out may equal in). Returns nothing; total in out[count].
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t count, cudaStream_t s);

// Transpose structure: for CSR g (n_rows x n_cols) build the CSR of g^T and the
// map tmap[q] = position in g of the entry that lands at q in g^T.
void transpose_map(const DeviceCSR& g, DeviceCSR& gt, DevBuf& tmap, cudaStream_t s);

// ---- backward pass ----------------------------------------------------------------
// CSC view of P (the CSR of P^T) for the adjoint: structure built once per
// graph, values gathered from P's current values through tmap.
struct Adjoint {
  DeviceCSR t;    // P^T: indptr int64[n+1], indices int32[nnz], values vtype[nnz]
  DevBuf tmap;    // int32[nnz]: entry q of P^T is entry tmap[q] of P
  DevBuf tinv;    // int32[nnz]: entry p of P is entry tinv[p] of P^T
  bool values_ok = false;
  bool sym_structure = false;  // P^T has P's indptr and indices (P's values need no remap)
  DevBuf order;   // uint32[n]: rows of P^T in the order the backward steps take them
                  // (rows over twice the mean length first, longest first; then the rest in index order)
};
void build_adjoint(const DeviceCSR& g, Adjoint& a, cudaStream_t s);
void adjoint_values(const void* vals, DType t, Adjoint& a, cudaStream_t s);

// Checkpoint slots the forward fills: X_s for s = every, 2*every, ... < steps,
// plus (keep_last) the iterates of the last segment after its checkpoint.
int64_t checkpoint_slots(int64_t steps, int64_t every, bool keep_last);
// Y = P^steps X0 (f32 or f64, original row order), storing the checkpoints in
// ckpt (checkpoint_slots(...) blocks of n x F). X0 != Y.
void diffuse_checkpointed(const CsrView& g, const void* X0, void* Y, DType t, int64_t F, int64_t steps,
                          int64_t every, bool keep_last, void* ckpt, cudaStream_t s);
// Given dY = dL/dX_T: dX0 = dL/dX_0 and, when gPt is non-null, the SDDMM
// gradient dL/dP accumulated in P^T's (CSC) entry order.
void diffuse_backward(const CsrView& g, const Adjoint& adj, const void* X0, const void* ckpt, const void* dY,
                      DType t, int64_t F, int64_t steps, int64_t every, bool keep_last, void* dX0, void* gPt,
                      cudaStream_t s);
// dW (CSR order of P) from dL/dP in CSC order, through the row or symmetric
// normalisation with the FP64 degrees kept by normalize().
void normalize_backward(const CsrView& P, const Adjoint& adj, const void* gPt, const double* degrees, int symmetric,
                        void* dW, cudaStream_t s);
// Median time (ms) over `reps` of gathering one row_bytes-wide row per entry of
// idx[0..M) from an n_rows-row block — the memory-system floor of an SpMM step
// that visits the same column sequence (probe.cu).
double gather_floor_ms(const int32_t* idx, int64_t M, int64_t n_rows, int64_t row_bytes, int reps, cudaStream_t s);

// Imputation (impute.cu): the dense cells x genes block of a sparse expression
// matrix (csr: primary = cells, else primary = genes), and MAGIC's t steps
// X <- W X with W the row-normalised affinity (rows with sum < 1e-12 copy X).
void densify_expression(const CsrView& m, bool csr, int64_t n_cells, int64_t n_genes, void* dense, cudaStream_t s);
void magic_diffuse(const CsrView& aff, void* X, int64_t F, int64_t steps, cudaStream_t s);
// kNN imputation: out (n_cells x n_genes) = the dense block with every value
// not above threshold replaced by the Gaussian-weighted mean of the neighbours
// (nbr, dist: n_cells x K) that store the gene.
void knn_impute(const CsrView& m, bool csr, int64_t n_cells, int64_t n_genes, const void* nbr, DType it,
                const void* dist, int K, double bandwidth, double threshold, void* out, cudaStream_t s);
// Y (A.n_rows x K) <- alpha A X + beta Y, X: A.n_cols x K (scl_algebra_spmm's arithmetic).
void algebra_spmm(const CsrView& A, const void* X, int64_t K, void* Y, double alpha, double beta, cudaStream_t s);

// Brute-force kNN over the rows of a dense n x d block: indices (kI32/kI64)
// and sqrt distances [n, k], ascending, missing slots (inf, -1); and the
// squared row norms as sequential fma chains. knn_dense picks the CUDA-core
// kernel (knn.cu, d <= 128, k <= 64) for small sample counts and the
// tensor-core filter (knn_tc.cu, any d and k) otherwise, unless
// knn_set_kernel(1 or 2) fixed one; both give the same bits.
int knn_max_features();
int knn_set_kernel(int kernel);  // returns the previous choice
void knn_dense(const void* X, const void* norms, DType t, int64_t n, int d, int k, void* idx, DType it, void* dist,
               cudaStream_t s);
void knn_tensor(const void* X, const void* norms, DType t, int64_t n, int d, int k, void* idx, DType it, void* dist,
                cudaStream_t s);
// test hook: CTA `cta` of the next tensor-core kNN launches never sees its first accumulator (-1 = off)
void knn_tensor_inject_stall(int64_t cta, cudaStream_t s);
void row_norms_dense(const void* X, DType t, int64_t n, int d, void* out, cudaStream_t s);

// Vector walks (walks.cu). walk_linear: x <- c_x x + c_p P x, `steps` times
// (lazy random walk, heat-kernel signature). walk_restart: the restart walk
// y = alpha P x + (1 - alpha) r until the L1 change is below tol or max_iter
// steps, scores holding r on entry; returns the steps taken.
void walk_linear(const CsrView& P, void* x, int64_t steps, double c_x, double c_p, cudaStream_t s);
int64_t walk_restart(const CsrView& P, const void* r, void* scores, double alpha, int64_t max_iter, double tol,
                     cudaStream_t s);
// Diffusion pseudotime from one root (out: n values) and the average of
// n_roots such rows (all: n_roots x n, summed in root order, times 1/n_roots).
void dpt(const CsrView& P, int64_t root, void* out, int64_t max_iter, double tol, cudaStream_t s);
void dpt_average(const void* all, int64_t n_roots, int64_t n, DType t, void* out, cudaStream_t s);
// Diffusion map embedding: K columns (row-major n x K in out) from a fixed
// cosine start, orthonormalised, then n_iter rounds of Q <- P Q + Gram-Schmidt.
void diffusion_map(const CsrView& P, void* out, int K, int64_t n_iter, cudaStream_t s);
// Diffusion distance: D (n x n) = pairwise L2 distances between the rows of
// P^steps (n <= 1000) or its columns (n > 1000), as the reference's two branches.
void diffusion_distance(const CsrView& P, void* D, int64_t steps, cudaStream_t s);

// FP64 error of a block X (f32/f64/bf16/f16, `total` elements) against an FP64
// reference R, reduced on the device in a fixed order (residual.cu). Writes to
// host memory: relative Frobenius error, max |x-r|/max(|r|, rel_floor), max
// |x-r|, ||r||. Synchronises s.
void residual_fp64(const void* X, DType xt, const double* R, int64_t total, double rel_floor, double* out_host,
                   cudaStream_t s);

// dL/dP in CSR order from its CSC-order accumulator.
void scatter_adjoint_entries(const Adjoint& adj, const void* gPt, DType t, void* gP, cudaStream_t s);

}  // namespace sclgpu

namespace sclgpu {

// ---- batched diffusion -------------------------------------------------------------
// Many independent f32 graphs, all diffusion steps in one persistent kernel
// launch replayed from a CUDA graph (batch.cu). The graphs' structure and
// values are copied into one block-diagonal CSR at init.
class BatchSolver {
 public:
  BatchSolver() = default;
  BatchSolver(const BatchSolver&) = delete;
  BatchSolver& operator=(const BatchSolver&) = delete;
  ~BatchSolver();

  void init(const std::vector<CsrView>& graphs, int64_t F, int64_t steps, cudaStream_t s);
  // tile_nnz: stored entries per tile; unroll: gathers in flight (4 or 8);
  // blocks_per_sm: resident CTAs per SM (0 = occupancy limit)
  void set_schedule(int64_t tile_nnz, int unroll, int blocks_per_sm, cudaStream_t s);
  // times every candidate schedule on (X0, Y) and keeps the fastest
  void autotune(const float* X0, float* Y, int reps, cudaStream_t s);
  // Y = P_b^steps X0_b for every graph b, one CUDA-graph launch (asynchronous)
  void solve(const float* X0, float* Y, cudaStream_t s);
  // plain launch of the same kernel (no graph), for timing candidates
  void launch_direct(const float* X0, float* Y, cudaStream_t s);
  // syncs s; returns the kernel's status word (0 ok) and clears it
  int32_t status(cudaStream_t s, int32_t* item);
  // test hook: graph `graph`'s waits can never complete (-1 = off), so they run
  // into their time limit and report an error
  void inject_stall(int graph);

  int64_t n_graphs() const { return n_graphs_; }
  int64_t n_total() const { return n_total_; }
  int64_t nnz_total() const { return nnz_total_; }
  int64_t n_tiles() const { return n_tiles_; }
  int64_t tile_nnz() const { return tile_nnz_; }
  int unroll() const { return unroll_; }
  int grid() const { return grid_; }
  int group() const { return group_; }
  int vec() const { return vec_; }
  double tuned_ms() const { return tuned_ms_; }
  const std::vector<int64_t>& row_offsets() const { return row_off_; }

 private:
  void build_tiles(int64_t tile_nnz, cudaStream_t s);
  void invalidate_graph();
  void* params_for(const float* X0, float* Y, void* storage) const;
  double time_solve(const float* X0, float* Y, int reps, cudaStream_t s);

  int64_t F_ = 0, steps_ = 0, n_graphs_ = 0, n_total_ = 0, nnz_total_ = 0, n_tiles_ = 0, tile_nnz_ = 0;
  int unroll_ = 8, grid_ = 1, group_ = 1, vec_ = 1, blocks_per_sm_ = 0, stall_graph_ = -1;
  double tuned_ms_ = 0.0;
  std::vector<int64_t> row_off_, nnz_off_, h_indptr_;
  DevBuf indptr_, indices_, values_, tiles_, tile_graph_, graph_tiles_, counters_, status_, scratch_, row_order_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  cudaGraphNode_t knode_ = nullptr;
  const float* cap_x0_ = nullptr;
  float* cap_y_ = nullptr;
};

}  // namespace sclgpu
