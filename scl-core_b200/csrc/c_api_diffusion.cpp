// Drop-in diffusion C ABI executed on the GPU.
// Replaces scl/binding/c_api/diffusion.cpp:36-116 and 318-341 (argument
// checks, defaults and messages kept) with uploads + CUDA kernels.
#include <functional>
#include <cstring>
#include <vector>

#include "abi.hpp"
#include "scl_diffusion.h"
#include "scl_impute.h"
#include "scl_algebra.h"
#include "scl_neighbors.h"

using sclabi::Index;
using sclabi::Real;
using namespace sclgpu;

namespace sclabi {

// Device copy of a handle's primary-major arrays.
struct DeviceMirror {
  int device = -1;
  DeviceCSR g;
  std::unique_ptr<Reordered> reo;  // locality reordering (built on demand)
};

}  // namespace sclabi

namespace {

thread_local int t_degree_mode = 0;
// -1 = automatic (reorder when X is at least kReorderMinBytes and >= 2 steps),
//  0 = never, 1 = always (square matrices only).
thread_local int t_reorder_mode = -1;
constexpr int64_t kReorderMinBytes = 32ll << 20;

bool want_reorder(const DeviceCSR& g, int64_t F, int64_t steps, size_t esz) {
  if (g.n_rows != g.n_cols || g.n_rows < 2 || t_reorder_mode == 0) return false;
  if (t_reorder_mode == 1) return true;
  return steps >= 2 && g.n_rows * F * (int64_t)esz >= kReorderMinBytes;
}
struct Stats {
  double device_ms = 0, h2d = 0, d2h = 0;
};
thread_local Stats t_stats;

// Host -> device copy of the handle (indptr int64, indices int32, values Real).
// Rows whose storage is adjacent are copied as one run.
// `after_copies` (optional) runs once the host->device copies are issued on
// s, before the validation that waits for them, so the caller can start work
// on other streams right behind the copies.
std::shared_ptr<sclabi::DeviceMirror> upload(const scl_sparse_matrix& m, cudaStream_t s, double& h2d,
                                             const std::function<void()>& after_copies = {}) {
  auto mir = std::make_shared<sclabi::DeviceMirror>();
  mir->device = current_device();
  DeviceCSR& g = mir->g;
  const Index pdim = m.primary_dim();
  const std::vector<int64_t> off = sclabi::offsets_of(m);
  const int64_t nnz = off[pdim];
  g.n_rows = pdim;
  g.n_cols = m.secondary_dim();
  g.nnz = nnz;
  g.vtype = sclabi::kRealDType;
  g.indptr = DevBuf((pdim + 1) * sizeof(int64_t), s);
  g.indices = DevBuf(std::max<int64_t>(nnz, 1) * sizeof(int32_t), s);
  g.values = DevBuf(std::max<int64_t>(nnz, 1) * sizeof(Real), s);
  SCL_REQUIRE(m.secondary_dim() <= 0x7fffffff, SCL_ERROR_INVALID_ARGUMENT, "dimension exceeds the int32 column range");
  SCL_CUDA(cudaMemcpyAsync(g.indptr.p, off.data(), (pdim + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  h2d += (double)(pdim + 1) * sizeof(int64_t);
  DevBuf idx_tmp;
  void* idx_dst = g.indices.p;
  if (sizeof(Index) != sizeof(int32_t)) {
    idx_tmp = DevBuf(std::max<int64_t>(nnz, 1) * sizeof(Index), s);
    idx_dst = idx_tmp.p;
  }
  Index i = 0;
  while (i < pdim) {
    if (m.lengths[i] == 0) { ++i; continue; }
    Index j = i + 1;
    int64_t run = m.lengths[i];
    while (j < pdim && (m.lengths[j] == 0 ||
                        (m.data_ptrs[j] == m.data_ptrs[i] + run && m.index_ptrs[j] == m.index_ptrs[i] + run))) {
      run += m.lengths[j];
      ++j;
    }
    SCL_CUDA(cudaMemcpyAsync(static_cast<char*>(g.values.p) + off[i] * sizeof(Real), m.data_ptrs[i], run * sizeof(Real),
                             cudaMemcpyHostToDevice, s));
    SCL_CUDA(cudaMemcpyAsync(static_cast<char*>(idx_dst) + off[i] * sizeof(Index), m.index_ptrs[i], run * sizeof(Index),
                             cudaMemcpyHostToDevice, s));
    h2d += (double)run * (sizeof(Real) + sizeof(Index));
    i = j;
  }
  if (after_copies) after_copies();
  if (idx_tmp.p) convert_indices(idx_tmp.p, sclabi::kIndexDType, g.indices.as<int32_t>(), nnz, s);
  DevStatus st(s);
  validate_csr(g, st.ptr(), s);
  st.check(s, "invalid sparse structure: column index out of range or malformed offsets");
  return mir;
}

std::shared_ptr<sclabi::DeviceMirror> device_graph(scl_sparse_matrix& m, cudaStream_t s, double& h2d,
                                                   const std::function<void()>& after_copies = {}) {
  if (m.mirror && m.mirror->device == current_device()) {
    if (after_copies) after_copies();
    return m.mirror;
  }
  return upload(m, s, h2d, after_copies);
}

struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit EventTimer(cudaStream_t st) : s(st) {
    SCL_CUDA(cudaEventCreate(&a));
    SCL_CUDA(cudaEventCreate(&b));
  }
  ~EventTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  void start() { SCL_CUDA(cudaEventRecord(a, s)); }
  void stop() { SCL_CUDA(cudaEventRecord(b, s)); }
  double ms() {
    SCL_CUDA(cudaEventSynchronize(b));
    float t = 0;
    SCL_CUDA(cudaEventElapsedTime(&t, a, b));
    return t;
  }
};

// X (n x F) <- P^steps X on the device; shared by diffuse_matrix / magic_impute.
void diffuse_host_block(scl_sparse_matrix& m, Real* X, Index n_nodes, Index n_features, Index n_steps) {
  SCL_REQUIRE(m.valid, SCL_ERROR_INVALID_ARGUMENT, "Transition matrix is not valid");
  SCL_REQUIRE(n_nodes == m.primary_dim(), SCL_ERROR_DIMENSION_MISMATCH,
              "Diffusion: n_nodes must equal the transition matrix's primary dimension");
  SCL_REQUIRE(m.secondary_dim() <= n_nodes, SCL_ERROR_DIMENSION_MISMATCH,
              "Diffusion: column indices would address rows beyond n_nodes");
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  cudaStream_t cs = library_copy_stream(dev);
  Stats st;
  // The graph is uploaded on the main stream; the dense block follows on the
  // copy stream as soon as the graph's copies are issued, so its transfer
  // overlaps the graph's validation and the locality reordering built on the
  // main stream; the diffusion waits for both.
  const int64_t total = (int64_t)n_nodes * n_features;
  DevBuf Xd(total * sizeof(Real), cs);
  // on every exit (errors included) the copy stream is drained before the
  // caller's X can be released, and the events are destroyed
  struct CopyGuard {
    cudaStream_t s;
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~CopyGuard() {
      cudaStreamSynchronize(s);
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } guard{cs};
  SCL_CUDA(cudaEventCreateWithFlags(&guard.e[0], cudaEventDisableTiming));
  SCL_CUDA(cudaEventCreateWithFlags(&guard.e[1], cudaEventDisableTiming));
  cudaEvent_t graph_copied = guard.e[0], x_ready = guard.e[1];
  auto issue_x = [&]() {  // behind the graph's copies, ahead of its validation
    SCL_CUDA(cudaEventRecord(graph_copied, s));
    SCL_CUDA(cudaStreamWaitEvent(cs, graph_copied, 0));
    SCL_CUDA(cudaMemcpyAsync(Xd.p, X, total * sizeof(Real), cudaMemcpyHostToDevice, cs));
    st.h2d += (double)total * sizeof(Real);
    SCL_CUDA(cudaEventRecord(x_ready, cs));
  };
  auto mir = device_graph(m, s, st.h2d, issue_x);
  EventTimer tm(s);
  tm.start();
  if (want_reorder(mir->g, n_features, n_steps, sizeof(Real))) {
    if (!mir->reo) {
      mir->reo = std::make_unique<Reordered>();
      build_reorder(mir->g.view(), *mir->reo, s);
    }
    if (!mir->reo->values_ok) reorder_values(mir->g.values.p, mir->g.vtype, *mir->reo, s);
    SCL_CUDA(cudaStreamWaitEvent(s, x_ready, 0));
    diffuse_reordered(*mir->reo, Xd.p, sclabi::kRealDType, Xd.p, sclabi::kRealDType, n_features, n_steps, s);
  } else {
    SCL_CUDA(cudaStreamWaitEvent(s, x_ready, 0));
    diffuse(mir->g.view(), Xd.p, sclabi::kRealDType, Xd.p, sclabi::kRealDType, sclabi::kRealDType, n_features,
            n_steps, s);
  }
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(X, Xd.p, total * sizeof(Real), cudaMemcpyDeviceToHost, s));
  st.d2h += (double)total * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(s));
  SCL_CUDA(cudaStreamSynchronize(cs));  // Xd is returned to the pool on the copy stream
  st.device_ms = tm.ms();
  t_stats = st;
}

// Imputation (scl/binding/c_api/impute.cpp:93-157): the sparse expression
// matrix becomes a dense n_cells x n_genes block on the device, which is
// diffused over the cells graph and copied back into X_imputed.
void impute_host(scl_sparse_matrix& X, scl_sparse_matrix& T, Index n_cells, Index n_genes, Index n_steps,
                 Real* X_imputed, bool magic) {
  SCL_REQUIRE(X.valid, SCL_ERROR_INVALID_ARGUMENT, "Expression matrix is not valid");
  SCL_REQUIRE(T.valid, SCL_ERROR_INVALID_ARGUMENT, "Transition matrix is not valid");
  SCL_REQUIRE(T.primary_dim() == n_cells, SCL_ERROR_DIMENSION_MISMATCH,
              "Imputation: n_cells must equal the transition matrix's primary dimension");
  SCL_REQUIRE(T.secondary_dim() <= n_cells, SCL_ERROR_DIMENSION_MISMATCH,
              "Imputation: column indices would address cells beyond n_cells");
  SCL_REQUIRE(X.primary_dim() >= (X.is_csr ? n_cells : n_genes), SCL_ERROR_DIMENSION_MISMATCH,
              "Imputation: the expression matrix has fewer cells (CSR rows) or genes (CSC columns) than requested");
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  Stats st;
  const bool seed = !magic || X.is_csr;  // MAGIC starts from zero for a CSC matrix, as the reference
  std::shared_ptr<sclabi::DeviceMirror> xm;
  if (seed) xm = device_graph(X, s, st.h2d);
  auto tm = device_graph(T, s, st.h2d);
  const int64_t total = (int64_t)n_cells * n_genes;
  DevBuf D(std::max<int64_t>(total, 1) * sizeof(Real), s);
  EventTimer tmr(s);
  tmr.start();
  if (seed) densify_expression(xm->g.view(), X.is_csr, n_cells, n_genes, D.p, s);
  else SCL_CUDA(cudaMemsetAsync(D.p, 0, total * sizeof(Real), s));
  if (magic)
    magic_diffuse(tm->g.view(), D.p, n_genes, n_steps, s);
  else
    diffuse(tm->g.view(), D.p, sclabi::kRealDType, D.p, sclabi::kRealDType, sclabi::kRealDType, n_genes, n_steps, s);
  tmr.stop();
  SCL_CUDA(cudaMemcpyAsync(X_imputed, D.p, total * sizeof(Real), cudaMemcpyDeviceToHost, s));
  st.d2h += (double)total * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(s));
  st.device_ms = tmr.ms();
  t_stats = st;
}

// Vector walks (diffusion.cpp:179-248, 285-312, 375-399): the handle's
// primary dimension n is the walk's size; the caller's vector must hold at
// least n entries (only those are read and written).
struct WalkSetup {
  int dev;
  cudaStream_t s;
  std::shared_ptr<sclabi::DeviceMirror> mir;
  Index n;
};

WalkSetup walk_setup(scl_sparse_matrix& m, size_t n_nodes, const char* too_small, Stats& st) {
  SCL_REQUIRE(m.valid, SCL_ERROR_INVALID_ARGUMENT, "Transition matrix is not valid");
  const Index n = m.primary_dim();
  SCL_REQUIRE(n_nodes >= (size_t)n, SCL_ERROR_DIMENSION_MISMATCH, too_small);
  SCL_REQUIRE(m.secondary_dim() <= n, SCL_ERROR_DIMENSION_MISMATCH,
              "Walk: column indices would address entries beyond the vector");
  WalkSetup w;
  w.dev = current_device();
  w.s = library_stream(w.dev);
  w.mir = device_graph(m, w.s, st.h2d);
  w.n = n;
  return w;
}

// x <- c_x x + c_p P x, `steps` times, on the first n entries of x.
void walk_linear_host(scl_sparse_matrix& m, Real* x, size_t n_nodes, Index steps, Real c_x, Real c_p,
                      const char* too_small) {
  Stats st;
  WalkSetup w = walk_setup(m, n_nodes, too_small, st);
  if (w.n == 0 || steps <= 0) return;
  DevBuf xd(w.n * sizeof(Real), w.s);
  SCL_CUDA(cudaMemcpyAsync(xd.p, x, w.n * sizeof(Real), cudaMemcpyHostToDevice, w.s));
  st.h2d += (double)w.n * sizeof(Real);
  EventTimer tm(w.s);
  tm.start();
  walk_linear(w.mir->g.view(), xd.p, steps, (double)c_x, (double)c_p, w.s);
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(x, xd.p, w.n * sizeof(Real), cudaMemcpyDeviceToHost, w.s));
  st.d2h += (double)w.n * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(w.s));
  st.device_ms = tm.ms();
  t_stats = st;
}

// random_walk_with_restart (diffusion.hpp:833-895): restart = 1 / (number of
// in-range seeds, repeats counted) on every in-range seed; no in-range seed
// gives zero scores.
void walk_restart_host(scl_sparse_matrix& m, const Index* seeds, size_t n_seeds, Real* scores, size_t n_nodes,
                       Real alpha, Index max_iter, Real tol) {
  Stats st;
  WalkSetup w = walk_setup(m, n_nodes, "RWR: output buffer too small", st);
  if (w.n == 0) return;
  std::vector<Real> r((size_t)w.n, Real(0));
  size_t count = 0;
  for (size_t i = 0; i < n_seeds; ++i) {
    const Index idx = seeds[i];
    if (idx >= 0 && idx < w.n) {
      r[(size_t)idx] = Real(1);
      ++count;
    }
  }
  if (count == 0) {
    std::memset(scores, 0, (size_t)w.n * sizeof(Real));
    return;
  }
  const Real inv = Real(1) / static_cast<Real>(count);
  for (Real& v : r) v *= inv;
  DevBuf rd(w.n * sizeof(Real), w.s), sd(w.n * sizeof(Real), w.s);
  SCL_CUDA(cudaMemcpyAsync(rd.p, r.data(), w.n * sizeof(Real), cudaMemcpyHostToDevice, w.s));
  SCL_CUDA(cudaMemcpyAsync(sd.p, rd.p, w.n * sizeof(Real), cudaMemcpyDeviceToDevice, w.s));
  st.h2d += (double)w.n * sizeof(Real);
  EventTimer tm(w.s);
  tm.start();
  walk_restart(w.mir->g.view(), rd.p, sd.p, (double)alpha, max_iter, (double)tol, w.s);
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(scores, sd.p, w.n * sizeof(Real), cudaMemcpyDeviceToHost, w.s));
  st.d2h += (double)w.n * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(w.s));
  st.device_ms = tm.ms();
  t_stats = st;
}

// kNN imputation (impute.cpp:19-87, impute.hpp:400-510).
void knn_impute_host(scl_sparse_matrix& X, const Index* nbr, const Real* dist, Index n_cells, Index n_genes, Index K,
                     Real* X_imputed, Real bandwidth, Real threshold) {
  SCL_REQUIRE(X.valid, SCL_ERROR_INVALID_ARGUMENT, "Expression matrix is not valid");
  SCL_REQUIRE(X.primary_dim() >= (X.is_csr ? n_cells : n_genes), SCL_ERROR_DIMENSION_MISMATCH,
              "Imputation: the expression matrix has fewer cells (CSR rows) or genes (CSC columns) than requested");
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  Stats st;
  auto xm = device_graph(X, s, st.h2d);
  const int64_t nk = (int64_t)n_cells * K, total = (int64_t)n_cells * n_genes;
  DevBuf nb(std::max<int64_t>(nk, 1) * sizeof(Index), s), ds(std::max<int64_t>(nk, 1) * sizeof(Real), s);
  DevBuf out(std::max<int64_t>(total, 1) * sizeof(Real), s);
  SCL_CUDA(cudaMemcpyAsync(nb.p, nbr, nk * sizeof(Index), cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaMemcpyAsync(ds.p, dist, nk * sizeof(Real), cudaMemcpyHostToDevice, s));
  st.h2d += (double)nk * (sizeof(Index) + sizeof(Real));
  EventTimer tm(s);
  tm.start();
  knn_impute(xm->g.view(), X.is_csr, n_cells, n_genes, nb.p, sclabi::kIndexDType, ds.p, (int)K, (double)bandwidth,
             (double)threshold, out.p, s);
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(X_imputed, out.p, total * sizeof(Real), cudaMemcpyDeviceToHost, s));
  st.d2h += (double)total * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(s));
  st.device_ms = tm.ms();
  t_stats = st;
}

// kNN (neighbors.cpp): the handle's primary rows made dense on the device.
struct DenseSamples {
  cudaStream_t s;
  DevBuf X;
  int64_t n;
  int d;
};

DenseSamples dense_samples(scl_sparse_matrix& m, Stats& st) {
  SCL_REQUIRE(m.valid, SCL_ERROR_INVALID_ARGUMENT, "Invalid sparse matrix");
  DenseSamples ds;
  ds.s = library_stream(current_device());
  ds.n = m.primary_dim();
  const int64_t d = m.secondary_dim();
  SCL_REQUIRE(d >= 1 && d <= 0x7fffffff, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  ds.d = (int)d;
  auto mir = device_graph(m, ds.s, st.h2d);
  ds.X = DevBuf(std::max<int64_t>(ds.n * d, 1) * sizeof(Real), ds.s);
  densify_expression(mir->g.view(), true, ds.n, d, ds.X.p, ds.s);
  return ds;
}

void knn_host(scl_sparse_matrix& m, const Real* norms, size_t n_samples, size_t k, Index* out_idx, Real* out_dist) {
  Stats st;
  SCL_REQUIRE(n_samples == (size_t)m.primary_dim(), SCL_ERROR_DIMENSION_MISMATCH,
              "kNN: n_samples must equal the matrix's primary dimension");
  SCL_REQUIRE(k >= 1, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  DenseSamples ds = dense_samples(m, st);
  DevBuf nd(std::max<int64_t>(ds.n, 1) * sizeof(Real), ds.s);
  if (norms) {
    SCL_CUDA(cudaMemcpyAsync(nd.p, norms, ds.n * sizeof(Real), cudaMemcpyHostToDevice, ds.s));
    st.h2d += (double)ds.n * sizeof(Real);
  } else {
    row_norms_dense(ds.X.p, sclabi::kRealDType, ds.n, ds.d, nd.p, ds.s);
  }
  const int64_t total = ds.n * (int64_t)k;
  DevBuf di(std::max<int64_t>(total, 1) * sizeof(Index), ds.s), dd(std::max<int64_t>(total, 1) * sizeof(Real), ds.s);
  EventTimer tm(ds.s);
  tm.start();
  knn_dense(ds.X.p, nd.p, sclabi::kRealDType, ds.n, ds.d, (int)k, di.p, sclabi::kIndexDType, dd.p, ds.s);
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(out_idx, di.p, total * sizeof(Index), cudaMemcpyDeviceToHost, ds.s));
  SCL_CUDA(cudaMemcpyAsync(out_dist, dd.p, total * sizeof(Real), cudaMemcpyDeviceToHost, ds.s));
  st.d2h += (double)total * (sizeof(Index) + sizeof(Real));
  SCL_CUDA(cudaStreamSynchronize(ds.s));
  st.device_ms = tm.ms();
  t_stats = st;
}

constexpr Real kDefaultAlpha = Real(0.85);  // diffusion.cpp:20-27
constexpr Real kDefaultTol = Real(1e-6);
constexpr Index kDefaultMaxIter = 100;
constexpr Index kDefaultStepsHks = 10;
constexpr Real kDefaultLaziness = Real(0.5);

}  // namespace

extern "C" {

SCL_EXPORT scl_error_t scl_diffusion_compute_transition_matrix(scl_sparse_t adjacency, int symmetric) {
  SCL_API_CHECK_NULL(adjacency, "Adjacency matrix is null");
  SCL_API_TRY
  Real* values = adjacency->contiguous_data();
  SCL_API_CHECK(values != nullptr, SCL_ERROR_INVALID_ARGUMENT,
                "Matrix must be contiguous for transition matrix computation");
  SCL_API_CHECK(!symmetric || adjacency->rows == adjacency->cols, SCL_ERROR_DIMENSION_MISMATCH,
                "Symmetric normalization needs a square matrix");
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  Stats st;
  auto mir = device_graph(*adjacency, s, st.h2d);
  EventTimer tm(s);
  tm.start();
  normalize(mir->g, symmetric != 0, t_degree_mode, nullptr, s);
  if (mir->reo) mir->reo->values_ok = false;
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(values, mir->g.values.p, mir->g.nnz * sizeof(Real), cudaMemcpyDeviceToHost, s));
  st.d2h += (double)mir->g.nnz * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_diffuse_vector(scl_sparse_t transition, scl_real_t* x, scl_size_t n_nodes,
                                                    scl_index_t n_steps) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(x, "Vector x is null");
  SCL_API_CHECK(n_nodes > 0 && n_steps > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  scl_sparse_matrix& m = *transition;
  SCL_REQUIRE(m.valid, SCL_ERROR_INVALID_ARGUMENT, "Transition matrix is not valid");
  const int64_t N = m.primary_dim();
  // diffusion.hpp:617: SCL_CHECK_DIM(x.len >= N, ...)
  SCL_REQUIRE((int64_t)n_nodes >= N, SCL_ERROR_DIMENSION_MISMATCH, "Diffusion: vector size mismatch");
  SCL_REQUIRE((int64_t)m.secondary_dim() <= (int64_t)n_nodes, SCL_ERROR_DIMENSION_MISMATCH,
              "Diffusion: column indices would address entries beyond n_nodes");
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  Stats st;
  auto mir = device_graph(m, s, st.h2d);
  const int64_t nn = (int64_t)n_nodes;
  DevBuf xd(nn * sizeof(Real), s);
  SCL_CUDA(cudaMemcpyAsync(xd.p, x, nn * sizeof(Real), cudaMemcpyHostToDevice, s));
  st.h2d += (double)nn * sizeof(Real);
  EventTimer tm(s);
  tm.start();
  if (nn == N) {
    diffuse(mir->g.view(), xd.p, sclabi::kRealDType, xd.p, sclabi::kRealDType, sclabi::kRealDType, 1, n_steps, s);
  } else {
    // Entries beyond the primary dimension keep their input values and are
    // read by later steps, as in the reference's memcpy of N entries.
    DevBuf tmp(std::max<int64_t>(N, 1) * sizeof(Real), s);
    SpmmArgs a{};
    const CsrView v = mir->g.view();
    a.indptr = v.indptr; a.indices = v.indices; a.values = v.values; a.vtype = v.vtype;
    a.n_rows = N; a.F = 1;
    a.X = xd.p; a.xtype = sclabi::kRealDType; a.Y = tmp.p; a.ytype = sclabi::kRealDType;
    for (Index t = 0; t < n_steps; ++t) {
      spmm(a, s);
      SCL_CUDA(cudaMemcpyAsync(xd.p, tmp.p, N * sizeof(Real), cudaMemcpyDeviceToDevice, s));
    }
  }
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(x, xd.p, nn * sizeof(Real), cudaMemcpyDeviceToHost, s));
  st.d2h += (double)nn * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_diffuse_matrix(scl_sparse_t transition, scl_real_t* X, scl_index_t n_nodes,
                                                    scl_index_t n_features, scl_index_t n_steps) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(X, "Matrix X is null");
  SCL_API_CHECK(n_nodes > 0 && n_features > 0 && n_steps > 0, SCL_ERROR_INVALID_ARGUMENT,
                "Dimensions must be positive");
  SCL_API_TRY
  diffuse_host_block(*transition, X, n_nodes, n_features, n_steps);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_magic_impute(scl_sparse_t transition, scl_real_t* X, scl_index_t n_nodes,
                                                  scl_index_t n_features, scl_index_t t) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(X, "Matrix X is null");
  SCL_API_CHECK(n_nodes > 0 && n_features > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  const Index steps = (t == 0) ? 3 : t;  // diffusion.cpp:26 DEFAULT_N_STEPS
  if (steps > 0) diffuse_host_block(*transition, X, n_nodes, n_features, steps);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_compute_dpt(scl_sparse_t transition, scl_index_t root_cell,
                                                 scl_real_t* pseudotime, scl_size_t n_nodes, scl_index_t max_iter,
                                                 scl_real_t tol) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(pseudotime, "Output pseudotime array is null");
  SCL_API_CHECK(n_nodes > 0, SCL_ERROR_INVALID_ARGUMENT, "Number of nodes must be positive");
  SCL_API_TRY
  Stats st;
  WalkSetup w = walk_setup(*transition, n_nodes, "DPT: output buffer too small", st);
  SCL_REQUIRE(root_cell >= 0 && root_cell < w.n, SCL_ERROR_INVALID_ARGUMENT, "DPT: root_cell out of range");
  DevBuf out(w.n * sizeof(Real), w.s);
  EventTimer tm(w.s);
  tm.start();
  dpt(w.mir->g.view(), root_cell, out.p, max_iter == 0 ? kDefaultMaxIter : max_iter,
      (double)(tol == Real(0) ? kDefaultTol : tol), w.s);
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(pseudotime, out.p, w.n * sizeof(Real), cudaMemcpyDeviceToHost, w.s));
  st.d2h += (double)w.n * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(w.s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_compute_dpt_multi_root(scl_sparse_t transition, const scl_index_t* root_cells,
                                                            scl_size_t n_roots, scl_real_t* pseudotime,
                                                            scl_size_t n_nodes, scl_index_t max_iter) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(root_cells, "Root cells array is null");
  SCL_API_CHECK_NULL(pseudotime, "Output pseudotime array is null");
  SCL_API_CHECK(n_roots > 0 && n_nodes > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  Stats st;
  WalkSetup w = walk_setup(*transition, n_nodes, "DPT: output buffer too small", st);
  if (w.n == 0) SCL_API_RETURN_OK;
  std::vector<Index> valid;  // diffusion.hpp:794-800: out-of-range roots are skipped
  for (size_t r = 0; r < n_roots; ++r)
    if (root_cells[r] >= 0 && root_cells[r] < w.n) valid.push_back(root_cells[r]);
  if (valid.empty()) {
    for (Index i = 0; i < w.n; ++i) pseudotime[i] = Real(1);
    SCL_API_RETURN_OK;
  }
  const Index it = (max_iter == 0) ? kDefaultMaxIter : max_iter;
  DevBuf all((size_t)valid.size() * w.n * sizeof(Real), w.s), out(w.n * sizeof(Real), w.s);
  EventTimer tm(w.s);
  tm.start();
  for (size_t r = 0; r < valid.size(); ++r)  // each root with the kernel's default tolerance (diffusion.hpp:805-808)
    dpt(w.mir->g.view(), valid[r], all.as<Real>() + r * (size_t)w.n, it, (double)kDefaultTol, w.s);
  dpt_average(all.p, (int64_t)valid.size(), w.n, sclabi::kRealDType, out.p, w.s);
  tm.stop();
  SCL_CUDA(cudaMemcpyAsync(pseudotime, out.p, w.n * sizeof(Real), cudaMemcpyDeviceToHost, w.s));
  st.d2h += (double)w.n * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(w.s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}
SCL_EXPORT scl_error_t scl_diffusion_random_walk_with_restart(scl_sparse_t transition, const scl_index_t* seed_nodes,
                                                              scl_size_t n_seeds, scl_real_t* scores,
                                                              scl_size_t n_nodes, scl_real_t alpha,
                                                              scl_index_t max_iter, scl_real_t tol) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(seed_nodes, "Seed nodes array is null");
  SCL_API_CHECK_NULL(scores, "Output scores array is null");
  SCL_API_CHECK(n_seeds > 0 && n_nodes > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_CHECK(alpha >= 0 && alpha <= 1, SCL_ERROR_INVALID_ARGUMENT, "Alpha must be in [0, 1]");
  SCL_API_TRY
  walk_restart_host(*transition, seed_nodes, n_seeds, scores, n_nodes, alpha == Real(0) ? kDefaultAlpha : alpha,
                    max_iter == 0 ? kDefaultMaxIter : max_iter, tol == Real(0) ? kDefaultTol : tol);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}
SCL_EXPORT scl_error_t scl_diffusion_personalized_pagerank(scl_sparse_t transition, scl_index_t seed_node,
                                                           scl_real_t* scores, scl_size_t n_nodes, scl_real_t alpha,
                                                           scl_index_t max_iter, scl_real_t tol) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(scores, "Output scores array is null");
  SCL_API_CHECK(n_nodes > 0, SCL_ERROR_INVALID_ARGUMENT, "Number of nodes must be positive");
  SCL_API_CHECK(alpha >= 0 && alpha <= 1, SCL_ERROR_INVALID_ARGUMENT, "Alpha must be in [0, 1]");
  SCL_API_TRY
  const Index seed = seed_node;
  walk_restart_host(*transition, &seed, 1, scores, n_nodes, alpha == Real(0) ? kDefaultAlpha : alpha,
                    max_iter == 0 ? kDefaultMaxIter : max_iter, tol == Real(0) ? kDefaultTol : tol);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}
SCL_EXPORT scl_error_t scl_diffusion_diffusion_map_embedding(scl_sparse_t transition, scl_real_t* embedding,
                                                             scl_index_t n_nodes, scl_index_t n_components,
                                                             scl_index_t n_iter) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(embedding, "Output embedding array is null");
  SCL_API_CHECK(n_nodes > 0 && n_components > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  Stats st;
  WalkSetup w = walk_setup(*transition, (size_t)n_nodes, "DiffusionMap: embedding buffer too small", st);
  SCL_REQUIRE(n_components <= 4096, SCL_ERROR_INVALID_ARGUMENT, "diffusion map: at most 4096 components");
  const int64_t total = (int64_t)w.n * n_components;
  DevBuf out(std::max<int64_t>(total, 1) * sizeof(Real), w.s);
  EventTimer tm(w.s);
  tm.start();
  diffusion_map(w.mir->g.view(), out.p, (int)n_components, n_iter == 0 ? 50 : n_iter, w.s);  // diffusion.cpp:24
  tm.stop();
  if (total > 0) SCL_CUDA(cudaMemcpyAsync(embedding, out.p, total * sizeof(Real), cudaMemcpyDeviceToHost, w.s));
  st.d2h += (double)total * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(w.s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}
SCL_EXPORT scl_error_t scl_diffusion_heat_kernel_signature(scl_sparse_t transition, scl_real_t* signature,
                                                           scl_size_t n_nodes, scl_real_t t, scl_index_t n_steps) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(signature, "Output signature array is null");
  SCL_API_CHECK(n_nodes > 0, SCL_ERROR_INVALID_ARGUMENT, "Number of nodes must be positive");
  SCL_API_CHECK(t > 0, SCL_ERROR_INVALID_ARGUMENT, "Time parameter t must be positive");
  SCL_API_TRY
  const Index steps = (n_steps == 0) ? kDefaultStepsHks : n_steps;
  const Index n = transition->primary_dim();
  SCL_REQUIRE(n_nodes >= (size_t)n, SCL_ERROR_DIMENSION_MISMATCH, "HKS: output buffer too small");
  for (Index i = 0; i < n; ++i) signature[i] = Real(1);  // diffusion.hpp:975 (identity diagonal)
  const Real dt = t / static_cast<Real>(steps);
  walk_linear_host(*transition, signature, n_nodes, steps, Real(1) - dt, dt, "HKS: output buffer too small");
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}
SCL_EXPORT scl_error_t scl_diffusion_diffusion_distance(scl_sparse_t transition, scl_real_t* distances,
                                                        scl_size_t n_nodes, scl_index_t n_steps) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(distances, "Output distances array is null");
  SCL_API_CHECK(n_nodes > 0 && n_steps > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  Stats st;
  WalkSetup w = walk_setup(*transition, n_nodes, "DiffusionDist: output buffer too small", st);
  const int64_t total = (int64_t)w.n * w.n;  // written with row stride n, as the reference
  DevBuf D(std::max<int64_t>(total, 1) * sizeof(Real), w.s);
  EventTimer tm(w.s);
  tm.start();
  diffusion_distance(w.mir->g.view(), D.p, n_steps, w.s);
  tm.stop();
  if (total > 0) SCL_CUDA(cudaMemcpyAsync(distances, D.p, total * sizeof(Real), cudaMemcpyDeviceToHost, w.s));
  st.d2h += (double)total * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(w.s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}
SCL_EXPORT scl_error_t scl_diffusion_lazy_random_walk(scl_sparse_t transition, scl_real_t* x, scl_size_t n_nodes,
                                                      scl_index_t n_steps, scl_real_t laziness) {
  SCL_API_CHECK_NULL(transition, "Transition matrix is null");
  SCL_API_CHECK_NULL(x, "Vector x is null");
  SCL_API_CHECK(n_nodes > 0 && n_steps > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_CHECK(laziness >= 0 && laziness <= 1, SCL_ERROR_INVALID_ARGUMENT, "Laziness must be in [0, 1]");
  SCL_API_TRY
  const Real lazy = (laziness == Real(0)) ? kDefaultLaziness : laziness;
  walk_linear_host(*transition, x, n_nodes, n_steps, lazy, Real(1) - lazy, "LazyRW: vector size mismatch");
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_gpu_set_degree_mode(int mode) {
  SCL_API_CHECK(mode == 0 || mode == 1, SCL_ERROR_INVALID_ARGUMENT, "degree mode must be 0 (FP64) or 1 (native)");
  t_degree_mode = mode;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_diffusion_gpu_set_reorder(int mode) {
  SCL_API_CHECK(mode >= -1 && mode <= 1, SCL_ERROR_INVALID_ARGUMENT,
                "reorder mode must be -1 (automatic), 0 (off) or 1 (on)");
  t_reorder_mode = mode;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_diffusion_gpu_attach(scl_sparse_t handle) {
  SCL_API_CHECK_NULL(handle, "Matrix is null");
  SCL_API_TRY
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  double h2d = 0;
  handle->mirror = upload(*handle, s, h2d);
  SCL_CUDA(cudaStreamSynchronize(s));
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_gpu_detach(scl_sparse_t handle) {
  SCL_API_CHECK_NULL(handle, "Matrix is null");
  SCL_API_TRY
  handle->mirror.reset();
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_diffusion_gpu_last_stats(double* device_ms, double* h2d_bytes, double* d2h_bytes) {
  if (device_ms) *device_ms = t_stats.device_ms;
  if (h2d_bytes) *h2d_bytes = t_stats.h2d;
  if (d2h_bytes) *d2h_bytes = t_stats.d2h;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_impute_diffusion(scl_sparse_t matrix, scl_sparse_t transition_matrix, scl_index_t n_cells,
                                            scl_index_t n_genes, scl_index_t n_steps, scl_real_t* X_imputed) {
  SCL_API_CHECK_NULL(matrix, "Matrix is null");
  SCL_API_CHECK_NULL(transition_matrix, "Transition matrix is null");
  SCL_API_CHECK_NULL(X_imputed, "Output imputed matrix is null");
  SCL_API_CHECK(n_cells > 0 && n_genes > 0 && n_steps > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  impute_host(*matrix, *transition_matrix, n_cells, n_genes, n_steps, X_imputed, false);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_impute_magic(scl_sparse_t matrix, scl_sparse_t affinity_matrix, scl_index_t n_cells,
                                        scl_index_t n_genes, scl_index_t t, scl_real_t* X_imputed) {
  SCL_API_CHECK_NULL(matrix, "Matrix is null");
  SCL_API_CHECK_NULL(affinity_matrix, "Affinity matrix is null");
  SCL_API_CHECK_NULL(X_imputed, "Output imputed matrix is null");
  SCL_API_CHECK(n_cells > 0 && n_genes > 0 && t > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  impute_host(*matrix, *affinity_matrix, n_cells, n_genes, t, X_imputed, true);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_algebra_spmm(scl_sparse_t A, const scl_real_t* X, scl_index_t n_cols, scl_real_t* Y,
                                        scl_real_t alpha, scl_real_t beta) {
  SCL_API_CHECK_NULL(A, "Matrix A is null");
  SCL_API_CHECK_NULL(X, "Input matrix X is null");
  SCL_API_CHECK_NULL(Y, "Output matrix Y is null");
  SCL_API_CHECK(n_cols > 0, SCL_ERROR_INVALID_ARGUMENT, "Number of columns must be positive");
  SCL_API_TRY
  SCL_REQUIRE(A->valid, SCL_ERROR_INVALID_ARGUMENT, "Matrix A is not valid");
  const int dev = current_device();
  cudaStream_t s = library_stream(dev);
  Stats st;
  auto mir = device_graph(*A, s, st.h2d);
  const int64_t m = A->primary_dim(), kx = A->secondary_dim(), K = n_cols;
  DevBuf Xd(std::max<int64_t>(kx * K, 1) * sizeof(Real), s), Yd(std::max<int64_t>(m * K, 1) * sizeof(Real), s);
  if (kx > 0) SCL_CUDA(cudaMemcpyAsync(Xd.p, X, kx * K * sizeof(Real), cudaMemcpyHostToDevice, s));
  st.h2d += (double)kx * K * sizeof(Real);
  if (beta != Real(0) && m > 0) {
    SCL_CUDA(cudaMemcpyAsync(Yd.p, Y, m * K * sizeof(Real), cudaMemcpyHostToDevice, s));
    st.h2d += (double)m * K * sizeof(Real);
  }
  EventTimer tm(s);
  tm.start();
  algebra_spmm(mir->g.view(), Xd.p, K, Yd.p, (double)alpha, (double)beta, s);
  tm.stop();
  if (m > 0) SCL_CUDA(cudaMemcpyAsync(Y, Yd.p, m * K * sizeof(Real), cudaMemcpyDeviceToHost, s));
  st.d2h += (double)m * K * sizeof(Real);
  SCL_CUDA(cudaStreamSynchronize(s));
  st.device_ms = tm.ms();
  t_stats = st;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_neighbors_compute_norms(scl_sparse_t matrix, scl_real_t* norms_sq) {
  SCL_API_CHECK_NULL(matrix, "Matrix handle is null");
  SCL_API_CHECK_NULL(norms_sq, "Norms output pointer is null");
  SCL_API_TRY
  Stats st;
  DenseSamples ds = dense_samples(*matrix, st);
  DevBuf nd(std::max<int64_t>(ds.n, 1) * sizeof(Real), ds.s);
  row_norms_dense(ds.X.p, sclabi::kRealDType, ds.n, ds.d, nd.p, ds.s);
  if (ds.n > 0) SCL_CUDA(cudaMemcpyAsync(norms_sq, nd.p, ds.n * sizeof(Real), cudaMemcpyDeviceToHost, ds.s));
  SCL_CUDA(cudaStreamSynchronize(ds.s));
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_knn(scl_sparse_t matrix, const scl_real_t* norms_sq, scl_size_t n_samples, scl_size_t k,
                               scl_index_t* out_indices, scl_real_t* out_distances) {
  SCL_API_CHECK_NULL(matrix, "Matrix handle is null");
  SCL_API_CHECK_NULL(norms_sq, "Norms input pointer is null");
  SCL_API_CHECK_NULL(out_indices, "Indices output pointer is null");
  SCL_API_CHECK_NULL(out_distances, "Distances output pointer is null");
  SCL_API_CHECK(n_samples > 0 && k > 0, SCL_ERROR_INVALID_ARGUMENT, "Dimensions must be positive");
  SCL_API_TRY
  knn_host(*matrix, norms_sq, n_samples, k, out_indices, out_distances);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_knn_simple(scl_sparse_t matrix, scl_size_t n_samples, scl_size_t k,
                                      scl_index_t* out_indices, scl_real_t* out_distances) {
  SCL_API_CHECK_NULL(matrix, "Matrix handle is null");
  SCL_API_CHECK_NULL(out_indices, "Indices output pointer is null");
  SCL_API_CHECK_NULL(out_distances, "Distances output pointer is null");
  SCL_API_TRY
  knn_host(*matrix, nullptr, n_samples, k, out_indices, out_distances);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_impute_knn(scl_sparse_t matrix, const scl_index_t* knn_indices,
                                      const scl_real_t* knn_distances, scl_index_t n_cells, scl_index_t n_genes,
                                      scl_index_t k_neighbors, scl_real_t* X_imputed, scl_real_t bandwidth,
                                      scl_real_t threshold) {
  SCL_API_CHECK_NULL(matrix, "Matrix is null");
  SCL_API_CHECK_NULL(knn_indices, "KNN indices array is null");
  SCL_API_CHECK_NULL(knn_distances, "KNN distances array is null");
  SCL_API_CHECK_NULL(X_imputed, "Output imputed matrix is null");
  SCL_API_CHECK(n_cells > 0 && n_genes > 0 && k_neighbors > 0, SCL_ERROR_INVALID_ARGUMENT,
                "Dimensions must be positive");
  SCL_API_TRY
  knn_impute_host(*matrix, knn_indices, knn_distances, n_cells, n_genes, k_neighbors, X_imputed, bandwidth, threshold);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

// impute.cpp:54-87: the reference's weighted entry point runs the same kernel
// (knn_impute_dense, Gaussian weights of the given distances).
SCL_EXPORT scl_error_t scl_impute_knn_weighted(scl_sparse_t matrix, const scl_index_t* knn_indices,
                                               const scl_real_t* knn_distances, scl_index_t n_cells,
                                               scl_index_t n_genes, scl_index_t k_neighbors, scl_real_t* X_imputed,
                                               scl_real_t bandwidth, scl_real_t threshold) {
  SCL_API_CHECK_NULL(matrix, "Matrix is null");
  SCL_API_CHECK_NULL(knn_indices, "KNN indices array is null");
  SCL_API_CHECK_NULL(knn_distances, "KNN distances array is null");
  SCL_API_CHECK_NULL(X_imputed, "Output imputed matrix is null");
  SCL_API_CHECK(n_cells > 0 && n_genes > 0 && k_neighbors > 0, SCL_ERROR_INVALID_ARGUMENT,
                "Dimensions must be positive");
  SCL_API_TRY
  knn_impute_host(*matrix, knn_indices, knn_distances, n_cells, n_genes, k_neighbors, X_imputed, bandwidth, threshold);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

}  // extern "C"
