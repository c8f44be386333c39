// Diffusion and MAGIC imputation on the device (scl/kernel/impute.hpp:599-735).
//
// Both start from a dense cells x genes block built from a sparse expression
// matrix and then run t SpMM steps over the cells graph; the steps are this
// library's SpMM kernels (each output element the sequential fma chain over its
// row's entries, as scl-core's axpy_simd forms it with MulAdd). MAGIC first
// normalises the affinity rows the way impute.hpp:700-735 does: a sequential
// row sum in the storage precision, w = a * (1 / sum) per entry, and rows whose
// sum is below 1e-12 copy their input row instead of averaging.
#include <algorithm>

#include "engine.hpp"

namespace sclgpu {
namespace {

// Zero-initialised X_imputed, then every stored (cell, gene) with cell <
// n_cells and gene < n_genes written in stored order; a later duplicate of the
// same position overwrites an earlier one (impute.hpp:608-640, 680-697). A warp
// walks one primary row (a cell for CSR, a gene for CSC) in chunks of 32; in a
// chunk only the last lane holding a position writes it, and chunks are
// ordered by __syncwarp.
template <class T>
__global__ void k_densify(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val,
                          int64_t n_primary, int64_t n_cells, int64_t n_genes, int csr, T* __restrict__ dense) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_primary; p += nw) {
    const int64_t s0 = ptr[p], s1 = ptr[p + 1];
    for (int64_t base = s0; base < s1; base += 32) {
      const int64_t k = base + lane;
      int32_t sec = -1;
      T v = T(0);
      if (k < s1) {
        sec = idx[k];
        v = val[k];
      }
      const bool ok = sec >= 0 && (csr ? (int64_t)sec < n_genes : (int64_t)sec < n_cells);
      const unsigned grp = __match_any_sync(0xffffffffu, ok ? sec : -2 - lane);
      if (ok && lane == 31 - __clz(grp)) {
        const int64_t c = csr ? p : (int64_t)sec;
        const int64_t g = csr ? (int64_t)sec : p;
        dense[c * n_genes + g] = v;
      }
      __syncwarp();
    }
  }
}

// The lookup side of kNN imputation: the FIRST stored value of every
// (cell, gene) inside the block (the reference's has_expression finds the
// first match) and a mask of the stored positions (a stored zero counts).
template <class T>
__global__ void k_densify_first(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                const T* __restrict__ val, int64_t n_primary, int64_t n_cells, int64_t n_genes,
                                int csr, T* __restrict__ dense, unsigned char* __restrict__ mask) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_primary; p += nw) {
    const int64_t s0 = ptr[p], s1 = ptr[p + 1];
    for (int64_t base = s0; base < s1; base += 32) {
      const int64_t k = base + lane;
      int32_t sec = -1;
      T v = T(0);
      if (k < s1) {
        sec = idx[k];
        v = val[k];
      }
      const bool ok = sec >= 0 && (csr ? (int64_t)sec < n_genes : (int64_t)sec < n_cells);
      const unsigned grp = __match_any_sync(0xffffffffu, ok ? sec : -2 - lane);
      if (ok && lane == __ffs(grp) - 1) {
        const int64_t c = csr ? p : (int64_t)sec;
        const int64_t g = csr ? (int64_t)sec : p;
        if (!mask[c * n_genes + g]) {
          dense[c * n_genes + g] = v;
          mask[c * n_genes + g] = 1;
        }
      }
      __syncwarp();
    }
  }
}

// w = exp(-(d / (bandwidth + 1e-12))^2) per neighbour (impute.hpp:156-159).
template <class T>
__global__ void k_knn_weights(const T* __restrict__ dist, int64_t m, T bw, T* __restrict__ w) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
    const T scaled = dist[e] / (bw + (T)1e-12);
    w[e] = exp(-scaled * scaled);
  }
}

// impute.hpp:468-508 for one (cell, gene): values above the threshold stay;
// otherwise the weighted mean of the neighbours that store the gene
// (sum w v as an fma chain, sum w, neighbours in list order) replaces the
// value when the weight sum exceeds 1e-12 and the mean exceeds 1e-10.
template <class T, class IT>
__global__ void k_knn_impute(T* __restrict__ D, const T* __restrict__ L, const unsigned char* __restrict__ M,
                             const IT* __restrict__ nbr, const T* __restrict__ w, int64_t n, int64_t G, int K,
                             T threshold) {
  const int64_t total = n * G;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / G, g = e - c * G;
    const T x = D[e];
    if (x > threshold) continue;
    T sv = T(0), sw = T(0);
    int found = 0;
    for (int k = 0; k < K; ++k) {
      const int64_t j = (int64_t)nbr[c * K + k];
      if (j < 0 || j >= n || !M[j * G + g]) continue;
      const T wk = w[c * K + k];
      sv = fma(wk, L[j * G + g], sv);
      sw = sw + wk;
      ++found;
    }
    if (found == 0 || !(sw > (T)1e-12)) continue;
    const T imp = sv / sw;
    if (imp > (T)1e-10) D[e] = imp;
  }
}

// One thread per affinity row: sum its values in stored order (storage
// precision), then w = a * (1 / sum) for every entry; rows with sum < eps are
// marked to copy their input row and listed in copy_rows.
template <class T>
__global__ void k_magic_weights(const int64_t* __restrict__ ptr, const T* __restrict__ val, int64_t n, T eps,
                                T* __restrict__ w, int32_t* __restrict__ copy_rows, unsigned long long* n_copy) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s0 = ptr[i], s1 = ptr[i + 1];
    T sum = T(0);
    for (int64_t k = s0; k < s1; ++k) sum += val[k];
    if (sum < eps) {
      copy_rows[atomicAdd(n_copy, 1ull)] = (int32_t)i;
      for (int64_t k = s0; k < s1; ++k) w[k] = T(0);
    } else {
      const T inv = T(1) / sum;
      for (int64_t k = s0; k < s1; ++k) w[k] = val[k] * inv;
    }
  }
}

template <class T>
__global__ void k_copy_rows(const int32_t* __restrict__ rows, int64_t n_copy, const T* __restrict__ in,
                            T* __restrict__ out, int64_t F) {
  const int64_t total = n_copy * F;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = rows[e / F];
    out[r * F + e % F] = in[r * F + e % F];
  }
}

unsigned grid_for(int64_t threads) {
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const int64_t want = (threads + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count(dev) * 16));
}

}  // namespace

void densify_expression(const CsrView& m, bool csr, int64_t n_cells, int64_t n_genes, void* dense, cudaStream_t s) {
  SCL_REQUIRE(m.vtype == kF32 || m.vtype == kF64, kErrTypeMismatch, "expression values must be f32 or f64");
  const size_t esz = dtype_size(m.vtype);
  SCL_CUDA(cudaMemsetAsync(dense, 0, (size_t)n_cells * (size_t)n_genes * esz, s));
  const int64_t n_primary = std::min<int64_t>(m.n_rows, csr ? n_cells : n_genes);
  if (n_primary <= 0 || m.nnz == 0) return;
  const unsigned grid = grid_for(n_primary * 32);
  if (m.vtype == kF32)
    k_densify<float><<<grid, 256, 0, s>>>(m.indptr, m.indices, static_cast<const float*>(m.values), n_primary,
                                          n_cells, n_genes, csr ? 1 : 0, static_cast<float*>(dense));
  else
    k_densify<double><<<grid, 256, 0, s>>>(m.indptr, m.indices, static_cast<const double*>(m.values), n_primary,
                                           n_cells, n_genes, csr ? 1 : 0, static_cast<double*>(dense));
  SCL_CUDA(cudaGetLastError());
}

void knn_impute(const CsrView& m, bool csr, int64_t n_cells, int64_t n_genes, const void* nbr, DType it,
                const void* dist, int K, double bandwidth, double threshold, void* out, cudaStream_t s) {
  SCL_REQUIRE(m.vtype == kF32 || m.vtype == kF64, kErrTypeMismatch, "expression values must be f32 or f64");
  densify_expression(m, csr, n_cells, n_genes, out, s);  // the block, later duplicates winning
  const size_t esz = dtype_size(m.vtype);
  const int64_t total = n_cells * n_genes;
  DevBuf L(std::max<int64_t>(total, 1) * esz, s), M(std::max<int64_t>(total, 1), s), W(std::max<int64_t>(n_cells * K, 1) * esz, s);
  SCL_CUDA(cudaMemsetAsync(M.p, 0, total, s));
  const int64_t n_primary = std::min<int64_t>(m.n_rows, csr ? n_cells : n_genes);
  if (n_primary > 0 && m.nnz > 0) {
    const unsigned gp = grid_for(n_primary * 32);
    if (m.vtype == kF32)
      k_densify_first<float><<<gp, 256, 0, s>>>(m.indptr, m.indices, static_cast<const float*>(m.values), n_primary,
                                                n_cells, n_genes, csr ? 1 : 0, L.as<float>(), M.as<unsigned char>());
    else
      k_densify_first<double><<<gp, 256, 0, s>>>(m.indptr, m.indices, static_cast<const double*>(m.values), n_primary,
                                                 n_cells, n_genes, csr ? 1 : 0, L.as<double>(), M.as<unsigned char>());
    SCL_CUDA(cudaGetLastError());
  }
  const unsigned gw = grid_for(n_cells * K), ge = grid_for(total);
#define SCL_KNN_IMPUTE(T)                                                                                  \
  k_knn_weights<T><<<gw, 256, 0, s>>>(static_cast<const T*>(dist), n_cells * K, (T)bandwidth, W.as<T>());  \
  if (it == kI32)                                                                                          \
    k_knn_impute<T, int32_t><<<ge, 256, 0, s>>>(static_cast<T*>(out), L.as<T>(), M.as<unsigned char>(),      \
                                                static_cast<const int32_t*>(nbr), W.as<T>(), n_cells,        \
                                                n_genes, K, (T)threshold);                                    \
  else                                                                                                     \
    k_knn_impute<T, int64_t><<<ge, 256, 0, s>>>(static_cast<T*>(out), L.as<T>(), M.as<unsigned char>(),      \
                                                static_cast<const int64_t*>(nbr), W.as<T>(), n_cells,        \
                                                n_genes, K, (T)threshold);
  if (m.vtype == kF32) {
    SCL_KNN_IMPUTE(float)
  } else {
    SCL_KNN_IMPUTE(double)
  }
#undef SCL_KNN_IMPUTE
  SCL_CUDA(cudaGetLastError());
}

void magic_diffuse(const CsrView& aff, void* X, int64_t F, int64_t steps, cudaStream_t s) {
  SCL_REQUIRE(aff.vtype == kF32 || aff.vtype == kF64, kErrTypeMismatch, "affinity values must be f32 or f64");
  SCL_REQUIRE(aff.n_cols <= aff.n_rows, kErrDimensionMismatch, "affinity columns must address rows of X");
  const int64_t n = aff.n_rows;
  if (steps <= 0 || n == 0 || F == 0) return;
  const size_t esz = dtype_size(aff.vtype);
  DevBuf w(std::max<int64_t>(aff.nnz, 1) * esz, s);
  DevBuf rows(std::max<int64_t>(n, 1) * sizeof(int32_t), s);
  DevBuf cnt(sizeof(unsigned long long), s);
  SCL_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), s));
  const unsigned g = grid_for(n);
  if (aff.vtype == kF32)
    k_magic_weights<float><<<g, 256, 0, s>>>(aff.indptr, static_cast<const float*>(aff.values), n, 1e-12f,
                                             w.as<float>(), rows.as<int32_t>(), cnt.as<unsigned long long>());
  else
    k_magic_weights<double><<<g, 256, 0, s>>>(aff.indptr, static_cast<const double*>(aff.values), n, 1e-12,
                                              w.as<double>(), rows.as<int32_t>(), cnt.as<unsigned long long>());
  SCL_CUDA(cudaGetLastError());
  unsigned long long n_copy = 0;
  SCL_CUDA(cudaMemcpyAsync(&n_copy, cnt.p, sizeof(n_copy), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  DevBuf tmp(std::max<int64_t>(n * F, 1) * esz, s);
  SpmmArgs a{};
  a.indptr = aff.indptr;
  a.indices = aff.indices;
  a.values = w.p;
  a.vtype = aff.vtype;
  a.n_rows = n;
  a.F = F;
  a.xtype = aff.vtype;
  a.ytype = aff.vtype;
  void* in = X;
  void* out = tmp.p;
  for (int64_t st = 0; st < steps; ++st) {
    a.X = in;
    a.Y = out;
    spmm(a, s);
    if (n_copy > 0) {
      const unsigned gc = grid_for((int64_t)n_copy * F);
      if (aff.vtype == kF32)
        k_copy_rows<float><<<gc, 256, 0, s>>>(rows.as<int32_t>(), (int64_t)n_copy, static_cast<const float*>(in),
                                              static_cast<float*>(out), F);
      else
        k_copy_rows<double><<<gc, 256, 0, s>>>(rows.as<int32_t>(), (int64_t)n_copy, static_cast<const double*>(in),
                                               static_cast<double*>(out), F);
      SCL_CUDA(cudaGetLastError());
    }
    std::swap(in, out);
  }
  if (in != X) SCL_CUDA(cudaMemcpyAsync(X, in, (size_t)n * (size_t)F * esz, cudaMemcpyDeviceToDevice, s));
}

}  // namespace sclgpu

// ---- general SpMM, Y = alpha A X + beta Y (scl/kernel/algebra.hpp:546-600) -------
namespace sclgpu {
namespace {

// A warp per row of A, lane l owning columns l, l+32, ...: y starts as beta y
// (beta 0: zero, beta 1: y) and every stored entry with w = a * alpha != 0
// adds fma(w, x_row, y) in stored order, as scl_algebra_spmm's axpy does.
template <class T>
__global__ void __launch_bounds__(256)
k_algebra_spmm(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val, int64_t m,
               const T* __restrict__ X, int64_t K, T* __restrict__ Y, T alpha, T beta) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += nw) {
    const int64_t s0 = ptr[i], s1 = ptr[i + 1];
    for (int64_t c = lane; c < K; c += 32) {
      T y = (beta == T(0)) ? T(0) : (beta == T(1) ? Y[i * K + c] : Y[i * K + c] * beta);
      if (alpha != T(0)) {
        for (int64_t k = s0; k < s1; ++k) {
          const T w = val[k] * alpha;
          if (w != T(0)) y = fma(w, X[(int64_t)idx[k] * K + c], y);
        }
      }
      Y[i * K + c] = y;
    }
  }
}

}  // namespace

void algebra_spmm(const CsrView& A, const void* X, int64_t K, void* Y, double alpha, double beta, cudaStream_t s) {
  const int64_t m = A.n_rows;
  if (m == 0 || K == 0) return;
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((m + 7) / 8, (int64_t)sm_count(dev) * 8));
  if (A.vtype == kF32)
    k_algebra_spmm<float><<<grid, 256, 0, s>>>(A.indptr, A.indices, static_cast<const float*>(A.values), m,
                                               static_cast<const float*>(X), K, static_cast<float*>(Y), (float)alpha,
                                               (float)beta);
  else
    k_algebra_spmm<double><<<grid, 256, 0, s>>>(A.indptr, A.indices, static_cast<const double*>(A.values), m,
                                                static_cast<const double*>(X), K, static_cast<double*>(Y), alpha,
                                                beta);
  SCL_CUDA(cudaGetLastError());
}

}  // namespace sclgpu
