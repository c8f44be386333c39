// Transition-matrix build on the device:
//   * FP64 row degrees + row / symmetric normalisation
//       (replaces scl/kernel/diffusion.hpp:452-484 compute_row_sums_parallel and
//        diffusion.hpp:492-603 compute_transition_matrix)
//   * Gaussian kNN weights with adaptive sigma
//       (scl/kernel/kernel.hpp:403-453 local_bandwidth: sigma_i = max of the row's
//        kNN distances floored at 1e-10; weight exp(-(d/sigma_i)^2) as in
//        scl/kernel/impute.hpp:156-159 without its +1e-12)
//   * (W + W^T)/2 union symmetrisation of the kNN graph — the reference only
//       has a dense n x n version (scl/kernel/transition.hpp:529-563); here it is
//       a radix sort of the 2nk COO keys followed by a run reduction.
//   * structural transpose with a value map (CSC view for the backward pass).
#include <cuda_runtime.h>

#include <algorithm>

#include "engine.hpp"

namespace sclgpu {
namespace {

constexpr double kMinProb = 1e-15;       // diffusion.hpp:41 config::MIN_PROB
constexpr float kMinBandwidth = 1e-10f;  // kernel.hpp:28 config::MIN_BANDWIDTH
constexpr float kDefaultBandwidth = 1.0f;  // kernel.hpp:27 config::DEFAULT_BANDWIDTH

inline unsigned blocks_for(int64_t items, int per_block) {
  int64_t b = (items + per_block - 1) / per_block;
  return (unsigned)std::max<int64_t>(1, b);
}

// ---- degrees ------------------------------------------------------------------
// One thread per row, sequential sum in the row's stored order — the same
// summation order as the reference, so an f64 graph reproduces its degrees
// bit for bit.
template <class T>
__global__ void k_degrees_fp64(const int64_t* __restrict__ indptr, const T* __restrict__ v, int64_t n,
                               double* __restrict__ d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int64_t p = indptr[i], e = indptr[i + 1]; p < e; ++p) s += (double)v[p];
  d[i] = s;
}

template <class T>
__global__ void k_degrees_native(const int64_t* __restrict__ indptr, const T* __restrict__ v, int64_t n,
                                 T* __restrict__ d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  T s = T(0);
  for (int64_t p = indptr[i], e = indptr[i + 1]; p < e; ++p) s = s + v[p];
  d[i] = s;
}

// scale factors: row -> 1/d, symmetric -> 1/sqrt(d); 0 where d <= 1e-15
template <class S>
__global__ void k_scale_factors(const S* __restrict__ d, int64_t n, int symmetric, S* __restrict__ f) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const S di = d[i];
  S r = S(0);
  if (di > (S)kMinProb) r = symmetric ? S(1) / sqrt(di) : S(1) / di;
  f[i] = r;
}

// Warp per row; lanes stride the row's entries (coalesced). The product
// (scale_i * scale_j) is formed first, as the reference does (diffusion.hpp:545).
template <class T, class S>
__global__ void k_apply_scale(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                              T* __restrict__ v, const S* __restrict__ f, int64_t n, int symmetric) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const S fi = f[row];
  for (int64_t p = indptr[row] + lane, e = indptr[row + 1]; p < e; p += 32) {
    const S sc = symmetric ? fi * f[idx[p]] : fi;
    v[p] = (T)((S)v[p] * sc);
  }
}

// ---- Gaussian weights ---------------------------------------------------------
__global__ void k_gauss(const int32_t* __restrict__ knn_idx, const float* __restrict__ knn_dist, int64_t n,
                        int64_t k, float* __restrict__ sigma, float* __restrict__ w) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const int32_t* ir = knn_idx + row * k;
  const float* dr = knn_dist + row * k;
  float mx = 0.0f;
  int any = 0;
  for (int64_t m = lane; m < k; m += 32) {
    if (ir[m] >= 0) {
      any = 1;
      mx = fmaxf(mx, dr[m]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    any |= __shfl_xor_sync(0xffffffffu, any, o);
  }
  const float s = any ? fmaxf(mx, kMinBandwidth) : kDefaultBandwidth;
  if (lane == 0) sigma[row] = s;
  for (int64_t m = lane; m < k; m += 32) {
    float out = 0.0f;
    if (ir[m] >= 0) {
      const float q = dr[m] / s;
      out = expf(-(q * q));
    }
    w[row * k + m] = out;
  }
}

// ---- symmetrisation -----------------------------------------------------------
// COO layout: entries [0, nk) are W[i, j] ("out", payload p), entries [nk, 2nk)
// are W^T[j, i] ("in", payload p | 0x80000000). Key = (row << cbits) | col.
// Invalid neighbours (index < 0) get an all-ones key so they sort last.
__global__ void k_build_coo(const int32_t* __restrict__ knn_idx, int64_t n, int64_t k, int cbits,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ pay, int32_t* __restrict__ status,
                            unsigned long long* __restrict__ n_invalid) {
  const int64_t nk = n * k;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nk; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p / k;
    const int32_t j = knn_idx[p];
    uint64_t ko = ~0ull, ki = ~0ull;
    if (j < 0) atomicAdd(n_invalid, 2ull);
    if (j >= 0) {
      if ((int64_t)j >= n) {
        if (atomicCAS(status, 0, (int32_t)kErrIndexOutOfBounds) == 0) status[1] = (int32_t)p;
      } else {
        ko = ((uint64_t)i << cbits) | (uint64_t)j;
        ki = ((uint64_t)j << cbits) | (uint64_t)i;
      }
    }
    keys[p] = ko;
    pay[p] = (uint32_t)p;
    keys[nk + p] = ki;
    pay[nk + p] = (uint32_t)p | 0x80000000u;
  }
}

// head[q] = 1 when sorted key q starts a run (and is valid)
__global__ void k_run_heads(const uint64_t* __restrict__ keys, int64_t m, int64_t* __restrict__ head) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t kq = keys[q];
    head[q] = (kq != ~0ull && (q == 0 || keys[q - 1] != kq)) ? 1 : 0;
  }
}

// One thread per run head: value = 0.5 * (sum of out weights + sum of in
// weights), each partial sum in sorted (= original) order.
__global__ void k_reduce_runs(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ pay,
                              const int64_t* __restrict__ head_pos, const float* __restrict__ w, int64_t m,
                              int cbits, int64_t n, int32_t* __restrict__ out_idx, float* __restrict__ out_val,
                              int64_t* __restrict__ indptr) {
  const uint64_t cmask = (cbits >= 64) ? ~0ull : ((1ull << cbits) - 1ull);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t kq = keys[q];
    if (kq == ~0ull) continue;
    if (q > 0 && keys[q - 1] == kq) continue;
    const int64_t u = head_pos[q];
    float so = 0.0f, si = 0.0f;
    for (int64_t r = q; r < m && keys[r] == kq; ++r) {
      const uint32_t pl = pay[r];
      const float wv = w[pl & 0x7fffffffu];
      if (pl & 0x80000000u) si += wv; else so += wv;
    }
    out_idx[u] = (int32_t)(kq & cmask);
    out_val[u] = 0.5f * (so + si);
    // row offsets: this head owns rows (prev_row, row]
    const int64_t row = (int64_t)(kq >> cbits);
    int64_t prev_row = -1;
    if (u > 0) {
      // find the previous valid head's row: the key just before q is valid
      prev_row = (int64_t)(keys[q - 1] >> cbits);
    }
    for (int64_t r = prev_row + 1; r <= row; ++r) indptr[r] = u;
    (void)n;
  }
}

__global__ void k_indptr_tail(const uint64_t* __restrict__ keys, int64_t m_valid, int cbits, int64_t n,
                              int64_t nnz, int64_t* __restrict__ indptr) {
  int64_t last_row = -1;
  if (m_valid > 0) last_row = (int64_t)(keys[m_valid - 1] >> cbits);
  for (int64_t r = last_row + 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= n;
       r += (int64_t)gridDim.x * blockDim.x)
    indptr[r] = nnz;
}

// ---- transpose ------------------------------------------------------------------
__global__ void k_transpose_keys(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx, int64_t n,
                                 int rbits, uint64_t* __restrict__ keys, uint32_t* __restrict__ pay) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  for (int64_t p = indptr[row] + lane, e = indptr[row + 1]; p < e; p += 32) {
    keys[p] = ((uint64_t)(uint32_t)idx[p] << rbits) | (uint64_t)row;
    pay[p] = (uint32_t)p;
  }
}

__global__ void k_transpose_fill(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ pay, int64_t nnz,
                                 int rbits, int64_t n_cols, int32_t* __restrict__ t_idx, int32_t* __restrict__ tmap,
                                 int64_t* __restrict__ t_indptr) {
  const uint64_t rmask = (1ull << rbits) - 1ull;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t kq = keys[q];
    t_idx[q] = (int32_t)(kq & rmask);
    tmap[q] = (int32_t)pay[q];
    const int64_t col = (int64_t)(kq >> rbits);
    const int64_t prev = (q == 0) ? -1 : (int64_t)(keys[q - 1] >> rbits);
    for (int64_t c = prev + 1; c <= col; ++c) t_indptr[c] = q;
    if (q == nnz - 1)
      for (int64_t c = col + 1; c <= n_cols; ++c) t_indptr[c] = nnz;
  }
}

int bits_for(int64_t n) {
  int b = 1;
  while ((1ll << b) < n) ++b;
  return b;
}

}  // namespace

// ============================================================================
void row_degrees_fp64(const DeviceCSR& g, double* degrees, cudaStream_t s) {
  if (g.n_rows == 0) return;
  const unsigned b = blocks_for(g.n_rows, 256);
  if (g.vtype == kF32)
    k_degrees_fp64<float><<<b, 256, 0, s>>>(g.indptr.as<int64_t>(), g.values.as<float>(), g.n_rows, degrees);
  else if (g.vtype == kF64)
    k_degrees_fp64<double><<<b, 256, 0, s>>>(g.indptr.as<int64_t>(), g.values.as<double>(), g.n_rows, degrees);
  else
    throw Error(kErrTypeMismatch, "degrees need f32 or f64 weights");
  SCL_CUDA(cudaGetLastError());
}

void normalize(DeviceCSR& g, int symmetric, int degree_mode, double* degrees_out, cudaStream_t s) {
  const int64_t n = g.n_rows;
  if (n == 0) return;
  SCL_REQUIRE(g.vtype == kF32 || g.vtype == kF64, kErrTypeMismatch, "normalisation needs f32 or f64 weights");
  if (symmetric) SCL_REQUIRE(g.n_rows == g.n_cols, kErrDimensionMismatch, "symmetric normalisation needs a square matrix");
  const unsigned bt = blocks_for(n, 256);
  const unsigned bw = blocks_for(n * 32, 256);
  const int64_t* ip = g.indptr.as<int64_t>();
  const int32_t* ix = g.indices.as<int32_t>();
  if (degree_mode == 0 || g.vtype == kF64) {
    // FP64 degrees and scale factors; for an f64 graph this is exactly the
    // reference's own arithmetic.
    DevBuf d(n * sizeof(double), s), f(n * sizeof(double), s);
    row_degrees_fp64(g, d.as<double>(), s);
    k_scale_factors<double><<<bt, 256, 0, s>>>(d.as<double>(), n, symmetric, f.as<double>());
    if (g.vtype == kF32)
      k_apply_scale<float, double><<<bw, 256, 0, s>>>(ip, ix, g.values.as<float>(), f.as<double>(), n, symmetric);
    else
      k_apply_scale<double, double><<<bw, 256, 0, s>>>(ip, ix, g.values.as<double>(), f.as<double>(), n, symmetric);
    SCL_CUDA(cudaGetLastError());
    if (degrees_out) SCL_CUDA(cudaMemcpyAsync(degrees_out, d.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return;
  }
  // native f32: float sums, 1.0f/d or 1.0f/sqrtf(d), v *= scale — the f32
  // reference build's arithmetic (IEEE division and square root).
  if (degrees_out) row_degrees_fp64(g, degrees_out, s);  // FP64 degrees of the weights, before scaling
  DevBuf d(n * sizeof(float), s), f(n * sizeof(float), s);
  k_degrees_native<float><<<bt, 256, 0, s>>>(ip, g.values.as<float>(), n, d.as<float>());
  k_scale_factors<float><<<bt, 256, 0, s>>>(d.as<float>(), n, symmetric, f.as<float>());
  k_apply_scale<float, float><<<bw, 256, 0, s>>>(ip, ix, g.values.as<float>(), f.as<float>(), n, symmetric);
  SCL_CUDA(cudaGetLastError());
}

void gauss_weights(const int32_t* knn_idx, const float* knn_dist, int64_t n, int64_t k, float* sigma, float* w,
                   cudaStream_t s) {
  if (n == 0 || k == 0) return;
  k_gauss<<<blocks_for(n * 32, 256), 256, 0, s>>>(knn_idx, knn_dist, n, k, sigma, w);
  SCL_CUDA(cudaGetLastError());
}

void symmetrize_knn(const int32_t* knn_idx, const float* w, int64_t n, int64_t k, DeviceCSR& out, cudaStream_t s) {
  SCL_REQUIRE(n > 0 && k > 0, kErrInvalidArgument, "kNN graph needs n > 0 and k > 0");
  SCL_REQUIRE(n * k < (1ll << 31), kErrInvalidArgument, "n * k must be below 2^31");
  const int64_t nk = n * k, m = 2 * nk;
  const int cbits = bits_for(n);
  const int key_bits = 2 * cbits;
  SCL_REQUIRE(key_bits <= 62, kErrInvalidArgument, "graph too large for 64-bit sort keys");
  DevBuf keys(m * 8, s), pay(m * 4, s), keys2(m * 8, s), pay2(m * 4, s);
  DevStatus st(s);
  DevBuf inval(8, s);
  SCL_CUDA(cudaMemsetAsync(inval.p, 0, 8, s));
  const unsigned gb = blocks_for(nk, 256) > 148u * 16u ? 148u * 16u : blocks_for(nk, 256);
  k_build_coo<<<gb, 256, 0, s>>>(knn_idx, n, k, cbits, keys.as<uint64_t>(), pay.as<uint32_t>(), st.ptr(),
                                 inval.as<unsigned long long>());
  SCL_CUDA(cudaGetLastError());
  st.check(s, "kNN index out of range");
  unsigned long long invalid = 0;
  SCL_CUDA(cudaMemcpyAsync(&invalid, inval.p, 8, cudaMemcpyDeviceToHost, s));
  // Invalid entries have all-ones keys; sorting on key_bits would wrap them,
  // so sort on one extra bit (the all-ones key has it set, valid keys do not).
  radix_sort_pairs(keys.as<uint64_t>(), pay.as<uint32_t>(), keys2.as<uint64_t>(), pay2.as<uint32_t>(), m,
                   key_bits + 1, s);
  const uint64_t* sk = keys2.as<uint64_t>();
  const uint32_t* sp = pay2.as<uint32_t>();
  DevBuf head((m + 1) * 8, s);
  const unsigned gm = blocks_for(m, 256) > 148u * 16u ? 148u * 16u : blocks_for(m, 256);
  k_run_heads<<<gm, 256, 0, s>>>(sk, m, head.as<int64_t>());
  exclusive_scan_i64(head.as<int64_t>(), head.as<int64_t>(), m, s);
  int64_t nnz = 0;
  SCL_CUDA(cudaMemcpyAsync(&nnz, head.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  // valid entries form a prefix of the sorted array (invalid keys sort last)
  const int64_t m_valid = m - (int64_t)invalid;
  out.n_rows = n;
  out.n_cols = n;
  out.nnz = nnz;
  out.vtype = kF32;
  out.indptr = DevBuf((n + 1) * 8, s);
  out.indices = DevBuf(std::max<int64_t>(nnz, 1) * 4, s);
  out.values = DevBuf(std::max<int64_t>(nnz, 1) * 4, s);
  if (m_valid > 0) {
    const unsigned gv = blocks_for(m_valid, 256) > 148u * 16u ? 148u * 16u : blocks_for(m_valid, 256);
    k_reduce_runs<<<gv, 256, 0, s>>>(sk, sp, head.as<int64_t>(), w, m_valid, cbits, n, out.indices.as<int32_t>(),
                                     out.values.as<float>(), out.indptr.as<int64_t>());
  }
  k_indptr_tail<<<blocks_for(n + 1, 256), 256, 0, s>>>(sk, m_valid, cbits, n, nnz, out.indptr.as<int64_t>());
  SCL_CUDA(cudaGetLastError());
}

void transpose_map(const DeviceCSR& g, DeviceCSR& gt, DevBuf& tmap, cudaStream_t s) {
  const int64_t nnz = g.nnz;
  SCL_REQUIRE(nnz < (1ll << 31), kErrInvalidArgument, "transpose map needs nnz < 2^31");
  const int rbits = bits_for(std::max<int64_t>(g.n_rows, 2));
  const int cbits = bits_for(std::max<int64_t>(g.n_cols, 2));
  gt.n_rows = g.n_cols;
  gt.n_cols = g.n_rows;
  gt.nnz = nnz;
  gt.vtype = g.vtype;
  gt.indptr = DevBuf((g.n_cols + 1) * 8, s);
  gt.indices = DevBuf(std::max<int64_t>(nnz, 1) * 4, s);
  tmap = DevBuf(std::max<int64_t>(nnz, 1) * 4, s);
  if (nnz == 0) {
    SCL_CUDA(cudaMemsetAsync(gt.indptr.p, 0, (g.n_cols + 1) * 8, s));
    return;
  }
  DevBuf keys(nnz * 8, s), pay(nnz * 4, s), keys2(nnz * 8, s), pay2(nnz * 4, s);
  k_transpose_keys<<<blocks_for(g.n_rows * 32, 256), 256, 0, s>>>(g.indptr.as<int64_t>(), g.indices.as<int32_t>(),
                                                                 g.n_rows, rbits, keys.as<uint64_t>(),
                                                                 pay.as<uint32_t>());
  SCL_CUDA(cudaGetLastError());
  radix_sort_pairs(keys.as<uint64_t>(), pay.as<uint32_t>(), keys2.as<uint64_t>(), pay2.as<uint32_t>(), nnz,
                   rbits + cbits, s);
  const unsigned gb = blocks_for(nnz, 256) > 148u * 16u ? 148u * 16u : blocks_for(nnz, 256);
  k_transpose_fill<<<gb, 256, 0, s>>>(keys2.as<uint64_t>(), pay2.as<uint32_t>(), nnz, rbits, g.n_cols,
                                      gt.indices.as<int32_t>(), tmap.as<int32_t>(), gt.indptr.as<int64_t>());
  SCL_CUDA(cudaGetLastError());
}

}  // namespace sclgpu
