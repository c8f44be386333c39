// Vector walks on the transition graph (scl/kernel/diffusion.hpp:833-900,
// 961-1007, 1136-1194): lazy random walk, heat-kernel signature, random walk
// with restart and personalized PageRank.
//
// Every step is one fused kernel: a thread per row forms (P x)_i as the
// sequential fma chain over the row's entries in stored order, then the
// step's linear combination with one explicit rounding pattern:
//   lazy / heat kernel:  y_i = fma(c_x, x_i, c_p * (P x)_i)
//   restart:             y_i = fma(c_p, (P x)_i, c_r * r_i)
// and, for the restart walk, the L1 change sum |y_i - x_i| (differences in
// the storage precision, summed in FP64) for the convergence test.
#include <algorithm>

#include "engine.hpp"

namespace sclgpu {
namespace {

__device__ __forceinline__ float wfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double wfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float wmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double wmul(double a, double b) { return __dmul_rn(a, b); }

template <class T, bool RESTART>
__global__ void __launch_bounds__(256)
k_walk_step(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val, int64_t n,
            const T* __restrict__ x, const T* __restrict__ r, T c1, T c2, T* __restrict__ y,
            double* __restrict__ l1) {
  __shared__ double part[8];
  double d = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    T s = T(0);
    for (int64_t k = ptr[i], e = ptr[i + 1]; k < e; ++k) s = wfma(val[k], x[idx[k]], s);
    T out;
    if constexpr (RESTART) out = wfma(c1, s, wmul(c2, r[i]));
    else out = wfma(c1, x[i], wmul(c2, s));
    y[i] = out;
    if constexpr (RESTART) {
      const T diff = out - x[i];
      d += (double)(diff >= T(0) ? diff : -diff);
    }
  }
  if constexpr (RESTART) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
      atomicAdd(l1, t);
    }
  }
}

unsigned walk_grid(int64_t n) {
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const int64_t want = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count(dev) * 8));
}

template <class T>
void walk_linear_typed(const CsrView& P, T* x, int64_t steps, T c_x, T c_p, cudaStream_t s) {
  const int64_t n = P.n_rows;
  DevBuf tmp(std::max<int64_t>(n, 1) * sizeof(T), s);
  T* in = x;
  T* out = tmp.as<T>();
  for (int64_t st = 0; st < steps; ++st) {
    k_walk_step<T, false><<<walk_grid(n), 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n, in,
                                                        nullptr, c_x, c_p, out, nullptr);
    SCL_CUDA(cudaGetLastError());
    std::swap(in, out);
  }
  if (in != x) SCL_CUDA(cudaMemcpyAsync(x, in, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
}

template <class T>
int64_t walk_restart_typed(const CsrView& P, const T* r, T* scores, T alpha, int64_t max_iter, T tol,
                           cudaStream_t s) {
  const int64_t n = P.n_rows;
  DevBuf other(std::max<int64_t>(n, 1) * sizeof(T), s);
  DevBuf l1(sizeof(double), s);
  double* host_l1 = nullptr;
  SCL_CUDA(cudaMallocHost(&host_l1, sizeof(double)));
  struct Free {
    double* p;
    ~Free() { cudaFreeHost(p); }
  } guard{host_l1};
  const T beta = T(1) - alpha;
  // scores holds the restart vector; the two buffers swap roles after every
  // step that has not converged, so the caller's buffer ends up holding the
  // last iterate written into it (the reference's pointer swap)
  T* cur = scores;
  T* nxt = other.as<T>();
  int64_t it = 0;
  for (; it < max_iter; ++it) {
    SCL_CUDA(cudaMemsetAsync(l1.p, 0, sizeof(double), s));
    k_walk_step<T, true><<<walk_grid(n), 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n, cur,
                                                       r, alpha, beta, nxt, l1.as<double>());
    SCL_CUDA(cudaGetLastError());
    SCL_CUDA(cudaMemcpyAsync(host_l1, l1.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    SCL_CUDA(cudaStreamSynchronize(s));
    if (*host_l1 < (double)tol) {
      SCL_CUDA(cudaMemcpyAsync(cur, nxt, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
      return it + 1;
    }
    std::swap(cur, nxt);
  }
  return it;
}

}  // namespace

void walk_linear(const CsrView& P, void* x, int64_t steps, double c_x, double c_p, cudaStream_t s) {
  SCL_REQUIRE(P.n_cols <= P.n_rows, kErrDimensionMismatch, "walk: column indices must address rows of x");
  if (steps <= 0 || P.n_rows == 0) return;
  if (P.vtype == kF32) return walk_linear_typed<float>(P, static_cast<float*>(x), steps, (float)c_x, (float)c_p, s);
  SCL_REQUIRE(P.vtype == kF64, kErrTypeMismatch, "walk values must be f32 or f64");
  walk_linear_typed<double>(P, static_cast<double*>(x), steps, c_x, c_p, s);
}

int64_t walk_restart(const CsrView& P, const void* r, void* scores, double alpha, int64_t max_iter, double tol,
                     cudaStream_t s) {
  SCL_REQUIRE(P.n_cols <= P.n_rows, kErrDimensionMismatch, "walk: column indices must address rows of x");
  if (P.n_rows == 0 || max_iter <= 0) return 0;
  if (P.vtype == kF32)
    return walk_restart_typed<float>(P, static_cast<const float*>(r), static_cast<float*>(scores), (float)alpha,
                                     max_iter, (float)tol, s);
  SCL_REQUIRE(P.vtype == kF64, kErrTypeMismatch, "walk values must be f32 or f64");
  return walk_restart_typed<double>(P, static_cast<const double*>(r), static_cast<double*>(scores), alpha, max_iter,
                                    tol, s);
}

}  // namespace sclgpu
