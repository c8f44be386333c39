// FP64 error check of a diffused block against an FP64 reference block.
//
// The precision forms store edge values and iterates in 16 bits (or 32) and
// accumulate in FP32; their accuracy is stated against an FP64 diffusion of
// the same graph. This reduction runs on the device in FP64 so that checking a
// 500k x 64 result costs one pass over the two blocks instead of a host copy:
//
//   sum_sq_diff = sum (x - r)^2        sum_sq_ref = sum r^2
//   max_abs     = max |x - r|          max_rel    = max |x - r| / max(|r|, floor)
//
// Each CTA folds a fixed, strided set of elements and writes one partial; one
// CTA then folds the partials in index order. The grid depends only on the
// element count, so the sums are the same bits on every run.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <type_traits>

#include "engine.hpp"

namespace sclgpu {
namespace {

constexpr int kResThreads = 256;

template <class T>
__device__ __forceinline__ double load_as_f64(const T* p, int64_t i) {
  if constexpr (std::is_same_v<T, __nv_bfloat16>) return (double)__bfloat162float(p[i]);
  else if constexpr (std::is_same_v<T, __half>) return (double)__half2float(p[i]);
  else return (double)p[i];
}

struct Partial {
  double sq_diff, sq_ref, max_abs, max_rel;
};

__device__ __forceinline__ Partial combine(const Partial& a, const Partial& b) {
  return {a.sq_diff + b.sq_diff, a.sq_ref + b.sq_ref, fmax(a.max_abs, b.max_abs), fmax(a.max_rel, b.max_rel)};
}

// Tree reduction over the CTA in shared memory (fixed order).
__device__ Partial cta_reduce(Partial p) {
  __shared__ Partial sh[kResThreads];
  sh[threadIdx.x] = p;
  __syncthreads();
  for (int w = kResThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = combine(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  return sh[0];
}

template <class T>
__global__ void __launch_bounds__(kResThreads)
k_residual_partials(const T* __restrict__ X, const double* __restrict__ R, int64_t total, double floor_,
                    Partial* __restrict__ parts) {
  Partial p{0.0, 0.0, 0.0, 0.0};
  const int64_t stride = (int64_t)gridDim.x * kResThreads;
  for (int64_t i = (int64_t)blockIdx.x * kResThreads + threadIdx.x; i < total; i += stride) {
    const double r = R[i];
    const double d = load_as_f64(X, i) - r;
    const double ad = fabs(d);
    p.sq_diff = fma(d, d, p.sq_diff);
    p.sq_ref = fma(r, r, p.sq_ref);
    p.max_abs = fmax(p.max_abs, ad);
    p.max_rel = fmax(p.max_rel, ad / fmax(fabs(r), floor_));
  }
  const Partial t = cta_reduce(p);
  if (threadIdx.x == 0) parts[blockIdx.x] = t;
}

// One CTA: thread t folds partials t, t + 256, ... in order, then the tree.
__global__ void __launch_bounds__(kResThreads)
k_residual_final(const Partial* __restrict__ parts, int n_parts, double* __restrict__ out) {
  Partial p{0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < n_parts; i += kResThreads) p = combine(p, parts[i]);
  const Partial t = cta_reduce(p);
  if (threadIdx.x == 0) {
    out[0] = t.sq_diff;
    out[1] = t.sq_ref;
    out[2] = t.max_abs;
    out[3] = t.max_rel;
  }
}

template <class T>
void launch_residual(const void* X, const double* R, int64_t total, double floor_, Partial* parts, int grid,
                     double* out, cudaStream_t s) {
  k_residual_partials<T><<<grid, kResThreads, 0, s>>>(static_cast<const T*>(X), R, total, floor_, parts);
  SCL_CUDA(cudaGetLastError());
  k_residual_final<<<1, kResThreads, 0, s>>>(parts, grid, out);
  SCL_CUDA(cudaGetLastError());
}

}  // namespace

// out (host, 4 doubles): relative Frobenius error ||x - r|| / ||r|| (0 when
// r == 0 and x == r), max relative error, max absolute error, ||r||.
void residual_fp64(const void* X, DType xt, const double* R, int64_t total, double rel_floor, double* out_host,
                   cudaStream_t s) {
  SCL_REQUIRE(total > 0, kErrInvalidArgument, "Dimensions must be positive");
  SCL_REQUIRE(rel_floor >= 0.0, kErrInvalidArgument, "rel_floor must be non-negative");
  const int dev = current_device();
  const int64_t want = (total + (int64_t)kResThreads * 8 - 1) / ((int64_t)kResThreads * 8);
  const int64_t cap = (int64_t)sm_count(dev) * 4;
  const int grid = (int)(want < 1 ? 1 : (want > cap ? cap : want));
  DevBuf parts((size_t)grid * sizeof(Partial), s);
  DevBuf res(4 * sizeof(double), s);
  switch (xt) {
    case kF32: launch_residual<float>(X, R, total, rel_floor, parts.as<Partial>(), grid, res.as<double>(), s); break;
    case kF64: launch_residual<double>(X, R, total, rel_floor, parts.as<Partial>(), grid, res.as<double>(), s); break;
    case kBF16:
      launch_residual<__nv_bfloat16>(X, R, total, rel_floor, parts.as<Partial>(), grid, res.as<double>(), s);
      break;
    case kF16: launch_residual<__half>(X, R, total, rel_floor, parts.as<Partial>(), grid, res.as<double>(), s); break;
    default: throw Error(kErrTypeMismatch, "residual: X must be f32, f64, bf16 or f16");
  }
  double h[4];
  SCL_CUDA(cudaMemcpyAsync(h, res.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  const double nrm_d = std::sqrt(h[0]), nrm_r = std::sqrt(h[1]);
  out_host[0] = nrm_r > 0.0 ? nrm_d / nrm_r : (nrm_d > 0.0 ? INFINITY : 0.0);
  out_host[1] = h[3];
  out_host[2] = h[2];
  out_host[3] = nrm_r;
}

}  // namespace sclgpu
