// Vector walks on the transition graph (scl/kernel/diffusion.hpp:670-831,
// 833-900, 961-1007, 1136-1194): lazy random walk, heat-kernel signature,
// random walk with restart, personalized PageRank and diffusion pseudotime.
//
// Lazy walk, heat kernel and restart walk: one fused kernel per step with a
// warp per row. Lane l runs the fma chain over the row's entries l, l+32, ...
// and the 32 partial sums are combined by a fixed xor butterfly (offsets 16,
// 8, 4, 2, 1), so (P x)_i is deterministic; then the step's linear combination
// with one explicit rounding pattern:
//   lazy / heat kernel:  y_i = fma(c_x, x_i, c_p * (P x)_i)
//   restart:             y_i = fma(c_p, (P x)_i, c_r * r_i)
// and, for the restart walk, the L1 change sum |y_i - x_i| (differences in
// the storage precision, summed in FP64) for the convergence test.
// Diffusion pseudotime keeps a thread per row and the sequential fma chain in
// stored order.
#include <algorithm>
#include <cstring>

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
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double d = 0.0;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    T s = T(0);
    for (int64_t k = ptr[i] + lane, e = ptr[i + 1]; k < e; k += 32) s = wfma(__ldcs(val + k), x[__ldcs(idx + k)], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      T out;
      if constexpr (RESTART) out = wfma(c1, s, wmul(c2, r[i]));
      else out = wfma(c1, x[i], wmul(c2, s));
      y[i] = out;
      if constexpr (RESTART) {
        const T diff = out - x[i];
        d += (double)(diff >= T(0) ? diff : -diff);
      }
    }
  }
  if constexpr (RESTART) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == 0) part[threadIdx.x >> 5] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
      atomicAdd(l1, t);
    }
  }
}

// Atomic max of a non-negative value through its bit pattern (for such
// values the unsigned order of the bits is the numeric order).
__device__ __forceinline__ void max_nonneg(float v, unsigned long long* word) {
  atomicMax(reinterpret_cast<unsigned int*>(word), __float_as_uint(v));
}
__device__ __forceinline__ void max_nonneg(double v, unsigned long long* word) {
  atomicMax(word, (unsigned long long)__double_as_longlong(v));
}
template <class T> T from_bits(unsigned long long w);
template <> float from_bits<float>(unsigned long long w) {
  const unsigned int u = (unsigned int)w;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
template <> double from_bits<double>(unsigned long long w) {
  double d;
  std::memcpy(&d, &w, 8);
  return d;
}

// One diffusion-pseudotime step (diffusion.hpp:706-738): p_new = P p, then for
// rows not yet (almost) visited the hitting time and visit probability grow by
// the newly arriving mass; the largest unvisited probability 1 - visited is
// max-reduced for the convergence test.
template <class T>
__global__ void __launch_bounds__(256)
k_dpt_step(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val, int64_t n,
           const T* __restrict__ p, T* __restrict__ p_new, T* __restrict__ hit, T* __restrict__ vis, T step,
           unsigned long long* __restrict__ max_unvisited) {
  T m = T(0);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    T s = T(0);
    for (int64_t k = ptr[i], e = ptr[i + 1]; k < e; ++k) s = wfma(val[k], p[idx[k]], s);
    p_new[i] = s;
    T v = vis[i];
    if (v < T(0.99) && s > T(1e-15)) {
      const T np = wmul(s, T(1) - v);
      hit[i] = wfma(step, np, hit[i]);
      v = v + np;
      v = v < T(1) ? v : T(1);
      vis[i] = v;
    }
    const T u = T(1) - v;
    m = u > m ? u : m;
  }
  max_nonneg(m, max_unvisited);
}

// hitting time / visit probability on the visited rows (> 0.5), max-reduced
template <class T>
__global__ void k_dpt_scale(int64_t n, T* __restrict__ hit, const T* __restrict__ vis,
                            unsigned long long* __restrict__ max_time) {
  T m = T(0);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (vis[i] > T(0.5)) {
      const T h = hit[i] / vis[i];
      hit[i] = h;
      m = h > m ? h : m;
    }
  }
  max_nonneg(m, max_time);
}

template <class T>
__global__ void k_dpt_output(int64_t n, const T* __restrict__ hit, const T* __restrict__ vis, T inv_max,
                             T* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = vis[i] > T(0.5) ? wmul(hit[i], inv_max) : T(1);
}

template <class T>
__global__ void k_add_scaled_rows(int64_t n, int64_t n_rows, const T* __restrict__ all, T scale, T* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    T s = T(0);
    for (int64_t r = 0; r < n_rows; ++r) s = s + all[r * n + i];
    out[i] = wmul(s, scale);
  }
}

unsigned walk_grid(int64_t n) {
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const int64_t want = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count(dev) * 8));
}

unsigned warp_row_grid(int64_t n) {  // a warp per row, 8 warps per block
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const int64_t want = (n + 7) / 8;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sm_count(dev) * 8));
}

template <class T>
void walk_linear_typed(const CsrView& P, T* x, int64_t steps, T c_x, T c_p, cudaStream_t s) {
  const int64_t n = P.n_rows;
  DevBuf tmp(std::max<int64_t>(n, 1) * sizeof(T), s);
  T* in = x;
  T* out = tmp.as<T>();
  for (int64_t st = 0; st < steps; ++st) {
    k_walk_step<T, false><<<warp_row_grid(n), 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n, in,
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
    k_walk_step<T, true><<<warp_row_grid(n), 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n, cur,
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

template <class T>
void dpt_typed(const CsrView& P, int64_t root, T* out, int64_t max_iter, T tol, cudaStream_t s) {
  const int64_t n = P.n_rows;
  const size_t bytes = (size_t)n * sizeof(T);
  DevBuf pa(bytes, s), pb(bytes, s), hit(bytes, s), vis(bytes, s), word(sizeof(unsigned long long), s);
  SCL_CUDA(cudaMemsetAsync(pa.p, 0, bytes, s));
  SCL_CUDA(cudaMemsetAsync(hit.p, 0, bytes, s));
  SCL_CUDA(cudaMemsetAsync(vis.p, 0, bytes, s));
  const T one = T(1);
  SCL_CUDA(cudaMemcpyAsync(pa.as<T>() + root, &one, sizeof(T), cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaMemcpyAsync(vis.as<T>() + root, &one, sizeof(T), cudaMemcpyHostToDevice, s));
  unsigned long long* hw = nullptr;
  SCL_CUDA(cudaMallocHost(&hw, sizeof(unsigned long long)));
  struct Free {
    unsigned long long* p;
    ~Free() { cudaFreeHost(p); }
  } guard{hw};
  T* p = pa.as<T>();
  T* q = pb.as<T>();
  for (int64_t it = 1; it <= max_iter; ++it) {
    SCL_CUDA(cudaMemsetAsync(word.p, 0, sizeof(unsigned long long), s));
    k_dpt_step<T><<<walk_grid(n), 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n, p, q,
                                                hit.as<T>(), vis.as<T>(), static_cast<T>(it),
                                                word.as<unsigned long long>());
    SCL_CUDA(cudaGetLastError());
    SCL_CUDA(cudaMemcpyAsync(hw, word.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    SCL_CUDA(cudaStreamSynchronize(s));
    if (from_bits<T>(*hw) < tol) break;
    std::swap(p, q);
  }
  SCL_CUDA(cudaMemsetAsync(word.p, 0, sizeof(unsigned long long), s));
  k_dpt_scale<T><<<walk_grid(n), 256, 0, s>>>(n, hit.as<T>(), vis.as<T>(), word.as<unsigned long long>());
  SCL_CUDA(cudaGetLastError());
  SCL_CUDA(cudaMemcpyAsync(hw, word.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  const T max_time = from_bits<T>(*hw);
  const T inv_max = (max_time > T(0)) ? T(1) / max_time : T(1);
  k_dpt_output<T><<<walk_grid(n), 256, 0, s>>>(n, hit.as<T>(), vis.as<T>(), inv_max, out);
  SCL_CUDA(cudaGetLastError());
}

}  // namespace

void dpt(const CsrView& P, int64_t root, void* out, int64_t max_iter, double tol, cudaStream_t s) {
  SCL_REQUIRE(P.n_cols <= P.n_rows, kErrDimensionMismatch, "DPT: column indices must address rows");
  SCL_REQUIRE(root >= 0 && root < P.n_rows, kErrInvalidArgument, "DPT: root_cell out of range");
  if (P.vtype == kF32) return dpt_typed<float>(P, root, static_cast<float*>(out), max_iter, (float)tol, s);
  SCL_REQUIRE(P.vtype == kF64, kErrTypeMismatch, "DPT values must be f32 or f64");
  dpt_typed<double>(P, root, static_cast<double*>(out), max_iter, tol, s);
}

void dpt_average(const void* all, int64_t n_roots, int64_t n, DType t, void* out, cudaStream_t s) {
  if (t == kF32) {
    k_add_scaled_rows<float><<<walk_grid(n), 256, 0, s>>>(n, n_roots, static_cast<const float*>(all),
                                                          1.0f / (float)n_roots, static_cast<float*>(out));
  } else {
    k_add_scaled_rows<double><<<walk_grid(n), 256, 0, s>>>(n, n_roots, static_cast<const double*>(all),
                                                           1.0 / (double)n_roots, static_cast<double*>(out));
  }
  SCL_CUDA(cudaGetLastError());
}

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
