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
// the storage precision, summed in FP64) for the convergence test. The
// restart walk decides convergence on the device: every block stores its
// partial sum, the last block to finish adds the partials in block order (a
// fixed order, so the sum is deterministic) and, below tol, records the step
// and raises a flag that makes the later steps' launches return at once. The
// host queues steps in chunks and reads the flag once per chunk instead of
// once per step.
// Diffusion pseudotime keeps one sequential fma chain per row in stored order
// (a lane per row over entries staged by its warp) and also decides
// convergence on the device.
#include <algorithm>
#include <cstring>

#include "engine.hpp"

namespace sclgpu {
namespace {

__device__ __forceinline__ float wfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double wfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float wmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double wmul(double a, double b) { return __dmul_rn(a, b); }

// Convergence state of a restart walk, in device memory.
struct WalkCtl {
  unsigned int arrived;  // blocks of the current step that have stored their partial sum
  int done;              // set by the step whose L1 change fell below tol
  long long step;        // that step's index
};

template <class T, bool RESTART>
__global__ void __launch_bounds__(256)
k_walk_step(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val, int64_t n,
            const T* __restrict__ x, const T* __restrict__ r, T c1, T c2, T* __restrict__ y, WalkCtl* ctl,
            double* __restrict__ partials, long long step, double tol) {
  __shared__ double part[8];
  __shared__ bool last;
  if constexpr (RESTART) {
    // a converged walk's later steps do nothing (the flag only changes after
    // every block of the converging step has passed this point)
    if (*reinterpret_cast<volatile int*>(&ctl->done)) return;
  }
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
      partials[blockIdx.x] = t;
      __threadfence();
      last = atomicAdd(&ctl->arrived, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x < 32) {
      __threadfence();
      double t = 0.0;
      for (unsigned b = lane; b < gridDim.x; b += 32) t += __ldcg(partials + b);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) {
        if (t < tol) {
          ctl->step = step;
          ctl->done = 1;
        }
        ctl->arrived = 0;
      }
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
template <class T> __device__ T from_bits_dev(unsigned long long w);
template <> __device__ float from_bits_dev<float>(unsigned long long w) { return __uint_as_float((unsigned int)w); }
template <> __device__ double from_bits_dev<double>(unsigned long long w) { return __longlong_as_double((long long)w); }
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
// Convergence state of a DPT walk, in device memory.
struct DptCtl {
  unsigned int arrived;  // blocks of the current step that have max-reduced their rows
  int done;              // set by the step whose largest unvisited probability fell below tol
};

constexpr int kDptWarps = 8;      // warps per block
constexpr int kDptHubLen = 256;   // rows longer than this get a warp of their own

// The row update after p_new[i] = s: hitting time and visit probability of
// rows still below 0.99 visited; returns 1 - visited.
template <class T>
__device__ __forceinline__ T dpt_update(int64_t i, T s, T* __restrict__ p_new, T* __restrict__ hit,
                                        T* __restrict__ vis, T step) {
  p_new[i] = s;
  T v = vis[i];
  if (v < T(0.99) && s > T(1e-15)) {
    const T np = wmul(s, T(1) - v);
    hit[i] = wfma(step, np, hit[i]);
    v = v + np;
    v = v < T(1) ? v : T(1);
    vis[i] = v;
  }
  return T(1) - v;
}

// Rows are taken longest first (`order`, a permutation by decreasing length,
// computed once per walk). Every row's sum is the sequential fma chain over
// its entries in stored order, as a thread walking the row would form it.
// * The n_hub longest rows (> kDptHubLen entries) get a warp each: the lanes
//   gather the row's values and p values into shared memory 256 entries at a
//   time, with all loads in flight together, and lane 0 runs the chain.
// * The other rows go 32 to a warp, neighbours in length order, so the lanes
//   finish together; a lane reads its row's values and indices in 16-byte
//   blocks, two at a time, gathers their p values, then consumes them.
// The largest unvisited probability is max-reduced per block into one word
// (one atomic per block); the last block of the step compares it with tol,
// raises the done flag (the later steps' launches then return at once) and
// clears the word for the next step.
template <class T>
__global__ void __launch_bounds__(kDptWarps * 32)
k_dpt_step(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val, int64_t n,
           const int32_t* __restrict__ order, int64_t n_hub, const T* __restrict__ p, T* __restrict__ p_new,
           T* __restrict__ hit, T* __restrict__ vis, T step, unsigned long long* __restrict__ max_unvisited,
           DptCtl* ctl, T tol) {
  if (*reinterpret_cast<volatile int*>(&ctl->done)) return;
  __shared__ T sv[kDptWarps][kDptHubLen];
  __shared__ T sp[kDptWarps][kDptHubLen];
  __shared__ T part[kDptWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t gw = (int64_t)blockIdx.x * kDptWarps + w, nw = (int64_t)gridDim.x * kDptWarps;
  T m = T(0);
  for (int64_t hr = gw; hr < n_hub; hr += nw) {
    const int64_t i = order[hr];
    const int64_t rb = ptr[i], re = ptr[i + 1];
    T s = T(0);
    for (int64_t c0 = rb; c0 < re; c0 += kDptHubLen) {
      const int cn = (re - c0) < (int64_t)kDptHubLen ? (int)(re - c0) : kDptHubLen;
#pragma unroll
      for (int q = 0; q < kDptHubLen / 32; ++q) {
        const int j = q * 32 + lane;
        if (j < cn) {
          sv[w][j] = val[c0 + j];
          sp[w][j] = p[idx[c0 + j]];
        }
      }
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < cn; ++k) s = wfma(sv[w][k], sp[w][k], s);
      __syncwarp();
    }
    if (lane == 0) {
      const T u = dpt_update<T>(i, s, p_new, hit, vis, step);
      m = u > m ? u : m;
    }
  }
  // values and indices in 16-byte blocks (aligned to the block, entries outside the row skipped),
  // two blocks per round, then the round's p gathers, then its fmas in order
  constexpr int V = 16 / (int)sizeof(T);
  const int64_t nnz = ptr[n];
  const int64_t groups = (n - n_hub + 31) / 32;
  for (int64_t g = gw; g < groups; g += nw) {
    const int64_t r = n_hub + g * 32 + lane;
    if (r < n) {
      const int64_t i = order[r];
      const int64_t rb = ptr[i], re = ptr[i + 1];
      T s = T(0);
      for (int64_t k0 = rb & ~(int64_t)(V - 1); k0 < re; k0 += 2 * V) {
        T vv[2 * V];
        int32_t jj[2 * V];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t kb = k0 + h * V;
          if (kb + V <= nnz) {
            if constexpr (sizeof(T) == 4) {
              const float4 a = __ldg(reinterpret_cast<const float4*>(val + kb));
              const int4 b = __ldg(reinterpret_cast<const int4*>(idx + kb));
              vv[h * V] = a.x, vv[h * V + 1] = a.y, vv[h * V + 2] = a.z, vv[h * V + 3] = a.w;
              jj[h * V] = b.x, jj[h * V + 1] = b.y, jj[h * V + 2] = b.z, jj[h * V + 3] = b.w;
            } else {
              const double2 a = __ldg(reinterpret_cast<const double2*>(val + kb));
              const int2 b = __ldg(reinterpret_cast<const int2*>(idx + kb));
              vv[h * V] = a.x, vv[h * V + 1] = a.y;
              jj[h * V] = b.x, jj[h * V + 1] = b.y;
            }
          } else {
#pragma unroll
            for (int q = 0; q < V; ++q) {
              const bool in = kb + q < nnz;
              vv[h * V + q] = in ? val[kb + q] : T(0);
              jj[h * V + q] = in ? idx[kb + q] : 0;
            }
          }
        }
        T pp[2 * V];
#pragma unroll
        for (int q = 0; q < 2 * V; ++q)
          if (k0 + q >= rb && k0 + q < re) pp[q] = p[jj[q]];
#pragma unroll
        for (int q = 0; q < 2 * V; ++q)
          if (k0 + q >= rb && k0 + q < re) s = wfma(vv[q], pp[q], s);
      }
      const T u = dpt_update<T>(i, s, p_new, hit, vis, step);
      m = u > m ? u : m;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T x = __shfl_xor_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  if (lane == 0) part[w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kDptWarps; ++k) m = part[k] > m ? part[k] : m;
    max_nonneg(m, max_unvisited);
    __threadfence();
    if (atomicAdd(&ctl->arrived, 1u) == gridDim.x - 1) {
      __threadfence();
      const T mx = from_bits_dev<T>(atomicAdd(max_unvisited, 0ull));
      if (mx < tol) ctl->done = 1;
      *max_unvisited = 0ull;
      ctl->arrived = 0;
    }
  }
}

// Sort keys of the DPT row order: decreasing length, ties by row index.
__global__ void k_dpt_keys(const int64_t* __restrict__ ptr, int64_t n, uint64_t* __restrict__ keys,
                           uint32_t* __restrict__ vals, unsigned long long* __restrict__ n_hub) {
  unsigned long long hubs = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t len = ptr[i + 1] - ptr[i];
    const uint64_t l = len < (int64_t)0xffffffff ? (uint64_t)len : 0xffffffffull;
    keys[i] = 0xffffffffull - l;
    vals[i] = (uint32_t)i;
    hubs += len > kDptHubLen ? 1ull : 0ull;
  }
  if (hubs) atomicAdd(n_hub, hubs);
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
                                                        nullptr, c_x, c_p, out, nullptr, nullptr, 0, 0.0);
    SCL_CUDA(cudaGetLastError());
    std::swap(in, out);
  }
  if (in != x) SCL_CUDA(cudaMemcpyAsync(x, in, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
}

template <class T>
int64_t walk_restart_typed(const CsrView& P, const T* r, T* scores, T alpha, int64_t max_iter, T tol,
                           cudaStream_t s) {
  const int64_t n = P.n_rows;
  const unsigned grid = warp_row_grid(n);
  DevBuf other(std::max<int64_t>(n, 1) * sizeof(T), s);
  DevBuf ctl(sizeof(WalkCtl), s), partials(grid * sizeof(double), s);
  SCL_CUDA(cudaMemsetAsync(ctl.p, 0, sizeof(WalkCtl), s));
  WalkCtl host{};  // read back once per chunk (a few bytes: pageable memory, no pinned allocation per call)
  const T beta = T(1) - alpha;
  // scores holds the restart vector; the two buffers swap roles after every
  // step that has not converged, so step `it` reads from scores when `it` is
  // even and the caller's buffer ends up holding the last iterate written
  // into it (the reference's pointer swap)
  T* bufs[2] = {scores, other.as<T>()};
  constexpr int64_t kChunk = 8;  // steps queued between reads of the flag
  for (int64_t c0 = 0; c0 < max_iter; c0 += kChunk) {
    const int64_t c1 = std::min<int64_t>(max_iter, c0 + kChunk);
    for (int64_t it = c0; it < c1; ++it) {
      k_walk_step<T, true><<<grid, 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n,
                                                bufs[it & 1], r, alpha, beta, bufs[(it + 1) & 1],
                                                ctl.as<WalkCtl>(), partials.as<double>(), (long long)it, (double)tol);
      SCL_CUDA(cudaGetLastError());
    }
    SCL_CUDA(cudaMemcpyAsync(&host, ctl.p, sizeof(WalkCtl), cudaMemcpyDeviceToHost, s));
    SCL_CUDA(cudaStreamSynchronize(s));
    if (host.done) {
      const int64_t it = host.step;  // the converged step wrote bufs[(it + 1) & 1]; it lands in bufs[it & 1]
      SCL_CUDA(cudaMemcpyAsync(bufs[it & 1], bufs[(it + 1) & 1], n * sizeof(T), cudaMemcpyDeviceToDevice, s));
      return it + 1;
    }
  }
  return max_iter;
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
  unsigned long long hw = 0;  // the max-reduced hitting time, read back once (pageable: 8 bytes)
  DevBuf ctl(sizeof(DptCtl), s);
  SCL_CUDA(cudaMemsetAsync(ctl.p, 0, sizeof(DptCtl), s));
  SCL_CUDA(cudaMemsetAsync(word.p, 0, sizeof(unsigned long long), s));
  T* bufs[2] = {pa.as<T>(), pb.as<T>()};  // step it reads bufs[(it + 1) & 1] and writes the other one
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_REQUIRE((reinterpret_cast<uintptr_t>(P.values) & 15u) == 0 && (reinterpret_cast<uintptr_t>(P.indices) & 15u) == 0,
              kErrInternal, "DPT: the step reads values and indices in 16-byte blocks");
  // rows longest first; the hub rows (one warp each) lead the order
  DevBuf keys(std::max<int64_t>(n, 1) * 8, s), keys2(std::max<int64_t>(n, 1) * 8, s);
  DevBuf rows(std::max<int64_t>(n, 1) * 4, s), order(std::max<int64_t>(n, 1) * 4, s), hubs(8, s);
  SCL_CUDA(cudaMemsetAsync(hubs.p, 0, 8, s));
  k_dpt_keys<<<walk_grid(n), 256, 0, s>>>(P.indptr, n, keys.as<uint64_t>(), rows.as<uint32_t>(),
                                          hubs.as<unsigned long long>());
  SCL_CUDA(cudaGetLastError());
  radix_sort_pairs(keys.as<uint64_t>(), rows.as<uint32_t>(), keys2.as<uint64_t>(), order.as<uint32_t>(), n, 32, s);
  unsigned long long n_hub = 0;
  SCL_CUDA(cudaMemcpyAsync(&n_hub, hubs.p, 8, cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  const int64_t groups = (int64_t)n_hub + (n - (int64_t)n_hub + 31) / 32;
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>((groups + kDptWarps - 1) / kDptWarps, (int64_t)sm_count(dev) * 8));
  constexpr int64_t kChunk = 8;  // steps queued between reads of the flag
  DptCtl host{};
  for (int64_t c0 = 1; c0 <= max_iter; c0 += kChunk) {
    const int64_t c1 = std::min<int64_t>(max_iter, c0 + kChunk - 1);
    for (int64_t it = c0; it <= c1; ++it) {
      k_dpt_step<T><<<grid, kDptWarps * 32, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), n,
                                                    reinterpret_cast<const int32_t*>(order.p), (int64_t)n_hub,
                                                    bufs[(it + 1) & 1], bufs[it & 1], hit.as<T>(), vis.as<T>(),
                                                    static_cast<T>(it), word.as<unsigned long long>(),
                                                    ctl.as<DptCtl>(), tol);
      SCL_CUDA(cudaGetLastError());
    }
    SCL_CUDA(cudaMemcpyAsync(&host, ctl.p, sizeof(DptCtl), cudaMemcpyDeviceToHost, s));
    SCL_CUDA(cudaStreamSynchronize(s));
    if (host.done) break;
  }
  SCL_CUDA(cudaMemsetAsync(word.p, 0, sizeof(unsigned long long), s));
  k_dpt_scale<T><<<walk_grid(n), 256, 0, s>>>(n, hit.as<T>(), vis.as<T>(), word.as<unsigned long long>());
  SCL_CUDA(cudaGetLastError());
  SCL_CUDA(cudaMemcpyAsync(&hw, word.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  const T max_time = from_bits<T>(hw);
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

// ---- diffusion map embedding (scl/kernel/diffusion.hpp:366-446, 901-955) -------------
namespace sclgpu {
namespace {

template <class T>
__global__ void k_dmap_init(T* __restrict__ Q, int64_t n, int K) {
  const int64_t total = n * K;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / K;
    const int c = (int)(e % K);
    const T t = (T)i / (T)n;
    const T phase = (T)(c + 1) * (T)3.14159265358979323846;
    Q[e] = wfma((T)0.1, sin(phase * t * (T)2.7), cos(phase * t));
  }
}

// Block-wide sum of a per-thread double, returned to every thread.
__device__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
  return s;
}

// Modified Gram-Schmidt with re-orthogonalisation over the K columns of the
// row-major n x K block Q, with the reference's control flow: each column is
// projected off the previous ones (coefficients dot / |q_p|^2 when
// |q_p|^2 > 1e-15), re-projected (up to 2 more passes) while its largest
// cosine with them is at least 0.7 after the first pass, and normalised; a
// column of norm^2 <= 1e-15 becomes the unit vector e_(v mod n). One CTA runs
// the whole loop; the sums are FP64 block reductions.
template <class T>
__global__ void __launch_bounds__(1024) k_gram_schmidt(T* __restrict__ Q, int64_t n, int K, T* __restrict__ w) {
  __shared__ double red[32];
  const int tid = threadIdx.x;
  const int NT = blockDim.x;
  for (int v = 0; v < K; ++v) {
    for (int64_t i = tid; i < n; i += NT) w[i] = Q[i * K + v];
    __syncthreads();
    for (int reorth = 0; reorth <= 2; ++reorth) {
      for (int p = 0; p < v; ++p) {
        double a = 0.0, b = 0.0;
        for (int64_t i = tid; i < n; i += NT) {
          const double q = (double)Q[i * K + p];
          a += (double)w[i] * q;
          b += q * q;
        }
        const T dot = (T)block_sum(a, red);
        const T norm_p = (T)block_sum(b, red);
        if (norm_p > (T)1e-15) {
          const T coeff = dot / norm_p;
          for (int64_t i = tid; i < n; i += NT) w[i] = wfma(-coeff, Q[i * K + p], w[i]);
        }
        __syncthreads();
      }
      double c = 0.0;
      for (int64_t i = tid; i < n; i += NT) c += (double)w[i] * (double)w[i];
      const T norm_v = (T)block_sum(c, red);
      if (reorth == 0 && v > 0) {
        T max_cos = T(0);
        for (int p = 0; p < v; ++p) {
          double a = 0.0;
          for (int64_t i = tid; i < n; i += NT) a += (double)w[i] * (double)Q[i * K + p];
          const T dot = (T)block_sum(a, red);
          const T cv = (norm_v > (T)1e-15) ? (dot < T(0) ? -dot : dot) / sqrt(norm_v) : T(0);
          max_cos = cv > max_cos ? cv : max_cos;
        }
        if (max_cos < (T)0.7) break;
      } else {
        break;
      }
    }
    double c = 0.0;
    for (int64_t i = tid; i < n; i += NT) c += (double)w[i] * (double)w[i];
    const T norm = (T)block_sum(c, red);
    if (norm > (T)1e-15) {
      const T inv = T(1) / sqrt(norm);
      for (int64_t i = tid; i < n; i += NT) Q[i * K + v] = wmul(w[i], inv);
    } else {
      for (int64_t i = tid; i < n; i += NT) Q[i * K + v] = (i == (int64_t)v % n) ? T(1) : T(0);
    }
    __syncthreads();
  }
}

template <class T>
void dmap_typed(const CsrView& P, T* out, int K, int64_t n_iter, cudaStream_t s) {
  const int64_t n = P.n_rows;
  const size_t bytes = (size_t)n * K * sizeof(T);
  DevBuf qa(bytes, s), qb(bytes, s), w((size_t)n * sizeof(T), s);
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n * K + 255) / 256, (int64_t)sm_count(dev) * 8));
  k_dmap_init<T><<<g, 256, 0, s>>>(qa.as<T>(), n, K);
  SCL_CUDA(cudaGetLastError());
  k_gram_schmidt<T><<<1, 1024, 0, s>>>(qa.as<T>(), n, K, w.as<T>());
  SCL_CUDA(cudaGetLastError());
  SpmmArgs a{};
  a.indptr = P.indptr;
  a.indices = P.indices;
  a.values = P.values;
  a.vtype = P.vtype;
  a.n_rows = n;
  a.F = K;
  a.xtype = P.vtype;
  a.ytype = P.vtype;
  T* q = qa.as<T>();
  T* qn = qb.as<T>();
  for (int64_t it = 0; it < n_iter; ++it) {
    a.X = q;
    a.Y = qn;
    spmm(a, s);
    k_gram_schmidt<T><<<1, 1024, 0, s>>>(qn, n, K, w.as<T>());
    SCL_CUDA(cudaGetLastError());
    std::swap(q, qn);
  }
  SCL_CUDA(cudaMemcpyAsync(out, q, bytes, cudaMemcpyDeviceToDevice, s));
}

}  // namespace

void diffusion_map(const CsrView& P, void* out, int K, int64_t n_iter, cudaStream_t s) {
  SCL_REQUIRE(P.n_cols <= P.n_rows, kErrDimensionMismatch, "diffusion map: column indices must address rows");
  if (P.n_rows == 0 || K <= 0) return;
  if (P.vtype == kF32) return dmap_typed<float>(P, static_cast<float*>(out), K, n_iter, s);
  SCL_REQUIRE(P.vtype == kF64, kErrTypeMismatch, "diffusion map values must be f32 or f64");
  dmap_typed<double>(P, static_cast<double*>(out), K, n_iter, s);
}

}  // namespace sclgpu

// ---- diffusion distance (scl/kernel/diffusion.hpp:1024-1130) ---------------------------
namespace sclgpu {
namespace {

template <class T>
__global__ void k_identity(T* __restrict__ Z, int64_t n) {
  const int64_t total = n * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    Z[e] = (e / n == e % n) ? T(1) : T(0);
}

template <class T>
__global__ void k_transpose_sq(const T* __restrict__ A, T* __restrict__ B, int64_t n) {
  __shared__ T tile[32][33];
  const int64_t bx = (int64_t)blockIdx.x * 32, by = (int64_t)blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t i = by + r, j = bx + threadIdx.x;
    if (i < n && j < n) tile[r][threadIdx.x] = A[i * n + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t i = bx + r, j = by + threadIdx.x;
    if (i < n && j < n) B[i * n + j] = tile[threadIdx.x][r];
  }
}

// D[i][j] = D[j][i] = sqrt(sum_k (Z[i][k] - Z[j][k])^2) for i < j, summed over
// k in order with each square rounded before it is added; D[i][i] = 0. A CTA takes a 32 x 32 block of
// (i, j) above the diagonal and stages 32-column slices of both row sets.
template <class T>
__global__ void k_pair_dist(const T* __restrict__ Z, int64_t n, T* __restrict__ D) {
  __shared__ T A[32][33], B[32][33];
  const int64_t bi = (int64_t)blockIdx.y * 32, bj = (int64_t)blockIdx.x * 32;
  if (bj + 31 < bi) return;  // block entirely below the diagonal
  const int ty = threadIdx.y, tx = threadIdx.x;
  const int64_t i = bi + ty, j = bj + tx;
  T acc = T(0);
  for (int64_t k0 = 0; k0 < n; k0 += 32) {
    const int64_t k = k0 + tx;
    A[ty][tx] = (bi + ty < n && k < n) ? Z[(bi + ty) * n + k] : T(0);
    B[ty][tx] = (bj + ty < n && k < n) ? Z[(bj + ty) * n + k] : T(0);
    __syncthreads();
    const int kn = (n - k0) < 32 ? (int)(n - k0) : 32;
    for (int kk = 0; kk < kn; ++kk) {
      const T diff = A[ty][kk] - B[tx][kk];
      acc = acc + wmul(diff, diff);  // a rounded product, then the sum (no fma), as the reference
    }
    __syncthreads();
  }
  if (i < n && j < n) {
    if (i == j) D[i * n + i] = T(0);
    else if (i < j) {
      const T dist = sqrt(acc);
      D[i * n + j] = dist;
      D[j * n + i] = dist;
    }
  }
}

template <class T>
void ddist_typed(const CsrView& P, T* D, int64_t steps, cudaStream_t s) {
  const int64_t n = P.n_rows;
  const size_t bytes = (size_t)n * (size_t)n * sizeof(T);
  DevBuf za(bytes, s), zb(bytes, s);
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n * n + 255) / 256, (int64_t)sm_count(dev) * 16));
  k_identity<T><<<g, 256, 0, s>>>(za.as<T>(), n);
  SCL_CUDA(cudaGetLastError());
  SpmmArgs a{};
  a.indptr = P.indptr;
  a.indices = P.indices;
  a.values = P.values;
  a.vtype = P.vtype;
  a.n_rows = n;
  a.F = n;
  a.xtype = P.vtype;
  a.ytype = P.vtype;
  T* z = za.as<T>();
  T* zn = zb.as<T>();
  for (int64_t st = 0; st < steps; ++st) {  // Z <- P Z: the rows of P^t
    a.X = z;
    a.Y = zn;
    spmm(a, s);
    std::swap(z, zn);
  }
  const dim3 blocks((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
  if (n > 1000) {  // the reference's large-n branch compares columns of P^t (P^t e_i)
    k_transpose_sq<T><<<blocks, dim3(32, 8), 0, s>>>(z, zn, n);
    SCL_CUDA(cudaGetLastError());
    std::swap(z, zn);
  }
  k_pair_dist<T><<<blocks, dim3(32, 32), 0, s>>>(z, n, D);
  SCL_CUDA(cudaGetLastError());
}

}  // namespace

void diffusion_distance(const CsrView& P, void* D, int64_t steps, cudaStream_t s) {
  SCL_REQUIRE(P.n_cols <= P.n_rows, kErrDimensionMismatch, "diffusion distance: column indices must address rows");
  SCL_REQUIRE(P.n_rows <= 46340, kErrInvalidArgument, "diffusion distance: at most 46,340 nodes (n^2 < 2^31)");
  if (P.n_rows == 0) return;
  if (P.vtype == kF32) return ddist_typed<float>(P, static_cast<float*>(D), steps, s);
  SCL_REQUIRE(P.vtype == kF64, kErrTypeMismatch, "diffusion distance values must be f32 or f64");
  ddist_typed<double>(P, static_cast<double*>(D), steps, s);
}

}  // namespace sclgpu
