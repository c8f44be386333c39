// Brute-force k-nearest neighbours (scl/kernel/neighbors.hpp:302-478): the
// graph-building step before the transition matrix.
//
// The samples (the handle's primary rows) are made dense on the device, n x d
// with d <= 128 features. A thread owns one query and walks every candidate j
// in increasing order, exactly as the reference's per-query loop does, so the
// result (ties included) is the reference's: the same Cauchy-Schwarz skip
// ((sqrt(norm_i) - sqrt(norm_j))^2 >= the current k-th distance), the same
// dist_sq = fma(-2, dot, norm_i + norm_j) clamped at 0 with the dot an fma
// chain over the features in order, the same max-heap of k entries (a
// candidate enters while the heap is short, else when strictly below the
// top), and the same heap sort at the end, so equal distances leave in the
// same order. The CTA's queries are staged column-major in shared memory and
// a tile of 64 candidate rows is staged row-major; every thread reads the
// candidate values at the same address (a broadcast) and forms four dot
// products per pass over the features. The heaps live in shared memory,
// column-major, one column per thread.
#include <algorithm>
#include <cmath>
#include <limits>
#include <type_traits>

#include "engine.hpp"

namespace sclgpu {
namespace {

constexpr int kKnnTile = 64;  // candidates per tile
constexpr int kKnnMaxD = 128;

__device__ __forceinline__ float kfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double kfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float ksqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double ksqrt(double a) { return __dsqrt_rn(a); }

// DR > 0 (16 or 32 features at most): the query row is held in DR registers
// (features zero-padded to DR, which leaves every fma chain unchanged) and the
// candidate rows are staged with pitch DR, read 16 bytes per load; DR == 0:
// queries in shared memory, any d up to 128 (a 64-register query spilled and
// ran slower than this path at 50 features).
template <class T, class IT, int NT, int KMAX, int DR>
__global__ void __launch_bounds__(NT)
k_knn_dense(const T* __restrict__ X, const T* __restrict__ norms, const T* __restrict__ snorms, int64_t n, int d,
            int k, IT* __restrict__ out_idx, T* __restrict__ out_dist) {
  extern __shared__ __align__(16) unsigned char knn_smem[];
  const int dp = DR > 0 ? DR : d + 1;
  T* Qs = reinterpret_cast<T*>(knn_smem);                          // [d][NT] (DR == 0)
  T* Cs = Qs + (DR > 0 ? 0 : (size_t)d * NT);                      // [kKnnTile][dp]
  T* Hd = Cs + (size_t)kKnnTile * dp;                              // [KMAX][NT]
  int32_t* Hj = reinterpret_cast<int32_t*>(Hd + (size_t)KMAX * NT);  // [KMAX][NT]
  const int tid = threadIdx.x;
  const int64_t i = (int64_t)blockIdx.x * NT + tid;
  const bool live = i < n;
  const int64_t q0 = (int64_t)blockIdx.x * NT;
  const int nq = (n - q0) < (int64_t)NT ? (int)(n - q0) : NT;
  T qr[DR > 0 ? DR : 1];
  if constexpr (DR > 0) {
#pragma unroll
    for (int f = 0; f < DR; ++f) qr[f] = (live && f < d) ? X[i * (int64_t)d + f] : T(0);
  } else {
    for (int e = tid; e < nq * d; e += NT) {  // queries, column-major
      const int r = e / d, f = e - r * d;
      Qs[f * NT + r] = X[(q0 + r) * (int64_t)d + f];
    }
  }
  const T ni = live ? norms[i] : T(0);
  const T si = live ? snorms[i] : T(0);
  T maxd = std::numeric_limits<T>::max();
  int cnt = 0;
#define HD(p) Hd[(p) * NT + tid]
#define HJ(p) Hj[(p) * NT + tid]
  auto swap_at = [&](int a, int b) {
    const T td = HD(a);
    const int32_t tj = HJ(a);
    HD(a) = HD(b);
    HJ(a) = HJ(b);
    HD(b) = td;
    HJ(b) = tj;
  };
  for (int64_t t0 = 0; t0 < n; t0 += kKnnTile) {
    const int tn = (n - t0) < (int64_t)kKnnTile ? (int)(n - t0) : kKnnTile;
    __syncthreads();  // the previous tile is consumed (and the queries are staged)
    if constexpr (DR > 0) {
      for (int e = tid; e < kKnnTile * DR; e += NT) {  // rows past the tile and features past d are zero
        const int r = e / DR, f = e - r * DR;
        Cs[e] = (r < tn && f < d) ? X[(t0 + r) * (int64_t)d + f] : T(0);
      }
    } else {
      for (int e = tid; e < tn * d; e += NT) {
        const int r = e / d, f = e - r * d;
        Cs[r * dp + f] = X[(t0 + r) * (int64_t)d + f];
      }
    }
    __syncthreads();
    if (!live) continue;
    for (int c0 = 0; c0 < tn; c0 += 4) {
      T dot[4] = {T(0), T(0), T(0), T(0)};
      const int cl = (tn - c0) < 4 ? (tn - c0) : 4;
      if constexpr (DR > 0) {
        using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
        constexpr int PER = 16 / (int)sizeof(T);  // values per 16-byte load
#pragma unroll
        for (int f = 0; f < DR; f += PER) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const V4 v = *reinterpret_cast<const V4*>(Cs + (c0 + u) * DR + f);
            if constexpr (sizeof(T) == 4) {
              dot[u] = kfma(qr[f], v.x, dot[u]);
              dot[u] = kfma(qr[f + 1], v.y, dot[u]);
              dot[u] = kfma(qr[f + 2], v.z, dot[u]);
              dot[u] = kfma(qr[f + 3], v.w, dot[u]);
            } else {
              dot[u] = kfma(qr[f], v.x, dot[u]);
              dot[u] = kfma(qr[f + 1], v.y, dot[u]);
            }
          }
        }
      } else {
        for (int f = 0; f < d; ++f) {
          const T a = Qs[f * NT + tid];
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (u < cl) dot[u] = kfma(a, Cs[(c0 + u) * dp + f], dot[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (u >= cl) break;
        const int64_t j = t0 + c0 + u;
        if (j == i) continue;
        const T nd = si - snorms[j];
        if (nd * nd >= maxd) continue;  // reference's lower-bound skip
        T ds = kfma(T(-2), dot[u], ni + norms[j]);
        if (ds < T(0)) ds = T(0);
        if (cnt < k) {
          int pos = cnt;
          HD(pos) = ds;
          HJ(pos) = (int32_t)j;
          while (pos > 0) {  // sift up
            const int parent = (pos - 1) / 2;
            if (HD(pos) <= HD(parent)) break;
            swap_at(pos, parent);
            pos = parent;
          }
          ++cnt;
          if (cnt == k) maxd = HD(0);
        } else if (ds < HD(0)) {
          HD(0) = ds;
          HJ(0) = (int32_t)j;
          int pos = 0;
          while (true) {  // sift down
            int largest = pos;
            const int l = 2 * pos + 1, r = 2 * pos + 2;
            if (l < cnt && HD(l) > HD(largest)) largest = l;
            if (r < cnt && HD(r) > HD(largest)) largest = r;
            if (largest == pos) break;
            swap_at(pos, largest);
            pos = largest;
          }
          maxd = HD(0);
        }
      }
    }
  }
  if (!live) return;
  // heap sort ascending (neighbors.hpp:437-466): min-heap sift, extract, reverse
  auto sort_sift = [&](int pos, int size) {
    while (true) {
      int smallest = pos;
      const int l = 2 * pos + 1, r = 2 * pos + 2;
      if (l < size && HD(l) < HD(smallest)) smallest = l;
      if (r < size && HD(r) < HD(smallest)) smallest = r;
      if (smallest == pos) break;
      swap_at(pos, smallest);
      pos = smallest;
    }
  };
  if (cnt >= 2)
    for (int m = cnt / 2; m > 0; --m) sort_sift(m - 1, cnt);
  for (int m = cnt; m > 1; --m) {
    swap_at(0, m - 1);
    sort_sift(0, m - 1);
  }
  for (int m = 0; m < cnt / 2; ++m) swap_at(m, cnt - 1 - m);
  for (int m = 0; m < k; ++m) {
    out_dist[i * k + m] = m < cnt ? ksqrt(HD(m)) : std::numeric_limits<T>::infinity();
    out_idx[i * k + m] = m < cnt ? (IT)HJ(m) : (IT)-1;
  }
#undef HD
#undef HJ
}

template <class T>
__global__ void k_sqrt(const T* __restrict__ a, int64_t n, T* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = ksqrt(a[i]);
}

template <class T>
__global__ void k_row_norms(const T* __restrict__ X, int64_t n, int d, T* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    T s = T(0);
    for (int f = 0; f < d; ++f) s = kfma(X[i * d + f], X[i * d + f], s);
    out[i] = s;
  }
}

template <class T, class IT, int NT, int KMAX, int DR>
void launch_knn(const T* X, const T* norms, const T* snorms, int64_t n, int d, int k, IT* idx, T* dist,
                cudaStream_t s) {
  const size_t smem = (DR > 0 ? (size_t)kKnnTile * DR * sizeof(T)
                              : (size_t)d * NT * sizeof(T) + (size_t)kKnnTile * (d + 1) * sizeof(T)) +
                      (size_t)KMAX * NT * (sizeof(T) + sizeof(int32_t));
  auto kern = k_knn_dense<T, IT, NT, KMAX, DR>;
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t grid = (n + NT - 1) / NT;
  kern<<<(unsigned)grid, NT, smem, s>>>(X, norms, snorms, n, d, k, idx, dist);
  SCL_CUDA(cudaGetLastError());
}

template <class T, class IT>
void knn_typed(const T* X, const T* norms, int64_t n, int d, int k, IT* idx, T* dist, cudaStream_t s) {
  DevBuf sn(std::max<int64_t>(n, 1) * sizeof(T), s);
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  k_sqrt<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(dev) * 8)), 256, 0,
              s>>>(norms, n, sn.as<T>());
  SCL_CUDA(cudaGetLastError());
  constexpr int NT = sizeof(T) == 4 ? 128 : 64;
  const T* sp = sn.as<T>();
  if (k <= 32) {
    if (d <= 16) return launch_knn<T, IT, NT, 32, 16>(X, norms, sp, n, d, k, idx, dist, s);
    if (d <= 32) return launch_knn<T, IT, NT, 32, 32>(X, norms, sp, n, d, k, idx, dist, s);
    return launch_knn<T, IT, NT, 32, 0>(X, norms, sp, n, d, k, idx, dist, s);
  }
  if (d <= 32) return launch_knn<T, IT, NT, 64, 32>(X, norms, sp, n, d, k, idx, dist, s);
  return launch_knn<T, IT, NT, 64, 0>(X, norms, sp, n, d, k, idx, dist, s);
}

}  // namespace

int knn_max_features() { return kKnnMaxD; }

void knn_dense(const void* X, const void* norms, DType t, int64_t n, int d, int k, void* idx, DType it, void* dist,
               cudaStream_t s) {
  SCL_REQUIRE(d >= 1 && d <= kKnnMaxD, kErrInvalidArgument, "kNN on the device takes 1 to 128 features");
  SCL_REQUIRE(k >= 1 && k <= 64, kErrInvalidArgument, "kNN on the device takes k from 1 to 64");
  SCL_REQUIRE(n < (int64_t)0x7fffffff, kErrInvalidArgument, "kNN sample count exceeds the int32 range");
  if (n == 0) return;
  if (t == kF32) {
    if (it == kI32)
      return knn_typed<float, int32_t>(static_cast<const float*>(X), static_cast<const float*>(norms), n, d, k,
                                       static_cast<int32_t*>(idx), static_cast<float*>(dist), s);
    return knn_typed<float, int64_t>(static_cast<const float*>(X), static_cast<const float*>(norms), n, d, k,
                                     static_cast<int64_t*>(idx), static_cast<float*>(dist), s);
  }
  if (it == kI32)
    return knn_typed<double, int32_t>(static_cast<const double*>(X), static_cast<const double*>(norms), n, d, k,
                                      static_cast<int32_t*>(idx), static_cast<double*>(dist), s);
  knn_typed<double, int64_t>(static_cast<const double*>(X), static_cast<const double*>(norms), n, d, k,
                             static_cast<int64_t*>(idx), static_cast<double*>(dist), s);
}

void row_norms_dense(const void* X, DType t, int64_t n, int d, void* out, cudaStream_t s) {
  if (n == 0) return;
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(dev) * 8));
  if (t == kF32)
    k_row_norms<float><<<grid, 256, 0, s>>>(static_cast<const float*>(X), n, d, static_cast<float*>(out));
  else
    k_row_norms<double><<<grid, 256, 0, s>>>(static_cast<const double*>(X), n, d, static_cast<double*>(out));
  SCL_CUDA(cudaGetLastError());
}

}  // namespace sclgpu
