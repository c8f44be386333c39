// Brute-force k-nearest neighbours on CUDA cores (scl/kernel/neighbors.hpp:302-478):
// the graph-building step before the transition matrix. This kernel computes
// every distance exactly; it runs for small sample counts (up to 128 features,
// k up to 64), the tensor-core filter of knn_tc.cu for the rest.
//
// The samples (the handle's primary rows) are made dense on the device, n x d
// with d <= 128 features. Every query walks every candidate j in increasing
// order, exactly as the reference's per-query loop does, so the result (ties
// included) is the reference's: the same Cauchy-Schwarz skip
// ((sqrt(norm_i) - sqrt(norm_j))^2 >= the current k-th distance), the same
// dist_sq = fma(-2, dot, norm_i + norm_j) clamped at 0 with the dot an fma
// chain over the features in order, the same max-heap of k entries (a
// candidate enters while the heap is short, else when strictly below the
// top), and the same heap sort at the end, so equal distances leave in the
// same order. The heap replay is sequential per query; the dot products
// around it are not, and they are the bulk of the work, so a CTA splits the
// two between warps (k_knn_ws below).
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

// k_knn_ws: a CTA owns 32 queries. Warp 0 replays their heaps (one lane per
// query: the reference's skip test, max-heap and heap sort, in candidate
// order) while four dot warps produce the squared distances of the tiles of
// 64 candidates ahead of it. A dot thread holds a 4 x 4 register tile (four
// queries x four consecutive candidates, sixteen independent fma chains over
// the features in order); per feature it reads the four queries (stored
// feature-major) and the four candidates (stored feature-major in 16-byte
// rows) as one 16-byte load each. It writes dist_sq = max(0, fma(-2, dot,
// norm_i + norm_j)) into a shared tile together with a keep mask per query,
// so the heap lane visits only the candidates it may act on. The candidate
// tiles, their norms and root norms are copied into shared memory with
// cp.async one tile ahead of the dot products.
//
// Hand-off: the dist_sq tiles are double-buffered between the two roles with
// named barriers, FULL[b] (the dot warps arrive, the heap warp waits) and
// EMPTY[b] (the heap warp arrives, the dot warps wait), so the dot warps run
// up to two tiles ahead of the replay and neither role waits for the other
// tile by tile; a third barrier, among the dot warps alone, guards their
// candidate buffers. Every barrier phase gets exactly one arrival per thread
// of the two roles for each tile (all trip counts are the CTA-wide tile
// count), so every wait is met.
constexpr int kWsQ = 32;                   // queries per CTA (the heap warp's lanes)
constexpr int kWsDotThreads = 128;         // four dot warps
constexpr int kWsThreads = 32 + kWsDotThreads;
// feature-major candidate pitch and dist_sq row pitch: 16-byte rows (68 floats, 66 doubles)
template <class T>
constexpr int kWsPitch = kKnnTile + 16 / (int)sizeof(T);
constexpr int kBarDot = 1, kBarFull = 2, kBarEmpty = 4;  // named barrier ids (0 is __syncthreads)

template <class T>
size_t knn_ws_smem(int d, int kmax) {
  return (2 * (size_t)kWsQ * kWsPitch<T> + 3 * (size_t)kKnnTile + 2 * (size_t)kKnnTile + (size_t)d * kWsQ +
          2 * (size_t)d * kWsPitch<T> + 3 * kWsQ + (size_t)kmax * kWsQ) * sizeof(T) +
         ((size_t)kmax * kWsQ + kWsQ) * sizeof(int32_t) + 2 * kWsQ * 16;
}

template <class T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}
template <int ID>
__device__ __forceinline__ void bar_sync(int count) {
  asm volatile("bar.sync %0, %1;\n" ::"n"(ID), "r"(count) : "memory");
}
template <int ID>
__device__ __forceinline__ void bar_arrive(int count) {
  asm volatile("bar.arrive %0, %1;\n" ::"n"(ID), "r"(count) : "memory");
}
// barrier ID0 or ID0 + 1 by the parity of a tile index (immediate operands)
template <int ID0>
__device__ __forceinline__ void bar_sync_pair(int64_t u, int count) {
  if (u & 1) bar_sync<ID0 + 1>(count);
  else bar_sync<ID0>(count);
}
template <int ID0>
__device__ __forceinline__ void bar_arrive_pair(int64_t u, int count) {
  if (u & 1) bar_arrive<ID0 + 1>(count);
  else bar_arrive<ID0>(count);
}

// four values from a 16-byte aligned shared address (one or two vector loads)
template <class T>
__device__ __forceinline__ void load4(const T* p, T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
  }
}
template <class T>
__device__ __forceinline__ void store4(T* p, const T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
  }
}

template <class T, class IT, int KMAX>
__global__ void __launch_bounds__(kWsThreads)
k_knn_ws(const T* __restrict__ X, const T* __restrict__ norms, const T* __restrict__ snorms, int64_t n, int d, int k,
         IT* __restrict__ out_idx, T* __restrict__ out_dist) {
  extern __shared__ __align__(16) unsigned char knn_smem[];
  // the regions read with 16-byte vector loads come first, each a multiple of 16 bytes long
  T* Ds = reinterpret_cast<T*>(knn_smem);      // [2][32][pitch] dist_sq
  T* Ss = Ds + 2 * kWsQ * kWsPitch<T>;         // [3][64] candidate root norms
  T* Ns = Ss + 3 * kKnnTile;                   // [2][64] candidate norms
  T* Qs = Ns + 2 * kKnnTile;                   // [d][32] queries, feature-major
  T* Cs = Qs + (size_t)d * kWsQ;               // [2][d][pitch] candidates, feature-major
  T* Qn = Cs + 2 * (size_t)d * kWsPitch<T>;    // [32] query norms
  T* Qr = Qn + kWsQ;                           // [32] query root norms
  volatile T* Mx = Qr + kWsQ;                  // [32] published k-th distance (max while the heap fills)
  T* Hd = const_cast<T*>(Mx) + kWsQ;           // [KMAX][32] heap distances
  int32_t* Hj = reinterpret_cast<int32_t*>(Hd + (size_t)KMAX * kWsQ);  // [KMAX][32] heap indices
  volatile int32_t* Fl = Hj + (size_t)KMAX * kWsQ;  // [32] published heap-full flag
  uint8_t* Km = reinterpret_cast<uint8_t*>(const_cast<int32_t*>(Fl) + kWsQ);  // [2][32][16] keep nibbles
  const int tid = threadIdx.x;
  const int64_t q0 = (int64_t)blockIdx.x * kWsQ;
  const int nq = (n - q0) < (int64_t)kWsQ ? (int)(n - q0) : kWsQ;
  const int64_t ntiles = (n + kKnnTile - 1) / kKnnTile;

  for (int e = tid; e < kWsQ * d; e += kWsThreads) {  // queries past n are zero
    const int r = e / d, f = e - r * d;
    Qs[f * kWsQ + r] = r < nq ? X[(q0 + r) * (int64_t)d + f] : T(0);
  }
  if (tid < kWsQ) {
    Qn[tid] = tid < nq ? norms[q0 + tid] : T(0);
    Qr[tid] = tid < nq ? snorms[q0 + tid] : T(0);
    Mx[tid] = std::numeric_limits<T>::max();
    Fl[tid] = 0;
  }
  __syncthreads();

  if (tid >= 32) {
    // ---------------- dot warps ----------------
    const int dt = tid - 32;
    // copy candidate tile u into its buffers (asynchronous)
    auto stage = [&](int64_t u) {
      const int64_t t0 = u * kKnnTile;
      const int tn = (n - t0) < (int64_t)kKnnTile ? (int)(n - t0) : kKnnTile;
      T* cs = Cs + (size_t)(u & 1) * d * kWsPitch<T>;
      const T* src = X + t0 * (int64_t)d;
      int r = dt / d, f = dt - (dt / d) * d;
      const int sr = kWsDotThreads / d, sf = kWsDotThreads - sr * d;
      for (int e = dt; e < tn * d; e += kWsDotThreads) {
        cp_async_elem(cs + f * kWsPitch<T> + r, src + e);
        f += sf;
        r += sr;
        if (f >= d) {
          f -= d;
          ++r;
        }
      }
      if (dt < tn) {
        cp_async_elem(Ns + (u & 1) * kKnnTile + dt, norms + t0 + dt);
        cp_async_elem(Ss + (u % 3) * kKnnTile + dt, snorms + t0 + dt);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    const int qg = (dt >> 4) * 4, c4 = (dt & 15) * 4;
    T qn[4], qr[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) qn[a] = Qn[qg + a], qr[a] = Qr[qg + a];
    stage(0);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    for (int64_t u = 0; u < ntiles; ++u) {
      // every dot thread's copy of tile u has landed and every dot thread is
      // done with tile u - 1, whose candidate buffers the copy of u + 1 reuses
      bar_sync<kBarDot>(kWsDotThreads);
      // the heap warp is done with tile u - 2: its dist_sq buffer is free, and
      // so is the root-norm slot (u + 1) % 3 == (u - 2) % 3
      if (u >= 2) bar_sync_pair<kBarEmpty>(u, kWsThreads);
      if (u + 1 < ntiles) stage(u + 1);
      const T* cs = Cs + (size_t)(u & 1) * d * kWsPitch<T> + c4;
      const T* qs = Qs + qg;
      T acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int m = 0; m < 4; ++m) acc[a][m] = T(0);
#pragma unroll 2
      for (int f = 0; f < d; ++f) {
        T qv[4], cv[4];
        load4(qs + f * kWsQ, qv);
        load4(cs + f * kWsPitch<T>, cv);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int m = 0; m < 4; ++m) acc[a][m] = kfma(qv[a], cv[m], acc[a][m]);
      }
      T nv[4], sv[4];
      load4(Ns + (u & 1) * kKnnTile + c4, nv);
      load4(Ss + (u % 3) * kKnnTile + c4, sv);
      T* ds = Ds + (size_t)(u & 1) * kWsQ * kWsPitch<T> + c4;
      const int64_t t0 = u * kKnnTile;
      const int tn = (n - t0) < (int64_t)kKnnTile ? (int)(n - t0) : kKnnTile;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        // The keep mask of these four candidates for query qg + a, from the
        // k-th distance and count the heap lane last published. Both only
        // move one way (the distance down, the count up), and the heap lane
        // is at most two tiles behind, so the mask keeps every candidate the
        // replay could act on; the heap lane re-tests the kept ones exactly.
        const T M = Mx[qg + a];
        const bool full = Fl[qg + a] != 0;
        const int64_t self = q0 + qg + a - t0;
        T o[4];
        unsigned nib = 0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const T v = kfma(T(-2), acc[a][m], qn[a] + nv[m]);
          o[m] = v < T(0) ? T(0) : v;
          const T nd = qr[a] - sv[m];
          const bool act = c4 + m < tn && (int64_t)(c4 + m) != self && !(nd * nd >= M) && (!full || o[m] < M);
          nib |= act ? (1u << m) : 0u;
        }
        store4(ds + (qg + a) * kWsPitch<T>, o);
        Km[((u & 1) * kWsQ + qg + a) * 16 + (c4 >> 2)] = (uint8_t)nib;
      }
      bar_arrive_pair<kBarFull>(u, kWsThreads);  // tile u's dist_sq is ready
      asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    return;
  }

  // ---------------- heap warp ----------------
  const int64_t i = q0 + tid;
  const bool live = i < n;
  const T si = live ? snorms[i] : T(0);
  T maxd = std::numeric_limits<T>::max();
  int cnt = 0;
#define HD(p) Hd[(p) * kWsQ + tid]
#define HJ(p) Hj[(p) * kWsQ + tid]
  auto swap_at = [&](int a, int b) {
    const T td = HD(a);
    const int32_t tj = HJ(a);
    HD(a) = HD(b);
    HJ(a) = HJ(b);
    HD(b) = td;
    HJ(b) = tj;
  };
  for (int64_t t = 0; t < ntiles; ++t) {
    bar_sync_pair<kBarFull>(t, kWsThreads);  // tile t's dist_sq (and its root norms) are in place
    if (live) {
      const int64_t t0 = t * kKnnTile;
      const T* dsr = Ds + (size_t)(t & 1) * kWsQ * kWsPitch<T> + tid * kWsPitch<T>;
      const T* ss = Ss + (t % 3) * kKnnTile;
      // the kept candidates of this tile in increasing order: byte j of the
      // row holds the nibble of candidates 4j .. 4j + 3
      const uint4 km = *reinterpret_cast<const uint4*>(Km + ((t & 1) * kWsQ + tid) * 16);
      const unsigned words[4] = {km.x, km.y, km.z, km.w};
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        unsigned keep = words[w];
        while (keep) {
          const int bit = __ffs(keep) - 1;
          keep &= keep - 1;
          const int c = 16 * w + 4 * (bit >> 3) + (bit & 7);
          const T nd = si - ss[c];
          if (nd * nd >= maxd) continue;  // reference's lower-bound skip
          const T ds = dsr[c];
          if (cnt < k) {
            int pos = cnt;
            HD(pos) = ds;
            HJ(pos) = (int32_t)(t0 + c);
            while (pos > 0) {  // sift up
              const int parent = (pos - 1) / 2;
              if (HD(pos) <= HD(parent)) break;
              swap_at(pos, parent);
              pos = parent;
            }
            ++cnt;
            if (cnt == k) maxd = HD(0);
          } else if (ds < maxd) {  // maxd is the heap top once the heap is full
            HD(0) = ds;
            HJ(0) = (int32_t)(t0 + c);
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
    if (live) {
      Mx[tid] = maxd;
      Fl[tid] = cnt >= k ? 1 : 0;
    }
    __syncwarp();
    if (t + 2 < ntiles) bar_arrive_pair<kBarEmpty>(t, kWsThreads);  // the dot warps may refill this buffer
  }

  if (!live) return;
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

template <class T, class IT, int KMAX>
void launch_knn_ws(const T* X, const T* norms, const T* snorms, int64_t n, int d, int k, IT* idx, T* dist,
                   cudaStream_t s) {
  const size_t smem = knn_ws_smem<T>(d, KMAX);
  int dev = 0, optin = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  SCL_REQUIRE(smem <= (size_t)optin, kErrInvalidArgument, "kNN tile buffers exceed the device's shared memory");
  auto kern = k_knn_ws<T, IT, KMAX>;
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)((n + kWsQ - 1) / kWsQ), kWsThreads, smem, s>>>(X, norms, snorms, n, d, k, idx, dist);
  SCL_CUDA(cudaGetLastError());
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

template <class T, class IT>
void knn_typed(const T* X, const T* norms, int64_t n, int d, int k, IT* idx, T* dist, cudaStream_t s) {
  DevBuf sn(std::max<int64_t>(n, 1) * sizeof(T), s);
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  k_sqrt<T><<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count(dev) * 8)), 256, 0,
              s>>>(norms, n, sn.as<T>());
  SCL_CUDA(cudaGetLastError());
  const T* sp = sn.as<T>();
  if (k <= 32) return launch_knn_ws<T, IT, 32>(X, norms, sp, n, d, k, idx, dist, s);
  launch_knn_ws<T, IT, 64>(X, norms, sp, n, d, k, idx, dist, s);
}

}  // namespace

int knn_max_features() { return kKnnMaxD; }

namespace {
// 0: automatic, 1: the warp-specialised CUDA-core kernel above, 2: the tensor-core filter (knn_tc.cu)
int g_knn_kernel = 0;
// below this many samples the CUDA-core kernel fills the GPU better (a tensor-core CTA takes 256 queries)
constexpr int64_t kKnnTensorMinSamples = 24576;
}

int knn_set_kernel(int kernel) {
  SCL_REQUIRE(kernel >= 0 && kernel <= 2, kErrInvalidArgument,
              "kNN kernel must be 0 (automatic), 1 (CUDA cores) or 2 (tensor cores)");
  const int prev = g_knn_kernel;
  g_knn_kernel = kernel;
  return prev;
}

void knn_dense(const void* X, const void* norms, DType t, int64_t n, int d, int k, void* idx, DType it, void* dist,
               cudaStream_t s) {
  SCL_REQUIRE(d >= 1 && k >= 1, kErrInvalidArgument, "Dimensions must be positive");
  SCL_REQUIRE(n < (int64_t)0x7fffffff, kErrInvalidArgument, "kNN sample count exceeds the int32 range");
  if (n == 0) return;
  const bool cuda_cores_fit = d <= kKnnMaxD && k <= 64;
  const bool tensor = g_knn_kernel == 2 || (g_knn_kernel == 0 && (!cuda_cores_fit || n >= kKnnTensorMinSamples));
  if (tensor) return knn_tensor(X, norms, t, n, d, k, idx, it, dist, s);
  SCL_REQUIRE(d <= kKnnMaxD, kErrInvalidArgument, "the CUDA-core kNN kernel takes 1 to 128 features");
  SCL_REQUIRE(k <= 64, kErrInvalidArgument, "the CUDA-core kNN kernel takes k from 1 to 64");
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
