// CSR x dense SpMM for the diffusion power iteration X_{s+1} = P X_s.
//
// Replaces scl-core's spmm_block (scl/kernel/diffusion.hpp:227-278) and the
// diffuse_matrix loop (diffusion.hpp:638-664).
//
// Mapping: a group of G lanes owns one output row; lane l of the group owns a
// VEC-wide column chunk (16 bytes of X per lane when the row pitch allows it,
// else one element). The group walks the row's nonzeros in stored order:
// G (index, value) pairs are fetched cooperatively with one coalesced load and
// broadcast by shuffles, then U gathered X rows are loaded back-to-back before
// their FMAs, so each lane keeps U 16-byte loads in flight. Every output
// element is therefore the sequential chain acc = fma(v_k, X[j_k, c], acc) over
// the row's nonzeros in CSR order — the same rounding sequence as the
// reference's axpy_simd (Highway MulAdd), which makes FP32/FP64 results
// bit-identical to scl-core on the same P and X.
//
// Precision forms: values/X in f32, f64, bf16 or f16 (storage), accumulation
// in f32 (f64 when either operand is f64), output in the storage type or f32.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdio>
#include <type_traits>

#include "chunk_cursor.cuh"
#include "engine.hpp"

namespace sclgpu {
namespace {

// ---- element conversions ---------------------------------------------------
template <class T> __device__ __forceinline__ float tof(T v);
template <> __device__ __forceinline__ float tof<float>(float v) { return v; }
template <> __device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float tof<__half>(__half v) { return __half2float(v); }

template <class A, class T> __device__ __forceinline__ A to_acc(T v) { return (A)tof<T>(v); }
template <> __device__ __forceinline__ double to_acc<double, double>(double v) { return v; }
template <> __device__ __forceinline__ float to_acc<float, float>(float v) { return v; }

template <class Y, class A> __device__ __forceinline__ Y from_acc(A v);
template <> __device__ __forceinline__ float from_acc<float, float>(float v) { return v; }
template <> __device__ __forceinline__ double from_acc<double, double>(double v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_acc<__nv_bfloat16, float>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_acc<__half, float>(float v) { return __float2half_rn(v); }

__device__ __forceinline__ float fma_acc(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_acc(double a, double b, double c) { return __fma_rn(a, b, c); }

// ---- vector load / store of VEC contiguous elements ------------------------
// Lane chunks of 4, 8 or 16 bytes are loaded with one vector instruction.
template <int BYTES> struct RawVec;
template <> struct RawVec<4> { using type = unsigned int; };
template <> struct RawVec<8> { using type = uint2; };
template <> struct RawVec<16> { using type = uint4; };

template <class T, int VEC>
struct VecIO {
  static constexpr int BYTES = VEC * (int)sizeof(T);
  static_assert(VEC == 1 || BYTES == 4 || BYTES == 8 || BYTES == 16, "lane chunk must be 4, 8 or 16 bytes");
  template <class A>
  static __device__ __forceinline__ void load(const T* __restrict__ p, A (&out)[VEC]) {
    if constexpr (VEC == 1) {
      out[0] = to_acc<A, T>(__ldg(p));
    } else {
      using R = typename RawVec<BYTES>::type;
      const R raw = __ldg(reinterpret_cast<const R*>(p));
      const T* e = reinterpret_cast<const T*>(&raw);
#pragma unroll
      for (int i = 0; i < VEC; ++i) out[i] = to_acc<A, T>(e[i]);
    }
  }
};

template <class T, int VEC>
struct VecStore {
  template <class A>
  static __device__ __forceinline__ void store(T* __restrict__ p, const A (&in)[VEC]) {
    constexpr int BYTES = VEC * (int)sizeof(T);
    if constexpr (VEC == 1) {
      p[0] = from_acc<T, A>(in[0]);
    } else if constexpr (BYTES == 16) {
      uint4 raw;
      T* e = reinterpret_cast<T*>(&raw);
#pragma unroll
      for (int i = 0; i < VEC; ++i) e[i] = from_acc<T, A>(in[i]);
      __stcs(reinterpret_cast<uint4*>(p), raw);  // streaming store: Y is not re-read this step
    } else if constexpr (BYTES == 32) {  // f32 output of a bf16/f16 (8-wide) chunk
      uint4 raw[2];
      T* e = reinterpret_cast<T*>(raw);
#pragma unroll
      for (int i = 0; i < VEC; ++i) e[i] = from_acc<T, A>(in[i]);
      __stcs(reinterpret_cast<uint4*>(p), raw[0]);
      __stcs(reinterpret_cast<uint4*>(p) + 1, raw[1]);
    } else if constexpr (BYTES == 8 || BYTES == 4) {
      using R = typename RawVec<BYTES>::type;
      R raw;
      T* e = reinterpret_cast<T*>(&raw);
#pragma unroll
      for (int i = 0; i < VEC; ++i) e[i] = from_acc<T, A>(in[i]);
      *reinterpret_cast<R*>(p) = raw;
    } else {
#pragma unroll
      for (int i = 0; i < VEC; ++i) p[i] = from_acc<T, A>(in[i]);
    }
  }
};

template <class V>
__device__ __forceinline__ V shfl_val(unsigned mask, V v, int src, int width) {
  return __shfl_sync(mask, v, src, width);
}
template <>
__device__ __forceinline__ __nv_bfloat16 shfl_val<__nv_bfloat16>(unsigned mask, __nv_bfloat16 v, int src, int width) {
  unsigned short u = __bfloat16_as_ushort(v);
  u = (unsigned short)__shfl_sync(mask, (unsigned)u, src, width);
  return __ushort_as_bfloat16(u);
}
template <>
__device__ __forceinline__ __half shfl_val<__half>(unsigned mask, __half v, int src, int width) {
  unsigned short u = __half_as_ushort(v);
  u = (unsigned short)__shfl_sync(mask, (unsigned)u, src, width);
  return __ushort_as_half(u);
}

// ---- the kernel -------------------------------------------------------------
// G lanes per row, VEC elements per lane per pass, U gathers in flight.
template <class VT, class XT, class YT, class AT, int G, int VEC, int U>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
       const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows,
       int64_t F) {
  const int lane = threadIdx.x & 31;
  const int lg = lane & (G - 1);                       // lane within group
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  // Persistent grid: each lane group walks rows gid, gid + n_groups, ... so a
  // group that finishes a short row immediately takes another (row lengths
  // are heavily skewed; whole groups advance together since G divides 32).
  const int64_t n_groups = ((int64_t)gridDim.x * kSpmmThreads) / G;
  for (int64_t row = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) / G; row < n_rows; row += n_groups) {
  const int64_t start = indptr[row];
  const int64_t end = indptr[row + 1];
  const int64_t out_row = row_map ? (int64_t)row_map[row] : row;
  constexpr int CPP = G * VEC;  // columns per pass

  for (int64_t c0 = 0; c0 < F; c0 += CPP) {
    const int64_t col = c0 + (int64_t)lg * VEC;
    const bool active = col < F;  // VEC divides F on the vector path
    AT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
    const XT* __restrict__ Xc = X + col;

    for (int64_t base = start; base < end; base += G) {
      const int64_t m = base + lg;
      int32_t j_l = 0;
      VT v_l = VT(0);
      if (m < end) {
        // the CSR stream is read once per step: evict-first, keep L2 for X
        j_l = __ldcs(indices + m);
        v_l = __ldcs(values + m);
      }
      const int cnt = (int)((end - base) < G ? (end - base) : G);
      int t = 0;
      if constexpr (U > 1) {
        for (; t + U <= cnt; t += U) {
          AT xv[U][VEC];
          AT vv[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int32_t jj = __shfl_sync(gmask, j_l, t + u, G);
            vv[u] = to_acc<AT, VT>(shfl_val<VT>(gmask, v_l, t + u, G));
            if (active) VecIO<XT, VEC>::load(Xc + (int64_t)jj * F, xv[u]);
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vv[u], xv[u][i], acc[i]);
          }
        }
      }
      for (; t < cnt; ++t) {
        const int32_t jj = __shfl_sync(gmask, j_l, t, G);
        const AT vv = to_acc<AT, VT>(shfl_val<VT>(gmask, v_l, t, G));
        AT xv[VEC];
        if (active) {
          VecIO<XT, VEC>::load(Xc + (int64_t)jj * F, xv);
#pragma unroll
          for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vv, xv[i], acc[i]);
        }
      }
    }
    if (active) VecStore<YT, VEC>::store(Y + out_row * F + col, acc);
  }
  }  // rows
}

// ---- pipelined variant: gathered rows land in shared memory via cp.async ----
// Same lane mapping and the same per-element fma order as k_spmm. A group of G
// lanes processes its row in chunks of S entries: lane t of the group loads
// entry t's (index, value) (one coalesced load), then every lane issues S
// 16-byte cp.async copies of ITS column chunk of the S gathered X rows into a
// double-buffered stage. While stage c is consumed (ld.shared + fma), stage
// c+1's indices and copies are already in flight, so memory latency overlaps
// the math and in-flight data costs no registers. Each lane only reads back the
// bytes it copied itself, so per-thread cp.async.wait_group is the only
// synchronisation needed. Requires the 16-byte vector mapping (VEC*sizeof(XT)
// == 16) and S <= G.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int S>
constexpr int pipe_smem_bytes() { return kSpmmThreads * 2 * S * 16; }

template <class VT, class XT, class YT, class AT, int G, int VEC, int S>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_pipe(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
            const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows,
            int64_t F) {
  static_assert(VEC * sizeof(XT) == 16, "pipelined SpMM needs 16-byte lane chunks");
  static_assert(S <= G, "stage size must not exceed the group size");
  extern __shared__ uint4 smem_pipe[];
  const int lane = threadIdx.x & 31;
  const int lg = lane & (G - 1);
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  // this lane's slots: stage b, entry t -> smem_pipe[((b * S + t) * kSpmmThreads) + threadIdx.x]
  uint4* my = smem_pipe + threadIdx.x;
  const int64_t n_groups = ((int64_t)gridDim.x * kSpmmThreads) / G;
  for (int64_t row = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) / G; row < n_rows; row += n_groups) {
  const int64_t start = indptr[row];
  const int64_t end = indptr[row + 1];
  const int64_t out_row = row_map ? (int64_t)row_map[row] : row;
  constexpr int CPP = G * VEC;

  for (int64_t c0 = 0; c0 < F; c0 += CPP) {
    const int64_t col = c0 + (int64_t)lg * VEC;
    const bool active = col < F;
    const XT* __restrict__ Xc = X + col;
    AT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = AT(0);

    // chunk c covers entries [start + c*S, start + c*S + S)
    int32_t j_cur = 0;
    VT v_cur = VT(0);
    {
      const int64_t m = start + lg;
      if (lg < S && m < end) {
        j_cur = __ldcs(indices + m);
        v_cur = __ldcs(values + m);
      }
    }
    auto issue = [&](int stage, int32_t jreg, int64_t base) {
      const int cnt = (int)((end - base) < S ? (end - base) : S);
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const int32_t jj = __shfl_sync(gmask, jreg, t, G);
        if (t < cnt && active) cp_async16(my + (stage * S + t) * kSpmmThreads, Xc + (int64_t)jj * F);
      }
      cp_async_commit();
    };
    if (start < end) issue(0, j_cur, start);
    int stage = 0;
    for (int64_t base = start; base < end; base += S) {
      const int cnt = (int)((end - base) < S ? (end - base) : S);
      const int64_t nbase = base + S;
      int32_t j_nxt = 0;
      VT v_nxt = VT(0);
      if (nbase < end) {
        const int64_t m = nbase + lg;
        if (lg < S && m < end) {
          j_nxt = __ldcs(indices + m);
          v_nxt = __ldcs(values + m);
        }
        issue(stage ^ 1, j_nxt, nbase);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
#pragma unroll
      for (int t = 0; t < S; ++t) {
        if (t < cnt) {
          const AT vv = to_acc<AT, VT>(shfl_val<VT>(gmask, v_cur, t, G));
          if (active) {
            const uint4 raw = my[(stage * S + t) * kSpmmThreads];
            const XT* e = reinterpret_cast<const XT*>(&raw);
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vv, to_acc<AT, XT>(e[i]), acc[i]);
          }
        }
      }
      j_cur = j_nxt;
      v_cur = v_nxt;
      stage ^= 1;
    }
    if (active) VecStore<YT, VEC>::store(Y + out_row * F + col, acc);
  }
  }  // rows
}

// ---- streaming variant: a warp walks the nonzero stream of a row block --------
// A warp takes a task of up to 31 consecutive rows (lane l holds indptr[r0+l])
// and walks their contiguous entries [indptr[r0], indptr[r1]) in chunks of 32:
// each chunk's (index, value) pairs are loaded one chunk ahead, and gathers are
// issued in predicated batches of U regardless of where rows begin or end, so
// no row pays a fresh index->gather latency chain and no tail runs one load at
// a time. A warp-uniform test e >= row_end flushes the finished row (its
// accumulator is stored and reset) — rows with no entries are flushed as
// zeros. Every row still accumulates exactly its own entries in stored order,
// the same fma sequence as k_spmm. One warp covers a row with VEC elements per
// lane (4-, 8- or 16-byte chunks); wider rows take several column passes.
constexpr int kStreamRows = 31;

template <class VT, class XT, class YT, class AT, int VEC, int U>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_stream(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
              const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows,
              int64_t F) {
  const int lane = threadIdx.x & 31;
  const int64_t n_warps = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  const int64_t n_tasks = (n_rows + kStreamRows - 1) / kStreamRows;
  constexpr int CPP = 32 * VEC;
  for (int64_t task = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5; task < n_tasks; task += n_warps) {
    const int64_t r0 = task * kStreamRows;
    const int nr = (int)((n_rows - r0) < kStreamRows ? (n_rows - r0) : kStreamRows);
    const int64_t ptr_l = (lane <= nr) ? __ldcs(indptr + r0 + lane) : 0;
    const int64_t p0 = __shfl_sync(0xffffffffu, ptr_l, 0);
    const int64_t p1 = __shfl_sync(0xffffffffu, ptr_l, nr);
    for (int64_t c0 = 0; c0 < F; c0 += CPP) {
      const int64_t col = c0 + (int64_t)lane * VEC;
      const bool active = col < F;
      const XT* __restrict__ Xc = X + col;
      AT acc[VEC];
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
      int ri = 0;  // current row = r0 + ri
      int64_t row_end = __shfl_sync(0xffffffffu, ptr_l, 1);
      auto flush = [&]() {
        if (active) {
          const int64_t r = r0 + ri;
          const int64_t orow = row_map ? (int64_t)row_map[r] : r;
          VecStore<YT, VEC>::store(Y + orow * F + col, acc);
        }
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
        ++ri;
        if (ri < nr) row_end = __shfl_sync(0xffffffffu, ptr_l, ri + 1);
      };
      int32_t j_n = 0;
      VT v_n = VT(0);
      if (p0 + lane < p1) {
        j_n = __ldcs(indices + p0 + lane);
        v_n = __ldcs(values + p0 + lane);
      }
      for (int64_t c = p0; c < p1; c += 32) {
        const int32_t j_l = j_n;
        const VT v_l = v_n;
        const int64_t mn = c + 32 + lane;
        if (mn < p1) {  // next chunk's pairs are in flight during this chunk
          j_n = __ldcs(indices + mn);
          v_n = __ldcs(values + mn);
        }
        const int cnt = (int)((p1 - c) < 32 ? (p1 - c) : 32);
#pragma unroll
        for (int t = 0; t < 32; t += U) {
          if (t >= cnt) break;
          AT xv[U][VEC];
          AT vv[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int32_t jj = __shfl_sync(0xffffffffu, j_l, t + u);
            vv[u] = to_acc<AT, VT>(shfl_val<VT>(0xffffffffu, v_l, t + u, 32));
            if (t + u < cnt && active) VecIO<XT, VEC>::load(Xc + (int64_t)jj * F, xv[u]);
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (t + u < cnt) {
              const int64_t e = c + t + u;
              while (e >= row_end) flush();
              if (active) {
#pragma unroll
                for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vv[u], xv[u][i], acc[i]);
              }
            }
          }
        }
      }
      while (ri < nr) flush();  // last row with entries, then trailing empty rows
    }
  }
}

// ---- stream + cp.async pipeline ------------------------------------------------
// The row-block stream of k_spmm_stream with the gathers decoupled from the
// consumer: for each chunk of S entries every lane fires S cp.async copies of
// its LB-byte column chunk of the gathered X rows into a double-buffered stage
// (lane-private slots, so the per-thread cp.async.wait_group is the only
// synchronisation), then consumes the previous stage in entry order — fma into
// the current row's accumulator, flushing rows as the stream crosses indptr.
// Index/value pairs are prefetched two chunks ahead, so neither the index loads
// nor the gathers sit on the consumer's critical path. Same fma sequence per
// row as every other variant.
template <int LB>
__device__ __forceinline__ void cp_async_lb(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (LB == 16) asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else if constexpr (LB == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <int LB, int S>
constexpr int stream_pipe_smem_bytes() { return (kSpmmThreads / 32) * 2 * S * 32 * LB; }

template <class VT, class XT, class YT, class AT, int VEC, int S>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_spipe(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
             const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows,
             int64_t F) {
  constexpr int LB = VEC * (int)sizeof(XT);
  static_assert(LB == 4 || LB == 8 || LB == 16, "lane chunk must be 4, 8 or 16 bytes");
  static_assert(S <= 32, "a stage holds at most one chunk of 32 entries");
  using R = typename RawVec<LB>::type;
  extern __shared__ uint4 smem_spipe[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  // slot (stage b, entry t) of this lane: base + ((b * S + t) * 32 + lane) * LB bytes
  char* wbase = reinterpret_cast<char*>(smem_spipe) + (size_t)warp_in_block * 2 * S * 32 * LB;
  auto slot = [&](int b, int t) -> R* { return reinterpret_cast<R*>(wbase + ((size_t)(b * S + t) * 32 + lane) * LB); };
  const int64_t n_warps = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  const int64_t n_tasks = (n_rows + kStreamRows - 1) / kStreamRows;
  constexpr int CPP = 32 * VEC;
  for (int64_t task = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5; task < n_tasks; task += n_warps) {
    const int64_t r0 = task * kStreamRows;
    const int nr = (int)((n_rows - r0) < kStreamRows ? (n_rows - r0) : kStreamRows);
    const int64_t ptr_l = (lane <= nr) ? __ldcs(indptr + r0 + lane) : 0;
    const int64_t p0 = __shfl_sync(0xffffffffu, ptr_l, 0);
    const int64_t p1 = __shfl_sync(0xffffffffu, ptr_l, nr);
    for (int64_t c0 = 0; c0 < F; c0 += CPP) {
      const int64_t col = c0 + (int64_t)lane * VEC;
      const bool active = col < F;
      const XT* __restrict__ Xc = X + (active ? col : 0);
      AT acc[VEC];
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
      int ri = 0;
      int64_t row_end = __shfl_sync(0xffffffffu, ptr_l, 1);
      // pairs of chunk k live in lane t < S as (j_k, v_k); chunks start at p0 + k*S
      auto load_pair = [&](int64_t base, int32_t& j, VT& v) {
        const int64_t m = base + lane;
        j = 0;
        v = VT(0);
        if (lane < S && m < p1) {
          j = __ldcs(indices + m);
          v = __ldcs(values + m);
        }
      };
      auto issue = [&](int b, int32_t j, int64_t base) {
        const int cnt = (int)((p1 - base) < S ? (p1 - base) : S);
#pragma unroll
        for (int t = 0; t < S; ++t) {
          const int32_t jj = __shfl_sync(0xffffffffu, j, t);
          if (t < cnt && active) cp_async_lb<LB>(slot(b, t), Xc + (int64_t)jj * F);
        }
        cp_async_commit();
      };
      int32_t j0, j1;
      VT v0, v1;
      load_pair(p0, j0, v0);
      load_pair(p0 + S, j1, v1);
      if (p0 < p1) issue(0, j0, p0);
      int b = 0;
      for (int64_t c = p0; c < p1; c += S) {
        // chunk c: pairs (j0, v0), data in stage b; chunk c+S: pairs (j1, v1)
        int32_t j2;
        VT v2;
        load_pair(c + 2 * S, j2, v2);
        if (c + S < p1) {
          issue(b ^ 1, j1, c + S);
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        const int cnt = (int)((p1 - c) < S ? (p1 - c) : S);
#pragma unroll
        for (int t = 0; t < S; ++t) {
          if (t < cnt) {
            const int64_t e = c + t;
            while (e >= row_end) {
              if (active) {
                const int64_t r = r0 + ri;
                const int64_t orow = row_map ? (int64_t)row_map[r] : r;
                VecStore<YT, VEC>::store(Y + orow * F + col, acc);
              }
#pragma unroll
              for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
              ++ri;
              row_end = __shfl_sync(0xffffffffu, ptr_l, ri + 1 <= nr ? ri + 1 : nr);
            }
            const AT vv = to_acc<AT, VT>(shfl_val<VT>(0xffffffffu, v0, t, 32));
            if (active) {
              const R raw = *slot(b, t);
              const XT* ex = reinterpret_cast<const XT*>(&raw);
#pragma unroll
              for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vv, to_acc<AT, XT>(ex[i]), acc[i]);
            }
          }
        }
        j0 = j1; v0 = v1;
        j1 = j2; v1 = v2;
        b ^= 1;
      }
      // the row holding the last entry, then trailing empty rows
      while (ri < nr) {
        if (active) {
          const int64_t r = r0 + ri;
          const int64_t orow = row_map ? (int64_t)row_map[r] : r;
          VecStore<YT, VEC>::store(Y + orow * F + col, acc);
        }
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
        ++ri;
      }
    }
  }
}

// ---- fixed-pitch warp-per-row kernel (the hot path for 128/256/512-byte rows) --
// One warp per row, lane l owning bytes [l*LB, (l+1)*LB) of every gathered row,
// with the row pitch ROWB = 32*LB a compile-time constant: a gather address is
// one wide multiply-add of the 32-bit column index and the lane offset folds
// into the load. The row's (index, value) pairs are staged 32 at a time in a
// per-warp shared-memory double buffer (values already widened to the
// accumulator type) and read back with 128-bit broadcast loads, 4 entries per
// load — shuffles would cost two shared-pipe operations per entry. Full
// batches of U gathers issue without predicates; only a row's last batch is
// predicated. While a chunk is consumed the next one (the rest of the row, or
// the next row's first chunk) is already in flight, and row bounds are fetched
// a row ahead, so a row start costs one gather latency. Same per-element fma
// order as every other variant.
// OFF32: X spans < 4 GiB, so gather offsets are 32-bit from the uniform base.
template <class VT, class XT, class YT, class AT, int ROWB, int U, bool OFF32>
__global__ void __launch_bounds__(kSpmmThreads, (U == 8) ? 4 : ((U == 16) ? 3 : 1))
k_spmm_row(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
           const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows) {
  constexpr int LB = ROWB / 32;
  constexpr int VEC = LB / (int)sizeof(XT);
  constexpr int WARPS = kSpmmThreads / 32;
  static_assert(LB == 4 || LB == 8 || LB == 16, "row pitch must be 128, 256 or 512 bytes");
  static_assert(U == 8 || U == 16 || U == 32, "batch must divide 32");
  static_assert(sizeof(AT) == 4 || sizeof(AT) == 8, "accumulator is f32 or f64");
  using R = typename RawVec<LB>::type;
  __shared__ __align__(16) int32_t s_j[WARPS][2][32];
  __shared__ __align__(16) AT s_v[WARPS][2][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  int64_t row = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5;
  if (row >= n_rows) return;
  const char* __restrict__ Xb = reinterpret_cast<const char*>(X);
  const char* __restrict__ Xl = Xb + lane * LB;
  const uint32_t lofs = (uint32_t)(lane * LB);
  auto gather = [&](int32_t j) -> R {
    if constexpr (OFF32) return __ldg(reinterpret_cast<const R*>(Xb + ((uint32_t)j * (uint32_t)ROWB + lofs)));
    else return __ldg(reinterpret_cast<const R*>(Xl + (size_t)(uint32_t)j * ROWB));
  };
  // bounds of this row and the next are known; the one after is fetched a row ahead
  int64_t s_cur = indptr[row], e_cur = indptr[row + 1];
  int64_t s_nx = 0, e_nx = 0;
  if (row + nw < n_rows) {
    s_nx = indptr[row + nw];
    e_nx = indptr[row + nw + 1];
  }
  auto fetch = [&](int64_t pos, int64_t end, int32_t& j, AT& v) {
    j = 0;
    v = AT(0);
    if (pos < end) {
      j = __ldcs(indices + pos);
      v = to_acc<AT, VT>(__ldcs(values + pos));
    }
  };
  int buf = 0;
  {
    int32_t j;
    AT v;
    fetch(s_cur + lane, e_cur, j, v);
    s_j[w][0][lane] = j;
    s_v[w][0][lane] = v;
    __syncwarp();
  }
  for (; row < n_rows; row += nw) {
    const int64_t nn = row + 2 * nw;
    int64_t s_nn = 0, e_nn = 0;
    if (nn < n_rows) {
      s_nn = indptr[nn];
      e_nn = indptr[nn + 1];
    }
    AT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
    const int len = (int)(e_cur - s_cur);
    for (int base = 0; base < len; base += 32) {
      // next chunk in flight: the rest of this row, else the next row's first
      int32_t j_n;
      AT v_n;
      if (base + 32 < len) fetch(s_cur + base + 32 + lane, e_cur, j_n, v_n);
      else fetch(s_nx + lane, e_nx, j_n, v_n);
      const int cnt = (len - base) < 32 ? (len - base) : 32;
      const int32_t* __restrict__ jb = s_j[w][buf];
      const AT* __restrict__ vb = s_v[w][buf];
#pragma unroll
      for (int t = 0; t < 32; t += U) {
        if (t >= cnt) break;
        // gather phase: indices from shared memory, U loads in flight
        R xr[U];
        const bool full = (t + U <= cnt);
#pragma unroll
        for (int q = 0; q < U; q += 4) {
          const int4 j4 = *reinterpret_cast<const int4*>(jb + t + q);
          if (full) {
            xr[q] = gather(j4.x);
            xr[q + 1] = gather(j4.y);
            xr[q + 2] = gather(j4.z);
            xr[q + 3] = gather(j4.w);
          } else {
            if (t + q < cnt) xr[q] = gather(j4.x);
            if (t + q + 1 < cnt) xr[q + 1] = gather(j4.y);
            if (t + q + 2 < cnt) xr[q + 2] = gather(j4.z);
            if (t + q + 3 < cnt) xr[q + 3] = gather(j4.w);
          }
        }
        // fma phase: values read from shared memory as they are needed
#pragma unroll
        for (int q = 0; q < U; q += 4) {
          AT vq[4];
          if constexpr (sizeof(AT) == 4) {
            const float4 v4 = *reinterpret_cast<const float4*>(vb + t + q);
            vq[0] = v4.x; vq[1] = v4.y; vq[2] = v4.z; vq[3] = v4.w;
          } else {
            const double2 va = *reinterpret_cast<const double2*>(vb + t + q);
            const double2 vc = *reinterpret_cast<const double2*>(vb + t + q + 2);
            vq[0] = va.x; vq[1] = va.y; vq[2] = vc.x; vq[3] = vc.y;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (full || t + q + r < cnt) {
              const XT* ex = reinterpret_cast<const XT*>(&xr[q + r]);
#pragma unroll
              for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vq[r], to_acc<AT, XT>(ex[i]), acc[i]);
            }
          }
        }
      }
      // publish the next chunk into the other buffer (its previous contents
      // were consumed one chunk ago, before the last __syncwarp)
      s_j[w][buf ^ 1][lane] = j_n;
      s_v[w][buf ^ 1][lane] = v_n;
      __syncwarp();
      buf ^= 1;
    }
    if (len == 0) {  // empty row: nothing was prefetched, stage the next row's first chunk
      int32_t j;
      AT v;
      fetch(s_nx + lane, e_nx, j, v);
      s_j[w][buf][lane] = j;
      s_v[w][buf][lane] = v;
      __syncwarp();
    }
    const int64_t orow = row_map ? (int64_t)row_map[row] : row;
    VecStore<YT, VEC>::store(Y + orow * (ROWB / (int)sizeof(XT)) + lane * VEC, acc);
    s_cur = s_nx;
    e_cur = e_nx;
    s_nx = s_nn;
    e_nx = e_nn;
  }
}

// ---- multi-row kernel with 16-byte lanes (FP32/FP64, 128/256-byte rows) ------------
// A gathered row is covered by L = ROWB/16 lanes with one 16-byte chunk each,
// so one load instruction of the warp fetches R = 32/L rows: the warp advances
// R consecutive output rows together, lane group q (lanes q*L .. q*L+L-1)
// owning row q of the group and lane lq of it the VEC columns
// [lq*VEC, (lq+1)*VEC). Each lane runs its columns' sequential fma chains over
// its row's entries in stored order (the same bits as k_spmm_row). Per chunk
// of 32 entries a row's (index, value) pairs are staged in shared memory and
// read back 4 at a time; the group's rows run in lockstep to the longest one,
// shorter rows predicated off, and batches where every row of the group still
// has U entries issue their U gathers without predicates. The next chunk's
// pairs (or the next group's first) are in flight while a chunk is consumed,
// and row bounds are fetched a group ahead, as in k_spmm_row.
template <class T, int ROWB, int U, int MINB>
__global__ void __launch_bounds__(kSpmmThreads, MINB)
k_spmm_rows16(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const T* __restrict__ values,
              const T* __restrict__ X, T* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows,
              const int32_t* __restrict__ sched) {
  constexpr int L = ROWB / 16;
  constexpr int R = 32 / L;
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int WARPS = kSpmmThreads / 32;
  static_assert(L == 8 || L == 16 || L == 32, "row pitch must be 128, 256 or 512 bytes");
  static_assert(U == 4 || U == 8 || U == 16, "batch must be 4, 8 or 16");
  __shared__ __align__(16) int32_t s_j[WARPS][2][32 * R];
  __shared__ __align__(16) T s_v[WARPS][2][32 * R];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int q = lane / L;
  const int lq = lane % L;
  const int64_t n_grp = (n_rows + R - 1) / R;
  const int64_t nw = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  const int64_t w_id = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5;
  // Groups of R rows: without a schedule warp w takes groups w, w + nw, ...
  // (a static grid stride); with one it takes its list sched[w] ..
  // sched[w + 1] - 1 of the group ids stored after the nw + 1 offsets. The
  // lists balance the warps' work (the longest groups first, each on a
  // lightly loaded warp); on the grid stride the warps that drew the longest
  // rows finished last. n_grp means no group is left.
  const int32_t* __restrict__ glist = sched ? sched + nw + 1 : nullptr;
  int64_t g_seq = w_id, q_next = 0, q_end = 0;
  auto next_group = [&]() -> int64_t {
    if (sched == nullptr) {
      g_seq += nw;
      return g_seq < n_grp ? g_seq : n_grp;
    }
    const int64_t qp = q_next++;
    return qp < q_end ? (int64_t)glist[qp] : n_grp;
  };
  int64_t grp = w_id;
  if (sched != nullptr) {
    q_next = sched[w_id];
    q_end = sched[w_id + 1];
    grp = q_next < q_end ? (int64_t)glist[q_next++] : n_grp;
  }
  if (grp >= n_grp) return;
  const char* __restrict__ Xl = reinterpret_cast<const char*>(X) + lq * 16;
  auto gather = [&](int32_t j) -> uint4 {
    return __ldg(reinterpret_cast<const uint4*>(Xl + (size_t)(uint32_t)j * ROWB));
  };
  auto bounds = [&](int64_t g, int64_t& b0, int64_t& b1) {
    const int64_t r = g * R + q;
    b0 = b1 = 0;
    if (g < n_grp && r < n_rows) {
      b0 = indptr[r];
      b1 = indptr[r + 1];
    }
  };
  // pairs [b0 + base, b0 + base + 32) of a row, R per lane of its group
  auto fetch = [&](int64_t b0, int64_t b1, int base, int32_t (&j)[R], T (&v)[R]) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int64_t p = b0 + base + lq + L * k;
      j[k] = 0;
      v[k] = T(0);
      if (p < b1) {
        j[k] = __ldcs(indices + p);
        v[k] = __ldcs(values + p);
      }
    }
  };
  auto publish = [&](int b, const int32_t (&j)[R], const T (&v)[R]) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      s_j[w][b][q * 32 + lq + L * k] = j[k];
      s_v[w][b][q * 32 + lq + L * k] = v[k];
    }
  };
  int64_t g_nx = next_group();
  int64_t g_nn = next_group();
  int64_t s_cur, e_cur, s_nx, e_nx;
  bounds(grp, s_cur, e_cur);
  bounds(g_nx, s_nx, e_nx);
  int buf = 0;
  {
    int32_t j[R];
    T v[R];
    fetch(s_cur, e_cur, 0, j, v);
    publish(0, j, v);
    __syncwarp();
  }
  while (grp < n_grp) {
    const int64_t g_n3 = next_group();  // its id is read a group ahead of its bounds
    int64_t s_nn, e_nn;
    bounds(g_nn, s_nn, e_nn);
    const int len = (int)(e_cur - s_cur);
    int maxlen = len, minlen = len;
#pragma unroll
    for (int o = L; o < 32; o <<= 1) {
      maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
      minlen = min(minlen, __shfl_xor_sync(0xffffffffu, minlen, o));
    }
    T acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = T(0);
    for (int base = 0; base < maxlen; base += 32) {
      int32_t jn[R];
      T vn[R];
      if (base + 32 < maxlen) fetch(s_cur, e_cur, base + 32, jn, vn);
      else fetch(s_nx, e_nx, 0, jn, vn);
      const int cnt = len - base;  // this lane's row: entries left (may be <= 0)
      const int cmax = min(maxlen - base, 32);
      const int cmin = min(minlen - base, 32);
      const int32_t* __restrict__ jb = &s_j[w][buf][q * 32];
      const T* __restrict__ vb = &s_v[w][buf][q * 32];
#pragma unroll 1
      for (int t = 0; t < cmax; t += U) {
        uint4 xr[U];
        const bool full = (t + U <= cmin);
#pragma unroll
        for (int u = 0; u < U; u += 4) {
          const int4 j4 = *reinterpret_cast<const int4*>(jb + t + u);
          if (full) {
            xr[u] = gather(j4.x);
            xr[u + 1] = gather(j4.y);
            xr[u + 2] = gather(j4.z);
            xr[u + 3] = gather(j4.w);
          } else {
            if (t + u < cnt) xr[u] = gather(j4.x);
            if (t + u + 1 < cnt) xr[u + 1] = gather(j4.y);
            if (t + u + 2 < cnt) xr[u + 2] = gather(j4.z);
            if (t + u + 3 < cnt) xr[u + 3] = gather(j4.w);
          }
        }
#pragma unroll
        for (int u = 0; u < U; u += 4) {
          T vq[4];
          if constexpr (sizeof(T) == 4) {
            const float4 v4 = *reinterpret_cast<const float4*>(vb + t + u);
            vq[0] = v4.x; vq[1] = v4.y; vq[2] = v4.z; vq[3] = v4.w;
          } else {
            const double2 va = *reinterpret_cast<const double2*>(vb + t + u);
            const double2 vc = *reinterpret_cast<const double2*>(vb + t + u + 2);
            vq[0] = va.x; vq[1] = va.y; vq[2] = vc.x; vq[3] = vc.y;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (full || t + u + r < cnt) {
              const T* ex = reinterpret_cast<const T*>(&xr[u + r]);
#pragma unroll
              for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vq[r], ex[i], acc[i]);
            }
          }
        }
      }
      // the other buffer was last read one chunk ago, before the last __syncwarp
      publish(buf ^ 1, jn, vn);
      __syncwarp();
      buf ^= 1;
    }
    if (maxlen == 0) {  // empty rows only: nothing was prefetched, stage the next group's first chunk
      int32_t j[R];
      T v[R];
      fetch(s_nx, e_nx, 0, j, v);
      publish(buf, j, v);
      __syncwarp();
    }
    const int64_t r = grp * R + q;
    if (r < n_rows) {
      const int64_t orow = row_map ? (int64_t)row_map[r] : r;
      uint4 o;
      T* op = reinterpret_cast<T*>(&o);
#pragma unroll
      for (int i = 0; i < VEC; ++i) op[i] = acc[i];
      *reinterpret_cast<uint4*>(reinterpret_cast<char*>(Y) + orow * ROWB + lq * 16) = o;
    }
    s_cur = s_nx;
    e_cur = e_nx;
    s_nx = s_nn;
    e_nx = e_nn;
    grp = g_nx;
    g_nx = g_nn;
    g_nn = g_n3;
  }
}

// ---- multi-row kernel for 16-bit storage (BF16/FP16, 128/256-byte rows) -----------
// k_spmm_rows16's layout with 16-bit values and X: L = ROWB/16 lanes cover a
// gathered row (8 values per lane), one warp advances Q = 32/L rows in
// lockstep, and every row keeps Q interleaved FP32 fma chains over its
// entries: entry p of the row feeds chain p mod Q, and the chains are summed
// pairwise at the end ((c0 + c1) + (c2 + c3) for Q = 4). That is the
// summation order of the other 16-bit kernels (kinds 5, 6, 9, 10), which the
// restatement oracle_diffuse_lowp_chains states, so all give the same bits.
// On rows ordered by length the lockstep costs little, and one load
// instruction gathers Q entries.
template <class VT, class YT, int ROWB, int U, int MINB>
__global__ void __launch_bounds__(kSpmmThreads, MINB)
k_spmm_rows16_lp(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                 const VT* __restrict__ values, const VT* __restrict__ X, YT* __restrict__ Y,
                 const int32_t* __restrict__ row_map, int64_t n_rows, const int32_t* __restrict__ sched) {
  constexpr int L = ROWB / 16;
  constexpr int Q = 32 / L;  // rows per warp = chains per row
  constexpr int VEC = 8;     // 16-bit values per lane
  constexpr int WARPS = kSpmmThreads / 32;
  constexpr int F = ROWB / 2;
  static_assert(L == 8 || L == 16, "16-bit rows of 128 or 256 bytes");
  static_assert(U == 4 || U == 8 || U == 16, "batch must be 4, 8 or 16");
  __shared__ __align__(16) int32_t s_j[WARPS][2][32 * Q];
  __shared__ __align__(16) float s_v[WARPS][2][32 * Q];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int q = lane / L;
  const int lq = lane % L;
  const int64_t n_grp = (n_rows + Q - 1) / Q;
  const int64_t nw = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  const int64_t w_id = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5;
  // groups of Q rows: a static grid stride, or this warp's list of a
  // balanced schedule (as in k_spmm_rows16)
  const int32_t* __restrict__ glist = sched ? sched + nw + 1 : nullptr;
  int64_t g_seq = w_id, q_next = 0, q_end = 0;
  auto next_group = [&]() -> int64_t {
    if (sched == nullptr) {
      g_seq += nw;
      return g_seq < n_grp ? g_seq : n_grp;
    }
    const int64_t qp = q_next++;
    return qp < q_end ? (int64_t)glist[qp] : n_grp;
  };
  int64_t grp = w_id;
  if (sched != nullptr) {
    q_next = sched[w_id];
    q_end = sched[w_id + 1];
    grp = q_next < q_end ? (int64_t)glist[q_next++] : n_grp;
  }
  if (grp >= n_grp) return;
  const char* __restrict__ Xl = reinterpret_cast<const char*>(X) + lq * 16;
  auto gather = [&](int32_t j) -> uint4 {
    return __ldg(reinterpret_cast<const uint4*>(Xl + (size_t)(uint32_t)j * ROWB));
  };
  auto bounds = [&](int64_t g, int64_t& b0, int64_t& b1) {
    const int64_t r = g * Q + q;
    b0 = b1 = 0;
    if (g < n_grp && r < n_rows) {
      b0 = indptr[r];
      b1 = indptr[r + 1];
    }
  };
  auto fetch = [&](int64_t b0, int64_t b1, int base, int32_t (&j)[Q], float (&v)[Q]) {
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int64_t p = b0 + base + lq + L * k;
      j[k] = 0;
      v[k] = 0.0f;
      if (p < b1) {
        j[k] = __ldcs(indices + p);
        v[k] = to_acc<float, VT>(__ldcs(values + p));
      }
    }
  };
  auto publish = [&](int b, const int32_t (&j)[Q], const float (&v)[Q]) {
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      s_j[w][b][q * 32 + lq + L * k] = j[k];
      s_v[w][b][q * 32 + lq + L * k] = v[k];
    }
  };
  int64_t g_nx = next_group();
  int64_t g_nn = next_group();
  int64_t s_cur, e_cur, s_nx, e_nx;
  bounds(grp, s_cur, e_cur);
  bounds(g_nx, s_nx, e_nx);
  int buf = 0;
  {
    int32_t j[Q];
    float v[Q];
    fetch(s_cur, e_cur, 0, j, v);
    publish(0, j, v);
    __syncwarp();
  }
  while (grp < n_grp) {
    const int64_t g_n3 = next_group();
    int64_t s_nn, e_nn;
    bounds(g_nn, s_nn, e_nn);
    const int len = (int)(e_cur - s_cur);
    int maxlen = len, minlen = len;
#pragma unroll
    for (int o = L; o < 32; o <<= 1) {
      maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
      minlen = min(minlen, __shfl_xor_sync(0xffffffffu, minlen, o));
    }
    float acc[Q][VEC];
#pragma unroll
    for (int c = 0; c < Q; ++c)
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[c][i] = 0.0f;
    for (int base = 0; base < maxlen; base += 32) {
      int32_t jn[Q];
      float vn[Q];
      if (base + 32 < maxlen) fetch(s_cur, e_cur, base + 32, jn, vn);
      else fetch(s_nx, e_nx, 0, jn, vn);
      const int cnt = len - base;  // this lane's row: entries left (may be <= 0)
      const int cmax = min(maxlen - base, 32);
      const int cmin = min(minlen - base, 32);
      const int32_t* __restrict__ jb = &s_j[w][buf][q * 32];
      const float* __restrict__ vb = &s_v[w][buf][q * 32];
#pragma unroll 1
      for (int t = 0; t < cmax; t += U) {
        uint4 xr[U];
        const bool full = (t + U <= cmin);
#pragma unroll
        for (int u = 0; u < U; u += 4) {
          const int4 j4 = *reinterpret_cast<const int4*>(jb + t + u);
          if (full) {
            xr[u] = gather(j4.x);
            xr[u + 1] = gather(j4.y);
            xr[u + 2] = gather(j4.z);
            xr[u + 3] = gather(j4.w);
          } else {
            if (t + u < cnt) xr[u] = gather(j4.x);
            if (t + u + 1 < cnt) xr[u + 1] = gather(j4.y);
            if (t + u + 2 < cnt) xr[u + 2] = gather(j4.z);
            if (t + u + 3 < cnt) xr[u + 3] = gather(j4.w);
          }
        }
#pragma unroll
        for (int u = 0; u < U; u += 4) {
          const float4 v4 = *reinterpret_cast<const float4*>(vb + t + u);
          const float vq[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (full || t + u + r < cnt) {
              // entry base + t + u + r of the row; base and t are multiples of 4, so its chain is (u + r) mod Q
              const uint32_t wv[4] = {xr[u + r].x, xr[u + r].y, xr[u + r].z, xr[u + r].w};
              float x[VEC];
#pragma unroll
              for (int h = 0; h < 4; ++h) {
                if constexpr (std::is_same_v<VT, __nv_bfloat16>) {
                  x[2 * h] = __uint_as_float(wv[h] << 16);
                  x[2 * h + 1] = __uint_as_float(wv[h] & 0xffff0000u);
                } else {
                  const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&wv[h]));
                  x[2 * h] = f.x;
                  x[2 * h + 1] = f.y;
                }
              }
#pragma unroll
              for (int i = 0; i < VEC; ++i) acc[(u + r) % Q][i] = __fmaf_rn(vq[r], x[i], acc[(u + r) % Q][i]);
            }
          }
        }
      }
      // the other buffer was last read one chunk ago, before the last __syncwarp
      publish(buf ^ 1, jn, vn);
      __syncwarp();
      buf ^= 1;
    }
    if (maxlen == 0) {  // empty rows only: nothing was prefetched, stage the next group's first chunk
      int32_t j[Q];
      float v[Q];
      fetch(s_nx, e_nx, 0, j, v);
      publish(buf, j, v);
      __syncwarp();
    }
    const int64_t r = grp * Q + q;
    if (r < n_rows) {
      float y[VEC];
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        if constexpr (Q == 4) y[i] = (acc[0][i] + acc[1][i]) + (acc[2][i] + acc[3][i]);
        else y[i] = acc[0][i] + acc[1][i];
      }
      const int64_t orow = row_map ? (int64_t)row_map[r] : r;
      YT* dst = Y + orow * F + lq * VEC;
      if constexpr (std::is_same_v<YT, float>) {
        *reinterpret_cast<float4*>(dst) = make_float4(y[0], y[1], y[2], y[3]);
        *reinterpret_cast<float4*>(dst + 4) = make_float4(y[4], y[5], y[6], y[7]);
      } else {
        uint32_t o[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          if constexpr (std::is_same_v<YT, __nv_bfloat16>) {
            const __nv_bfloat162 b = __floats2bfloat162_rn(y[2 * h], y[2 * h + 1]);
            o[h] = *reinterpret_cast<const uint32_t*>(&b);
          } else {
            const __half2 b = __floats2half2_rn(y[2 * h], y[2 * h + 1]);
            o[h] = *reinterpret_cast<const uint32_t*>(&b);
          }
        }
        *reinterpret_cast<uint4*>(dst) = make_uint4(o[0], o[1], o[2], o[3]);
      }
    }
    s_cur = s_nx;
    e_cur = e_nx;
    s_nx = s_nn;
    e_nx = e_nn;
    grp = g_nx;
    g_nx = g_nn;
    g_nn = g_n3;
  }
}

// ---- flat-stream kernel: a warp walks the entries of a block of rows ---------------
// A task is R consecutive rows; their entries [indptr[r0], indptr[r0+R]) are
// one contiguous stream that the warp consumes in batches of U gathers, with
// no regard for where rows begin or end — every batch but the stream's last is
// full, so U loads are always in flight, whatever the row lengths. The lane
// layout is k_spmm_row's (lane l owns bytes [l*LB, (l+1)*LB) of every
// gathered row, compile-time pitch), and entries are consumed in stream order:
// when the stream passes a row's end the row's accumulator is stored and
// reset, so every output element is still the sequential fma chain over its
// row's entries in stored order (bit-identical to the other variants). Row
// bounds of the task live in shared memory; (index, value) pairs are staged
// 32 at a time in a per-warp double buffer, the next chunk always in flight.
template <class VT, class XT, class YT, class AT, int ROWB, int U, int R>
__global__ void __launch_bounds__(kSpmmThreads, (U * ROWB <= 2048) ? 4 : ((U * ROWB <= 4096) ? 3 : 2))
k_spmm_flow(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
            const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows) {
  constexpr int LB = ROWB / 32;
  constexpr int VEC = LB / (int)sizeof(XT);
  constexpr int WARPS = kSpmmThreads / 32;
  constexpr int ROWE = ROWB / (int)sizeof(XT);
  static_assert(LB == 4 || LB == 8 || LB == 16, "row pitch must be 128, 256 or 512 bytes");
  static_assert(U == 8 || U == 16 || U == 32, "batch must divide 32");
  static_assert(R >= 1 && R <= 31, "a task holds at most 31 rows");
  using Rw = typename RawVec<LB>::type;
  __shared__ __align__(16) int32_t s_j[WARPS][2][32];
  __shared__ __align__(16) AT s_v[WARPS][2][32];
  __shared__ int64_t s_ptr[WARPS][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int64_t n_tasks = (n_rows + R - 1) / R;
  const int64_t nw = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  const char* __restrict__ Xb = reinterpret_cast<const char*>(X) + lane * LB;
  for (int64_t task = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5; task < n_tasks; task += nw) {
    const int64_t r0 = task * R;
    const int nr = (int)((n_rows - r0) < R ? (n_rows - r0) : R);
    if (lane <= nr) s_ptr[w][lane] = indptr[r0 + lane];
    __syncwarp();
    const int64_t p0 = s_ptr[w][0], p1 = s_ptr[w][nr];
    int ri = 0;                      // current row r0 + ri
    int64_t row_end = s_ptr[w][1];
    AT acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
    auto flush = [&]() {
      const int64_t r = r0 + ri;
      const int64_t orow = row_map ? (int64_t)row_map[r] : r;
      VecStore<YT, VEC>::store(Y + orow * ROWE + lane * VEC, acc);
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[i] = AT(0);
      ++ri;
      row_end = (ri < nr) ? s_ptr[w][ri + 1] : p1;
    };
    int buf = 0;
    if (p0 + lane < p1) {
      s_j[w][0][lane] = __ldcs(indices + p0 + lane);
      s_v[w][0][lane] = to_acc<AT, VT>(__ldcs(values + p0 + lane));
    }
    __syncwarp();
    for (int64_t c = p0; c < p1; c += 32) {
      int32_t j_n = 0;
      AT v_n = AT(0);
      if (c + 32 + lane < p1) {
        j_n = __ldcs(indices + c + 32 + lane);
        v_n = to_acc<AT, VT>(__ldcs(values + c + 32 + lane));
      }
      const int cnt = (p1 - c) < 32 ? (int)(p1 - c) : 32;
      const int32_t* __restrict__ jb = s_j[w][buf];
      const AT* __restrict__ vb = s_v[w][buf];
#pragma unroll
      for (int t = 0; t < 32; t += U) {
        if (t >= cnt) break;
        Rw xr[U];
        const bool full = (t + U <= cnt);
#pragma unroll
        for (int q = 0; q < U; q += 4) {
          const int4 j4 = *reinterpret_cast<const int4*>(jb + t + q);
          const int jj[4] = {j4.x, j4.y, j4.z, j4.w};
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (full || t + q + r < cnt)
              xr[q + r] = __ldg(reinterpret_cast<const Rw*>(Xb + (size_t)(uint32_t)jj[r] * ROWB));
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (full || t + u < cnt) {
            const int64_t e = c + t + u;
            while (e >= row_end) flush();  // rows that end before entry e (empty rows included)
            const AT vv = vb[t + u];
            const XT* ex = reinterpret_cast<const XT*>(&xr[u]);
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = fma_acc(vv, to_acc<AT, XT>(ex[i]), acc[i]);
          }
        }
      }
      s_j[w][buf ^ 1][lane] = j_n;
      s_v[w][buf ^ 1][lane] = v_n;
      __syncwarp();
      buf ^= 1;
    }
    while (ri < nr) flush();  // the row holding the last entry, then trailing empty rows
    __syncwarp();
  }
}

// ---- split-chain warp-per-row kernel (16-bit storage) --------------------------------
// One warp per row as in k_spmm_row, but every lane loads 16 bytes: a row of
// ROWB bytes takes L = ROWB/16 lanes, so one 128-bit load instruction of the
// warp gathers Q = 32/L entries at once — quarter q of the warp (lanes
// [qL, qL+L)) takes entries q, q+Q, q+2Q, ... of the row and keeps its own
// sequential fma chain over them. At the row end the Q chains are summed
// pairwise by shuffles over the lane bits L, 2L, ... (Q=2: c0+c1; Q=4:
// (c0+c1)+(c2+c3)), the order the oracle's chain restatement uses. Pairs are
// staged 32 at a time in a per-warp shared-memory double buffer, the next
// chunk (or the next row's first chunk) and the next row's bounds are fetched
// one step ahead, exactly as in k_spmm_row. MIXED forms the products with
// fma.rn.f32.{bf16,f16} straight from the stored operands (exact product, one
// rounding: the bits of widening both to f32 first).
template <class T>
__device__ __forceinline__ float fma_mixed(unsigned short a, unsigned short b, float c);
template <>
__device__ __forceinline__ float fma_mixed<__nv_bfloat16>(unsigned short a, unsigned short b, float c) {
  asm("fma.rn.f32.bf16 %0, %1, %2, %0;" : "+f"(c) : "h"(a), "h"(b));
  return c;
}
template <>
__device__ __forceinline__ float fma_mixed<__half>(unsigned short a, unsigned short b, float c) {
  asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(c) : "h"(a), "h"(b));
  return c;
}

// One batch of the split-chain kernel: lane quarter q gathers entries
// t + u*Q + q (u < U) and adds them to its chain; only a row's last batch
// tests each entry against the chunk count.
template <bool FULL, int U, int Q, int ROWB, class VT, class XT, bool MIXED>
__device__ __forceinline__ void split_batch(const char* __restrict__ Xb, const int32_t* __restrict__ jb,
                                            const unsigned short* __restrict__ vb, int t, int q, int cnt,
                                            float (&acc)[8]) {
  uint4 xr[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int e = t + u * Q + q;
    if (FULL || e < cnt) xr[u] = __ldg(reinterpret_cast<const uint4*>(Xb + (size_t)(uint32_t)jb[e] * (size_t)ROWB));
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int e = t + u * Q + q;
    if (FULL || e < cnt) {
      const unsigned short vbits = vb[e];
      const unsigned short* ex = reinterpret_cast<const unsigned short*>(&xr[u]);
      if constexpr (MIXED) {
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = fma_mixed<XT>(vbits, ex[i], acc[i]);
      } else {
        const float vf = tof<VT>(*reinterpret_cast<const VT*>(&vbits));
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = __fmaf_rn(vf, tof<XT>(*reinterpret_cast<const XT*>(&ex[i])), acc[i]);
      }
    }
  }
}

// Resident CTAs per SM of the split-chain kernel with 2 gathers per lane per
// batch (the 128-byte-row default): a compile-time tuning constant.
#ifndef SCL_SPLIT_MIN_BLOCKS_U2
#define SCL_SPLIT_MIN_BLOCKS_U2 4
#endif

template <class VT, class XT, class YT, int ROWB, int U, bool MIXED>
__global__ void __launch_bounds__(kSpmmThreads, (U <= 2) ? SCL_SPLIT_MIN_BLOCKS_U2 : ((U <= 8) ? 3 : 2))
k_spmm_split(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, const VT* __restrict__ values,
             const XT* __restrict__ X, YT* __restrict__ Y, const int32_t* __restrict__ row_map, int64_t n_rows) {
  static_assert(sizeof(XT) == 2 && sizeof(VT) == 2, "the split-chain kernel is for 16-bit storage");
  constexpr int L = ROWB / 16;        // lanes per gathered row
  constexpr int Q = 32 / L;           // entries per load instruction (chains)
  constexpr int VEC = 8;              // 16-bit elements per lane
  constexpr int WARPS = kSpmmThreads / 32;
  constexpr int STEP = U * Q;         // entries per batch
  static_assert(L == 8 || L == 16, "row pitch must be 128 or 256 bytes");
  static_assert(32 % STEP == 0, "a chunk of 32 entries holds whole batches");
  __shared__ __align__(16) int32_t s_j[WARPS][2][32];
  __shared__ __align__(16) unsigned short s_v[WARPS][2][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int q = lane / L;             // chain of this lane
  const int lq = lane & (L - 1);      // 16-byte chunk of the row
  const int64_t nw = ((int64_t)gridDim.x * kSpmmThreads) >> 5;
  int64_t row = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) >> 5;
  if (row >= n_rows) return;
  const char* __restrict__ Xb = reinterpret_cast<const char*>(X) + lq * 16;
  int64_t s_cur = indptr[row], e_cur = indptr[row + 1];
  int64_t s_nx = 0, e_nx = 0;
  if (row + nw < n_rows) {
    s_nx = indptr[row + nw];
    e_nx = indptr[row + nw + 1];
  }
  auto fetch = [&](int64_t pos, int64_t end, int32_t& j, unsigned short& v) {
    j = 0;
    v = 0;
    if (pos < end) {
      j = __ldcs(indices + pos);
      v = __ldcs(reinterpret_cast<const unsigned short*>(values) + pos);
    }
  };
  int buf = 0;
  {
    int32_t j;
    unsigned short v;
    fetch(s_cur + lane, e_cur, j, v);
    s_j[w][0][lane] = j;
    s_v[w][0][lane] = v;
    __syncwarp();
  }
  for (; row < n_rows; row += nw) {
    const int64_t nn = row + 2 * nw;
    int64_t s_nn = 0, e_nn = 0;
    if (nn < n_rows) {
      s_nn = indptr[nn];
      e_nn = indptr[nn + 1];
    }
    float acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
    const int len = (int)(e_cur - s_cur);
    for (int base = 0; base < len; base += 32) {
      int32_t j_n;
      unsigned short v_n;
      if (base + 32 < len) fetch(s_cur + base + 32 + lane, e_cur, j_n, v_n);
      else fetch(s_nx + lane, e_nx, j_n, v_n);
      const int cnt = (len - base) < 32 ? (len - base) : 32;
      const int32_t* __restrict__ jb = s_j[w][buf];
      const unsigned short* __restrict__ vb = s_v[w][buf];
      int t = 0;
#pragma unroll 1
      for (; t + STEP <= cnt; t += STEP) split_batch<true, U, Q, ROWB, VT, XT, MIXED>(Xb, jb, vb, t, q, cnt, acc);
      if (t < cnt) split_batch<false, U, Q, ROWB, VT, XT, MIXED>(Xb, jb, vb, t, q, cnt, acc);
      s_j[w][buf ^ 1][lane] = j_n;
      s_v[w][buf ^ 1][lane] = v_n;
      __syncwarp();
      buf ^= 1;
    }
    if (len == 0) {
      int32_t j;
      unsigned short v;
      fetch(s_nx + lane, e_nx, j, v);
      s_j[w][buf][lane] = j;
      s_v[w][buf][lane] = v;
      __syncwarp();
    }
    // sum the Q chains: lane bits L, 2L, ... from the lowest
#pragma unroll
    for (int o = L; o < 32; o <<= 1) {
#pragma unroll
      for (int i = 0; i < VEC; ++i) acc[i] = acc[i] + __shfl_xor_sync(0xffffffffu, acc[i], o);
    }
    if (q == 0) {
      const int64_t orow = row_map ? (int64_t)row_map[row] : row;
      VecStore<YT, VEC>::store(Y + orow * (ROWB / 2) + lq * VEC, acc);
    }
    s_cur = s_nx;
    e_cur = e_nx;
    s_nx = s_nn;
    e_nx = e_nn;
  }
}

// ---- pipelined split-chain kernel (16-bit storage, gathers land in shared memory) ---
// The lane layout and the chain order of k_spmm_split (quarter q of the warp
// takes entries q, q+Q, ... of the row, one 16-byte chunk per lane), but the
// gathered chunks are copied by cp.async straight into lane-private
// shared-memory slots instead of registers: the next chunk of 32 entries per
// warp is in flight while the current one is consumed, so deep batches cost no
// registers. The warp walks its chunk stream (chunk_cursor.cuh) three deep:
// (index, value) pairs of chunk k+2 load while chunk k+1's gathers are in
// flight and chunk k is consumed. Each lane only reads slots it filled itself,
// so the per-thread cp.async.wait_group is the only synchronisation. Same bits
// as k_spmm_split.
template <int ROWB>
constexpr int split_pipe_warps() { return ROWB == 128 ? 8 : 4; }
template <int ROWB>
constexpr int split_pipe_smem() { return split_pipe_warps<ROWB>() * 2 * 32 * ROWB; }

template <class VT, class XT, class YT, int ROWB, bool MIXED>
__global__ void __launch_bounds__(32 * split_pipe_warps<ROWB>(), ROWB == 128 ? 3 : 1)
k_spmm_split_pipe(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                  const VT* __restrict__ values, const XT* __restrict__ X, YT* __restrict__ Y,
                  const int32_t* __restrict__ row_map, int64_t n_rows, const int32_t* __restrict__ sched) {
  static_assert(sizeof(XT) == 2 && sizeof(VT) == 2, "the split-chain kernel is for 16-bit storage");
  constexpr int L = ROWB / 16;  // lanes per gathered row
  constexpr int Q = 32 / L;     // chains (entries per load instruction)
  constexpr int U = 32 / Q;     // copies per lane per chunk
  constexpr int VEC = 8;
  constexpr int NT = 32 * split_pipe_warps<ROWB>();
  extern __shared__ uint4 smem_split[];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int q = lane / L;
  const int lq = lane & (L - 1);
  uint4* __restrict__ my = smem_split + (size_t)w * 2 * U * 32 + lane;  // slot (st, u): my[(st * U + u) * 32]
  const char* __restrict__ Xb = reinterpret_cast<const char*>(X) + lq * 16;
  const unsigned short* __restrict__ vbits = reinterpret_cast<const unsigned short*>(values);
  const int64_t nw = ((int64_t)gridDim.x * NT) >> 5;
  const int64_t row0 = ((int64_t)blockIdx.x * NT + threadIdx.x) >> 5;
  if (row0 >= n_rows) return;
  ChunkCursor cur;
  cur.init(indptr, row0, n_rows, nw, sched);
  Chunk C = cur.next(indptr);  // pairs loading
  int32_t jC = 0;
  unsigned vC = 0;
  if (C.valid && lane < C.cnt) {
    jC = __ldcs(indices + C.pos + lane);
    vC = __ldcs(vbits + C.pos + lane);
  }
  Chunk B;  // gathers in flight
  unsigned vB = 0;
  int st = 0;
  float acc[VEC];
#pragma unroll
  for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
  while (B.valid || C.valid) {
    Chunk D = cur.next(indptr);
    int32_t jD = 0;
    unsigned vD = 0;
    if (D.valid && lane < D.cnt) {
      jD = __ldcs(indices + D.pos + lane);
      vD = __ldcs(vbits + D.pos + lane);
    }
    if (C.valid) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = u * Q + q;
        const int32_t jj = __shfl_sync(0xffffffffu, jC, e);
        if (e < C.cnt) {
          const unsigned s = (unsigned)__cvta_generic_to_shared(my + (st * U + u) * 32);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s),
                       "l"(Xb + (size_t)(uint32_t)jj * (size_t)ROWB) : "memory");
        }
      }
    }
    cp_async_commit_group();
    if (B.valid) {
      cp_async_wait_group<1>();
      if (B.first) {
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
      }
      const uint4* __restrict__ sb = my + (st ^ 1) * U * 32;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = u * Q + q;
        const unsigned short vv = (unsigned short)__shfl_sync(0xffffffffu, vB, e);
        if (e < B.cnt) {
          const uint4 raw = sb[u * 32];
          const unsigned short* ex = reinterpret_cast<const unsigned short*>(&raw);
          if constexpr (MIXED) {
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = fma_mixed<XT>(vv, ex[i], acc[i]);
          } else {
            const float vf = tof<VT>(*reinterpret_cast<const VT*>(&vv));
#pragma unroll
            for (int i = 0; i < VEC; ++i)
              acc[i] = __fmaf_rn(vf, tof<XT>(*reinterpret_cast<const XT*>(&ex[i])), acc[i]);
          }
        }
      }
      if (B.last) {
#pragma unroll
        for (int o = L; o < 32; o <<= 1) {
#pragma unroll
          for (int i = 0; i < VEC; ++i) acc[i] = acc[i] + __shfl_xor_sync(0xffffffffu, acc[i], o);
        }
        if (q == 0) {
          const int64_t orow = row_map ? (int64_t)row_map[B.row] : B.row;
          VecStore<YT, VEC>::store(Y + orow * (ROWB / 2) + lq * VEC, acc);
        }
      }
    }
    B = C;
    vB = vC;
    C = D;
    jC = jD;
    vC = vD;
    st ^= 1;
  }
  cp_async_wait_group<0>();
}

// ---- lean pipelined split-chain kernel (16-bit storage) -----------------------------
// k_spmm_split_pipe with the per-entry overhead cut: full chunks of 32
// entries (the common case) issue their copies and consume their slots with
// no per-entry predicate, every copy targets a constant offset from one
// shared-memory base address, and MODE selects the product form: 0 =
// fma.rn.f32.{bf16,f16} per element; 1 (bf16 only) = each 32-bit word's two
// bf16 values unpacked by a shift and a mask into an f32 pair and both
// accumulators advanced by one fma.rn.f32x2 (two independent IEEE fmas, so
// the bits equal mode 0's). Same chains and bits as k_spmm_split.
__device__ __forceinline__ void fma2_bf16_word(unsigned long long& acc2, unsigned long long v2, unsigned w) {
  unsigned long long x2;
  asm("{\n\t.reg .b32 lo, hi;\n\tshl.b32 lo, %1, 16;\n\tand.b32 hi, %1, 0xffff0000;\n\tmov.b64 %0, {lo, hi};\n\t}"
      : "=l"(x2)
      : "r"(w));
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc2) : "l"(v2), "l"(x2));
}

template <bool FULL, int MODE, int U, int Q, class XT>
__device__ __forceinline__ void lean_consume(const uint4* __restrict__ sb, const unsigned short (&vq)[U], int q,
                                             int cnt, float (&acc)[8], unsigned long long (&acc2)[4]) {
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int e = u * Q + q;
    const unsigned short vv = vq[u];
    if (FULL || e < cnt) {
      const uint4 raw = sb[u * 32];
      if constexpr (MODE == 1) {
        const float vf = __uint_as_float((unsigned)vv << 16);
        unsigned long long v2;
        asm("mov.b64 %0, {%1, %1};" : "=l"(v2) : "f"(vf));
        fma2_bf16_word(acc2[0], v2, raw.x);
        fma2_bf16_word(acc2[1], v2, raw.y);
        fma2_bf16_word(acc2[2], v2, raw.z);
        fma2_bf16_word(acc2[3], v2, raw.w);
      } else {
        const unsigned short* ex = reinterpret_cast<const unsigned short*>(&raw);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = fma_mixed<XT>(vv, ex[i], acc[i]);
      }
    }
  }
}

// For 256-byte rows (16 entries per lane per chunk) the chunk's (index, value)
// pairs are staged in shared memory quarter-major (entry e at position
// (e % Q) * U + e / Q), so a lane reads the U indices or values of its own
// entries with a few vector loads instead of U shuffles; for 128-byte rows the
// shuffles were measured faster and are kept.
template <class VT, class XT, class YT, int ROWB, int MODE>
__global__ void __launch_bounds__(32 * split_pipe_warps<ROWB>(), ROWB == 128 ? 3 : 1)
k_spmm_split_lean(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                  const VT* __restrict__ values, const XT* __restrict__ X, YT* __restrict__ Y,
                  const int32_t* __restrict__ row_map, int64_t n_rows, const int32_t* __restrict__ sched) {
  static_assert(sizeof(XT) == 2 && sizeof(VT) == 2, "the split-chain kernel is for 16-bit storage");
  constexpr int L = ROWB / 16;
  constexpr int Q = 32 / L;
  constexpr int U = 32 / Q;
  constexpr int VEC = 8;
  constexpr int WARPS = split_pipe_warps<ROWB>();
  constexpr int NT = 32 * WARPS;
  constexpr unsigned SLOT = 32 * 16;  // bytes between a lane's consecutive slots
  extern __shared__ uint4 smem_lean[];
  __shared__ __align__(16) int32_t s_j[WARPS][2][32];
  __shared__ __align__(16) unsigned short s_v[WARPS][2][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int q = lane / L;
  const int lq = lane & (L - 1);
  const int tpos = (lane % Q) * U + lane / Q;  // where this lane's pair goes in the staging
  const uint4* __restrict__ my = smem_lean + (size_t)w * 2 * U * 32 + lane;
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(my);
  const char* __restrict__ Xb = reinterpret_cast<const char*>(X) + lq * 16;
  const unsigned short* __restrict__ vbits = reinterpret_cast<const unsigned short*>(values);
  const int64_t nw = ((int64_t)gridDim.x * NT) >> 5;
  const int64_t row0 = ((int64_t)blockIdx.x * NT + threadIdx.x) >> 5;
  if (row0 >= n_rows) return;
  ChunkCursor cur;
  cur.init(indptr, row0, n_rows, nw, sched);
  Chunk C = cur.next(indptr);
  int32_t jC = 0;
  unsigned short vC = 0;
  if (C.valid && lane < C.cnt) {
    jC = __ldcs(indices + C.pos + lane);
    vC = __ldcs(vbits + C.pos + lane);
  }
  Chunk B;
  unsigned short vB = 0;  // B's values, one per lane (shuffle path)
  int st = 0;
  float acc[VEC];
  unsigned long long acc2[4];
#pragma unroll
  for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i) acc2[i] = 0ull;
  while (B.valid || C.valid) {
    Chunk D = cur.next(indptr);
    int32_t jD = 0;
    unsigned short vD = 0;
    if (D.valid && lane < D.cnt) {
      jD = __ldcs(indices + D.pos + lane);
      vD = __ldcs(vbits + D.pos + lane);
    }
    constexpr bool STG = (ROWB == 256);
    if constexpr (STG) {  // stage C's pairs (its stage was last read two iterations ago)
      __syncwarp();
      s_j[w][st][tpos] = jC;
      s_v[w][st][tpos] = vC;
      __syncwarp();
    }
    if (C.valid) {
      int32_t jq[U];
      if constexpr (STG) {
#pragma unroll
        for (int k = 0; k < U; k += 4) {
          const int4 j4 = *reinterpret_cast<const int4*>(&s_j[w][st][q * U + k]);
          jq[k] = j4.x; jq[k + 1] = j4.y; jq[k + 2] = j4.z; jq[k + 3] = j4.w;
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) jq[u] = __shfl_sync(0xffffffffu, jC, u * Q + q);
      }
      const unsigned sst = sbase + (unsigned)st * (U * SLOT);
      if (C.cnt == 32) {
#pragma unroll
        for (int u = 0; u < U; ++u)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sst + u * SLOT),
                       "l"(Xb + (size_t)(uint32_t)jq[u] * (size_t)ROWB) : "memory");
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (u * Q + q < C.cnt)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sst + u * SLOT),
                         "l"(Xb + (size_t)(uint32_t)jq[u] * (size_t)ROWB) : "memory");
        }
      }
    }
    cp_async_commit_group();
    if (B.valid) {
      cp_async_wait_group<1>();
      if (B.first) {
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) acc2[i] = 0ull;
      }
      unsigned short vq[U];
      if constexpr (STG) {
#pragma unroll
        for (int k = 0; k < U; k += 8) {
          const uint4 v8 = *reinterpret_cast<const uint4*>(&s_v[w][st ^ 1][q * U + k]);
          const unsigned short* pv = reinterpret_cast<const unsigned short*>(&v8);
#pragma unroll
          for (int i = 0; i < 8; ++i) vq[k + i] = pv[i];
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) vq[u] = (unsigned short)__shfl_sync(0xffffffffu, (unsigned)vB, u * Q + q);
      }
      const uint4* __restrict__ sb = my + (st ^ 1) * U * 32;
      if (B.cnt == 32) lean_consume<true, MODE, U, Q, XT>(sb, vq, q, 32, acc, acc2);
      else lean_consume<false, MODE, U, Q, XT>(sb, vq, q, B.cnt, acc, acc2);
      if (B.last) {
        if constexpr (MODE == 1) {
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            acc[2 * i] = __uint_as_float((unsigned)(acc2[i] & 0xffffffffull));
            acc[2 * i + 1] = __uint_as_float((unsigned)(acc2[i] >> 32));
          }
        }
#pragma unroll
        for (int o = L; o < 32; o <<= 1) {
#pragma unroll
          for (int i = 0; i < VEC; ++i) acc[i] = acc[i] + __shfl_xor_sync(0xffffffffu, acc[i], o);
        }
        if (q == 0) {
          const int64_t orow = row_map ? (int64_t)row_map[B.row] : B.row;
          VecStore<YT, VEC>::store(Y + orow * (ROWB / 2) + lq * VEC, acc);
        }
      }
    }
    B = C;
    vB = vC;
    C = D;
    jC = jD;
    vC = vD;
    st ^= 1;
  }
  cp_async_wait_group<0>();
}

// Persistent grid size: resident blocks per SM (from the occupancy
// calculator) times the SM count, capped by the blocks the rows need.
template <class K>
unsigned persistent_blocks(K kern, int smem, int64_t n_rows, int G) {
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSpmmThreads, smem));
  const int64_t need = (n_rows * G + kSpmmThreads - 1) / kSpmmThreads;
  int64_t b = (int64_t)std::max(per_sm, 1) * sm_count(dev);
  if (b > need) b = need;
  return (unsigned)std::max<int64_t>(b, 1);
}

template <class VT, class XT, class YT, class AT, int VEC, int S>
void launch_pipe_s(int G, const SpmmArgs& a, cudaStream_t s) {
  const int smem = pipe_smem_bytes<S>();
  const auto* ip = a.indptr;
  const auto* ix = a.indices;
  const auto* vv = static_cast<const VT*>(a.values);
  const auto* xx = static_cast<const XT*>(a.X);
  auto* yy = static_cast<YT*>(a.Y);
#define SCL_PIPE_CASE(GG)                                                                                \
  case GG: {                                                                                             \
    auto kern = k_spmm_pipe<VT, XT, YT, AT, GG, VEC, (S <= GG ? S : GG)>;                                 \
    SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));             \
    SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,                   \
                                  (int)cudaSharedmemCarveoutMaxShared));                                 \
    const dim3 grid(persistent_blocks(kern, smem, a.n_rows, GG));                                        \
    kern<<<grid, kSpmmThreads, smem, s>>>(ip, ix, vv, xx, yy, a.row_map, a.n_rows, a.F);                  \
    break;                                                                                               \
  }
  switch (G) {
    SCL_PIPE_CASE(4)
    SCL_PIPE_CASE(8)
    SCL_PIPE_CASE(16)
    SCL_PIPE_CASE(32)
    default: throw Error(kErrInvalidArgument, "pipelined SpMM needs a lane-group size of 4..32");
  }
#undef SCL_PIPE_CASE
  SCL_CUDA(cudaGetLastError());
}

// G == 1 needs no shuffles but the template handles it (width-1 shuffles are
// identity operations); keep one instantiation path for simplicity.

template <class VT, class XT, class YT, class AT, int VEC>
void launch_g(int G, const SpmmArgs& a, cudaStream_t s) {
  const auto* ip = a.indptr;
  const auto* ix = a.indices;
  const auto* vv = static_cast<const VT*>(a.values);
  const auto* xx = static_cast<const XT*>(a.X);
  auto* yy = static_cast<YT*>(a.Y);
#define SCL_SPMM_CASE(GG, UU)                                                                     \
  case GG: {                                                                                      \
    auto kern = k_spmm<VT, XT, YT, AT, GG, VEC, UU>;                                              \
    const dim3 grid(persistent_blocks(kern, 0, a.n_rows, GG));                                    \
    kern<<<grid, kSpmmThreads, 0, s>>>(ip, ix, vv, xx, yy, a.row_map, a.n_rows, a.F);             \
    break;                                                                                        \
  }
  switch (G) {
    SCL_SPMM_CASE(1, 1)
    SCL_SPMM_CASE(2, 2)
    SCL_SPMM_CASE(4, 4)
    SCL_SPMM_CASE(8, 8)
    SCL_SPMM_CASE(16, 8)
    SCL_SPMM_CASE(32, 8)
    default: throw Error(kErrInternal, "unsupported lane-group size");
  }
#undef SCL_SPMM_CASE
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, class AT, int VEC, int U>
void launch_stream_u(const SpmmArgs& a, cudaStream_t s) {
  auto kern = k_spmm_stream<VT, XT, YT, AT, VEC, U>;
  const int64_t tasks = (a.n_rows + kStreamRows - 1) / kStreamRows;
  // one warp per task: ask for tasks*32 "rows" of one lane each
  const dim3 grid(persistent_blocks(kern, 0, tasks, 32));
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                     static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows, a.F);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, class AT, int VEC, int S>
void launch_spipe_s(const SpmmArgs& a, cudaStream_t s) {
  constexpr int LB = VEC * (int)sizeof(XT);
  auto kern = k_spmm_spipe<VT, XT, YT, AT, VEC, S>;
  const int smem = stream_pipe_smem_bytes<LB, S>();
  int dev = 0, max_smem = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  SCL_REQUIRE(smem <= max_smem, kErrInvalidArgument, "stream pipeline stage does not fit in shared memory");
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  const int64_t tasks = (a.n_rows + kStreamRows - 1) / kStreamRows;
  const dim3 grid(persistent_blocks(kern, smem, tasks, 32));
  kern<<<grid, kSpmmThreads, smem, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                        static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows, a.F);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, class AT, int ROWB, int U>
void launch_row_u(const SpmmArgs& a, cudaStream_t s) {
  // rows of X addressed by the column indices: n_cols <= n_rows, X holds n_rows rows
  const bool off32 = (uint64_t)a.n_rows * (uint64_t)ROWB < (1ull << 32);
  auto kern = off32 ? k_spmm_row<VT, XT, YT, AT, ROWB, U, true> : k_spmm_row<VT, XT, YT, AT, ROWB, U, false>;
  const dim3 grid(persistent_blocks(kern, 0, a.n_rows, 32));
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                     static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows);
  SCL_CUDA(cudaGetLastError());
}

// kind 4: fixed-pitch warp-per-row kernel; stage = gathers per batch (8/16/32)
template <class VT, class XT, class YT, class AT>
void launch_row(const SpmmArgs& a, int U, cudaStream_t s) {
  const int64_t rowb = a.F * (int64_t)sizeof(XT);
#define SCL_ROW_CASE(RB)                                                         \
  if constexpr (RB / 32 >= (int)sizeof(XT)) {                                    \
    if (rowb == RB) {                                                            \
      if (U == 8) return launch_row_u<VT, XT, YT, AT, RB, 8>(a, s);              \
      if (U == 16) return launch_row_u<VT, XT, YT, AT, RB, 16>(a, s);            \
      if (U == 32) return launch_row_u<VT, XT, YT, AT, RB, 32>(a, s);            \
      throw Error(kErrInvalidArgument, "row SpMM batch must be 8, 16 or 32");    \
    }                                                                            \
  }
  SCL_ROW_CASE(128)
  SCL_ROW_CASE(256)
  SCL_ROW_CASE(512)
#undef SCL_ROW_CASE
  throw Error(kErrInvalidArgument, "the fixed-pitch SpMM needs 128-, 256- or 512-byte rows");
}

// kind 12: multi-row kernel with 16-byte lanes; stage = gathers per batch (4/8/16)
template <class T, int ROWB, int U, int MINB>
void launch_rows16_u(const SpmmArgs& a, cudaStream_t s) {
  constexpr int R = 32 / (ROWB / 16);
  auto kern = k_spmm_rows16<T, ROWB, U, MINB>;
  const int64_t groups = (a.n_rows + R - 1) / R;
  const dim3 grid(persistent_blocks(kern, 0, groups, 32));
  const int32_t* sched = a.reo ? warp_schedule_for(*a.reo, R, (int64_t)grid.x * (kSpmmThreads / 32), s) : nullptr;
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const T*>(a.values),
                                     static_cast<const T*>(a.X), static_cast<T*>(a.Y), a.row_map, a.n_rows, sched);
  SCL_CUDA(cudaGetLastError());
}

template <class T, int ROWB>
void launch_rows16_rb(const SpmmArgs& a, int U, cudaStream_t s) {
  if (U == 4) return launch_rows16_u<T, ROWB, 4, 4>(a, s);
  if (U == 8) return launch_rows16_u<T, ROWB, 8, 3>(a, s);
  if (U == 16) return launch_rows16_u<T, ROWB, 16, 2>(a, s);
  throw Error(kErrInvalidArgument, "multi-row SpMM batch must be 4, 8 or 16");
}

template <class T>
void launch_rows16(const SpmmArgs& a, int U, cudaStream_t s) {
  const int64_t rowb = a.F * (int64_t)sizeof(T);
  SCL_REQUIRE(reinterpret_cast<uintptr_t>(a.X) % 16 == 0 && reinterpret_cast<uintptr_t>(a.Y) % 16 == 0,
              kErrInvalidArgument, "the multi-row SpMM needs 16-byte aligned X and Y");
  if (rowb == 128) return launch_rows16_rb<T, 128>(a, U, s);
  if (rowb == 256) return launch_rows16_rb<T, 256>(a, U, s);
  if (rowb == 512) return launch_rows16_rb<T, 512>(a, U, s);
  throw Error(kErrInvalidArgument, "the multi-row SpMM needs 128-, 256- or 512-byte rows");
}

// kind 7: flat-stream kernel over tasks of 16 consecutive rows; stage = gathers per batch
template <class VT, class XT, class YT, class AT, int ROWB, int U>
void launch_flow_u(const SpmmArgs& a, cudaStream_t s) {
  constexpr int R = 16;
  auto kern = k_spmm_flow<VT, XT, YT, AT, ROWB, U, R>;
  const int64_t tasks = (a.n_rows + R - 1) / R;
  const dim3 grid(persistent_blocks(kern, 0, tasks, 32));
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                     static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, class AT>
void launch_flow(const SpmmArgs& a, int U, cudaStream_t s) {
  const int64_t rowb = a.F * (int64_t)sizeof(XT);
#define SCL_FLOW_CASE(RB)                                                          \
  if constexpr (RB / 32 >= (int)sizeof(XT)) {                                      \
    if (rowb == RB) {                                                              \
      if (U == 8) return launch_flow_u<VT, XT, YT, AT, RB, 8>(a, s);               \
      if (U == 16) return launch_flow_u<VT, XT, YT, AT, RB, 16>(a, s);             \
      if (U == 32) return launch_flow_u<VT, XT, YT, AT, RB, 32>(a, s);             \
      throw Error(kErrInvalidArgument, "flat-stream SpMM batch must be 8, 16 or 32"); \
    }                                                                              \
  }
  SCL_FLOW_CASE(128)
  SCL_FLOW_CASE(256)
  SCL_FLOW_CASE(512)
#undef SCL_FLOW_CASE
  throw Error(kErrInvalidArgument, "the flat-stream SpMM needs 128-, 256- or 512-byte rows");
}

// kind 9: pipelined split-chain kernel (16-bit storage); stage: 0 = plain fma, 1 = mixed-precision fma
template <class VT, class XT, class YT, int ROWB, bool MIXED>
void launch_split_pipe_r(const SpmmArgs& a, cudaStream_t s) {
  auto kern = k_spmm_split_pipe<VT, XT, YT, ROWB, MIXED>;
  constexpr int smem = split_pipe_smem<ROWB>();
  constexpr int nt = 32 * split_pipe_warps<ROWB>();
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem));
  const int64_t need = (a.n_rows * 32 + nt - 1) / nt;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)std::max(per_sm, 1) * sm_count(dev)));
  const int32_t* sched = a.reo ? warp_schedule_for(*a.reo, 1, grid * (nt / 32), s) : nullptr;
  kern<<<(unsigned)grid, nt, smem, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                        static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows,
                                        sched);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT>
void launch_split_pipe(const SpmmArgs& a, int mixed, cudaStream_t s) {
  const int64_t rowb = a.F * (int64_t)sizeof(XT);
  if (rowb == 128) {
    if (mixed) return launch_split_pipe_r<VT, XT, YT, 128, true>(a, s);
    return launch_split_pipe_r<VT, XT, YT, 128, false>(a, s);
  }
  if (rowb == 256) {
    if (mixed) return launch_split_pipe_r<VT, XT, YT, 256, true>(a, s);
    return launch_split_pipe_r<VT, XT, YT, 256, false>(a, s);
  }
  throw Error(kErrInvalidArgument, "the pipelined split-chain SpMM needs 128- or 256-byte rows");
}

// kind 10: lean pipelined split-chain kernel; stage = MODE (0 mixed fma, 1 bf16 f32x2 fma)
template <class VT, class XT, class YT, int ROWB, int MODE>
void launch_split_lean_r(const SpmmArgs& a, cudaStream_t s) {
  auto kern = k_spmm_split_lean<VT, XT, YT, ROWB, MODE>;
  constexpr int smem = split_pipe_smem<ROWB>();
  constexpr int nt = 32 * split_pipe_warps<ROWB>();
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem));
  const int64_t need = (a.n_rows * 32 + nt - 1) / nt;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)std::max(per_sm, 1) * sm_count(dev)));
  const int32_t* sched = a.reo ? warp_schedule_for(*a.reo, 1, grid * (nt / 32), s) : nullptr;
  kern<<<(unsigned)grid, nt, smem, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                        static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows,
                                        sched);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT>
void launch_split_lean(const SpmmArgs& a, int mode, cudaStream_t s) {
  const int64_t rowb = a.F * (int64_t)sizeof(XT);
  constexpr bool kBf16 = std::is_same<XT, __nv_bfloat16>::value && std::is_same<VT, __nv_bfloat16>::value;
  SCL_REQUIRE(mode == 0 || (mode == 1 && kBf16), kErrInvalidArgument,
              "lean split-chain SpMM: stage 1 (packed f32x2 fma) needs bf16 storage");
  if (rowb == 128) {
    if constexpr (kBf16) {
      if (mode == 1) return launch_split_lean_r<VT, XT, YT, 128, 1>(a, s);
    }
    return launch_split_lean_r<VT, XT, YT, 128, 0>(a, s);
  }
  if (rowb == 256) {
    if constexpr (kBf16) {
      if (mode == 1) return launch_split_lean_r<VT, XT, YT, 256, 1>(a, s);
    }
    return launch_split_lean_r<VT, XT, YT, 256, 0>(a, s);
  }
  throw Error(kErrInvalidArgument, "the lean split-chain SpMM needs 128- or 256-byte rows");
}

// kind 14: multi-row kernel for 16-bit storage; stage = gathers per batch (4/8/16)
template <class VT, class YT, int ROWB, int U, int MINB>
void launch_rows16_lp_u(const SpmmArgs& a, cudaStream_t s) {
  constexpr int R = 32 / (ROWB / 16);
  auto kern = k_spmm_rows16_lp<VT, YT, ROWB, U, MINB>;
  const int64_t groups = (a.n_rows + R - 1) / R;
  const dim3 grid(persistent_blocks(kern, 0, groups, 32));
  const int32_t* sched = a.reo ? warp_schedule_for(*a.reo, R, (int64_t)grid.x * (kSpmmThreads / 32), s) : nullptr;
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                     static_cast<const VT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows,
                                     sched);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class YT>
void launch_rows16_lp(const SpmmArgs& a, int U, cudaStream_t s) {
  const int64_t rowb = a.F * 2;
  SCL_REQUIRE(reinterpret_cast<uintptr_t>(a.X) % 16 == 0 && reinterpret_cast<uintptr_t>(a.Y) % 16 == 0,
              kErrInvalidArgument, "the 16-bit multi-row SpMM needs 16-byte aligned X and Y");
#define SCL_LP_CASE(RB)                                                               \
  if (rowb == RB) {                                                                   \
    if (U == 4) return launch_rows16_lp_u<VT, YT, RB, 4, 3>(a, s);                   \
    if (U == 8) return launch_rows16_lp_u<VT, YT, RB, 8, 2>(a, s);                   \
    if (U == 16) return launch_rows16_lp_u<VT, YT, RB, 16, 2>(a, s);                 \
    throw Error(kErrInvalidArgument, "16-bit multi-row SpMM batch must be 4, 8 or 16"); \
  }
  SCL_LP_CASE(128)
  SCL_LP_CASE(256)
#undef SCL_LP_CASE
  throw Error(kErrInvalidArgument, "the 16-bit multi-row SpMM needs 128- or 256-byte rows");
}

// kinds 5/6: split-chain kernel for 16-bit storage (6 = mixed-precision fma);
// stage = gathers per lane per batch (U * chains must divide 32)
template <class VT, class XT, class YT, int ROWB, int U, bool MIXED>
void launch_split_ru(const SpmmArgs& a, cudaStream_t s) {
  auto kern = k_spmm_split<VT, XT, YT, ROWB, U, MIXED>;
  const dim3 grid(persistent_blocks(kern, 0, a.n_rows, 32));
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                     static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, bool MIXED>
void launch_split(const SpmmArgs& a, int U, cudaStream_t s) {
  const int64_t rowb = a.F * (int64_t)sizeof(XT);
  if (rowb == 128) {  // 4 chains: U in {2, 4, 8}
    if (U == 2) return launch_split_ru<VT, XT, YT, 128, 2, MIXED>(a, s);
    if (U == 4) return launch_split_ru<VT, XT, YT, 128, 4, MIXED>(a, s);
    if (U == 8) return launch_split_ru<VT, XT, YT, 128, 8, MIXED>(a, s);
  } else if (rowb == 256) {  // 2 chains: U in {4, 8, 16}
    if (U == 4) return launch_split_ru<VT, XT, YT, 256, 4, MIXED>(a, s);
    if (U == 8) return launch_split_ru<VT, XT, YT, 256, 8, MIXED>(a, s);
    if (U == 16) return launch_split_ru<VT, XT, YT, 256, 16, MIXED>(a, s);
  } else {
    throw Error(kErrInvalidArgument, "the split-chain SpMM needs 128- or 256-byte rows");
  }
  throw Error(kErrInvalidArgument, "split-chain SpMM batch must be 2/4/8 (128-byte rows) or 4/8/16 (256-byte rows)");
}

// kind 2: register stream (stage = U in {8, 16}); kind 3: cp.async stream
// pipeline (stage = entries per stage in {16, 32}).
template <class VT, class XT, class YT, class AT, int VEC>
void launch_stream(const SpmmArgs& a, int kind, int stage, cudaStream_t s) {
  if (kind == 2 && stage == 8) return launch_stream_u<VT, XT, YT, AT, VEC, 8>(a, s);
  if (kind == 2 && stage == 16) return launch_stream_u<VT, XT, YT, AT, VEC, 16>(a, s);
  if (kind == 3 && stage == 16) return launch_spipe_s<VT, XT, YT, AT, VEC, 16>(a, s);
  if (kind == 3 && stage == 32) return launch_spipe_s<VT, XT, YT, AT, VEC, 32>(a, s);
  throw Error(kErrInvalidArgument, "stream SpMM stage must be 8/16 (kind 2) or 16/32 (kind 3)");
}

// Whole warp per row with a narrow lane chunk (4 or 8 bytes).
template <class VT, class XT, class YT, class AT, int VEC>
void launch_warp(const SpmmArgs& a, cudaStream_t s) {
  auto kern = k_spmm<VT, XT, YT, AT, 32, VEC, 8>;
  const dim3 grid(persistent_blocks(kern, 0, a.n_rows, 32));
  kern<<<grid, kSpmmThreads, 0, s>>>(a.indptr, a.indices, static_cast<const VT*>(a.values),
                                     static_cast<const XT*>(a.X), static_cast<YT*>(a.Y), a.row_map, a.n_rows, a.F);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, class AT>
void launch_typed(const SpmmArgs& a, const SpmmPlan& plan, cudaStream_t s) {
  constexpr int kVec = 16 / (int)sizeof(XT);
  if (plan.vec > 1 && plan.kind == 1) {
    switch (plan.stage) {
      case 4: return launch_pipe_s<VT, XT, YT, AT, kVec, 4>(plan.group, a, s);
      case 8: return launch_pipe_s<VT, XT, YT, AT, kVec, 8>(plan.group, a, s);
      case 16: return launch_pipe_s<VT, XT, YT, AT, kVec, 16>(plan.group, a, s);
      default: throw Error(kErrInvalidArgument, "pipeline stage must be 4, 8 or 16");
    }
  }
  constexpr int kVec8 = 8 / (int)sizeof(XT);  // 8-byte lane chunks
  constexpr int kVec4 = 4 / (int)sizeof(XT);  // 4-byte lane chunks
  if (plan.kind == 4) {
    SCL_REQUIRE(plan.group == 32 && plan.vec * (int64_t)sizeof(XT) * 32 == a.F * (int64_t)sizeof(XT),
                kErrInvalidArgument, "the fixed-pitch SpMM covers a row with one chunk per lane of a warp");
    return launch_row<VT, XT, YT, AT>(a, plan.stage, s);
  }
  if (plan.kind == 7) {
    SCL_REQUIRE(plan.group == 32 && plan.vec * 32 == a.F, kErrInvalidArgument,
                "the flat-stream SpMM covers a row with one chunk per lane of a warp");
    return launch_flow<VT, XT, YT, AT>(a, plan.stage, s);
  }
  if (plan.kind == 12) {
    SCL_REQUIRE((int64_t)plan.group * plan.vec == a.F && plan.vec * (int)sizeof(XT) == 16 &&
                    (plan.group == 8 || plan.group == 16 || plan.group == 32),
                kErrInvalidArgument, "the multi-row SpMM covers a row with 16-byte chunks, 8/16/32 lanes per row");
    if constexpr (std::is_same<VT, XT>::value && std::is_same<XT, YT>::value && std::is_same<YT, AT>::value &&
                  sizeof(AT) >= 4) {
      return launch_rows16<AT>(a, plan.stage, s);
    }
    throw Error(kErrInvalidArgument, "the multi-row SpMM is for FP32 or FP64 values, X and Y of one dtype");
  }
  if (plan.kind == 10) {
    SCL_REQUIRE(plan.vec == kVec && (int64_t)plan.group * kVec == a.F && (plan.stage == 0 || plan.stage == 1),
                kErrInvalidArgument, "the lean split-chain SpMM covers a row with one 16-byte chunk per lane");
    if constexpr (sizeof(XT) == 2 && sizeof(VT) == 2 && sizeof(AT) == 4) {
      return launch_split_lean<VT, XT, YT>(a, plan.stage, s);
    }
    throw Error(kErrInvalidArgument, "the lean split-chain SpMM is for bf16 or f16 storage");
  }
  if (plan.kind == 14) {
    SCL_REQUIRE(plan.vec == kVec && (int64_t)plan.group * kVec == a.F && (plan.group == 8 || plan.group == 16),
                kErrInvalidArgument, "the 16-bit multi-row SpMM covers a row with 16-byte chunks, 8 or 16 lanes per row");
    if constexpr (sizeof(XT) == 2 && std::is_same<VT, XT>::value && sizeof(AT) == 4 &&
                  (std::is_same<YT, XT>::value || std::is_same<YT, float>::value)) {
      return launch_rows16_lp<VT, YT>(a, plan.stage, s);
    }
    throw Error(kErrInvalidArgument, "the 16-bit multi-row SpMM is for bf16 or f16 values and X");
  }
  if (plan.kind == 9) {
    SCL_REQUIRE(plan.vec == kVec && (int64_t)plan.group * kVec == a.F && (plan.stage == 0 || plan.stage == 1),
                kErrInvalidArgument, "the pipelined split-chain SpMM covers a row with one 16-byte chunk per lane");
    if constexpr (sizeof(XT) == 2 && sizeof(VT) == 2 && sizeof(AT) == 4) {
      return launch_split_pipe<VT, XT, YT>(a, plan.stage, s);
    }
    throw Error(kErrInvalidArgument, "the pipelined split-chain SpMM is for bf16 or f16 storage");
  }
  if (plan.kind == 5 || plan.kind == 6) {
    SCL_REQUIRE(plan.vec == kVec && (int64_t)plan.group * kVec == a.F, kErrInvalidArgument,
                "the split-chain SpMM covers a row with one 16-byte chunk per lane of a group");
    if constexpr (sizeof(XT) == 2 && sizeof(VT) == 2 && sizeof(AT) == 4) {
      if (plan.kind == 6) return launch_split<VT, XT, YT, true>(a, plan.stage, s);
      return launch_split<VT, XT, YT, false>(a, plan.stage, s);
    }
    throw Error(kErrInvalidArgument, "the split-chain SpMM is for bf16 or f16 storage");
  }
  if (plan.kind == 2 || plan.kind == 3) {
    SCL_REQUIRE(plan.group == 32, kErrInvalidArgument, "the stream SpMM uses a whole warp per row block");
    const int k = plan.kind, st = plan.stage;
    if (plan.vec == kVec) return launch_stream<VT, XT, YT, AT, kVec>(a, k, st, s);
    if constexpr (kVec8 > 1) {
      if (plan.vec == kVec8) return launch_stream<VT, XT, YT, AT, (kVec8 > 1 ? kVec8 : 2)>(a, k, st, s);
    }
    if constexpr (kVec4 > 1) {
      if (plan.vec == kVec4) return launch_stream<VT, XT, YT, AT, (kVec4 > 1 ? kVec4 : 2)>(a, k, st, s);
    }
    if constexpr (sizeof(XT) >= 4) {
      if (plan.vec == 1) return launch_stream<VT, XT, YT, AT, 1>(a, k, st, s);
    }
    throw Error(kErrInvalidArgument, "unsupported lane chunk width for the stream SpMM");
  }
  if (plan.vec == kVec) return launch_g<VT, XT, YT, AT, kVec>(plan.group, a, s);
  if (plan.vec == 1) return launch_g<VT, XT, YT, AT, 1>(plan.group, a, s);
  // narrower chunks: one warp per row (no divergence between rows in a warp)
  SCL_REQUIRE(plan.group == 32, kErrInvalidArgument, "4- and 8-byte lane chunks need a whole warp per row");
  if constexpr (kVec8 > 1) {
    if (plan.vec == kVec8) return launch_warp<VT, XT, YT, AT, (kVec8 > 1 ? kVec8 : 2)>(a, s);
  }
  if constexpr (kVec4 > 1) {
    if (plan.vec == kVec4) return launch_warp<VT, XT, YT, AT, (kVec4 > 1 ? kVec4 : 2)>(a, s);
  }
  throw Error(kErrInvalidArgument, "unsupported lane chunk width");
}

}  // namespace

// ---- plan selection -----------------------------------------------------------
SpmmPlan default_spmm_plan(int64_t F, DType xtype, const void* X, const void* Y, DType ytype) {
  SpmmPlan p;
  const int xs = (int)dtype_size(xtype);
  const int ys = (int)dtype_size(ytype);
  // Rows of 128, 256 or 512 bytes: one warp per row, one 4/8/16-byte chunk per
  // lane — no divergence between rows sharing a warp, one load per entry.
  const int64_t rb = F * xs;
  if (xs == 2 && (rb == 128 || rb == 256) && (reinterpret_cast<uintptr_t>(X) & 15u) == 0 &&
      (reinterpret_cast<uintptr_t>(Y) % (uintptr_t)(8 * ys)) == 0) {
    // 16-bit storage: one 16-byte chunk per lane, 4 (128-byte rows) or 2
    // (256-byte rows) entries per load instruction, mixed-precision fma
    // (measured at 500k cells: the lean cp.async pipeline with mixed-precision
    // fma is fastest for both 128- and 256-byte rows)
    p.group = (int)(rb / 16);
    p.vec = 8;
    p.kind = 10;
    p.stage = 0;
    return p;
  }
  if (rb == 128 || rb == 256 || rb == 512) {
    const int lane_bytes = (int)(rb / 32);
    const int v = lane_bytes / xs;
    if (v >= 1 && (reinterpret_cast<uintptr_t>(X) % lane_bytes) == 0 &&
        (reinterpret_cast<uintptr_t>(Y) % (uintptr_t)(v * ys)) == 0) {
      p.group = 32;
      p.vec = v;
      p.kind = 4;
      p.stage = 16;  // 16 gathers in flight per lane (measured faster than 8 on B200)
      return p;
    }
  }
  const int vec = 16 / xs;
  const bool aligned = ((reinterpret_cast<uintptr_t>(X) & 15u) == 0) && ((reinterpret_cast<uintptr_t>(Y) & 15u) == 0) &&
                       ((F * xs) % 16 == 0) && ((F * ys) % 8 == 0) && (F % vec == 0);
  p.vec = aligned ? vec : 1;
  const int64_t lanes = (F + p.vec - 1) / p.vec;
  int g = 1;
  while (g < lanes && g < 32) g <<= 1;
  p.group = g;
  // the cp.async pipeline hides gather latency without register cost; it needs
  // 16-byte lane chunks and at least 4 lanes per row
  if (p.vec > 1 && p.group >= 4) {
    p.kind = 1;
    p.stage = p.group >= 8 ? 8 : 4;
  }
  return p;
}

std::vector<SpmmPlan> candidate_plans(int64_t F, DType xtype, const void* X, const void* Y, DType ytype) {
  const SpmmPlan d = default_spmm_plan(F, xtype, X, Y, ytype);
  std::vector<SpmmPlan> c{d};
  auto add = [&](int group, int vec, int kind, int stage) {
    SpmmPlan p;
    p.group = group;
    p.vec = vec;
    p.kind = kind;
    p.stage = stage;
    c.push_back(p);
  };
  if (d.kind == 5 || d.kind == 6 || d.kind == 9 || d.kind == 10) {
    // interleaved-chain family (16-bit storage): same bits for every member
    const int rb = (int)(F * (int64_t)dtype_size(xtype));
    const int group = rb / 16;
    const int stages128[] = {2, 4, 8}, stages256[] = {4, 8, 16};
    for (int st : (rb == 128 ? stages128 : stages256)) {
      add(group, 8, 6, st);
      add(group, 8, 5, st);
    }
    add(group, 8, 9, 1);
    add(group, 8, 10, 0);
    if (xtype == kBF16) add(group, 8, 10, 1);
    if ((reinterpret_cast<uintptr_t>(X) & 15u) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15u) == 0)
      for (int st : {4, 8, 16}) add(group, 8, 14, st);
  } else if (d.kind == 4) {
    // sequential-chain family, fixed row pitch
    for (int st : {8, 16, 32}) add(32, d.vec, 4, st);
    for (int st : {8, 16}) add(32, d.vec, 7, st);
    if (spmm_bulk_fits(F, xtype, X, Y) && xtype == ytype)
      for (int st : {2, 3}) add(32, d.vec, 11, st);
    const int rb = (int)(F * (int64_t)dtype_size(xtype));
    if (xtype == ytype && (rb == 128 || rb == 256) && (reinterpret_cast<uintptr_t>(X) & 15u) == 0 &&
        (reinterpret_cast<uintptr_t>(Y) & 15u) == 0)
      for (int st : {4, 8, 16}) add(rb / 16, 16 / (int)dtype_size(xtype), 12, st);
  }
  return c;
}

void spmm_with_plan(const SpmmArgs& a, const SpmmPlan& plan, cudaStream_t s) {
  if (a.n_rows <= 0 || a.F <= 0) return;
  SCL_REQUIRE(plan.kind != 13, kErrInvalidArgument,
              "plan kind 13 (grouped rows) runs on a reordered graph only (scl_gpu_graph_reorder)");
  SCL_REQUIRE(plan.group >= 1 && plan.group <= 32 && (plan.group & (plan.group - 1)) == 0, kErrInvalidArgument,
              "lane-group size must be a power of two in [1, 32]");
  SCL_REQUIRE(plan.kind == 0 || plan.kind == 2 || plan.kind == 3 || plan.kind == 4 || plan.kind == 5 ||
                  plan.kind == 6 || plan.kind == 7 || plan.kind == 9 || plan.kind == 10 || plan.kind == 11 ||
                  plan.kind == 12 || plan.kind == 14 ||
                  (plan.kind == 1 && plan.vec > 1 && plan.group >= 4),
              kErrInvalidArgument, "the pipelined SpMM needs 16-byte lane chunks and a lane group of at least 4");
  if (plan.kind == 11) {
    SCL_REQUIRE(plan.group == 32 && (int64_t)plan.vec * 32 == a.F, kErrInvalidArgument, "the bulk-copy SpMM covers a row with one chunk per lane of a warp");
    return spmm_bulk(a, plan.stage, s);
  }
  if (plan.vec > 1) {
    const int xs = (int)dtype_size(a.xtype), ys = (int)dtype_size(a.ytype);
    const int xb = plan.vec * xs, yb = plan.vec * ys;
    SCL_REQUIRE((xb == 4 || xb == 8 || xb == 16) && a.F % plan.vec == 0 &&
                    reinterpret_cast<uintptr_t>(a.X) % xb == 0 && reinterpret_cast<uintptr_t>(a.Y) % yb == 0,
                kErrInvalidArgument, "vector SpMM plan does not fit this feature block");
    SCL_REQUIRE(xb == 16 || plan.group == 32, kErrInvalidArgument,
                "4- and 8-byte lane chunks need a whole warp per row");
  }
  const DType v = a.vtype, x = a.xtype, y = a.ytype;
  if (v == kF32 && x == kF32 && y == kF32) return launch_typed<float, float, float, float>(a, plan, s);
  if (v == kF64 && x == kF64 && y == kF64) return launch_typed<double, double, double, double>(a, plan, s);
  if (v == kBF16 && x == kBF16 && y == kBF16) return launch_typed<__nv_bfloat16, __nv_bfloat16, __nv_bfloat16, float>(a, plan, s);
  if (v == kBF16 && x == kBF16 && y == kF32) return launch_typed<__nv_bfloat16, __nv_bfloat16, float, float>(a, plan, s);
  if (v == kF16 && x == kF16 && y == kF16) return launch_typed<__half, __half, __half, float>(a, plan, s);
  if (v == kF16 && x == kF16 && y == kF32) return launch_typed<__half, __half, float, float>(a, plan, s);
  throw Error(kErrTypeMismatch, "unsupported (values, X, Y) dtype combination for SpMM");
}

void spmm(const SpmmArgs& a, cudaStream_t s) {
  spmm_with_plan(a, default_spmm_plan(a.F, a.xtype, a.X, a.Y, a.ytype), s);
}

// ---- T-step power iteration --------------------------------------------------
void diffuse(const CsrView& g, const void* X0, DType xtype, void* Y, DType ytype, DType mtype, int64_t F,
             int64_t steps, cudaStream_t s, const SpmmPlan* plan_in) {
  SCL_REQUIRE(g.n_cols <= g.n_rows, kErrDimensionMismatch,
              "diffusion needs column indices within the iterate's rows (n_cols <= n_rows)");
  SCL_REQUIRE(g.vtype == mtype, kErrTypeMismatch, "graph storage dtype must match the iterate dtype");
  const int64_t n = g.n_rows;
  if (steps <= 0 || n == 0 || F == 0) {
    if (X0 != Y) convert_values(X0, xtype, Y, ytype, n * F, s);
    return;
  }
  const size_t esz = dtype_size(mtype);
  DevBuf bufA, bufB;
  const void* src = X0;
  if (xtype != mtype) {
    bufB = DevBuf(n * F * esz, s);
    convert_values(X0, xtype, bufB.p, mtype, n * F, s);
    src = bufB.p;
  }
  SpmmArgs a{};
  a.indptr = g.indptr;
  a.indices = g.indices;
  a.values = g.values;
  a.vtype = g.vtype;
  a.n_rows = n;
  a.F = F;
  for (int64_t st = 0; st < steps; ++st) {
    const bool last = (st == steps - 1);
    void* dst;
    DType dtype_out;
    if (last && Y != src) {
      dst = Y;
      dtype_out = ytype;
    } else if (last) {
      // in place with a single step: compute into scratch, then copy over X0
      if (!bufA.p) bufA = DevBuf(n * F * dtype_size(ytype), s);
      dst = bufA.p;
      dtype_out = ytype;
    } else {
      if (!bufA.p) bufA = DevBuf(n * F * esz, s);
      if (src == bufA.p) {
        if (!bufB.p) bufB = DevBuf(n * F * esz, s);
        dst = bufB.p;
      } else {
        dst = bufA.p;
      }
      dtype_out = mtype;
    }
    a.X = src;
    a.xtype = mtype;
    a.Y = dst;
    a.ytype = dtype_out;
    const SpmmPlan plan = plan_in ? *plan_in : default_spmm_plan(F, mtype, src, dst, dtype_out);
    spmm_with_plan(a, plan, s);
    src = dst;
  }
  if (src != Y) SCL_CUDA(cudaMemcpyAsync(Y, src, n * F * dtype_size(ytype), cudaMemcpyDeviceToDevice, s));
}

}  // namespace sclgpu
