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
template <class T, int VEC>
struct VecIO {
  static_assert(VEC * sizeof(T) == 16 || VEC == 1, "VEC must cover 16 bytes or be scalar");
  template <class A>
  static __device__ __forceinline__ void load(const T* __restrict__ p, A (&out)[VEC]) {
    if constexpr (VEC == 1) {
      out[0] = to_acc<A, T>(__ldg(p));
    } else {
      const uint4 raw = __ldg(reinterpret_cast<const uint4*>(p));
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
      *reinterpret_cast<uint4*>(p) = raw;
    } else if constexpr (BYTES == 32) {  // f32 output of a bf16/f16 (8-wide) chunk
      uint4 raw[2];
      T* e = reinterpret_cast<T*>(raw);
#pragma unroll
      for (int i = 0; i < VEC; ++i) e[i] = from_acc<T, A>(in[i]);
      reinterpret_cast<uint4*>(p)[0] = raw[0];
      reinterpret_cast<uint4*>(p)[1] = raw[1];
    } else {  // 8-byte chunks (e.g. bf16 output from a 4-wide f32 chunk)
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
  const int64_t row = ((int64_t)blockIdx.x * kSpmmThreads + threadIdx.x) / G;
  if (row >= n_rows) return;  // whole groups exit together (G divides 32)

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
        j_l = __ldg(indices + m);
        v_l = values[m];
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
}

// G == 1 needs no shuffles but the template handles it (width-1 shuffles are
// identity operations); keep one instantiation path for simplicity.

template <class VT, class XT, class YT, class AT, int VEC>
void launch_g(int G, const SpmmArgs& a, cudaStream_t s) {
  const int64_t rows_per_block = kSpmmThreads / G;
  const int64_t blocks = (a.n_rows + rows_per_block - 1) / rows_per_block;
  SCL_REQUIRE(blocks <= 0x7fffffffLL, kErrInvalidArgument, "too many rows for one launch");
  const auto* ip = a.indptr;
  const auto* ix = a.indices;
  const auto* vv = static_cast<const VT*>(a.values);
  const auto* xx = static_cast<const XT*>(a.X);
  auto* yy = static_cast<YT*>(a.Y);
  const dim3 grid((unsigned)blocks);
#define SCL_SPMM_CASE(GG, UU)                                                                      \
  case GG:                                                                                         \
    k_spmm<VT, XT, YT, AT, GG, VEC, UU><<<grid, kSpmmThreads, 0, s>>>(ip, ix, vv, xx, yy, a.row_map, \
                                                                     a.n_rows, a.F);               \
    break;
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

template <class VT, class XT, class YT, class AT>
void launch_typed(const SpmmArgs& a, const SpmmPlan& plan, cudaStream_t s) {
  constexpr int kVec = 16 / (int)sizeof(XT);
  if (plan.vec > 1) launch_g<VT, XT, YT, AT, kVec>(plan.group, a, s);
  else launch_g<VT, XT, YT, AT, 1>(plan.group, a, s);
}

}  // namespace

// ---- plan selection -----------------------------------------------------------
SpmmPlan default_spmm_plan(int64_t F, DType xtype, const void* X, const void* Y, DType ytype) {
  SpmmPlan p;
  const int xs = (int)dtype_size(xtype);
  const int ys = (int)dtype_size(ytype);
  const int vec = 16 / xs;
  const bool aligned = ((reinterpret_cast<uintptr_t>(X) & 15u) == 0) && ((reinterpret_cast<uintptr_t>(Y) & 15u) == 0) &&
                       ((F * xs) % 16 == 0) && ((F * ys) % 8 == 0) && (F % vec == 0);
  p.vec = aligned ? vec : 1;
  const int64_t lanes = (F + p.vec - 1) / p.vec;
  int g = 1;
  while (g < lanes && g < 32) g <<= 1;
  p.group = g;
  return p;
}

void spmm_with_plan(const SpmmArgs& a, const SpmmPlan& plan, cudaStream_t s) {
  if (a.n_rows <= 0 || a.F <= 0) return;
  SCL_REQUIRE(plan.group >= 1 && plan.group <= 32 && (plan.group & (plan.group - 1)) == 0, kErrInvalidArgument,
              "lane-group size must be a power of two in [1, 32]");
  if (plan.vec > 1) {
    const int xs = (int)dtype_size(a.xtype);
    SCL_REQUIRE(plan.vec == 16 / xs && a.F % plan.vec == 0 && (reinterpret_cast<uintptr_t>(a.X) & 15u) == 0 &&
                    (reinterpret_cast<uintptr_t>(a.Y) & 15u) == 0,
                kErrInvalidArgument, "vector SpMM plan does not fit this feature block");
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
