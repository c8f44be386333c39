// Grouped-row SpMM on the reordered structure (plan kind 13).
//
// One step Y = P X of scl-core's spmm_block (scl/kernel/diffusion.hpp:227-278):
// every output element is the sequential fma chain over its row's entries in
// stored order, the rounding sequence of the reference's axpy_simd, so results
// are bit-identical to the other sequential-chain kernels.
//
// Layout. A row of X is ROWB = 128, 256 or 512 bytes and is covered by
// LPR = ROWB/16 lanes holding 16 bytes each, so one warp serves C = 32/LPR
// rows at once and one 128-bit load instruction gathers C entries. The
// reordered rows (connected components together, longest rows first inside a
// component) are taken C at a time; group g owns rows [gC, gC+C). Its entries
// are stored as blocks of 32 slots: slot s of a block holds entry
// (block * LPR + s % LPR) of row gC + s / LPR, or padding past a row's end. A
// warp therefore loads a block's (index, value) pairs with one coalesced
// 128-byte load each, lane s holding exactly the pair its row segment needs
// LPR steps later; a width-LPR shuffle hands pair t of each row to that row's
// lanes. Rows of a group have nearly equal lengths because of the
// longest-first order, so little is padded and lanes rarely idle.
//
// Per entry this is one shuffle pair, one address, 1/C of a load and
// 16/sizeof(X) fmas per lane — about a third of the instructions of the
// warp-per-row kernel, which leaves the gathers in flight as the limit.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>

#include "engine.hpp"

namespace sclgpu {
namespace {

inline unsigned nblk(int64_t items, int per) {
  int64_t b = (items + per - 1) / per;
  if (b < 1) b = 1;
  if (b > 148LL * 64) b = 148LL * 64;
  return (unsigned)b;
}

template <class T>
__device__ __forceinline__ float widen(T v) {
  if constexpr (std::is_same_v<T, float>) return v;
  else if constexpr (std::is_same_v<T, __nv_bfloat16>) return __bfloat162float(v);
  else return __half2float(v);
}

// 16 bytes of X as VEC accumulator-type values.
template <class XT, int VEC>
__device__ __forceinline__ void unpack16(const uint4& r, float (&x)[VEC]) {
  if constexpr (std::is_same_v<XT, float>) {
    x[0] = __uint_as_float(r.x);
    x[1] = __uint_as_float(r.y);
    x[2] = __uint_as_float(r.z);
    x[3] = __uint_as_float(r.w);
  } else {
    const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if constexpr (std::is_same_v<XT, __nv_bfloat16>) {
        x[2 * i] = __uint_as_float(w[i] << 16);
        x[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
      } else {
        const __half2 h = *reinterpret_cast<const __half2*>(&w[i]);
        const float2 f = __half22float2(h);
        x[2 * i] = f.x;
        x[2 * i + 1] = f.y;
      }
    }
  }
}

template <class YT, int VEC>
__device__ __forceinline__ void store_row_chunk(YT* __restrict__ dst, const float (&acc)[VEC]) {
  if constexpr (std::is_same_v<YT, float>) {
#pragma unroll
    for (int i = 0; i < VEC; i += 4)
      *reinterpret_cast<float4*>(dst + i) = make_float4(acc[i], acc[i + 1], acc[i + 2], acc[i + 3]);
  } else {
    uint32_t w[VEC / 2];
#pragma unroll
    for (int i = 0; i < VEC / 2; ++i) {
      if constexpr (std::is_same_v<YT, __nv_bfloat16>) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(acc[2 * i], acc[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&h);
      } else {
        const __half2 h = __floats2half2_rn(acc[2 * i], acc[2 * i + 1]);
        w[i] = *reinterpret_cast<const uint32_t*>(&h);
      }
    }
#pragma unroll
    for (int i = 0; i < VEC / 2; i += 4) *reinterpret_cast<uint4*>(dst + 2 * i) = make_uint4(w[i], w[i + 1], w[i + 2], w[i + 3]);
  }
}

constexpr int kGroupedThreads = 256;

// MINB: resident CTAs per SM the register budget is sized for.
template <class VT, class XT, class YT, int ROWB, int U, int MINB>
__global__ void __launch_bounds__(kGroupedThreads, MINB)
k_spmm_grouped(const int32_t* __restrict__ lens, const int64_t* __restrict__ boff, const int32_t* __restrict__ gidx,
               const VT* __restrict__ gval, const XT* __restrict__ X, YT* __restrict__ Y,
               const int32_t* __restrict__ row_map, int64_t n_rows, int64_t n_groups, int64_t F) {
  constexpr int LPR = ROWB / 16;           // lanes per row
  constexpr int C = 32 / LPR;              // rows per warp
  constexpr int VEC = 16 / (int)sizeof(XT);  // X elements per lane
  static_assert(LPR == 8 || LPR == 16 || LPR == 32, "row pitch must be 128, 256 or 512 bytes");
  static_assert(LPR % U == 0, "batch must divide the block");
  const int lane = threadIdx.x & 31;
  const int c = lane / LPR;
  const int q = lane % LPR;
  const int64_t nw = ((int64_t)gridDim.x * kGroupedThreads) >> 5;
  const char* __restrict__ Xq = reinterpret_cast<const char*>(X) + q * 16;
  for (int64_t grp = ((int64_t)blockIdx.x * kGroupedThreads + threadIdx.x) >> 5; grp < n_groups; grp += nw) {
    const int64_t row = grp * C + c;
    const int len = row < n_rows ? lens[row] : 0;
    const int64_t b0 = boff[grp], b1 = boff[grp + 1];
    float acc[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
    int32_t j = 0;
    float v = 0.0f;
    if (b0 < b1) {
      j = __ldcs(gidx + b0 * 32 + lane);
      v = widen(__ldcs(gval + b0 * 32 + lane));
    }
    int left = len;  // entries of this lane's row not yet consumed
    for (int64_t b = b0; b < b1; ++b) {
      int32_t jn = 0;
      float vn = 0.0f;
      if (b + 1 < b1) {
        jn = __ldcs(gidx + (b + 1) * 32 + lane);
        vn = widen(__ldcs(gval + (b + 1) * 32 + lane));
      }
      const int kmax = left < LPR ? left : LPR;
      const bool full = __reduce_min_sync(0xffffffffu, (unsigned)(kmax < 0 ? 0 : kmax)) == (unsigned)LPR;
      const int kwarp = (int)__reduce_max_sync(0xffffffffu, (unsigned)(kmax < 0 ? 0 : kmax));
#pragma unroll
      for (int t = 0; t < LPR; t += U) {
        if (t >= kwarp) break;
        uint4 xr[U];
        float vv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int32_t jj = __shfl_sync(0xffffffffu, j, t + u, LPR);
          vv[u] = __shfl_sync(0xffffffffu, v, t + u, LPR);
          if (full || t + u < kmax)
            xr[u] = __ldg(reinterpret_cast<const uint4*>(Xq + (size_t)(uint32_t)jj * (size_t)ROWB));
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (full || t + u < kmax) {
            float x[VEC];
            unpack16<XT, VEC>(xr[u], x);
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = __fmaf_rn(vv[u], x[i], acc[i]);
          }
        }
      }
      left -= LPR;
      j = jn;
      v = vn;
    }
    if (row < n_rows) {
      const int64_t orow = row_map ? (int64_t)row_map[row] : row;
      store_row_chunk<YT, VEC>(Y + orow * F + q * VEC, acc);
    }
  }
}

// ---- layout build ----------------------------------------------------------------------
__global__ void k_group_lens(const int64_t* __restrict__ indptr, int64_t n, int C, int LPR,
                             int32_t* __restrict__ lens, int64_t* __restrict__ nblocks, int64_t n_groups) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_groups; g += (int64_t)gridDim.x * blockDim.x) {
    int64_t mx = 0;
    for (int c = 0; c < C; ++c) {
      const int64_t r = g * C + c;
      int64_t l = 0;
      if (r < n) {
        l = indptr[r + 1] - indptr[r];
        lens[r] = (int32_t)l;
      }
      mx = l > mx ? l : mx;
    }
    nblocks[g] = (mx + LPR - 1) / LPR;
  }
}

// Warp per group: slot s of block b holds entry b*LPR + s%LPR of row gC + s/LPR
// (gmap = its position in the reordered entry arrays, -1 for padding).
__global__ void k_group_fill(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices, int64_t n,
                             int C, int LPR, const int64_t* __restrict__ boff, int64_t n_groups,
                             int32_t* __restrict__ gidx, int32_t* __restrict__ gmap) {
  const int lane = threadIdx.x & 31;
  const int c = lane / LPR, k = lane % LPR;
  for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < n_groups;
       g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t r = g * C + c;
    const int64_t s = r < n ? indptr[r] : 0, e = r < n ? indptr[r + 1] : 0;
    for (int64_t b = boff[g]; b < boff[g + 1]; ++b) {
      const int64_t p = s + (b - boff[g]) * LPR + k;
      const int64_t slot = b * 32 + lane;
      if (p < e) {
        gidx[slot] = indices[p];
        gmap[slot] = (int32_t)p;
      } else {
        gidx[slot] = 0;
        gmap[slot] = -1;
      }
    }
  }
}

template <class T>
__global__ void k_group_values(const T* __restrict__ src, const int32_t* __restrict__ gmap, int64_t slots,
                               T* __restrict__ dst) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < slots; q += (int64_t)gridDim.x * blockDim.x) {
    const int32_t p = gmap[q];
    dst[q] = p >= 0 ? src[p] : T(0);
  }
}

template <class VT, class XT, class YT, int ROWB, int U>
void launch_grouped_u(const Grouped& gr, const SpmmArgs& a, cudaStream_t s) {
  constexpr int MINB = (U <= 4) ? 4 : (U == 8 ? 3 : 2);
  auto kern = k_spmm_grouped<VT, XT, YT, ROWB, U, MINB>;
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGroupedThreads, 0));
  const int64_t warps_needed = gr.n_groups;
  const int64_t blocks_needed = (warps_needed * 32 + kGroupedThreads - 1) / kGroupedThreads;
  const int64_t cap = (int64_t)sm_count(dev) * std::max(per_sm, 1);
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min(blocks_needed, cap));
  kern<<<grid, kGroupedThreads, 0, s>>>(gr.lens.as<int32_t>(), gr.boff.as<int64_t>(), gr.gidx.as<int32_t>(),
                                        static_cast<const VT*>(gr.gval.p), static_cast<const XT*>(a.X),
                                        static_cast<YT*>(a.Y), a.row_map, a.n_rows, gr.n_groups, a.F);
  SCL_CUDA(cudaGetLastError());
}

template <class VT, class XT, class YT, int ROWB>
void launch_grouped_r(const Grouped& gr, const SpmmArgs& a, int U, cudaStream_t s) {
  if (U == 4) return launch_grouped_u<VT, XT, YT, ROWB, 4>(gr, a, s);
  if (U == 8) return launch_grouped_u<VT, XT, YT, ROWB, 8>(gr, a, s);
  if constexpr (ROWB >= 256) {
    if (U == 16) return launch_grouped_u<VT, XT, YT, ROWB, 16>(gr, a, s);
  }
  throw Error(kErrInvalidArgument, "grouped SpMM batch must be 4, 8 or 16 (16 needs rows of at least 256 bytes)");
}

template <class VT, class XT, class YT>
void launch_grouped(const Grouped& gr, const SpmmArgs& a, int U, cudaStream_t s) {
  const int64_t rb = a.F * (int64_t)sizeof(XT);
  if (rb == 128) return launch_grouped_r<VT, XT, YT, 128>(gr, a, U, s);
  if (rb == 256) return launch_grouped_r<VT, XT, YT, 256>(gr, a, U, s);
  if (rb == 512) return launch_grouped_r<VT, XT, YT, 512>(gr, a, U, s);
  throw Error(kErrInvalidArgument, "the grouped SpMM needs 128-, 256- or 512-byte rows");
}

}  // namespace

int grouped_rows_per_warp(int64_t F, DType xtype) {
  const int64_t rb = F * (int64_t)dtype_size(xtype);
  if (rb == 128) return 4;
  if (rb == 256) return 2;
  if (rb == 512) return 1;
  return 0;
}

bool grouped_fits(int64_t F, DType xtype, const void* X, const void* Y, DType ytype) {
  if (grouped_rows_per_warp(F, xtype) == 0) return false;
  if (xtype == kF64) return false;  // FP32 accumulation only
  if ((reinterpret_cast<uintptr_t>(X) & 15u) != 0) return false;
  const int vec = 16 / (int)dtype_size(xtype);
  return (reinterpret_cast<uintptr_t>(Y) % (uintptr_t)(vec * dtype_size(ytype))) == 0 &&
         ((F * (int64_t)dtype_size(ytype)) % 16) == 0;
}

void build_grouped(const CsrView& r, int C, Grouped& gr, cudaStream_t s) {
  SCL_REQUIRE(C == 1 || C == 2 || C == 4, kErrInvalidArgument, "rows per group must be 1, 2 or 4");
  const int64_t n = r.n_rows;
  const int LPR = 32 / C;
  gr.C = C;
  gr.n_groups = (n + C - 1) / C;
  gr.lens = DevBuf(std::max<int64_t>(n, 1) * 4, s);
  DevBuf nb((gr.n_groups + 1) * 8, s);
  k_group_lens<<<nblk(gr.n_groups, 256), 256, 0, s>>>(r.indptr, n, C, LPR, gr.lens.as<int32_t>(),
                                                      nb.as<int64_t>(), gr.n_groups);
  SCL_CUDA(cudaGetLastError());
  gr.boff = DevBuf((gr.n_groups + 1) * 8, s);
  exclusive_scan_i64(nb.as<int64_t>(), gr.boff.as<int64_t>(), gr.n_groups, s);
  int64_t total = 0;
  SCL_CUDA(cudaMemcpyAsync(&total, gr.boff.as<int64_t>() + gr.n_groups, 8, cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  gr.n_blocks = total;
  const int64_t slots = std::max<int64_t>(total, 1) * 32;
  gr.gidx = DevBuf(slots * 4, s);
  gr.gmap = DevBuf(slots * 4, s);
  k_group_fill<<<nblk(gr.n_groups * 32, 256), 256, 0, s>>>(r.indptr, r.indices, n, C, LPR, gr.boff.as<int64_t>(),
                                                          gr.n_groups, gr.gidx.as<int32_t>(), gr.gmap.as<int32_t>());
  SCL_CUDA(cudaGetLastError());
  gr.values_version = 0;
  gr.vtype = kF32;
}

void grouped_values(const void* vals, DType t, uint64_t version, Grouped& gr, cudaStream_t s) {
  const size_t es = dtype_size(t);
  const int64_t slots = std::max<int64_t>(gr.n_blocks, 1) * 32;
  if (!gr.gval.p || gr.vtype != t) gr.gval = DevBuf(slots * es, s);
  gr.vtype = t;
  const unsigned b = nblk(slots, 256);
  if (es == 8)
    k_group_values<uint64_t><<<b, 256, 0, s>>>((const uint64_t*)vals, gr.gmap.as<int32_t>(), slots, gr.gval.as<uint64_t>());
  else if (es == 4)
    k_group_values<uint32_t><<<b, 256, 0, s>>>((const uint32_t*)vals, gr.gmap.as<int32_t>(), slots, gr.gval.as<uint32_t>());
  else
    k_group_values<uint16_t><<<b, 256, 0, s>>>((const uint16_t*)vals, gr.gmap.as<int32_t>(), slots, gr.gval.as<uint16_t>());
  SCL_CUDA(cudaGetLastError());
  gr.values_version = version;
}

void spmm_grouped(const Grouped& gr, const SpmmArgs& a, int U, cudaStream_t s) {
  if (a.n_rows <= 0 || a.F <= 0) return;
  SCL_REQUIRE(grouped_rows_per_warp(a.F, a.xtype) == gr.C, kErrInvalidArgument,
              "grouped layout does not match the row pitch");
  SCL_REQUIRE(grouped_fits(a.F, a.xtype, a.X, a.Y, a.ytype), kErrInvalidArgument,
              "grouped SpMM plan does not fit this feature block");
  SCL_REQUIRE(gr.vtype == a.vtype, kErrTypeMismatch, "grouped values are in another dtype");
  const DType v = a.vtype, x = a.xtype, y = a.ytype;
  if (v == kF32 && x == kF32 && y == kF32) return launch_grouped<float, float, float>(gr, a, U, s);
  if (v == kBF16 && x == kBF16 && y == kBF16) return launch_grouped<__nv_bfloat16, __nv_bfloat16, __nv_bfloat16>(gr, a, U, s);
  if (v == kBF16 && x == kBF16 && y == kF32) return launch_grouped<__nv_bfloat16, __nv_bfloat16, float>(gr, a, U, s);
  if (v == kF16 && x == kF16 && y == kF16) return launch_grouped<__half, __half, __half>(gr, a, U, s);
  if (v == kF16 && x == kF16 && y == kF32) return launch_grouped<__half, __half, float>(gr, a, U, s);
  throw Error(kErrTypeMismatch, "unsupported (values, X, Y) dtype combination for the grouped SpMM");
}

}  // namespace sclgpu
