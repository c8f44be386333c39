// Tensor-gather SpMM (plan kind 11): Y = P X for FP32 / FP64 storage with
// rows of 128, 256 or 512 bytes. Every output element is the sequential fma
// chain over its row's entries in stored order, the same bits as plan kinds
// 0-4 and 7 (scl-core's spmm_block, scl/kernel/diffusion.hpp:227-278).
//
// The row gathers go to the SM's tensor-memory-access engine instead of the
// load/store path: X is described by a 2-D tensor map (rows of F elements,
// box one row high) and one cp.async.bulk.tensor ... tile::gather4
// instruction copies the X rows of four entries into shared memory. A warp
// owns rows row0, row0 + nw, ... and walks their entries in chunks of at most
// 32 (chunk_cursor.cuh); lane 0 issues the chunk's gathers (eight for a full
// chunk) into one stage of the warp's shared-memory ring, and the stage's
// mbarrier counts the bytes in. No register holds data in flight: the bytes in
// flight are bounded by the ring (NS stages of 32 rows per warp, one CTA per
// SM filling its shared memory), not by the register file. The warp keeps NS-1
// chunks in flight while it consumes the oldest: lane l reads bytes
// [l*LB, (l+1)*LB) of each staged row with one shared load and advances its
// VEC column chains. The (index, value) pairs of the chunk after the one being
// issued are already loading, so a chunk's gathers never wait on its indices.
// A partial group of four is padded with row 0, whose copy lands in a slot
// that is never read.
//
// Every wait on an mbarrier is bounded (2 s of %globaltimer); a wait that gives
// up records kErrConvergence and the warp in the status word, waits a bounded
// time for the warp's other copies in flight, and returns. The host reads the
// word with spmm_bulk_status. A test hook (spmm_bulk_inject_stall) makes one
// warp expect 16 bytes more than it copies, so its first wait runs out.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "chunk_cursor.cuh"
#include "engine.hpp"

namespace sclgpu {
namespace {

constexpr unsigned long long kBulkWaitNs = 2000ull * 1000ull * 1000ull;   // 2 s
constexpr unsigned long long kDrainWaitNs = 200ull * 1000ull * 1000ull;   // 0.2 s
constexpr int kGatherRingBytes = 200 * 1024;  // ring bytes of the one CTA per SM

__device__ int32_t g_bulk_status[2];  // [0] error code, [1] global warp that gave up
__device__ long long g_bulk_stall_warp = -1;

__device__ __forceinline__ unsigned long long bulk_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait suspends the thread for a hardware-defined time before it reports
// failure, so this loop is not a hot spin; it gives up after `limit_ns`.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = bulk_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (bulk_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// Four X rows (coordinates {0, r0..r3} of the row-major tensor map) into four
// consecutive row slots at `dst`; completion counted on `bar`.
__device__ __forceinline__ void gather4_rows(unsigned dst, const CUtensorMap* map, int r0, int r1, int r2, int r3,
                                             unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(bar)
      : "memory");
}

__device__ __forceinline__ float bfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double bfma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <int B> struct BulkVec;
template <> struct BulkVec<4> { using type = unsigned int; };
template <> struct BulkVec<8> { using type = uint2; };
template <> struct BulkVec<16> { using type = uint4; };

template <int ROWB, int NS>
constexpr int bulk_warps() {
  return std::max(1, std::min(16, kGatherRingBytes / (NS * 32 * ROWB)));
}

// A chunk in flight: what consumption needs once its copies have landed.
struct Pend {
  int64_t row;
  int cnt;    // entries (0..32); -1 = no chunk (stream exhausted)
  bool first;
  bool last;
};

__device__ __forceinline__ Pend pend_of(const Chunk& c) {
  Pend p;
  p.row = c.row;
  p.cnt = c.valid ? c.cnt : -1;
  p.first = c.first;
  p.last = c.last;
  return p;
}

template <class T, int ROWB, int WARPS, int NS>
__global__ void __launch_bounds__(32 * WARPS)
k_spmm_gather4(const __grid_constant__ CUtensorMap xmap, const int64_t* __restrict__ indptr,
               const int32_t* __restrict__ indices, const T* __restrict__ values, T* __restrict__ Y,
               const int32_t* __restrict__ row_map, int64_t n_rows) {
  constexpr int LB = ROWB / 32;  // bytes of every row owned by one lane
  constexpr int VEC = LB / (int)sizeof(T);
  constexpr unsigned STAGE = 32u * ROWB;
  static_assert(NS >= 2 && NS <= 8, "ring of 2..8 stages");
  static_assert(VEC >= 1 && (LB == 4 || LB == 8 || LB == 16), "row pitch must be 128, 256 or 512 bytes");
  using R = typename BulkVec<LB>::type;
  extern __shared__ __align__(128) unsigned char smem_bulk[];
  __shared__ __align__(8) unsigned long long s_bar[WARPS][NS];
  __shared__ __align__(16) T s_v[WARPS][NS][32];
  __shared__ __align__(16) int32_t s_j[WARPS][NS][32];
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int64_t nw = (int64_t)gridDim.x * WARPS;
  const int64_t gw = (int64_t)blockIdx.x * WARPS + w;
  if (gw >= n_rows) return;
  unsigned char* ring = smem_bulk + (size_t)w * NS * STAGE;
  const unsigned ring_s = smem_addr(ring);
  const unsigned bar_s = smem_addr(&s_bar[w][0]);
  if ((ring_s & 127u) != 0u) {  // tensor copies want 128-byte aligned destinations
    if (lane == 0) atomicCAS(&g_bulk_status[0], 0, (int32_t)kErrInternal);
    return;
  }
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) mbar_init(bar_s + 8u * s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncwarp();
  const unsigned extra = (g_bulk_stall_warp == gw) ? 16u : 0u;  // test hook: this warp's first wait runs out

  ChunkCursor cur;
  cur.init(indptr, gw, n_rows, nw);
  // (index, value) of the chunk to issue next, loaded one iteration ahead
  auto load_pairs = [&](const Chunk& c, int32_t& j, T& v) {
    j = 0;
    v = T(0);
    if (c.valid && lane < c.cnt) {
      j = __ldcs(indices + c.pos + lane);
      v = __ldcs(values + c.pos + lane);
    }
  };
  unsigned parity = 0u;  // bit s: phase parity the next wait on stage s expects
  unsigned armed = 0u;   // bit s: stage s has copies in flight
  bool issued_any = false;
  auto issue = [&](const Chunk& c, int32_t j, T v, int st) {
    if (!c.valid || c.cnt == 0) return;
    s_v[w][st][lane] = v;
    s_j[w][st][lane] = j;  // lanes past the chunk hold row 0
    __syncwarp();
    if (lane == 0) {
      const int groups = (c.cnt + 3) >> 2;
      unsigned bytes = (unsigned)groups * 4u * ROWB;
      if (extra && !issued_any) bytes += extra;
      const unsigned bar = bar_s + 8u * st;
      mbar_arrive_expect(bar, bytes);
      const unsigned dst = ring_s + st * STAGE;
      for (int gi = 0; gi < groups; ++gi) {
        const int4 r = *reinterpret_cast<const int4*>(&s_j[w][st][4 * gi]);
        gather4_rows(dst + gi * 4u * ROWB, &xmap, r.x, r.y, r.z, r.w, bar);
      }
    }
    issued_any = true;
    armed |= 1u << st;
  };

  Pend q[NS - 1];
  Chunk nxt = cur.next(indptr);
  int32_t jn;
  T vn;
  load_pairs(nxt, jn, vn);
#pragma unroll
  for (int k = 0; k < NS - 1; ++k) {
    const Chunk c = nxt;
    const int32_t jc = jn;
    const T vc = vn;
    nxt = cur.next(indptr);
    load_pairs(nxt, jn, vn);
    issue(c, jc, vc, k);
    q[k] = pend_of(c);
  }
  int st_issue = NS - 1;
  int st_use = 0;
  T acc[VEC];
#pragma unroll
  for (int i = 0; i < VEC; ++i) acc[i] = T(0);
  while (q[0].cnt >= 0) {
    // refill the stage consumed last iteration (all lanes are past their reads)
    __syncwarp();
    {
      const Chunk c = nxt;
      const int32_t jc = jn;
      const T vc = vn;
      nxt = cur.next(indptr);
      load_pairs(nxt, jn, vn);
      issue(c, jc, vc, st_issue);
      const Pend pc = pend_of(c);
      const Pend p = q[0];
#pragma unroll
      for (int k = 0; k < NS - 2; ++k) q[k] = q[k + 1];
      q[NS - 2] = pc;
      // consume chunk p from stage st_use
      if (p.cnt > 0) {
        const unsigned bar = bar_s + 8u * st_use;
        const bool ok = mbar_wait(bar, (parity >> st_use) & 1u, kBulkWaitNs);
        if (!__all_sync(0xffffffffu, ok)) {  // warp-uniform: any lane that gave up fails the warp
          if (lane == 0 && atomicCAS(&g_bulk_status[0], 0, (int32_t)kErrConvergence) == 0)
            g_bulk_status[1] = (int32_t)gw;
          armed &= ~(1u << st_use);
          // bounded wait for this warp's other copies in flight, then leave
#pragma unroll
          for (int s = 0; s < NS; ++s)
            if (armed & (1u << s)) mbar_wait(bar_s + 8u * s, (parity >> s) & 1u, kDrainWaitNs);
          return;
        }
        parity ^= 1u << st_use;
        armed &= ~(1u << st_use);
      }
      if (p.first) {
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] = T(0);
      }
      const unsigned char* sb = ring + st_use * STAGE + lane * LB;
      const T* vb = s_v[w][st_use];
      if (p.cnt == 32) {
#pragma unroll
        for (int t = 0; t < 32; t += 4) {
          T vq[4];
          if constexpr (sizeof(T) == 4) {
            const float4 v4 = *reinterpret_cast<const float4*>(vb + t);
            vq[0] = v4.x; vq[1] = v4.y; vq[2] = v4.z; vq[3] = v4.w;
          } else {
            const double2 a = *reinterpret_cast<const double2*>(vb + t);
            const double2 b = *reinterpret_cast<const double2*>(vb + t + 2);
            vq[0] = a.x; vq[1] = a.y; vq[2] = b.x; vq[3] = b.y;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const R raw = *reinterpret_cast<const R*>(sb + (t + r) * ROWB);
            const T* ex = reinterpret_cast<const T*>(&raw);
#pragma unroll
            for (int i = 0; i < VEC; ++i) acc[i] = bfma(vq[r], ex[i], acc[i]);
          }
        }
      } else {
#pragma unroll 4
        for (int t = 0; t < p.cnt; ++t) {
          const T vv = vb[t];
          const R raw = *reinterpret_cast<const R*>(sb + t * ROWB);
          const T* ex = reinterpret_cast<const T*>(&raw);
#pragma unroll
          for (int i = 0; i < VEC; ++i) acc[i] = bfma(vv, ex[i], acc[i]);
        }
      }
      if (p.last) {
        const int64_t orow = row_map ? (int64_t)row_map[p.row] : p.row;
        R out;
        T* o = reinterpret_cast<T*>(&out);
#pragma unroll
        for (int i = 0; i < VEC; ++i) o[i] = acc[i];
        *reinterpret_cast<R*>(reinterpret_cast<char*>(Y) + orow * ROWB + lane * LB) = out;
      }
    }
    st_issue = (st_issue + 1 == NS) ? 0 : st_issue + 1;
    st_use = (st_use + 1 == NS) ? 0 : st_use + 1;
  }
}

}  // namespace

// The driver's tensor-map encoder, looked up once (shared with the kNN operand maps).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  SCL_REQUIRE(fn != nullptr, kErrFeatureUnavailable, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

namespace {

// X as a row-major [rows, F] tensor whose box is one row of F elements.
CUtensorMap row_gather_map(const void* X, DType t, int64_t rows, int64_t F) {
  alignas(64) CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)F, (cuuint64_t)std::max<int64_t>(rows, 1)};
  const cuuint64_t strides[1] = {(cuuint64_t)(F * (int64_t)dtype_size(t))};
  const cuuint32_t box[2] = {(cuuint32_t)F, 1u};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = tensor_map_encoder()(
      &m, t == kF64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(X), dims,
      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  SCL_REQUIRE(r == CUDA_SUCCESS, kErrInternal, "cuTensorMapEncodeTiled rejected the row-gather tensor map");
  return m;
}

template <class T, int ROWB, int NS>
void launch_bulk_r(const SpmmArgs& a, cudaStream_t s) {
  constexpr int W = bulk_warps<ROWB, NS>();
  constexpr int smem = W * NS * 32 * ROWB;
  auto kern = k_spmm_gather4<T, ROWB, W, NS>;
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * W, smem));
  const int64_t need = (a.n_rows + W - 1) / W;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)std::max(per_sm, 1) * sm_count(dev)));
  const CUtensorMap xmap = row_gather_map(a.X, a.xtype, a.n_rows, a.F);
  kern<<<(unsigned)grid, 32 * W, smem, s>>>(xmap, a.indptr, a.indices, static_cast<const T*>(a.values),
                                           static_cast<T*>(a.Y), a.row_map, a.n_rows);
  SCL_CUDA(cudaGetLastError());
}

template <class T, int ROWB>
void launch_bulk_rowb(const SpmmArgs& a, int ns, cudaStream_t s) {
  switch (ns) {
    case 2: return launch_bulk_r<T, ROWB, 2>(a, s);
    case 3: return launch_bulk_r<T, ROWB, 3>(a, s);
    case 4: return launch_bulk_r<T, ROWB, 4>(a, s);
    case 6: return launch_bulk_r<T, ROWB, 6>(a, s);
    default: throw Error(kErrInvalidArgument, "tensor-gather SpMM: stage (ring depth) must be 2, 3, 4 or 6");
  }
}

}  // namespace

bool spmm_bulk_fits(int64_t F, DType t, const void* X, const void* Y) {
  if (t != kF32 && t != kF64) return false;
  const int64_t rb = F * (int64_t)dtype_size(t);
  if (!(rb == 128 || rb == 256 || rb == 512) || (t == kF64 && rb == 128)) return false;
  const uintptr_t lb = (uintptr_t)(rb / 32);
  return (reinterpret_cast<uintptr_t>(X) % 16u) == 0 && (reinterpret_cast<uintptr_t>(Y) % lb) == 0;
}

void spmm_bulk(const SpmmArgs& a, int ns, cudaStream_t s) {
  SCL_REQUIRE(a.vtype == a.xtype && a.xtype == a.ytype && (a.xtype == kF32 || a.xtype == kF64), kErrTypeMismatch,
              "the tensor-gather SpMM is for FP32 or FP64 values, X and Y of one dtype");
  SCL_REQUIRE(spmm_bulk_fits(a.F, a.xtype, a.X, a.Y), kErrInvalidArgument,
              "the tensor-gather SpMM needs 128/256/512-byte rows (FP64: 256/512), X 16-byte aligned");
  if (a.n_rows <= 0) return;
  const int64_t rb = a.F * (int64_t)dtype_size(a.xtype);
  if (a.xtype == kF32) {
    if (rb == 128) return launch_bulk_rowb<float, 128>(a, ns, s);
    if (rb == 256) return launch_bulk_rowb<float, 256>(a, ns, s);
    return launch_bulk_rowb<float, 512>(a, ns, s);
  }
  if (rb == 256) return launch_bulk_rowb<double, 256>(a, ns, s);
  return launch_bulk_rowb<double, 512>(a, ns, s);
}

int32_t spmm_bulk_status(cudaStream_t s, int32_t* warp) {
  int32_t h[2] = {0, 0};
  SCL_CUDA(cudaMemcpyFromSymbolAsync(h, g_bulk_status, sizeof(h), 0, cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  if (h[0] != 0) {
    const int32_t z[2] = {0, 0};
    SCL_CUDA(cudaMemcpyToSymbolAsync(g_bulk_status, z, sizeof(z), 0, cudaMemcpyHostToDevice, s));
    SCL_CUDA(cudaStreamSynchronize(s));
  }
  if (warp) *warp = h[1];
  return h[0];
}

void spmm_bulk_inject_stall(int64_t warp, cudaStream_t s) {
  const long long w = (long long)warp;
  SCL_CUDA(cudaMemcpyToSymbolAsync(g_bulk_stall_warp, &w, sizeof(w), 0, cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaStreamSynchronize(s));
}

}  // namespace sclgpu
