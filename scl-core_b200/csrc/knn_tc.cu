// Brute-force k-nearest neighbours with a tensor-core filter
// (scl/kernel/neighbors.hpp:319-478), any feature count and any k.
//
// The reference walks every candidate j of a query i in increasing order:
// skip j when (sqrt(n_i) - sqrt(n_j))^2 >= the current k-th distance,
// otherwise dist_sq = max(0, n_i + n_j - 2 * dot) with dot the sequential fma
// chain over the features, and offer (dist_sq, j) to a max-heap of k entries.
// Only the candidates the heap can act on matter to the result: every
// candidate while the heap is short, afterwards those strictly below its top.
//
// Here the tensor cores find those candidates. A CTA owns 256 queries, two
// halves of 128 (the rows of one tcgen05.mma, M = 128), and streams every
// candidate tile of 256 rows (N = 256) through a TMA ring; both halves'
// MMAs read the same candidate tile, so each tile gives the 256 x 256
// approximate inner products, accumulated in FP32 in tensor memory (one
// accumulator of 256 columns per half, 512 in all; the epilogue releases it
// as soon as it has read it, so the MMAs of tile t + 1 overlap the rest of
// tile t's work). The operands are the samples rounded to
// BF16, K-major rows of 64 values (128 bytes) in the 128-byte swizzled layout
// both TMA and the MMA descriptors use. Two more K columns carry -n_j / 2 as a
// BF16 pair (hi + lo) against ones on the query side, so the accumulator
// holds s_ij ~ dot_ij - n_j / 2 and n_i - 2 s_ij approximates dist_sq.
//
// A rigorous bound B_it on |approximate - exact dist_sq| over query i and
// tile t (below) turns that into a filter: candidate j can only matter when
// s_ij > theta = (n_i - M_i - B_it) / 2, M_i being the heap's current top.
// The epilogue thread of query i reads its accumulator row from tensor memory
// and replays, in increasing j, exactly the candidates the filter keeps: the
// reference's skip test, the exact FP32/FP64 dot (the same fma chain over the
// same dense row), the same clamp and the same heap rules, with the heap in
// the caller's output arrays. Nothing the filter drops could have changed the
// heap, so indices and distances, ties included, are the reference's.
//
// Bound. With q~, c~ the BF16 roundings (relative error <= 2^-8 each),
// R_i = ||x_i|| (computed here, rounded up), hi + lo = -n_j / 2 to 2^-16
// relative, and the FP32 accumulation inside the tensor core taken at a
// generous (K / 16 + 4) * 2^-18 of the summed magnitudes:
//   |exact - (n_i - 2 s_ij)| <= beta R_i R_j + gamma_n |n_j|
//                               + 2^-20 (|n_i| + |n_j| + 2 R_i R_j + |M_i|)
// with beta = 2^-5 + (d + 64) 2^-19 and gamma_n = 2^-14 + (d + 64) 2^-18;
// R_j and |n_j| are replaced by their maxima over the tile. Inputs that would
// overflow BF16, or non-finite values or norms, switch the filter off (every
// candidate replayed).
//
// Every wait on an mbarrier is bounded (2 s of %globaltimer); a wait that
// runs out records kErrConvergence in the status word, raises an abort flag
// that ends the other roles' loops, and the CTA drains its copies and MMAs
// before freeing tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>

#include "engine.hpp"

namespace sclgpu {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();  // spmm_bulk.cu

namespace {

// Test hook: the MMA thread of this CTA never signals its first accumulator,
// so that CTA's epilogue wait runs out (the error path of the bounded waits,
// exercised without any fault). -1 = off.
__device__ long long g_knn_tc_stall_cta = -1;

constexpr int kTcQ = 256;                   // queries per CTA: two MMAs of M = 128 share every candidate tile
constexpr int kTcM = 128;                   // MMA M: tensor-memory lanes
constexpr int kTcEpiWarps = kTcQ / 32;      // one epilogue thread per query
constexpr int kTcN = 256;                   // candidates per tile: MMA N
constexpr int kTcK = 64;                    // BF16 values per 128-byte swizzled row chunk
constexpr int kTcMaxStages = 4;             // candidate ring depth (at most)
constexpr int kTcThreads = 32 * (kTcEpiWarps + 2);  // epilogue warps, a TMA warp, an MMA warp
constexpr int kTcProducerWarp = kTcEpiWarps, kTcMmaWarp = kTcEpiWarps + 1;
constexpr int kTcResidentChunks = 2;        // queries kept resident up to 128 K columns
constexpr unsigned kChunkA = kTcQ * 128u;   // 32 KB: 256 query rows x 128 bytes
constexpr unsigned kHalfA = kTcM * 128u;    // the rows of one MMA
constexpr unsigned kChunkB = kTcN * 128u;   // 32 KB: 256 candidate rows x 128 bytes
constexpr unsigned kTmemCols = 2 * kTcN;    // one FP32 accumulator of 256 columns per query half
constexpr unsigned long long kTcWaitNs = 2000ull * 1000ull * 1000ull;   // 2 s
constexpr unsigned long long kTcDrainNs = 200ull * 1000ull * 1000ull;   // 0.2 s

// instruction descriptor of tcgen05.mma kind::f16: BF16 A and B, FP32 D,
// both K-major, M = 128, N = 256
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ unsigned long long tc_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
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
// Bounded wait for the phase of `parity` to complete; false on time-out or
// when another role has aborted.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, const volatile int* abort_flag,
                                          unsigned long long limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = tc_ns();
  unsigned sleep_ns = 32;
  while (!mbar_try(bar, parity)) {
    if (*abort_flag) return false;
    if (tc_ns() - t0 > limit_ns) return false;
    __nanosleep(sleep_ns);  // a waiting role must not take issue slots from the epilogue warps
    if (sleep_ns < 512) sleep_ns <<= 1;
  }
  return true;
}

__device__ __forceinline__ void tma_tile2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (rows of 128 bytes), descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(unsigned addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ float tfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double tfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float tsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double tsqrt(double a) { return __dsqrt_rn(a); }

template <class T>
__device__ __forceinline__ __nv_bfloat16 to_bf16(T v) {
  if constexpr (sizeof(T) == 4) return __float2bfloat16_rn(v);
  else return __double2bfloat16(v);
}

// ---- preparation ---------------------------------------------------------------------------
// Warp per sample row j: the query operand row (x rounded to BF16, then two
// ones), the candidate operand row (x rounded to BF16, then -n_j / 2 as hi +
// lo), zero padding to Kp; the row again in T with a 16-byte pitch dp (zeros
// past d) for the exact dot products; R_j = ||x_j|| rounded up; flag[0] = 1
// when the filter cannot be trusted (non-finite values or norms, values near
// BF16's range).
template <class T>
__global__ void k_tc_prep(const T* __restrict__ X, const T* __restrict__ norms, int64_t n, int d, int Kp, int dp,
                          __nv_bfloat16* __restrict__ Qb, __nv_bfloat16* __restrict__ Cb, T* __restrict__ Xp,
                          float* __restrict__ Rn, int32_t* __restrict__ flag) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const double kBig = 1.0e30;  // far below BF16's overflow threshold, far above any sane sample value
  for (int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n; j += nw) {
    const T* x = X + j * (int64_t)d;
    const double nj = (double)norms[j];
    const float h = (float)(-0.5 * nj);
    const __nv_bfloat16 hi = __float2bfloat16_rn(h);
    const __nv_bfloat16 lo = __float2bfloat16_rn(h - __bfloat162float(hi));
    const __nv_bfloat16 one = __float2bfloat16_rn(1.0f);
    double ss = 0.0;
    bool bad = false;
    for (int f = lane; f < Kp; f += 32) {
      __nv_bfloat16 q, c;
      T xv = T(0);
      if (f < d) {
        xv = x[f];
        const double dv = (double)xv;
        bad |= !(fabs(dv) < kBig);
        ss += dv * dv;
        q = c = to_bf16(xv);
      } else if (f == d) {
        q = one;
        c = hi;
      } else if (f == d + 1) {
        q = one;
        c = lo;
      } else {
        q = c = __float2bfloat16_rn(0.0f);
      }
      Qb[j * (int64_t)Kp + f] = q;
      Cb[j * (int64_t)Kp + f] = c;
      if (f < dp) Xp[j * (int64_t)dp + f] = xv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      if (bad || !(fabs(nj) < kBig)) atomicExch(flag, 1);
      Rn[j] = __double2float_ru(sqrt(ss) * (1.0 + 1.0e-6));
    }
  }
}

// Per candidate tile: the largest R_j and |n_j| (rounded up to float).
template <class T>
__global__ void k_tc_tile_max(const float* __restrict__ Rn, const T* __restrict__ norms, int64_t n,
                              float* __restrict__ Rmax, float* __restrict__ Nmax) {
  const int64_t t = blockIdx.x;
  const int64_t j = t * kTcN + threadIdx.x;
  float r = 0.0f, m = 0.0f;
  if (j < n) {
    r = Rn[j];
    m = __double2float_ru(fabs((double)norms[j]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, o));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  __shared__ float sr[kTcN / 32], sm[kTcN / 32];
  if ((threadIdx.x & 31) == 0) {
    sr[threadIdx.x >> 5] = r;
    sm[threadIdx.x >> 5] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kTcN / 32; ++w) {
      r = fmaxf(r, sr[w]);
      m = fmaxf(m, sm[w]);
    }
    Rmax[t] = r;
    Nmax[t] = m;
  }
}

template <class T>
__global__ void k_tc_sqrt(const T* __restrict__ a, int64_t n, T* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = tsqrt(a[i]);
}

// ---- the search ------------------------------------------------------------------------------
struct TcParams {
  int64_t n;
  int d;
  int dp;         // pitch of the padded rows (16 bytes)
  int n_chunks;   // Kp / 64
  int k;
  int resident;   // queries loaded once (n_chunks <= kTcResidentChunks)
  int stages;     // candidate ring depth
  int heap_smem;  // heaps in shared memory ([k][128]); else in the output arrays
  int cap;        // kept candidates an epilogue lane queues before it computes their exact distances
  int per_cand;   // per-candidate thresholds (R_j, |n_j|) instead of the tile maxima
  int prefetch;   // bulk-prefetch each tile's padded rows into L2 ahead of the exact dot products
  unsigned off_warp, warp_bytes, off_heap;  // byte offsets in the aligned dynamic shared memory
  double beta, gamma_n;
  int32_t* status;  // [0] error code, [1] CTA that gave up
  const int32_t* flag;
};

// The filter threshold of one query against candidates whose R_j and |n_j|
// are at most rr_j and nn_j: candidates with s_ij at or below it cannot reach
// the heap. -inf (keep everything) while the heap fills or when it is NaN.
template <class T>
__device__ __forceinline__ float tc_theta(bool full, T ni, T maxd, float Ri, float Rj, float Nj, double beta,
                                          double gamma_n) {
  if (!full) return -INFINITY;
  const double n_i = (double)ni, M = (double)maxd, rr = (double)Ri * (double)Rj;
  const double B = beta * rr + gamma_n * (double)Nj + 0x1p-20 * (fabs(n_i) + (double)Nj + 2.0 * rr + fabs(M));
  const double th = 0.5 * (n_i - M - B);
  if (th != th) return -INFINITY;
  return __double2float_rd(th);
}

// 64 consecutive FP32 accumulator columns of this thread's tensor-memory lane:
// two loads, one wait. Empty asm statements after the wait take the registers
// as operands, so no use of them can be scheduled before the loads completed.
__device__ __forceinline__ void tmem_ld32_issue(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_pin32(uint32_t (&r)[32]) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  uint32_t a[32], b[32];
  tmem_ld32_issue(taddr, a);
  tmem_ld32_issue(taddr + 32u, b);
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  tmem_pin32(a);
  tmem_pin32(b);
#pragma unroll
  for (int c = 0; c < 32; ++c) {
    v[c] = __uint_as_float(a[c]);
    v[32 + c] = __uint_as_float(b[c]);
  }
}

// The reference's dist_sq for P candidate rows at once: each dot product is
// the sequential fma chain over the features in order (zeros past d change
// nothing), then max(0, fma(-2, dot, n_a + n_b)); the P chains are
// independent, so their row loads are in flight together.
template <class T, int P>
__device__ __forceinline__ void exact_dist_sq_multi(const T* const (&a)[P], const T* const (&b)[P], int dp,
                                                    const T (&na)[P], const T (&nb)[P], T (&out)[P]) {
  T dot[P];
#pragma unroll
  for (int q = 0; q < P; ++q) dot[q] = T(0);
  if constexpr (sizeof(T) == 4) {
#pragma unroll 2
    for (int v = 0; v < dp / 4; ++v) {
      float4 x[P], y[P];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        x[q] = __ldg(reinterpret_cast<const float4*>(a[q]) + v);
        y[q] = __ldg(reinterpret_cast<const float4*>(b[q]) + v);
      }
#pragma unroll
      for (int q = 0; q < P; ++q) {
        dot[q] = tfma(x[q].x, y[q].x, dot[q]);
        dot[q] = tfma(x[q].y, y[q].y, dot[q]);
        dot[q] = tfma(x[q].z, y[q].z, dot[q]);
        dot[q] = tfma(x[q].w, y[q].w, dot[q]);
      }
    }
  } else {
#pragma unroll 2
    for (int v = 0; v < dp / 2; ++v) {
      double2 x[P], y[P];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        x[q] = __ldg(reinterpret_cast<const double2*>(a[q]) + v);
        y[q] = __ldg(reinterpret_cast<const double2*>(b[q]) + v);
      }
#pragma unroll
      for (int q = 0; q < P; ++q) {
        dot[q] = tfma(x[q].x, y[q].x, dot[q]);
        dot[q] = tfma(x[q].y, y[q].y, dot[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const T ds = tfma(T(-2), dot[q], na[q] + nb[q]);
    out[q] = ds < T(0) ? T(0) : ds;
  }
}

// The eight epilogue warps: thread tid owns query q0 + tid, which is lane
// tid % 128 of the accumulator of query half tid / 128. Per tile it reads its
// 256 accumulator columns 64 at a time and keeps, in registers, a bit for
// every candidate whose s_ij is above the query's threshold (one subtraction
// and one funnel shift per candidate), then appends the kept candidates to
// its own queue in shared memory. When the queue would overflow, and after
// the last tile, the thread works through it in increasing j, four at a
// time: the four exact distances as independent chains, then for each in
// order the reference's skip test against the current heap top and the heap
// rules. Thresholds come from the heap top at the start of each tile, which
// only falls, so the filter never drops a candidate the replay would act on.
template <class T, class IT, bool PER_CAND>
__device__ __forceinline__ void tc_epilogue(const TcParams& p, const T* __restrict__ Xp, const T* __restrict__ norms,
                                            const T* __restrict__ snorms, const float* __restrict__ Rn,
                                            const float* __restrict__ Rmax, const float* __restrict__ Nmax,
                                            unsigned char* base, uint32_t tmem, int warp, int lane, int64_t q0,
                                            int64_t ntiles, unsigned long long* accf, unsigned long long* acce,
                                            volatile int* abort_flag, IT* __restrict__ out_idx,
                                            T* __restrict__ out_dist) {
  constexpr int kChunks = kTcN / 32;
  const int tid = warp * 32 + lane;
  const int64_t n = p.n;
  const int64_t i = q0 + tid;
  const bool live = i < n;
  const bool keep_all = *p.flag != 0;
  const int k = p.k, dp = p.dp, qcap = p.cap;
  const T ni = live ? norms[i] : T(0);
  const T si = live ? snorms[i] : T(0);
  const float Ri = live ? Rn[i] : 0.0f;
  // this warp's scratch: each lane's queue of kept candidates (slot s of lane l
  // at s * 32 + l) and the tile's (R_j, |n_j|) for per-candidate thresholds
  unsigned char* ws = base + p.off_warp + (size_t)warp * p.warp_bytes;
  int32_t* Qj = reinterpret_cast<int32_t*>(ws);
  float2* RN = reinterpret_cast<float2*>(Qj + (size_t)qcap * 32);
  const T* xi = Xp + (live ? i : 0) * (int64_t)dp;
  int qn = 0;  // candidates in this lane's queue
  T* Hd;
  IT* Hj;
  int hs;  // heap element m at Hd[m * hs], Hj[m * hs]
  if (p.heap_smem) {
    Hd = reinterpret_cast<T*>(base + p.off_heap) + tid;
    Hj = reinterpret_cast<IT*>(base + p.off_heap + (size_t)kTcQ * k * sizeof(T)) + tid;
    hs = kTcQ;
  } else {
    Hd = out_dist + (live ? i : 0) * (int64_t)k;
    Hj = out_idx + (live ? i : 0) * (int64_t)k;
    hs = 1;
  }
  T maxd = std::numeric_limits<T>::max();
  int cnt = 0;
  // warp w reads lane quarter w % 4 of the accumulator of query half w / 4
  const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * kTcN);

  auto swap_at = [&](int a, int b) {
    const T td = Hd[a * hs];
    const IT tj = Hj[a * hs];
    Hd[a * hs] = Hd[b * hs];
    Hj[a * hs] = Hj[b * hs];
    Hd[b * hs] = td;
    Hj[b * hs] = tj;
  };
  // the reference's heap rules for an offered (dist_sq, j)
  auto offer = [&](T ds, int64_t j) {
    if (cnt < k) {
      int pos = cnt;
      Hd[pos * hs] = ds;
      Hj[pos * hs] = (IT)j;
      while (pos > 0) {  // sift up
        const int parent = (pos - 1) / 2;
        if (Hd[pos * hs] <= Hd[parent * hs]) break;
        swap_at(pos, parent);
        pos = parent;
      }
      ++cnt;
      if (cnt == k) maxd = Hd[0];
      return;
    }
    if (!(ds < maxd)) return;  // maxd is the heap top once the heap is full
    Hd[0] = ds;
    Hj[0] = (IT)j;
    int pos = 0;
    while (true) {  // sift down
      int largest = pos;
      const int l = 2 * pos + 1, r = 2 * pos + 2;
      if (l < cnt && Hd[l * hs] > Hd[largest * hs]) largest = l;
      if (r < cnt && Hd[r * hs] > Hd[largest * hs]) largest = r;
      if (largest == pos) break;
      swap_at(pos, largest);
      pos = largest;
    }
    maxd = Hd[0];
  };

  // exact distances of up to four candidates of this query at once (independent fma chains), then
  // the reference's steps for each in order: the lower-bound skip against the current heap top, the
  // heap rules
  auto run4 = [&](const int64_t (&js)[4], int c) {
    const T* qa[4];
    const T* cb[4];
    T na[4], nb[4], dd[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t j = js[q < c ? q : 0];
      qa[q] = xi;
      cb[q] = Xp + j * dp;
      na[q] = ni;
      nb[q] = norms[j];
    }
    exact_dist_sq_multi<T, 4>(qa, cb, dp, na, nb, dd);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q >= c) break;
      const T ds = dd[q];
      if (cnt >= k && !(ds < maxd)) continue;  // a full heap takes only distances below its top
      const T nd = si - snorms[js[q]];
      if (nd * nd >= maxd) continue;  // the reference's lower-bound skip
      offer(ds, js[q]);
    }
  };
  auto flush_queue = [&]() {
    for (int s0 = 0; s0 < qn; s0 += 4) {
      int64_t js[4];
      const int c = qn - s0 < 4 ? qn - s0 : 4;
#pragma unroll
      for (int q = 0; q < 4; ++q) js[q] = q < c ? (int64_t)Qj[(s0 + q) * 32 + lane] : 0;
      run4(js, c);
    }
    qn = 0;
  };

  for (int64_t t = 0; t < ntiles; ++t) {
    // lane 0 waits for the warp, so the tensor-memory loads below stay warp-uniform
    int ok = 1;
    if (lane == 0) ok = mbar_wait(saddr(accf), (unsigned)(t & 1), abort_flag, kTcWaitNs) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) {
      if (lane == 0 && !*abort_flag) {
        if (atomicCAS(&p.status[0], 0, (int32_t)kErrConvergence) == 0) p.status[1] = (int32_t)blockIdx.x * 8 + 5;
        *abort_flag = 1;
      }
      break;
    }
    tc_fence_after();
    const int64_t tb = t * kTcN;
    const float theta = keep_all ? -INFINITY : tc_theta<T>(cnt >= k, ni, maxd, Ri, Rmax[t], Nmax[t], p.beta, p.gamma_n);
    const bool all = !(theta > -INFINITY);  // heap still filling, or the filter is off
    // per-candidate threshold base_i - b_i R_j - g |n_j|, every rounding downwards
    float base_i = -INFINITY, b_i = 0.0f, g = 0.0f;
    if constexpr (PER_CAND) {
      __syncwarp();
#pragma unroll
      for (int m = 0; m < kChunks; ++m) {
        const int64_t j = tb + m * 32 + lane;
        RN[m * 32 + lane] = j < n ? make_float2(Rn[j], __double2float_ru(fabs((double)norms[j]))) : make_float2(0.f, 0.f);
      }
      __syncwarp();
      if (!all) {
        const double n_i = (double)ni, M = (double)maxd;
        const double bs = 0.5 * (n_i - M - 0x1p-20 * (fabs(n_i) + fabs(M)));
        base_i = bs == bs ? __double2float_rd(bs) : -INFINITY;
        b_i = __double2float_ru(0.5 * (p.beta + 0x1p-19) * (double)Ri);
        g = __double2float_ru(0.5 * (p.gamma_n + 0x1p-20));
      }
    }
    uint32_t mk[kChunks];  // this query's keep bits, chunk by chunk
#pragma unroll
    for (int h = 0; h < kTcN / 64; ++h) {
      float v[64];
      __syncwarp();  // the tensor-memory load is warp-collective
      tmem_ld64(lane_base + (uint32_t)(h * 64), v);
      if (h == kTcN / 64 - 1) {  // the accumulator is read: the MMAs of tile t + 1 may overwrite it
        tc_fence_before();
        mbar_arrive(saddr(acce));
      }
      // bit c set when s_ic > threshold: the sign of threshold - s_ic (nonzero unless equal), shifted in
      // from the top (one funnel shift per candidate) and bit-reversed at the end
      uint32_t m0 = 0, m1 = 0;
      if constexpr (PER_CAND) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const float2 r0 = RN[h * 64 + c];
          m0 = __funnelshift_l(__float_as_uint(__fmaf_rd(-b_i, r0.x, __fmaf_rd(-g, r0.y, base_i)) - v[c]), m0, 1);
        }
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const float2 r1 = RN[h * 64 + 32 + c];
          m1 = __funnelshift_l(__float_as_uint(__fmaf_rd(-b_i, r1.x, __fmaf_rd(-g, r1.y, base_i)) - v[32 + c]), m1, 1);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          m0 = __funnelshift_l(__float_as_uint(theta - v[c]), m0, 1);
          m1 = __funnelshift_l(__float_as_uint(theta - v[32 + c]), m1, 1);
        }
      }
      m0 = __brev(m0);
      m1 = __brev(m1);
      if (all) m0 = m1 = 0xffffffffu;
      mk[2 * h] = m0;
      mk[2 * h + 1] = m1;
    }
    // drop candidates past n and the query itself
    int mine = 0;
#pragma unroll
    for (int ch = 0; ch < kChunks; ++ch) {
      const int64_t j0 = tb + ch * 32;
      uint32_t m = live ? mk[ch] : 0u;
      if (n - j0 < 32) m &= n - j0 <= 0 ? 0u : ((1u << (unsigned)(n - j0)) - 1u);
      if (i >= j0 && i < j0 + 32) m &= ~(1u << (unsigned)(i - j0));
      mk[ch] = m;
      mine += __popc(m);
    }
    // the warp's queues together (so their latencies overlap) when any lane's would overflow; then
    // each lane's candidates of this tile into its queue, or straight through when they alone exceed it
    if (__any_sync(0xffffffffu, qn + mine > qcap)) flush_queue();
    if (mine > qcap) {
      int64_t js[4];
      int c = 0;
#pragma unroll
      for (int ch = 0; ch < kChunks; ++ch)
        for (uint32_t m = mk[ch]; m; m &= m - 1) {
          js[c++] = tb + ch * 32 + (__ffs(m) - 1);
          if (c == 4) {
            run4(js, 4);
            c = 0;
          }
        }
      if (c) run4(js, c);
    } else if (mine) {
#pragma unroll
      for (int ch = 0; ch < kChunks; ++ch)
        for (uint32_t m = mk[ch]; m; m &= m - 1) Qj[(qn++) * 32 + lane] = (int32_t)(tb + ch * 32 + (__ffs(m) - 1));
    }
  }
  flush_queue();
  if (!live || *abort_flag) return;
  // heap sort as the reference does: min-heap build, extract to the back, reverse
  auto sort_sift = [&](int pos, int size) {
    while (true) {
      int smallest = pos;
      const int l = 2 * pos + 1, r = 2 * pos + 2;
      if (l < size && Hd[l * hs] < Hd[smallest * hs]) smallest = l;
      if (r < size && Hd[r * hs] < Hd[smallest * hs]) smallest = r;
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
  T* od = out_dist + i * (int64_t)k;
  IT* oi = out_idx + i * (int64_t)k;
  for (int m = 0; m < k; ++m) {
    if (m < cnt) {
      const T dsq = Hd[m * hs];
      const IT jj = Hj[m * hs];
      od[m] = tsqrt(dsq);
      oi[m] = jj;
    } else {
      od[m] = std::numeric_limits<T>::infinity();
      oi[m] = (IT)-1;
    }
  }
}

template <class T, class IT, bool PER_CAND>
__global__ void __launch_bounds__(kTcThreads, 1)
k_knn_tc(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap cmap,
         const T* __restrict__ Xp, const T* __restrict__ norms, const T* __restrict__ snorms,
         const float* __restrict__ Rn, const float* __restrict__ Rmax, const float* __restrict__ Nmax, TcParams p,
         IT* __restrict__ out_idx, T* __restrict__ out_dist) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  __shared__ __align__(8) unsigned long long s_full[kTcMaxStages], s_empty[kTcMaxStages], s_aload, s_accf, s_acce,
      s_drain;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;
  __shared__ volatile int s_never;  // drains wait for their copies and MMAs even after an abort

  // 1024-byte aligned operand area (the 128-byte swizzle repeats every 8 rows of 128 bytes)
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023u) & ~static_cast<uintptr_t>(1023u));
  const int nK = p.n_chunks;
  const int S = p.stages;
  const bool resident = p.resident != 0;
  unsigned char* a_res = base;  // resident queries: nK chunks of 16 KB
  unsigned char* ring = base + (resident ? (size_t)nK * kChunkA : 0);
  const unsigned stage_bytes = resident ? kChunkB : (kChunkA + kChunkB);  // stage: [B | A]

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int64_t n = p.n;
  const int64_t q0 = (int64_t)blockIdx.x * kTcQ;
  const int64_t ntiles = (n + kTcN - 1) / kTcN;

  if (tid == 32 * kTcProducerWarp) {
    for (int s = 0; s < S; ++s) {
      mbar_init(saddr(&s_full[s]), 1);
      mbar_init(saddr(&s_empty[s]), 1);
    }
    mbar_init(saddr(&s_aload), 1);
    mbar_init(saddr(&s_accf), 1);
    mbar_init(saddr(&s_acce), kTcQ);
    mbar_init(saddr(&s_drain), 1);
    s_abort = 0;
    s_never = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == kTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    tc_fence_before();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  auto give_up = [&](int where) {
    if (atomicCAS(&p.status[0], 0, (int32_t)kErrConvergence) == 0) p.status[1] = (int32_t)blockIdx.x * 8 + where;
    s_abort = 1;
  };

  if (warp == kTcProducerWarp) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int64_t issued = 0;
      if (resident) {
        mbar_expect(saddr(&s_aload), (unsigned)nK * kChunkA);
        for (int c = 0; c < nK; ++c)
          tma_tile2d(saddr(a_res + (size_t)c * kChunkA), &qmap, c * kTcK, (int)q0, saddr(&s_aload));
      }
      for (int64_t t = 0; t < ntiles && !s_abort; ++t) {
        for (int c = 0; c < nK; ++c, ++issued) {
          const int s = (int)(issued % S);
          const unsigned use = (unsigned)(issued / S);
          if (use > 0 && !mbar_wait(saddr(&s_empty[s]), (use - 1) & 1u, &s_abort, kTcWaitNs)) {
            if (!s_abort) give_up(1);
            break;
          }
          unsigned char* st = ring + (size_t)s * stage_bytes;
          mbar_expect(saddr(&s_full[s]), stage_bytes);
          tma_tile2d(saddr(st), &cmap, c * kTcK, (int)(t * kTcN), saddr(&s_full[s]));
          if (c == 0 && p.prefetch) {  // the rows the epilogue's exact dot products of this tile read
            const int64_t rows = (n - t * kTcN) < (int64_t)kTcN ? (n - t * kTcN) : (int64_t)kTcN;
            const T* src = Xp + t * kTcN * (int64_t)p.dp;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src),
                         "r"((unsigned)(rows * p.dp * (int64_t)sizeof(T)))
                         : "memory");
          }
          if (!resident) tma_tile2d(saddr(st + kChunkB), &qmap, c * kTcK, (int)q0, saddr(&s_full[s]));
        }
      }
      // drain: every copy issued into the ring has landed before the CTA ends
      for (int s = 0; s < S; ++s) {
        const int64_t uses = issued / S + ((issued % S) > s ? 1 : 0);
        if (uses > 0) mbar_wait(saddr(&s_full[s]), (unsigned)((uses - 1) & 1), &s_never, kTcDrainNs);
      }
      if (resident) mbar_wait(saddr(&s_aload), 0, &s_never, kTcDrainNs);
    }
  } else if (warp == kTcMmaWarp) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      bool ok = !resident || mbar_wait(saddr(&s_aload), 0, &s_abort, kTcWaitNs);
      if (!ok && !s_abort) give_up(2);
      int64_t it = 0;
      bool issued_any = false;
      for (int64_t t = 0; ok && t < ntiles; ++t) {
        if (t >= 1 && !mbar_wait(saddr(&s_acce), (unsigned)((t - 1) & 1), &s_abort, kTcWaitNs)) {
          if (!s_abort) give_up(3);
          break;
        }
        tc_fence_after();
        const bool stall = t == 0 && g_knn_tc_stall_cta == (long long)blockIdx.x;
        for (int c = 0; c < nK; ++c, ++it) {
          const int s = (int)(it % S);
          const unsigned use = (unsigned)(it / S);
          if (!mbar_wait(saddr(&s_full[s]), use & 1u, &s_abort, kTcWaitNs)) {
            if (!s_abort) give_up(4);
            ok = false;
            break;
          }
          tc_fence_after();
          unsigned char* st = ring + (size_t)s * stage_bytes;
          const unsigned a0 = saddr(resident ? a_res + (size_t)c * kChunkA : st + kChunkB);
          const unsigned b0 = saddr(st);
#pragma unroll
          for (int hq = 0; hq < 2; ++hq)  // the two query halves, each into its own accumulator
#pragma unroll
            for (int kk = 0; kk < kTcK / 16; ++kk)
              umma_bf16(tmem + (uint32_t)(hq * kTcN), sw128_desc(a0 + hq * kHalfA + 32u * kk),
                        sw128_desc(b0 + 32u * kk), (c | kk) != 0 ? 1u : 0u);
          umma_commit(saddr(&s_empty[s]));  // the stage is free once these MMAs have read it
          issued_any = true;
        }
        if (!ok) break;
        if (!stall) umma_commit(saddr(&s_accf));  // the accumulators hold tile t
      }
      if (issued_any) {  // no MMA in flight when the tensor memory is freed
        umma_commit(saddr(&s_drain));
        mbar_wait(saddr(&s_drain), 0, &s_never, kTcDrainNs);
      }
    }
  } else {
    tc_epilogue<T, IT, PER_CAND>(p, Xp, norms, snorms, Rn, Rmax, Nmax, base, tmem, warp, lane, q0, ntiles, &s_accf, &s_acce,
                       &s_abort, out_idx, out_dist);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kTcMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// Row-major [rows, Kp] BF16 operand whose box is 64 values x box_rows rows,
// 128-byte swizzled.
CUtensorMap operand_map(const void* base, int64_t rows, int Kp, int box_rows) {
  alignas(64) CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)std::max<int64_t>(rows, 1)};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * 2u};
  const cuuint32_t box[2] = {(cuuint32_t)kTcK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  SCL_REQUIRE(r == CUDA_SUCCESS, kErrInternal, "cuTensorMapEncodeTiled rejected a kNN operand map");
  return m;
}

template <class T, class IT>
void knn_tc_typed(const T* X, const T* norms, int64_t n, int d, int k, IT* idx, T* dist, cudaStream_t s) {
  int dev = 0, optin = 0, major = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  SCL_REQUIRE(major == 10, kErrFeatureUnavailable, "the tensor-core kNN needs an sm_100 device");
  const int Kp = ((d + 2 + kTcK - 1) / kTcK) * kTcK;
  const int nK = Kp / kTcK;
  constexpr int kVec = 16 / (int)sizeof(T);
  const int dp = ((d + kVec - 1) / kVec) * kVec;
  const int64_t ntiles = (n + kTcN - 1) / kTcN;

  // shared memory: [resident queries | ring | exact distances | pair lists | heaps], the first two
  // 1024-byte aligned; heaps move to the output arrays when they do not fit beside a 2-stage ring
  SCL_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t budget = (size_t)optin - 2048;  // static barriers and the alignment slack
  TcParams p;
  p.n = n;
  p.d = d;
  p.dp = dp;
  p.n_chunks = nK;
  p.k = k;
  p.resident = nK <= kTcResidentChunks ? 1 : 0;
  const size_t a_bytes = p.resident ? (size_t)nK * kChunkA : 0;
  const size_t stage = p.resident ? kChunkB : (size_t)(kChunkA + kChunkB);
  // per epilogue warp: a queue of cap candidates per lane and the tile's (R_j, |n_j|)
  p.cap = 16;
  const size_t warp_bytes = (size_t)p.cap * 32 * 4 + kTcN * 8;
  p.per_cand = d > 128 ? 1 : 0;
  p.prefetch = (size_t)dp * sizeof(T) <= 512 ? 1 : 0;
  const size_t heap_bytes = (size_t)kTcQ * (size_t)k * (sizeof(T) + sizeof(IT));
  p.stages = 0;
  for (int hs = 1; hs >= 0 && p.stages == 0; --hs)
    for (int S = kTcMaxStages; S >= 2; --S)
      if (a_bytes + S * stage + kTcEpiWarps * warp_bytes + (hs ? heap_bytes : 0) <= budget) {
        p.stages = S;
        p.heap_smem = hs;
        break;
      }
  SCL_REQUIRE(p.stages >= 2, kErrInternal, "kNN tile ring exceeds the device's shared memory");
  p.off_warp = (unsigned)(a_bytes + p.stages * stage);
  p.warp_bytes = (unsigned)warp_bytes;
  p.off_heap = p.off_warp + kTcEpiWarps * (unsigned)warp_bytes;
  const size_t smem = 1024 + p.off_heap + (p.heap_smem ? heap_bytes : 0);
  // |exact - approximate dist_sq| <= beta R_i R_j + gamma_n |n_j| + 2^-20 (...): BF16 rounding of both
  // operands (2^-6), the tensor core's FP32 accumulation and the exact chain's own rounding
  p.beta = 0x1p-6 + 0x1p-14 + (double)(d + 64) * 0x1p-17;
  p.gamma_n = 0x1p-14 + (double)(d + 64) * 0x1p-17;

  DevBuf Qb((size_t)n * Kp * 2, s), Cb((size_t)n * Kp * 2, s), Xp((size_t)n * dp * sizeof(T), s);
  DevBuf Rn((size_t)n * 4, s), sn((size_t)n * sizeof(T), s);
  DevBuf tiles((size_t)ntiles * 8, s), st(4 * sizeof(int32_t), s);
  SCL_CUDA(cudaMemsetAsync(st.p, 0, 4 * sizeof(int32_t), s));
  int32_t* status = st.as<int32_t>();
  int32_t* flag = status + 2;
  p.status = status;
  p.flag = flag;
  const int sms = sm_count(dev);
  const unsigned g1 = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  k_tc_sqrt<T><<<g1, 256, 0, s>>>(norms, n, sn.as<T>());
  SCL_CUDA(cudaGetLastError());
  const unsigned g2 = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n * 32 + 255) / 256, (int64_t)sms * 16));
  k_tc_prep<T><<<g2, 256, 0, s>>>(X, norms, n, d, Kp, dp, Qb.as<__nv_bfloat16>(), Cb.as<__nv_bfloat16>(),
                                  Xp.as<T>(), Rn.as<float>(), flag);
  SCL_CUDA(cudaGetLastError());
  float* Rmax = tiles.as<float>();
  float* Nmax = Rmax + ntiles;
  k_tc_tile_max<T><<<(unsigned)ntiles, kTcN, 0, s>>>(Rn.as<float>(), norms, n, Rmax, Nmax);
  SCL_CUDA(cudaGetLastError());

  const CUtensorMap qmap = operand_map(Qb.p, n, Kp, kTcQ);
  const CUtensorMap cmap = operand_map(Cb.p, n, Kp, kTcN);
  auto kern = p.per_cand ? k_knn_tc<T, IT, true> : k_knn_tc<T, IT, false>;
  SCL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)((n + kTcQ - 1) / kTcQ), kTcThreads, smem, s>>>(qmap, cmap, Xp.as<T>(), norms, sn.as<T>(),
                                                                   Rn.as<float>(), Rmax, Nmax, p, idx, dist);
  SCL_CUDA(cudaGetLastError());
  int32_t h[2] = {0, 0};
  SCL_CUDA(cudaMemcpyAsync(h, status, sizeof(h), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  SCL_REQUIRE(h[0] == 0, h[0], "tensor-core kNN: a pipeline wait timed out");
}

}  // namespace

void knn_tensor_inject_stall(int64_t cta, cudaStream_t s) {
  const long long v = cta;
  SCL_CUDA(cudaMemcpyToSymbolAsync(g_knn_tc_stall_cta, &v, sizeof(v), 0, cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaStreamSynchronize(s));
}

void knn_tensor(const void* X, const void* norms, DType t, int64_t n, int d, int k, void* idx, DType it, void* dist,
                cudaStream_t s) {
  if (n == 0) return;
  SCL_REQUIRE(n < (int64_t)0x7fffffff, kErrInvalidArgument, "kNN sample count exceeds the int32 range");
  if (t == kF32) {
    if (it == kI32)
      return knn_tc_typed<float, int32_t>(static_cast<const float*>(X), static_cast<const float*>(norms), n, d, k,
                                          static_cast<int32_t*>(idx), static_cast<float*>(dist), s);
    return knn_tc_typed<float, int64_t>(static_cast<const float*>(X), static_cast<const float*>(norms), n, d, k,
                                        static_cast<int64_t*>(idx), static_cast<float*>(dist), s);
  }
  if (it == kI32)
    return knn_tc_typed<double, int32_t>(static_cast<const double*>(X), static_cast<const double*>(norms), n, d, k,
                                         static_cast<int32_t*>(idx), static_cast<double*>(dist), s);
  knn_tc_typed<double, int64_t>(static_cast<const double*>(X), static_cast<const double*>(norms), n, d, k,
                                static_cast<int64_t*>(idx), static_cast<double*>(dist), s);
}

}  // namespace sclgpu
