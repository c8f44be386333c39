// Backward pass of the diffusion X_T = P^T X_0, P = normalise(W), for a loss
// L(X_T) whose gradient dL/dX_T the caller supplies.
//
//   G_T = dL/dX_T;   G_s = P^T G_{s+1};   dL/dX_0 = G_0
//   gP_ij = sum_s <G_{s+1}[i,:], X_s[j,:]>        (SDDMM over the stored entries)
//   row:  dW_ij = (gP_ij - u_i) / d_i,              u_i = sum_c gP_ic P_ic
//   sym:  dW_ij = gP_ij a_i a_j - (u_i + v_i)/(2 d_i), v_i = sum_r gP_ri P_ri, a = d^-1/2
//   rows with d_i <= 1e-15 were zeroed by the forward and get dW = 0.
//
// No scl-core counterpart (scl-core has no gradients); the forward it
// differentiates is scl/kernel/diffusion.hpp:492-603 (transition) and 638-664
// (diffuse_matrix). The FP64 restatement the tests check against is
// oracle_adjoint_f64 in the oracle.
//
// Kernels:
//   k_adj_step  one fused step over the CSC view of P (the CSR of P^T, built
//               once per graph by transpose_map): a warp owns row i of P^T,
//               keeps X_s[i] in registers, and for every stored entry (j, i) of
//               P gathers G_{s+1}[j] ONCE for both uses — the fma chain of
//               G_s[i] and the dot <G_{s+1}[j], X_s[i]> that is gP's term for
//               that entry. The 32 per-lane partial dots of a chunk of 32
//               entries are summed by a transposed butterfly (31 shuffles per
//               32 entries, lane l ends with entry l's total), and lane l adds
//               it to gPt[chunk + l] — a coalesced read-modify-write in CSC
//               order that no other warp touches (no atomics).
//   k_norm_*    normalisation backward in FP64 (degrees kept by normalize).
//   k_adj_quarter  the same step for rows of 1, 2 or 4 blocks of eight 16-byte
//               chunks: one load instruction gathers 4 entries (4 interleaved
//               chains of G_s[i], summed pairwise at the row end), partial
//               dots reduced within a quarter-warp (7 shuffles per 8 entries);
//               prefetch pipeline as in the forward row kernel. On a
//               structurally symmetric graph the pass also recomputes one
//               forward iterate of the previous segment (FUSE).
// Checkpointing: the forward stores X_s for s = every, 2*every, ... < T (and,
// with keep_last, the last segment's iterates); the backward recomputes every
// other iterate of a segment from its checkpoint with the forward SpMM (the
// same kernel, so the same bits) and walks the segment in reverse.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine.hpp"

namespace sclgpu {
namespace {

constexpr double kMinProbB = 1e-15;  // diffusion.hpp:41 config::MIN_PROB

inline unsigned nblk(int64_t items, int per) {
  return (unsigned)std::max<int64_t>(1, (items + per - 1) / per);
}

template <int BYTES> struct Raw;
template <> struct Raw<4> { using type = unsigned int; };
template <> struct Raw<8> { using type = uint2; };
template <> struct Raw<16> { using type = uint4; };

template <class T, int VEC>
__device__ __forceinline__ void load_vec(const T* __restrict__ p, T (&out)[VEC]) {
  if constexpr (VEC == 1) {
    out[0] = __ldg(p);
  } else {
    using R = typename Raw<VEC * (int)sizeof(T)>::type;
    const R raw = __ldg(reinterpret_cast<const R*>(p));
    const T* e = reinterpret_cast<const T*>(&raw);
#pragma unroll
    for (int i = 0; i < VEC; ++i) out[i] = e[i];
  }
}

template <class T, int VEC>
__device__ __forceinline__ void store_vec(T* __restrict__ p, const T (&in)[VEC]) {
  if constexpr (VEC == 1) {
    p[0] = in[0];
  } else {
    using R = typename Raw<VEC * (int)sizeof(T)>::type;
    R raw;
    T* e = reinterpret_cast<T*>(&raw);
#pragma unroll
    for (int i = 0; i < VEC; ++i) e[i] = in[i];
    *reinterpret_cast<R*>(p) = raw;
  }
}

__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

// Sum across the warp of 32 per-lane arrays: on return lane l holds
// sum over lanes of p[l]. Five butterfly rounds; in each a lane keeps the half
// of its live entries selected by its lane bit and sends the other half.
template <class T>
__device__ __forceinline__ T transpose_reduce32(T (&p)[32], int lane) {
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const bool hi = (lane & h) != 0;
#pragma unroll
    for (int k = 0; k < h; ++k) {
      const T send = hi ? p[k] : p[k + h];
      const T keep = hi ? p[k + h] : p[k];
      p[k] = keep + __shfl_xor_sync(0xffffffffu, send, h);
    }
  }
  return p[0];
}

// One backward step. Warp per row i of P^T (persistent grid-stride); lane l
// owns columns [c0 + l*VEC, c0 + l*VEC + VEC) of each column block of
// 32*VEC columns (VEC > 1 requires F % VEC == 0 and aligned rows).
// G0[i] = sum_q Pt[q] * G1[tidx[q]] in stored order (sequential fma chain);
// gPt[q] += <G1[tidx[q]], Xs[i]> when gPt is non-null.
template <class T, int VEC, int U>
__global__ void __launch_bounds__(256)
k_adj_step(const int64_t* __restrict__ tptr, const int32_t* __restrict__ tidx, const T* __restrict__ tval,
           const T* __restrict__ G1, const T* __restrict__ Xs, T* __restrict__ G0, T* __restrict__ gPt, int64_t n,
           int64_t F, int gp_accum) {
  static_assert(32 % U == 0, "batch must divide 32");
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  constexpr int CPB = 32 * VEC;  // columns per block
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += nw) {
    const int64_t start = tptr[row], end = tptr[row + 1];
    for (int64_t c0 = 0; c0 < F; c0 += CPB) {
      const int64_t col = c0 + (int64_t)lane * VEC;
      const bool active = col < F;
      T xi[VEC], acc[VEC];
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        xi[i] = T(0);
        acc[i] = T(0);
      }
      if (active) load_vec<T, VEC>(Xs + row * F + col, xi);
      const T* __restrict__ Gc = G1 + (active ? col : 0);
      for (int64_t base = start; base < end; base += 32) {
        const int64_t m = base + lane;
        int32_t j_l = 0;
        T v_l = T(0);
        if (m < end) {
          j_l = __ldcs(tidx + m);
          v_l = __ldcs(tval + m);
        }
        const int cnt = (int)((end - base) < 32 ? (end - base) : 32);
        T p[32];
#pragma unroll
        for (int t = 0; t < 32; ++t) p[t] = T(0);
#pragma unroll
        for (int t = 0; t < 32; t += U) {
          if (t < cnt) {
            T g[U][VEC];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int32_t jj = __shfl_sync(0xffffffffu, j_l, t + u);
              if (t + u < cnt && active) {
                load_vec<T, VEC>(Gc + (int64_t)jj * F, g[u]);
              } else {
#pragma unroll
                for (int i = 0; i < VEC; ++i) g[u][i] = T(0);
              }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const T vv = __shfl_sync(0xffffffffu, v_l, t + u);
              if (t + u < cnt) {
                T d = g[u][0] * xi[0];
#pragma unroll
                for (int i = 1; i < VEC; ++i) d = fma_t(g[u][i], xi[i], d);
                p[t + u] = d;
#pragma unroll
                for (int i = 0; i < VEC; ++i) acc[i] = fma_t(vv, g[u][i], acc[i]);
              }
            }
          }
        }
        if (gPt != nullptr) {
          const T tot = transpose_reduce32<T>(p, lane);
          // the first backward step overwrites (its first column block) instead of accumulating
          if (lane < cnt) gPt[m] = ((gp_accum || c0 > 0) ? gPt[m] : T(0)) + tot;
        }
      }
      if (active) store_vec<T, VEC>(G0 + row * F + col, acc);
    }
  }
}

// Quarter-warp form of the step for rows of NCB x 8 x (16 / sizeof(T))
// elements: 8 lanes cover a column block with one 16-byte chunk each, so one
// 128-bit load instruction gathers 4 entries (quarter q of the warp takes the
// chunk's entries q, q+4, ..., q+28). Quarter q keeps its own fma chain of
// G_s[i] over its entries; the 4 chains are summed (c0+c1)+(c2+c3) at the row
// end. The 8 per-lane partial dots of a lane's entries are summed inside the
// quarter by a transposed butterfly over lane bits 4, 2, 1 (7 shuffles for 8
// entries); lane l of quarter q then adds entry 4*l + q of the chunk to gPt.
// Summation order differs from the sequential chain only by the chain split.
template <int H, class T>
__device__ __forceinline__ void tr_round(T (&p)[8], int lq) {
  const bool hi = (lq & H) != 0;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const T send = hi ? p[k] : p[k + H];
    const T keep = hi ? p[k + H] : p[k];
    p[k] = keep + __shfl_xor_sync(0xffffffffu, send, H);
  }
}

// FUSE (structurally symmetric graphs, whose P and P^T share indptr/indices):
// the same pass also recomputes one forward iterate Xnew = P Xprev — a second
// value stream pval (P in the same entry order) and a second gather stream,
// 4 interleaved chains summed like G_s's — so a recompute step rides along
// with a backward step instead of running as its own launch.
template <class T, int NCB, int U, bool FUSE>
__global__ void __launch_bounds__(256, (NCB == 1 && sizeof(T) == 4 && !FUSE) ? 3 : 2)
k_adj_quarter(const int64_t* __restrict__ tptr, const int32_t* __restrict__ tidx, const T* __restrict__ tval,
              const T* __restrict__ G1, const T* __restrict__ Xs, T* __restrict__ G0, T* __restrict__ gPt,
              int64_t n, const T* __restrict__ pval, const T* __restrict__ Xprev, T* __restrict__ Xnew,
              int gp_accum, const uint32_t* __restrict__ order, unsigned int* __restrict__ ticket) {
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int CB = 8 * VEC;      // columns per block
  constexpr int F = NCB * CB;
  constexpr int NB = 8 / U;        // batches per chunk of 32 entries
  static_assert(U == 4 || U == 8, "batch of 4 or 8 gathers per lane");
  const int lane = threadIdx.x & 31;
  const int q = lane >> 3, lq = lane & 7;
  const int e_own = lq * 4 + q;    // chunk entry whose dot this lane finishes
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;
  // Rows are handed out dynamically: warp w starts with order[w], then takes
  // ticket numbers (order[nw + ticket]) from a counter the host zeroed. With
  // the long rows first in `order`, the warps finish within about one row of
  // each other; a static grid stride over these heavy-tailed row lengths
  // left the slowest warp with far more than the mean work. A row index of n
  // means none is left (ticket numbers only grow, so every later one is n too).
  auto take = [&]() -> unsigned {  // raw ticket, valid in lane 0
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(ticket, 1u);
    return t;
  };
  const int32_t nr = (int32_t)n;  // row indices are int32
  const unsigned nw32 = (unsigned)nw;
  auto row_at = [&](unsigned raw) -> int32_t {
    const unsigned id = __shfl_sync(0xffffffffu, raw, 0) + nw32;
    return id < (unsigned)nr ? (int32_t)order[id] : nr;
  };
  int32_t row = (int32_t)order[w];
  int32_t r_nx = row_at(take());
  int32_t r_nn = row_at(take());
  unsigned raw_n3 = take();
  // Prefetch pipeline (as in the forward row kernel): ticket three rows
  // ahead, its row two ahead, bounds two rows ahead, the next chunk's (index,
  // value) pairs one chunk ahead, the next row's X_s chunk one row ahead,
  // each chunk's accumulator values at its start.
  int64_t s_cur = tptr[row], e_cur = tptr[row + 1];
  int64_t s_nx = 0, e_nx = 0;
  if (r_nx < n) {
    s_nx = tptr[r_nx];
    e_nx = tptr[r_nx + 1];
  }
  auto fetch = [&](int64_t pos, int64_t end, int32_t& j, T& v, T& v2) {
    j = 0;
    v = T(0);
    v2 = T(0);
    if (pos < end) {
      j = __ldcs(tidx + pos);
      v = __ldcs(tval + pos);
      if constexpr (FUSE) v2 = __ldcs(pval + pos);
    }
  };
  T xi[NCB][VEC], xn[NCB][VEC];
#pragma unroll
  for (int c = 0; c < NCB; ++c) {
    load_vec<T, VEC>(Xs + (int64_t)row * F + c * CB + lq * VEC, xi[c]);
#pragma unroll
    for (int i = 0; i < VEC; ++i) xn[c][i] = T(0);
    if (r_nx < n) load_vec<T, VEC>(Xs + (int64_t)r_nx * F + c * CB + lq * VEC, xn[c]);
  }
  int32_t j_c;
  T v_c, w_c;
  fetch(s_cur + lane, e_cur, j_c, v_c, w_c);
  while (row < n) {
    const int32_t r_n3 = row_at(raw_n3);  // the ticket taken one row ago
    raw_n3 = take();
    int64_t s_nn = 0, e_nn = 0;
    if (r_nn < n) {
      s_nn = tptr[r_nn];
      e_nn = tptr[r_nn + 1];
    }
    T acc[NCB][VEC], accf[NCB][VEC];
#pragma unroll
    for (int c = 0; c < NCB; ++c) {
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        acc[c][i] = T(0);
        accf[c][i] = T(0);
      }
    }
    const int len = (int)(e_cur - s_cur);
    for (int base = 0; base < len; base += 32) {
      int32_t j_n;
      T v_n, w_n;
      if (base + 32 < len) fetch(s_cur + base + 32 + lane, e_cur, j_n, v_n, w_n);
      else fetch(s_nx + lane, e_nx, j_n, v_n, w_n);
      const int cnt = (len - base) < 32 ? (len - base) : 32;
      T old = T(0);  // the first backward step overwrites the accumulator (no memset)
      if (gPt != nullptr && gp_accum && e_own < cnt) old = gPt[s_cur + base + e_own];
      T p[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) p[u] = T(0);
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        if (b * U * 4 < cnt) {
#pragma unroll
          for (int c = 0; c < NCB; ++c) {
            T g[U][VEC];
            T gx[FUSE ? U : 1][VEC];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int e = (b * U + u) * 4 + q;
              const int32_t jj = __shfl_sync(0xffffffffu, j_c, e);
              if (e < cnt) {
                load_vec<T, VEC>(G1 + (int64_t)jj * F + c * CB + lq * VEC, g[u]);
                if constexpr (FUSE) load_vec<T, VEC>(Xprev + (int64_t)jj * F + c * CB + lq * VEC, gx[u]);
              } else {
#pragma unroll
                for (int i = 0; i < VEC; ++i) {
                  g[u][i] = T(0);
                  if constexpr (FUSE) gx[u][i] = T(0);
                }
              }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int e = (b * U + u) * 4 + q;
              const T vv = __shfl_sync(0xffffffffu, v_c, e);
              T d = p[b * U + u];
#pragma unroll
              for (int i = 0; i < VEC; ++i) d = fma_t(g[u][i], xi[c][i], d);
              p[b * U + u] = d;
              if (e < cnt) {
#pragma unroll
                for (int i = 0; i < VEC; ++i) acc[c][i] = fma_t(vv, g[u][i], acc[c][i]);
              }
              if constexpr (FUSE) {
                const T ww = __shfl_sync(0xffffffffu, w_c, e);
                if (e < cnt) {
#pragma unroll
                  for (int i = 0; i < VEC; ++i) accf[c][i] = fma_t(ww, gx[u][i], accf[c][i]);
                }
              }
            }
          }
        }
      }
      if (gPt != nullptr) {
        tr_round<4>(p, lq);
        tr_round<2>(p, lq);
        tr_round<1>(p, lq);
        if (e_own < cnt) gPt[s_cur + base + e_own] = old + p[0];
      }
      j_c = j_n;
      v_c = v_n;
      w_c = w_n;
    }
    if (len == 0) fetch(s_nx + lane, e_nx, j_c, v_c, w_c);  // nothing was prefetched for the next row
#pragma unroll
    for (int c = 0; c < NCB; ++c) {
#pragma unroll
      for (int i = 0; i < VEC; ++i) {
        acc[c][i] = acc[c][i] + __shfl_xor_sync(0xffffffffu, acc[c][i], 8);
        acc[c][i] = acc[c][i] + __shfl_xor_sync(0xffffffffu, acc[c][i], 16);
      }
      if (q == 0) store_vec<T, VEC>(G0 + (int64_t)row * F + c * CB + lq * VEC, acc[c]);
      if constexpr (FUSE) {
#pragma unroll
        for (int i = 0; i < VEC; ++i) {
          accf[c][i] = accf[c][i] + __shfl_xor_sync(0xffffffffu, accf[c][i], 8);
          accf[c][i] = accf[c][i] + __shfl_xor_sync(0xffffffffu, accf[c][i], 16);
        }
        if (q == 0) store_vec<T, VEC>(Xnew + (int64_t)row * F + c * CB + lq * VEC, accf[c]);
      }
    }
    // rotate: next row's X_s chunk is in xn; fetch the one after it
#pragma unroll
    for (int c = 0; c < NCB; ++c) {
#pragma unroll
      for (int i = 0; i < VEC; ++i) xi[c][i] = xn[c][i];
      if (r_nn < n) load_vec<T, VEC>(Xs + (int64_t)r_nn * F + c * CB + lq * VEC, xn[c]);
    }
    s_cur = s_nx;
    e_cur = e_nx;
    s_nx = s_nn;
    e_nx = e_nn;
    row = r_nx;
    r_nx = r_nn;
    r_nn = r_n3;
  }
}

// flag[0] = 1 when a and b (count entries) differ anywhere
template <class I>
__global__ void k_differ(const I* __restrict__ a, const I* __restrict__ b, int64_t count, int32_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    if (a[i] != b[i]) flag[0] = 1;
}

// sort key of a row of P^T: rows longer than thr by decreasing length, then
// every other row (one key, so a stable sort keeps their index order)
__global__ void k_order_keys(const int64_t* __restrict__ ptr, int64_t n, int64_t thr, uint64_t* __restrict__ keys,
                             uint32_t* __restrict__ rows) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t len = ptr[i + 1] - ptr[i];
    keys[i] = len > thr ? 0xffffffffull - (uint64_t)(len < 0xfffffffell ? len : 0xfffffffell) : 0xffffffffull;
    rows[i] = (uint32_t)i;
  }
}

__global__ void k_invert_map(const int32_t* __restrict__ map, int64_t nnz, int32_t* __restrict__ inv) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
    inv[map[q]] = (int32_t)q;
}

// Normalisation backward in one pass over P's rows: gP of entry p is read
// from the CSC-order accumulator through the inverse map, u_i = sum_p gP P is
// reduced in FP64, then every entry's dW is written; v (symmetric mode) is the
// CSC row dot computed beforehand. Sixteen lanes per row, two rows per warp:
// each lane holds up to KEEP entries of its row in registers, and every load
// a row needs (bounds, degree, v, inverse map, P, the gathers) is issued before
// the reduction, so the dependent chain per row is bounds -> map -> gather.
// Rows longer than LPR * KEEP entries gather the rest in batches of TB loads
// per lane and park gP in dW until u is known.
template <class T, bool SYM>
__global__ void __launch_bounds__(256) k_norm_bwd_gather(const int64_t* __restrict__ ptr,
                                                         const int32_t* __restrict__ idx, const T* __restrict__ P,
                                                         const T* __restrict__ gPt, const int32_t* __restrict__ inv,
                                                         const double* __restrict__ deg,
                                                         const double* __restrict__ v, int64_t n,
                                                         T* __restrict__ dW) {
  constexpr int KEEP = 8, LPR = 16, TB = 8;
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LPR;
  const int l = threadIdx.x & (LPR - 1);
  const bool has_row = row < n;
  int64_t s0 = 0, s1 = 0;
  double di = 0.0, vi = 0.0;
  if (has_row) {
    s0 = ptr[row];
    s1 = ptr[row + 1];
    di = deg[row];
    if (SYM) vi = v[row];
  }
  T gk[KEEP], pk[KEEP];
  double ak[SYM ? KEEP : 1];
  int32_t q[KEEP];
#pragma unroll
  for (int k = 0; k < KEEP; ++k) {
    const int64_t p = s0 + l + LPR * k;
    q[k] = 0;
    pk[k] = T(0);
    if (p < s1) {
      q[k] = inv[p];
      pk[k] = P[p];
    }
  }
  if (SYM) {
#pragma unroll
    for (int k = 0; k < KEEP; ++k) {
      const int64_t p = s0 + l + LPR * k;
      ak[k] = 0.0;
      if (p < s1) ak[k] = deg[idx[p]];
    }
  }
#pragma unroll
  for (int k = 0; k < KEEP; ++k) {
    const int64_t p = s0 + l + LPR * k;
    gk[k] = T(0);
    if (p < s1) gk[k] = gPt[q[k]];
  }
  double u = 0.0;
#pragma unroll
  for (int k = 0; k < KEEP; ++k) u += (double)gk[k] * (double)pk[k];  // zero past the row's end
  // rest of a long row: gathered once in batches of TB loads per lane; gP is
  // parked in dW and rewritten with the gradient below
  for (int64_t base = s0 + l + LPR * KEEP; base < s1; base += LPR * TB) {
    int32_t qt[TB];
    T pt[TB];
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int64_t p = base + LPR * k;
      qt[k] = 0;
      pt[k] = T(0);
      if (p < s1) {
        qt[k] = inv[p];
        pt[k] = P[p];
      }
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int64_t p = base + LPR * k;
      if (p < s1) {
        const T g = gPt[qt[k]];
        u += (double)g * (double)pt[k];
        dW[p] = g;
      }
    }
  }
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
  if (!has_row) return;
  const bool live = di > kMinProbB;
  const double ai = live ? 1.0 / sqrt(di) : 0.0;
  const double rdi = live ? 1.0 / di : 0.0;
  const double shift = live ? (SYM ? (u + vi) * (0.5 * rdi) : u) : 0.0;
  auto grad = [&](double gp, double dj) -> double {
    if (!live) return 0.0;
    if (SYM) return gp * ai * (dj > kMinProbB ? 1.0 / sqrt(dj) : 0.0) - shift;
    return (gp - shift) * rdi;
  };
#pragma unroll
  for (int k = 0; k < KEEP; ++k) {
    const int64_t p = s0 + l + LPR * k;
    if (p < s1) dW[p] = (T)grad((double)gk[k], SYM ? ak[k] : 0.0);
  }
  for (int64_t base = s0 + l + LPR * KEEP; base < s1; base += LPR * TB) {
    T gt[TB];
    double dj[TB];
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int64_t p = base + LPR * k;
      gt[k] = T(0);
      dj[k] = 0.0;
      if (p < s1) {
        gt[k] = dW[p];
        if (SYM) dj[k] = deg[idx[p]];
      }
    }
#pragma unroll
    for (int k = 0; k < TB; ++k) {
      const int64_t p = base + LPR * k;
      if (p < s1) dW[p] = (T)grad((double)gt[k], dj[k]);
    }
  }
}

template <class T>
__global__ void k_scatter_entries(const T* __restrict__ src, const int32_t* __restrict__ map, int64_t nnz,
                                  T* __restrict__ dst) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
    dst[map[q]] = src[q];
}

template <class T>
__global__ void k_gather_by_map(const T* __restrict__ src, const int32_t* __restrict__ map, int64_t nnz,
                                T* __restrict__ dst) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
    dst[q] = src[map[q]];
}

// out[i] = sum over row i of a[p] * b[p] in FP64 (warp per row).
template <class T>
__global__ void k_row_dot(const int64_t* __restrict__ ptr, const T* __restrict__ a, const T* __restrict__ b,
                          int64_t n, double* __restrict__ out) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int64_t p = ptr[row] + lane, e = ptr[row + 1]; p < e; p += 32) s += (double)a[p] * (double)b[p];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[row] = s;
}

template <class T, int VEC, int U>
void launch_adj(const CsrView& t, const T* G1, const T* Xs, T* G0, T* gPt, int gp_accum, int64_t F, cudaStream_t s) {
  auto kern = k_adj_step<T, VEC, U>;
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
  const int64_t need = (t.n_rows * 32 + 255) / 256;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)std::max(per_sm, 1) * sm_count(dev)));
  kern<<<(unsigned)grid, 256, 0, s>>>(t.indptr, t.indices, static_cast<const T*>(t.values), G1, Xs, G0, gPt,
                                      t.n_rows, F, gp_accum);
  SCL_CUDA(cudaGetLastError());
}

template <class T, int NCB, int U, bool FUSE = false>
void launch_adj_quarter(const CsrView& t, const uint32_t* order, unsigned int* ticket, const T* G1, const T* Xs,
                        T* G0, T* gPt, int gp_accum, cudaStream_t s, const T* pval = nullptr,
                        const T* Xprev = nullptr, T* Xnew = nullptr) {
  auto kern = k_adj_quarter<T, NCB, U, FUSE>;
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
  const int64_t need = (t.n_rows * 32 + 255) / 256;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)std::max(per_sm, 1) * sm_count(dev)));
  kern<<<(unsigned)grid, 256, 0, s>>>(t.indptr, t.indices, static_cast<const T*>(t.values), G1, Xs, G0, gPt,
                                      t.n_rows, pval, Xprev, Xnew, gp_accum, order, ticket);
  SCL_CUDA(cudaGetLastError());
}

// Whether the fused step (backward + one forward recompute) covers this width.
template <class T>
bool adj_fusable(int64_t F, const void* a, const void* b, const void* c, const void* d, const void* e) {
  constexpr int kV16 = 16 / (int)sizeof(T);
  for (const void* p : {a, b, c, d, e})
    if ((reinterpret_cast<uintptr_t>(p) & 15u) != 0) return false;
  return F == 8 * kV16;
}

template <class T>
void adj_step_fused(const CsrView& t, const uint32_t* order, unsigned int* ticket, const T* pval, const T* G1,
                    const T* Xs, T* G0, T* gPt, int gp_accum, const T* Xprev, T* Xnew, cudaStream_t s) {
  launch_adj_quarter<T, 1, 4, true>(t, order, ticket, G1, Xs, G0, gPt, gp_accum, s, pval, Xprev, Xnew);
}

// ticket: a zeroed counter of its own for the quarter-warp kernels' row hand-out
template <class T>
void adj_step(const CsrView& t, const uint32_t* order, unsigned int* ticket, const T* G1, const T* Xs, T* G0,
              T* gPt, int gp_accum, int64_t F, cudaStream_t s) {
  constexpr int kV16 = 16 / (int)sizeof(T);
  const auto al = [&](const void* p, int b) { return (reinterpret_cast<uintptr_t>(p) % (uintptr_t)b) == 0; };
  // quarter-warp kernel: rows of 1, 2 or 4 blocks of 8 sixteen-byte chunks
  if (al(G1, 16) && al(Xs, 16) && al(G0, 16)) {
    if (F == 8 * kV16) return launch_adj_quarter<T, 1, 4>(t, order, ticket, G1, Xs, G0, gPt, gp_accum, s);
    if (F == 16 * kV16) return launch_adj_quarter<T, 2, 4>(t, order, ticket, G1, Xs, G0, gPt, gp_accum, s);
    if (F == 32 * kV16) return launch_adj_quarter<T, 4, 4>(t, order, ticket, G1, Xs, G0, gPt, gp_accum, s);
  }
  // one 16-byte chunk per lane when the row fits one column block of the warp
  if (F % kV16 == 0 && F <= 32 * kV16 && F > 16 * kV16 && al(G1, 16) && al(Xs, 16) && al(G0, 16))
    return launch_adj<T, kV16, 8>(t, G1, Xs, G0, gPt, gp_accum, F, s);
  if constexpr (kV16 / 2 > 1) {
    constexpr int kV8 = kV16 / 2;
    if (F % kV8 == 0 && F <= 32 * kV8 && F > 16 * kV8 && al(G1, 8) && al(Xs, 8) && al(G0, 8))
      return launch_adj<T, kV8, 8>(t, G1, Xs, G0, gPt, gp_accum, F, s);
  }
  return launch_adj<T, 1, 8>(t, G1, Xs, G0, gPt, gp_accum, F, s);
}

}  // namespace

// ---- CSC view ---------------------------------------------------------------------
void build_adjoint(const DeviceCSR& g, Adjoint& a, cudaStream_t s) {
  transpose_map(g, a.t, a.tmap, s);
  a.values_ok = false;
  a.tinv = DevBuf(std::max<int64_t>(g.nnz, 1) * 4, s);
  if (g.nnz > 0) {
    k_invert_map<<<std::min<unsigned>(nblk(g.nnz, 256), 148u * 16u), 256, 0, s>>>(a.tmap.as<int32_t>(), g.nnz,
                                                                                   a.tinv.as<int32_t>());
    SCL_CUDA(cudaGetLastError());
  }
  // processing order of P^T's rows: those over twice the mean length first,
  // longest first, then the rest in index order (a stable sort on the key)
  const int64_t n = a.t.n_rows;
  a.order = DevBuf(std::max<int64_t>(n, 1) * 4, s);
  if (n > 0) {
    const int64_t thr = std::max<int64_t>(32, 2 * ((g.nnz + n - 1) / n));
    DevBuf keys(n * 8, s), keys2(n * 8, s), rows(n * 4, s);
    k_order_keys<<<std::min<unsigned>(nblk(n, 256), 148u * 8u), 256, 0, s>>>(a.t.indptr.as<int64_t>(), n, thr,
                                                                           keys.as<uint64_t>(),
                                                                           rows.as<uint32_t>());
    SCL_CUDA(cudaGetLastError());
    radix_sort_pairs(keys.as<uint64_t>(), rows.as<uint32_t>(), keys2.as<uint64_t>(), a.order.as<uint32_t>(), n,
                     32, s);
  }
  // a structurally symmetric P (the kNN union graphs) has P^T's structure:
  // then one pass over it can serve P and P^T together (fused recompute)
  a.sym_structure = false;
  if (g.n_rows == g.n_cols) {
    DevBuf flag(4, s);
    SCL_CUDA(cudaMemsetAsync(flag.p, 0, 4, s));
    const unsigned b1 = std::min<unsigned>(nblk(g.n_rows + 1, 256), 148u * 8u);
    k_differ<int64_t><<<b1, 256, 0, s>>>(g.indptr.as<int64_t>(), a.t.indptr.as<int64_t>(), g.n_rows + 1,
                                         flag.as<int32_t>());
    if (g.nnz > 0) {
      const unsigned b2 = std::min<unsigned>(nblk(g.nnz, 256), 148u * 8u);
      k_differ<int32_t><<<b2, 256, 0, s>>>(g.indices.as<int32_t>(), a.t.indices.as<int32_t>(), g.nnz,
                                           flag.as<int32_t>());
    }
    SCL_CUDA(cudaGetLastError());
    int32_t h = 1;
    SCL_CUDA(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, s));
    SCL_CUDA(cudaStreamSynchronize(s));
    a.sym_structure = (h == 0);
  }
}

void adjoint_values(const void* vals, DType t, Adjoint& a, cudaStream_t s) {
  SCL_REQUIRE(t == kF32 || t == kF64, kErrTypeMismatch, "the backward pass needs f32 or f64 values");
  const int64_t nnz = a.t.nnz;
  if (!a.t.values.p || a.t.vtype != t) a.t.values = DevBuf(std::max<int64_t>(nnz, 1) * dtype_size(t), s);
  a.t.vtype = t;
  if (nnz > 0) {
    const unsigned b = std::min<unsigned>(nblk(nnz, 256), 148u * 16u);
    if (t == kF32)
      k_gather_by_map<float><<<b, 256, 0, s>>>(static_cast<const float*>(vals), a.tmap.as<int32_t>(), nnz,
                                                a.t.values.as<float>());
    else
      k_gather_by_map<double><<<b, 256, 0, s>>>(static_cast<const double*>(vals), a.tmap.as<int32_t>(), nnz,
                                                 a.t.values.as<double>());
    SCL_CUDA(cudaGetLastError());
  }
  a.values_ok = true;
}

// ---- checkpointed forward -------------------------------------------------------------
// Slot layout: [0, nc) hold X_every, X_2every, ..., X_{nc*every} with
// nc = (steps-1)/every; with keep_last, slots [nc, nc + steps-1-nc*every) hold
// the last segment's iterates X_{nc*every+1} .. X_{steps-1}, which the
// backward then needs not recompute.
int64_t checkpoint_slots(int64_t steps, int64_t every, bool keep_last) {
  if (steps <= 0 || every < 1) return 0;
  const int64_t nc = (steps - 1) / every;
  return nc + (keep_last ? (steps - 1 - nc * every) : 0);
}

namespace {
// slot of iterate X_m (1 <= m < steps) or -1 when it is not kept
inline int64_t slot_of(int64_t m, int64_t steps, int64_t every, bool keep_last) {
  const int64_t nc = (steps - 1) / every;
  if (m % every == 0) return m / every - 1;
  if (keep_last && m > nc * every) return nc + (m - nc * every - 1);
  return -1;
}
}  // namespace

void diffuse_checkpointed(const CsrView& g, const void* X0, void* Y, DType t, int64_t F, int64_t steps,
                          int64_t every, bool keep_last, void* ckpt, cudaStream_t s) {
  SCL_REQUIRE(t == kF32 || t == kF64, kErrTypeMismatch, "checkpointed diffusion needs f32 or f64 values");
  SCL_REQUIRE(g.vtype == t, kErrTypeMismatch, "graph values and the iterate must have the same dtype");
  SCL_REQUIRE(g.n_rows == g.n_cols, kErrDimensionMismatch, "diffusion with checkpoints needs a square matrix");
  SCL_REQUIRE(every >= 1, kErrInvalidArgument, "checkpoint interval must be >= 1");
  const int64_t n = g.n_rows;
  const size_t blk = (size_t)n * (size_t)F * dtype_size(t);
  if (steps <= 0) {
    if (X0 != Y) SCL_CUDA(cudaMemcpyAsync(Y, X0, blk, cudaMemcpyDeviceToDevice, s));
    return;
  }
  SCL_REQUIRE(X0 != Y, kErrInvalidArgument, "checkpointed diffusion needs distinct input and output blocks");
  DevBuf A, B;
  SpmmArgs a{};
  a.indptr = g.indptr;
  a.indices = g.indices;
  a.values = g.values;
  a.vtype = t;
  a.n_rows = n;
  a.F = F;
  a.xtype = t;
  a.ytype = t;
  const void* src = X0;
  for (int64_t st = 0; st < steps; ++st) {
    const int64_t made = st + 1;  // index of the iterate this step produces
    void* dst;
    const int64_t slot = (made < steps) ? slot_of(made, steps, every, keep_last) : -1;
    if (made == steps) {
      dst = Y;
    } else if (slot >= 0) {
      dst = static_cast<char*>(ckpt) + (size_t)slot * blk;
    } else {
      if (!A.p) A = DevBuf(blk, s);
      if (src == A.p) {
        if (!B.p) B = DevBuf(blk, s);
        dst = B.p;
      } else {
        dst = A.p;
      }
    }
    a.X = src;
    a.Y = dst;
    spmm(a, s);
    src = dst;
  }
}

// ---- backward ---------------------------------------------------------------------------
template <class T>
static void backward_typed(const CsrView& g, const Adjoint& adj, const T* X0, const T* ckpt, const T* dY,
                           int64_t F, int64_t steps, int64_t every, bool keep_last, T* dX0, T* gPt,
                           cudaStream_t s) {
  const int64_t n = g.n_rows;
  const size_t blk = (size_t)n * (size_t)F * sizeof(T);
  const size_t elems = (size_t)n * (size_t)F;
  const CsrView tv = adj.t.view();
  if (steps <= 0) {
    if (gPt) SCL_CUDA(cudaMemsetAsync(gPt, 0, std::max<int64_t>(g.nnz, 1) * sizeof(T), s));
    SCL_CUDA(cudaMemcpyAsync(dX0, dY, blk, cudaMemcpyDeviceToDevice, s));
    return;
  }
  int gp_accum = 0;  // the first backward step writes the accumulator
  SCL_REQUIRE(adj.order.p != nullptr, kErrInternal, "adjoint row order is missing");
  const uint32_t* order = adj.order.as<uint32_t>();
  DevBuf tickets((size_t)steps * sizeof(unsigned int), s);  // one row counter per step
  SCL_CUDA(cudaMemsetAsync(tickets.p, 0, (size_t)steps * sizeof(unsigned int), s));
  const int64_t seg = std::min<int64_t>(every, steps);
  // recomputed iterates: two buffer sets, the segment being walked and the
  // (earlier) segment being recomputed alongside it
  std::vector<DevBuf> xs[2] = {std::vector<DevBuf>(seg), std::vector<DevBuf>(seg)};
  DevBuf Ga(blk, s), Gb(blk, s);
  const T* Gcur = dY;
  SpmmArgs a{};
  a.indptr = g.indptr;
  a.indices = g.indices;
  a.values = g.values;
  a.vtype = g.vtype;
  a.n_rows = n;
  a.F = F;
  a.xtype = g.vtype;
  a.ytype = g.vtype;
  const bool fuse = adj.sym_structure && adj_fusable<T>(F, dY, X0, Ga.p, Gb.p, ckpt ? (const void*)ckpt : X0);
  // kept iterates of segment c (checkpoint, X0 or keep_last slots); nullptr = to recompute
  auto kept = [&](int64_t c) {
    const int64_t e = std::min<int64_t>(c + every, steps);
    std::vector<const T*> X(e - c, nullptr);
    for (int64_t m = c; m < e; ++m) {
      if (m == 0) {
        X[0] = X0;
      } else {
        const int64_t slot = slot_of(m, steps, every, keep_last);
        if (slot >= 0) X[m - c] = ckpt + (size_t)slot * elems;
      }
    }
    return X;
  };
  auto recompute = [&](std::vector<const T*>& X, int64_t c, std::vector<DevBuf>& buf, int64_t m) {
    if (!buf[m - c].p) buf[m - c] = DevBuf(blk, s);
    a.X = X[m - c - 1];
    a.Y = buf[m - c].p;
    spmm(a, s);
    X[m - c] = buf[m - c].as<T>();
  };
  const int64_t last_c = ((steps - 1) / every) * every;
  std::vector<int64_t> segs;
  for (int64_t c = last_c; c >= 0; c -= every) segs.push_back(c);
  std::vector<const T*> X = kept(segs[0]);
  for (int64_t m = segs[0] + 1; m < std::min<int64_t>(segs[0] + every, steps); ++m)
    if (X[m - segs[0]] == nullptr) recompute(X, segs[0], xs[0], m);
  for (size_t k = 0; k < segs.size(); ++k) {
    const int64_t c = segs[k];
    const int64_t e = std::min<int64_t>(c + every, steps);
    const bool has_next = k + 1 < segs.size();
    const int64_t cn = has_next ? segs[k + 1] : 0;
    std::vector<const T*> Xn = has_next ? kept(cn) : std::vector<const T*>();
    std::vector<DevBuf>& bn = xs[(k + 1) & 1];
    int64_t mn = cn + 1;  // next iterate of segment cn to produce
    auto advance = [&]() {
      while (has_next && mn < c && Xn[mn - cn] != nullptr) ++mn;
    };
    advance();
    for (int64_t st = e - 1; st >= c; --st) {
      T* Gnext = (st == 0) ? dX0 : ((Gcur == Ga.as<T>()) ? Gb.as<T>() : Ga.as<T>());
      if (fuse && has_next && mn < c) {
        if (!bn[mn - cn].p) bn[mn - cn] = DevBuf(blk, s);
        adj_step_fused<T>(tv, order, tickets.as<unsigned int>() + st, static_cast<const T*>(g.values), Gcur,
                          X[st - c], Gnext, gPt, gp_accum, Xn[mn - cn - 1], bn[mn - cn].as<T>(), s);
        Xn[mn - cn] = bn[mn - cn].as<T>();
        ++mn;
        advance();
      } else {
        adj_step<T>(tv, order, tickets.as<unsigned int>() + st, Gcur, X[st - c], Gnext, gPt, gp_accum, F, s);
      }
      gp_accum = 1;
      Gcur = Gnext;
    }
    if (has_next) {
      for (int64_t m = cn + 1; m < c; ++m)
        if (Xn[m - cn] == nullptr) recompute(Xn, cn, bn, m);
      X = Xn;
    }
  }
}

void diffuse_backward(const CsrView& g, const Adjoint& adj, const void* X0, const void* ckpt, const void* dY,
                      DType t, int64_t F, int64_t steps, int64_t every, bool keep_last, void* dX0, void* gPt,
                      cudaStream_t s) {
  SCL_REQUIRE(t == kF32 || t == kF64, kErrTypeMismatch, "the backward pass needs f32 or f64 values");
  SCL_REQUIRE(g.vtype == t && adj.values_ok && adj.t.vtype == t, kErrInternal, "adjoint view is stale");
  SCL_REQUIRE(every >= 1, kErrInvalidArgument, "checkpoint interval must be >= 1");
  if (t == kF32)
    backward_typed<float>(g, adj, static_cast<const float*>(X0), static_cast<const float*>(ckpt),
                          static_cast<const float*>(dY), F, steps, every, keep_last, static_cast<float*>(dX0),
                          static_cast<float*>(gPt), s);
  else
    backward_typed<double>(g, adj, static_cast<const double*>(X0), static_cast<const double*>(ckpt),
                           static_cast<const double*>(dY), F, steps, every, keep_last, static_cast<double*>(dX0),
                           static_cast<double*>(gPt), s);
}

template <class T>
static void norm_bwd_typed(const CsrView& P, const Adjoint& adj, const T* gPt, const double* degrees, int symmetric,
                           T* dW, cudaStream_t s) {
  const int64_t n = P.n_rows, nnz = P.nnz;
  if (nnz == 0) return;
  DevBuf v(std::max<int64_t>(n, 1) * 8, s);
  if (symmetric)  // v_i = sum over column i of P of gP * P: a row dot over the CSC view
    k_row_dot<T><<<nblk(n * 32, 256), 256, 0, s>>>(adj.t.indptr.as<int64_t>(), gPt, adj.t.values.as<T>(), n,
                                                   v.as<double>());
  auto kern = symmetric ? k_norm_bwd_gather<T, true> : k_norm_bwd_gather<T, false>;
  kern<<<nblk(n * 16, 256), 256, 0, s>>>(P.indptr, P.indices, static_cast<const T*>(P.values), gPt,
                                        adj.tinv.as<int32_t>(), degrees, v.as<double>(), n, dW);
  SCL_CUDA(cudaGetLastError());
}

void normalize_backward(const CsrView& P, const Adjoint& adj, const void* gPt, const double* degrees, int symmetric,
                        void* dW, cudaStream_t s) {
  SCL_REQUIRE(P.vtype == adj.t.vtype, kErrInternal, "adjoint view is stale");
  if (P.vtype == kF32)
    norm_bwd_typed<float>(P, adj, static_cast<const float*>(gPt), degrees, symmetric, static_cast<float*>(dW), s);
  else
    norm_bwd_typed<double>(P, adj, static_cast<const double*>(gPt), degrees, symmetric, static_cast<double*>(dW), s);
}

void scatter_adjoint_entries(const Adjoint& adj, const void* gPt, DType t, void* gP, cudaStream_t s) {
  const int64_t nnz = adj.t.nnz;
  if (nnz == 0) return;
  const unsigned b = std::min<unsigned>(nblk(nnz, 256), 148u * 16u);
  if (t == kF32)
    k_scatter_entries<float><<<b, 256, 0, s>>>(static_cast<const float*>(gPt), adj.tmap.as<int32_t>(), nnz,
                                               static_cast<float*>(gP));
  else
    k_scatter_entries<double><<<b, 256, 0, s>>>(static_cast<const double*>(gPt), adj.tmap.as<int32_t>(), nnz,
                                                static_cast<double*>(gP));
  SCL_CUDA(cudaGetLastError());
}

}  // namespace sclgpu
