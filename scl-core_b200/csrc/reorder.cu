// Locality reordering for the diffusion SpMM.
//
// The X gather of Y = P X touches row j of X once per stored entry (nnz x F
// elements per step, ~14x the compulsory bytes at k=30, F=64). When rows are
// in arbitrary order the gather working set is all of X; grouping the rows of
// each connected component together shrinks it to one component, which stays
// resident in L2. The permutation is symmetric (P' = Pi P Pi^T, X' = Pi X), each
// row keeps its entries in their ORIGINAL stored order (column ids are only
// renamed), so every output element is the same fma sequence as without
// reordering — results are bit-identical.
//
// Components: min-label hooking (atomicMin on the larger label's slot) plus
// pointer jumping, a bounded number of rounds. Stopping early only yields a
// coarser grouping; any grouping is a valid permutation.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

#include <queue>
#include <vector>

#include "engine.hpp"

namespace sclgpu {
namespace {

inline unsigned nblocks(int64_t items, int per) {
  int64_t b = (items + per - 1) / per;
  if (b < 1) b = 1;
  if (b > 148LL * 64) b = 148LL * 64;
  return (unsigned)b;
}

__global__ void k_cc_init(int32_t* __restrict__ L, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    L[i] = (int32_t)i;
}

// Warp per row: hook the larger label onto the smaller one for every edge.
__global__ void k_cc_hook(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx, int64_t n,
                          int32_t* __restrict__ L, int32_t* __restrict__ changed) {
  const int lane = threadIdx.x & 31;
  for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; u < n;
       u += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    int any = 0;
    for (int64_t p = indptr[u] + lane, e = indptr[u + 1]; p < e; p += 32) {
      const int32_t v = idx[p];
      const int32_t lu = L[u], lv = L[v];
      if (lu != lv) {
        const int32_t lo = lu < lv ? lu : lv, hi = lu < lv ? lv : lu;
        atomicMin(&L[hi], lo);
        any = 1;
      }
    }
    if (__any_sync(0xffffffffu, any) && lane == 0) *changed = 1;
  }
}

// Pointer jumping: follow parents towards the root (labels only decrease).
__global__ void k_cc_jump(int32_t* __restrict__ L, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t p = L[i];
    for (int it = 0; it < 64; ++it) {
      const int32_t pp = L[p];
      if (pp == p) break;
      p = pp;
    }
    L[i] = p;
  }
}

// Sort key of row i: its component label, then its length, longest first
// (lengths saturate at 2^20 - 1; ties keep the original order).
constexpr int kLenBits = 20;
__global__ void k_label_keys(const int32_t* __restrict__ L, const int64_t* __restrict__ indptr, int64_t n,
                             uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  constexpr uint64_t kLenMax = (1ull << kLenBits) - 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t len = (uint64_t)(indptr[i + 1] - indptr[i]);
    keys[i] = ((uint64_t)(uint32_t)L[i] << kLenBits) | (kLenMax - (len < kLenMax ? len : kLenMax));
    vals[i] = (uint32_t)i;
  }
}

__global__ void k_perm_from_sort(const uint32_t* __restrict__ sorted_vals, int64_t n, int32_t* __restrict__ perm,
                                 int32_t* __restrict__ iperm, const int64_t* __restrict__ indptr,
                                 int64_t* __restrict__ lens) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t old = (int32_t)sorted_vals[r];
    perm[r] = old;
    iperm[old] = (int32_t)r;
    lens[r] = indptr[old + 1] - indptr[old];
  }
}

// Warp per new row: renamed column ids in the row's original entry order.
__global__ void k_fill_permuted(const int64_t* __restrict__ indptr, const int32_t* __restrict__ idx,
                                const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                                const int64_t* __restrict__ new_indptr, int64_t n, int32_t* __restrict__ new_idx,
                                int32_t* __restrict__ emap) {
  const int lane = threadIdx.x & 31;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < n;
       r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t os = indptr[perm[r]];
    const int64_t ns = new_indptr[r], ne = new_indptr[r + 1];
    for (int64_t q = ns + lane; q < ne; q += 32) {
      const int64_t p = os + (q - ns);
      new_idx[q] = iperm[idx[p]];
      emap[q] = (int32_t)p;
    }
  }
}

template <class T>
__global__ void k_gather_entries(const T* __restrict__ src, const int32_t* __restrict__ emap, int64_t nnz,
                                 T* __restrict__ dst) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
    dst[q] = src[emap[q]];
}

// dst row r = src row perm[r] (same dtype), 16-byte chunks when possible.
template <class C>
__global__ void k_gather_rows(const C* __restrict__ src, const int32_t* __restrict__ perm, int64_t n,
                              int64_t chunks_per_row, C* __restrict__ dst) {
  const int64_t total = n * chunks_per_row;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / chunks_per_row, c = t - r * chunks_per_row;
    dst[t] = src[(int64_t)perm[r] * chunks_per_row + c];
  }
}

void gather_rows(const void* src, const int32_t* perm, int64_t n, int64_t row_bytes, void* dst, cudaStream_t s) {
  if (n == 0 || row_bytes == 0) return;
  if (row_bytes % 16 == 0 && ((uintptr_t)src & 15) == 0 && ((uintptr_t)dst & 15) == 0) {
    const int64_t c = row_bytes / 16;
    k_gather_rows<uint4><<<nblocks(n * c, 256), 256, 0, s>>>((const uint4*)src, perm, n, c, (uint4*)dst);
  } else if (row_bytes % 4 == 0) {
    const int64_t c = row_bytes / 4;
    k_gather_rows<uint32_t><<<nblocks(n * c, 256), 256, 0, s>>>((const uint32_t*)src, perm, n, c, (uint32_t*)dst);
  } else {
    const int64_t c = row_bytes / 2;
    k_gather_rows<uint16_t><<<nblocks(n * c, 256), 256, 0, s>>>((const uint16_t*)src, perm, n, c, (uint16_t*)dst);
  }
  SCL_CUDA(cudaGetLastError());
}

int bits_for(int64_t n) {
  int b = 1;
  while ((1ll << b) < n) ++b;
  return b;
}

}  // namespace

void build_reorder(const CsrView& g, Reordered& r, cudaStream_t s, int mode) {
  SCL_REQUIRE(mode == 1 || mode == 2, kErrInvalidArgument, "reorder mode must be 1 (components) or 2 (lengths)");
  SCL_REQUIRE(g.n_rows == g.n_cols, kErrDimensionMismatch, "reordering needs a square matrix");
  SCL_REQUIRE(g.nnz < (1ll << 31) && g.n_rows < (1ll << 31), kErrInvalidArgument, "graph too large to reorder");
  const int64_t n = g.n_rows, nnz = g.nnz;
  r.n = n;
  r.nnz = nnz;
  r.values_ok = false;
  r.schedules.clear();
  DevBuf L(std::max<int64_t>(n, 1) * 4, s), changed(4, s);
  const int max_rounds = 4 * bits_for(std::max<int64_t>(n, 2)) + 16;
  int rounds = 0;
  if (mode == 2) SCL_CUDA(cudaMemsetAsync(L.p, 0, std::max<int64_t>(n, 1) * 4, s));  // one group: lengths only
  else k_cc_init<<<nblocks(n, 256), 256, 0, s>>>(L.as<int32_t>(), n);
  for (; mode == 1 && rounds < max_rounds; ++rounds) {
    SCL_CUDA(cudaMemsetAsync(changed.p, 0, 4, s));
    k_cc_hook<<<nblocks(n * 32, 256), 256, 0, s>>>(g.indptr, g.indices, n, L.as<int32_t>(), changed.as<int32_t>());
    k_cc_jump<<<nblocks(n, 256), 256, 0, s>>>(L.as<int32_t>(), n);
    int32_t h = 0;
    SCL_CUDA(cudaMemcpyAsync(&h, changed.p, 4, cudaMemcpyDeviceToHost, s));
    SCL_CUDA(cudaStreamSynchronize(s));
    if (!h) break;
  }
  r.cc_rounds = rounds;
  DevBuf keys(n * 8, s), vals(n * 4, s), keys2(n * 8, s), vals2(n * 4, s);
  k_label_keys<<<nblocks(n, 256), 256, 0, s>>>(L.as<int32_t>(), g.indptr, n, keys.as<uint64_t>(),
                                               vals.as<uint32_t>());
  radix_sort_pairs(keys.as<uint64_t>(), vals.as<uint32_t>(), keys2.as<uint64_t>(), vals2.as<uint32_t>(), n,
                   bits_for(std::max<int64_t>(n, 2)) + kLenBits, s);
  r.perm = DevBuf(n * 4, s);
  r.iperm = DevBuf(n * 4, s);
  DevBuf lens((n + 1) * 8, s);
  k_perm_from_sort<<<nblocks(n, 256), 256, 0, s>>>(vals2.as<uint32_t>(), n, r.perm.as<int32_t>(),
                                                   r.iperm.as<int32_t>(), g.indptr, lens.as<int64_t>());
  r.indptr = DevBuf((n + 1) * 8, s);
  exclusive_scan_i64(lens.as<int64_t>(), r.indptr.as<int64_t>(), n, s);
  r.indices = DevBuf(std::max<int64_t>(nnz, 1) * 4, s);
  r.emap = DevBuf(std::max<int64_t>(nnz, 1) * 4, s);
  k_fill_permuted<<<nblocks(n * 32, 256), 256, 0, s>>>(g.indptr, g.indices, r.perm.as<int32_t>(),
                                                       r.iperm.as<int32_t>(), r.indptr.as<int64_t>(), n,
                                                       r.indices.as<int32_t>(), r.emap.as<int32_t>());
  SCL_CUDA(cudaGetLastError());
}

std::vector<int32_t> warp_schedule_host(const int64_t* ip, int64_t n, int R, int64_t nw) {
  SCL_REQUIRE(R >= 1 && nw >= 1 && n >= 0 && n < (1ll << 31) && nw < (1ll << 31), kErrInvalidArgument,
              "bad warp schedule request");
  const int64_t ng = (n + R - 1) / R;
  std::vector<int64_t> len(ng, 0);
  for (int64_t g = 0; g < ng; ++g)
    for (int64_t r = g * R; r < std::min<int64_t>(n, g * R + R); ++r) len[g] = std::max(len[g], ip[r + 1] - ip[r]);
  const int64_t thr = 8 * std::max<int64_t>(1, (ip[n] - ip[0] + n - 1) / std::max<int64_t>(n, 1));
  std::vector<int32_t> hubs;
  for (int64_t g = 0; g < ng; ++g)
    if (len[g] > thr) hubs.push_back((int32_t)g);
  std::stable_sort(hubs.begin(), hubs.end(), [&](int32_t a, int32_t b) { return len[a] > len[b]; });
  using Slot = std::pair<int64_t, int64_t>;  // (load, warp): ties go to the lower warp
  std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
  for (int64_t w = 0; w < nw; ++w) heap.push({0, w});
  std::vector<int32_t> owner(ng);
  auto deal = [&](int64_t g) {
    Slot t = heap.top();
    heap.pop();
    owner[g] = (int32_t)t.second;
    heap.push({t.first + len[g] + 8, t.second});
  };
  std::vector<char> is_hub(ng, 0);
  for (int32_t g : hubs) {
    is_hub[g] = 1;
    deal(g);
  }
  for (int64_t g = 0; g < ng; ++g)
    if (!is_hub[g]) deal(g);
  // CSR of the lists: a warp's long groups first (in dealing order), then its others by index
  std::vector<int32_t> out(nw + 1 + ng), cnt(nw + 1, 0);
  for (int64_t g = 0; g < ng; ++g) ++cnt[owner[g] + 1];
  for (int64_t w = 0; w < nw; ++w) cnt[w + 1] += cnt[w];
  for (int64_t w = 0; w <= nw; ++w) out[w] = cnt[w];
  std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
  for (int32_t g : hubs) out[nw + 1 + fill[owner[g]]++] = g;
  for (int64_t g = 0; g < ng; ++g)
    if (!is_hub[g]) out[nw + 1 + fill[owner[g]]++] = (int32_t)g;
  return out;
}

DevBuf warp_schedule(const int64_t* indptr, int64_t n, int R, int64_t nw, cudaStream_t s) {
  std::vector<int64_t> ip(n + 1);
  SCL_CUDA(cudaMemcpyAsync(ip.data(), indptr, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  const std::vector<int32_t> out = warp_schedule_host(ip.data(), n, R, nw);
  DevBuf d(out.size() * sizeof(int32_t), s);
  SCL_CUDA(cudaMemcpyAsync(d.p, out.data(), out.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaStreamSynchronize(s));  // `out` is released on return
  return d;
}

const int32_t* warp_schedule_for(const Reordered& r, int R, int64_t nw, cudaStream_t s) {
  for (const Reordered::Schedule& e : r.schedules)
    if (e.R == R && e.nw == nw) return e.list.as<int32_t>();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  SCL_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return nullptr;
  Reordered::Schedule e;
  e.R = R;
  e.nw = nw;
  e.list = warp_schedule(r.indptr.as<int64_t>(), r.n, R, nw, s);
  r.schedules.push_back(std::move(e));
  return r.schedules.back().list.as<int32_t>();
}

void reorder_values(const void* vals, DType t, Reordered& r, cudaStream_t s) {
  const size_t es = dtype_size(t);
  if (!r.values.p || r.vtype != t) r.values = DevBuf(std::max<int64_t>(r.nnz, 1) * es, s);
  r.vtype = t;
  if (r.nnz > 0) {
    const unsigned b = nblocks(r.nnz, 256);
    if (es == 8)
      k_gather_entries<uint64_t><<<b, 256, 0, s>>>((const uint64_t*)vals, r.emap.as<int32_t>(), r.nnz, r.values.as<uint64_t>());
    else if (es == 4)
      k_gather_entries<uint32_t><<<b, 256, 0, s>>>((const uint32_t*)vals, r.emap.as<int32_t>(), r.nnz, r.values.as<uint32_t>());
    else
      k_gather_entries<uint16_t><<<b, 256, 0, s>>>((const uint16_t*)vals, r.emap.as<int32_t>(), r.nnz, r.values.as<uint16_t>());
    SCL_CUDA(cudaGetLastError());
  }
  r.values_ok = true;
  ++r.values_version;
}

const Grouped& reordered_grouped(const Reordered& r, int C, cudaStream_t s) {
  SCL_REQUIRE(C == 1 || C == 2 || C == 4, kErrInvalidArgument, "rows per group must be 1, 2 or 4");
  SCL_REQUIRE(r.values_ok, kErrInternal, "reordered values are stale");
  const int slot = C == 1 ? 0 : (C == 2 ? 1 : 2);
  std::unique_ptr<Grouped>& gp = r.grouped[slot];
  if (!gp) {
    CsrView v;
    v.n_rows = r.n;
    v.n_cols = r.n;
    v.nnz = r.nnz;
    v.indptr = r.indptr.as<int64_t>();
    v.indices = r.indices.as<int32_t>();
    auto g = std::make_unique<Grouped>();
    build_grouped(v, C, *g, s);
    gp = std::move(g);
  }
  if (gp->values_version != r.values_version || gp->vtype != r.vtype)
    grouped_values(r.values.p, r.vtype, r.values_version, *gp, s);
  return *gp;
}

void spmm_reordered(const Reordered& r, SpmmArgs a, const SpmmPlan& plan, cudaStream_t s) {
  if (plan.kind == 13) {
    const Grouped& gr = reordered_grouped(r, grouped_rows_per_warp(a.F, a.xtype), s);
    a.values = gr.gval.p;
    return spmm_grouped(gr, a, plan.stage, s);
  }
  spmm_with_plan(a, plan, s);
}

void diffuse_reordered(const Reordered& r, const void* X0, DType xtype, void* Y, DType ytype, int64_t F,
                       int64_t steps, cudaStream_t s, const SpmmPlan* plan_in) {
  SCL_REQUIRE(r.values_ok, kErrInternal, "reordered values are stale");
  const int64_t n = r.n;
  const DType mtype = r.vtype;
  if (steps <= 0 || n == 0 || F == 0) {
    if (X0 != Y) convert_values(X0, xtype, Y, ytype, n * F, s);
    return;
  }
  const size_t esz = dtype_size(mtype);
  DevBuf A(n * F * esz, s), B;
  // X' = Pi X0 in the iterate dtype
  if (xtype == mtype) {
    gather_rows(X0, r.perm.as<int32_t>(), n, F * (int64_t)esz, A.p, s);
  } else {
    DevBuf tmp(n * F * esz, s);
    convert_values(X0, xtype, tmp.p, mtype, n * F, s);
    gather_rows(tmp.p, r.perm.as<int32_t>(), n, F * (int64_t)esz, A.p, s);
  }
  SpmmArgs a{};
  a.indptr = r.indptr.as<int64_t>();
  a.indices = r.indices.as<int32_t>();
  a.values = r.values.p;
  a.vtype = mtype;
  a.n_rows = n;
  a.F = F;
  const void* src = A.p;
  for (int64_t st = 0; st < steps; ++st) {
    const bool last = (st == steps - 1);
    void* dst;
    DType ot;
    if (last) {
      dst = Y;  // Y[perm[r]] = row r: un-permute on the final store
      ot = ytype;
      a.row_map = r.perm.as<int32_t>();
    } else {
      if (!B.p) B = DevBuf(n * F * esz, s);
      dst = (src == A.p) ? B.p : A.p;
      ot = mtype;
      a.row_map = nullptr;
    }
    a.X = src;
    a.xtype = mtype;
    a.Y = dst;
    a.ytype = ot;
    const SpmmPlan plan = plan_in ? *plan_in : default_spmm_plan(F, mtype, src, dst, ot);
    a.reo = &r;
    spmm_reordered(r, a, plan, s);
    src = dst;
  }
}

}  // namespace sclgpu
