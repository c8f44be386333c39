// Batched diffusion: many independent graphs of uneven size, each with its own
// dense block, all T steps in ONE persistent kernel launch (replayed from a
// CUDA graph).
//
// No scl-core counterpart (scl-core diffuses one graph per call,
// scl/kernel/diffusion.hpp:638-664); each graph's arithmetic is exactly that
// call's: every output element is the sequential fma chain over its row's
// entries in stored order, so each graph's result is bit-identical to a
// separate diffusion of that graph.
//
// Layout: the graphs are concatenated into one block-diagonal CSR (row and
// column ids offset by the graph's first row), their blocks into one
// (sum n) x F row-major block. Each graph's rows are cut into tiles of about
// `tile_nnz` stored entries (never spanning graphs).
//
// Schedule: work item i = (step s, tile t) in step-major order, claimed by
// CTAs through one atomic counter. A tile of step s > 0 of graph b needs all
// of graph b's step s-1 tiles; those have smaller item ids, so they were
// claimed earlier by CTAs that are running and depend only on even earlier
// items — the wait always ends (no residency assumption, no grid barrier).
// A CTA that finishes a tile publishes it with a release (threadfence +
// atomicAdd on the graph's counter); a waiter spins with an acquire load and
// an iteration limit, after which it records an error in the status word,
// raises the abort flag and returns. Iterates written in this launch are
// read through L2 (ld.global.cg): L1 is not coherent across SMs and the two
// iterate buffers are reused every other step.
// Buffers: step s writes buf[(T-1-s) & 1] with buf[0] = Y, buf[1] = scratch,
// and reads X0 (s = 0) or buf[(T-s) & 1]; the last step therefore writes Y.
// A step-(s+1) tile of graph b overwrites X_s of graph b only after every
// step-s tile of b (its readers) has finished.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <numeric>
#include <vector>

#include "engine.hpp"

namespace sclgpu {
namespace {

constexpr int kBatchThreads = 256;
// A wait gives up after kWaitNs of wall time (read from %globaltimer) or
// kSpinLimit polls, whichever comes first. One wait normally lasts at most one
// step of one graph (microseconds to milliseconds).
constexpr unsigned long long kWaitNs = 2000ull * 1000ull * 1000ull;  // 2 s
constexpr unsigned kSpinLimit = 50u * 1000u * 1000u;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <int VEC>
__device__ __forceinline__ void load_x(const float* __restrict__ p, bool coherent, float (&o)[VEC]) {
  if constexpr (VEC == 4) {
    const float4 v = coherent ? __ldcg(reinterpret_cast<const float4*>(p)) : __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  } else if constexpr (VEC == 2) {
    const float2 v = coherent ? __ldcg(reinterpret_cast<const float2*>(p)) : __ldg(reinterpret_cast<const float2*>(p));
    o[0] = v.x; o[1] = v.y;
  } else {
    o[0] = coherent ? __ldcg(p) : __ldg(p);
  }
}

template <int VEC>
__device__ __forceinline__ void store_y(float* __restrict__ p, const float (&a)[VEC]) {
  if constexpr (VEC == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
  } else if constexpr (VEC == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(a[0], a[1]);
  } else {
    p[0] = a[0];
  }
}

struct BatchParams {
  const int64_t* indptr;    // [n_total + 1]
  const int32_t* indices;   // [nnz_total], global column ids
  const float* values;      // [nnz_total]
  const int64_t* tile_row;  // [2 n_tiles + 2]: first rows at [t], end rows at [n_tiles + 1 + t]
  const int32_t* tile_graph;     // [n_tiles]
  const int32_t* row_order;      // [n_total]: a tile's rows by decreasing length (positions = the tile's rows)
  const uint32_t* graph_tiles;   // [n_graphs] tiles per graph
  unsigned* done;                // [n_graphs] finished tiles per graph (cumulative over steps)
  unsigned* claim;               // [1] next work item
  int32_t* status;               // [0] error code, [1] item that gave up, [2] abort flag
  const float* X0;
  float* Y;
  float* scratch;
  int64_t F;
  int64_t n_tiles;
  int64_t steps;
  int32_t stall_graph;  // test hook: this graph's waits need one tile more than exists (-1 = off)
};

// G lanes per row (rows per warp = 32 / G), VEC floats per lane per pass, U
// gathers in flight per lane.
template <int G, int VEC, int U>
__global__ void __launch_bounds__(kBatchThreads, 3)
k_batch_diffuse(BatchParams p) {
  __shared__ long long s_item;
  __shared__ int s_go;
  const int lane = threadIdx.x & 31;
  const int lg = lane & (G - 1);
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  const int slot = threadIdx.x / G;                 // row slot within the CTA
  constexpr int kSlots = kBatchThreads / G;
  constexpr int CPP = G * VEC;
  constexpr int K = (U > G) ? (U / G) : 1;  // (index, value) pairs per lane per chunk
  constexpr int CH = G * K;                 // entries per chunk (a multiple of U)
  static_assert(CH % U == 0, "chunk must hold whole batches");
  const int64_t F = p.F;
  const int64_t n_items = p.n_tiles * p.steps;
  for (;;) {
    if (threadIdx.x == 0) {
      long long it = (long long)atomicAdd(p.claim, 1u);
      int go = 1;
      if (it >= n_items || *reinterpret_cast<volatile int32_t*>(p.status + 2) != 0) go = 0;
      if (go) {
        const int64_t s = it / p.n_tiles;
        const int64_t t = it - s * p.n_tiles;
        if (s > 0) {
          const int b = p.tile_graph[t];
          const unsigned need = (unsigned)s * p.graph_tiles[b] + (b == p.stall_graph ? 1u : 0u);
          unsigned spins = 0, ns = 32;
          const unsigned long long t0 = global_ns();
          while (ld_acquire(p.done + b) < need) {
            if (++spins > kSpinLimit || (spins & 63u) == 0u && global_ns() - t0 > kWaitNs ||
                *reinterpret_cast<volatile int32_t*>(p.status + 2) != 0) {
              if (atomicCAS(p.status, 0, (int32_t)kErrConvergence) == 0) p.status[1] = (int32_t)it;
              atomicExch(p.status + 2, 1);
              go = 0;
              break;
            }
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
          }
        }
      }
      s_item = it;
      s_go = go;
    }
    __syncthreads();
    const long long it = s_item;
    if (!s_go) break;
    const int64_t s = it / p.n_tiles;
    const int64_t t = it - s * p.n_tiles;
    const float* __restrict__ src = (s == 0) ? p.X0 : (((p.steps - s) & 1) ? p.scratch : p.Y);
    float* __restrict__ dst = ((p.steps - 1 - s) & 1) ? p.scratch : p.Y;
    const bool coherent = s > 0;
    const int64_t r0 = p.tile_row[t], r1 = p.tile_row[p.n_tiles + 1 + t];
    // The groups of a warp take consecutive rows of the tile's length order,
    // so rows processed side by side have about the same length. The next
    // row's id and bounds, and each row's next chunk of (index, value) pairs,
    // are fetched one step ahead.
    int64_t idx = r0 + slot;
    int64_t row = 0, start = 0, end = 0;
    if (idx < r1) {
      row = p.row_order[idx];
      start = p.indptr[row];
      end = p.indptr[row + 1];
    }
    while (idx < r1) {
      const int64_t nidx = idx + kSlots;
      int64_t nrow = 0, nstart = 0, nend = 0;
      if (nidx < r1) {
        nrow = p.row_order[nidx];
        nstart = p.indptr[nrow];
        nend = p.indptr[nrow + 1];
      }
      for (int64_t c0 = 0; c0 < F; c0 += CPP) {
        const int64_t col = c0 + (int64_t)lg * VEC;
        const bool active = col < F;
        float acc[VEC];
#pragma unroll
        for (int i = 0; i < VEC; ++i) acc[i] = 0.0f;
        const float* __restrict__ Xc = src + (active ? col : 0);
        // chunks of CH entries: lane lg of the group holds entries lg + G*k
        // (k < K), broadcast by shuffles; U gathers in flight per batch
        int32_t jl[K];
        float vl[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int64_t m = start + lg + (int64_t)G * k;
          jl[k] = 0;
          vl[k] = 0.0f;
          if (m < end) {
            jl[k] = __ldg(p.indices + m);
            vl[k] = __ldg(p.values + m);
          }
        }
        for (int64_t base = start; base < end; base += CH) {
          int32_t jn[K];
          float vn[K];
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const int64_t m = base + CH + lg + (int64_t)G * k;
            jn[k] = 0;
            vn[k] = 0.0f;
            if (m < end) {
              jn[k] = __ldg(p.indices + m);
              vn[k] = __ldg(p.values + m);
            }
          }
          const int cnt = (int)((end - base) < CH ? (end - base) : CH);
#pragma unroll
          for (int t = 0; t < CH; t += U) {
            if (t >= cnt) break;
            float xv[U][VEC];
            float vv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const int e = t + u;
              const int32_t jj = __shfl_sync(gmask, jl[e / G], e % G, G);
              vv[u] = __shfl_sync(gmask, vl[e / G], e % G, G);
              if (active && e < cnt) load_x<VEC>(Xc + (int64_t)jj * F, coherent, xv[u]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
              if (t + u < cnt && active) {
#pragma unroll
                for (int i = 0; i < VEC; ++i) acc[i] = __fmaf_rn(vv[u], xv[u][i], acc[i]);
              }
            }
          }
#pragma unroll
          for (int k = 0; k < K; ++k) {
            jl[k] = jn[k];
            vl[k] = vn[k];
          }
        }
        if (active) store_y<VEC>(dst + row * F + col, acc);
      }
      idx = nidx;
      row = nrow;
      start = nstart;
      end = nend;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(p.done + p.tile_graph[t], 1u);
    }
  }
}

// Lane groups narrower than a warp iterate rows in lock step; G must divide 32.
// Rows of a tile whose slot has no row left idle for that pass.
template <int G, int VEC, int U>
void launch_batch_gvu(const BatchParams& prm, int grid, cudaStream_t s, void** kernel_out) {
  auto kern = k_batch_diffuse<G, VEC, U>;
  if (kernel_out) *kernel_out = reinterpret_cast<void*>(kern);
  if (grid > 0) {
    kern<<<grid, kBatchThreads, 0, s>>>(prm);
    SCL_CUDA(cudaGetLastError());
  }
}

template <int VEC, int U>
void launch_batch_vu(int G, const BatchParams& prm, int grid, cudaStream_t s, void** k) {
  switch (G) {
    case 1: return launch_batch_gvu<1, VEC, U>(prm, grid, s, k);
    case 2: return launch_batch_gvu<2, VEC, U>(prm, grid, s, k);
    case 4: return launch_batch_gvu<4, VEC, U>(prm, grid, s, k);
    case 8: return launch_batch_gvu<8, VEC, U>(prm, grid, s, k);
    case 16: return launch_batch_gvu<16, VEC, U>(prm, grid, s, k);
    case 32: return launch_batch_gvu<32, VEC, U>(prm, grid, s, k);
    default: throw Error(kErrInvalidArgument, "batch lane group must be a power of two <= 32");
  }
}

void launch_batch(int G, int VEC, int U, const BatchParams& prm, int grid, cudaStream_t s, void** k) {
  if (VEC == 4 && U == 4) return launch_batch_vu<4, 4>(G, prm, grid, s, k);
  if (VEC == 4 && U == 8) return launch_batch_vu<4, 8>(G, prm, grid, s, k);
  if (VEC == 2 && U == 4) return launch_batch_vu<2, 4>(G, prm, grid, s, k);
  if (VEC == 2 && U == 8) return launch_batch_vu<2, 8>(G, prm, grid, s, k);
  if (VEC == 1 && U == 4) return launch_batch_vu<1, 4>(G, prm, grid, s, k);
  if (VEC == 1 && U == 8) return launch_batch_vu<1, 8>(G, prm, grid, s, k);
  throw Error(kErrInvalidArgument, "batch unroll must be 4 or 8");
}

__global__ void k_concat_structure(const int64_t* __restrict__ src_ptr, const int32_t* __restrict__ src_idx,
                                   const float* __restrict__ src_val, int64_t n, int64_t row_off, int64_t nnz_off,
                                   int64_t* __restrict__ dst_ptr, int32_t* __restrict__ dst_idx,
                                   float* __restrict__ dst_val) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i <= n; i += stride) dst_ptr[row_off + i] = src_ptr[i] + nnz_off;
  const int64_t nnz = src_ptr[n];
  for (int64_t q = tid; q < nnz; q += stride) {
    dst_idx[nnz_off + q] = src_idx[q] + (int32_t)row_off;
    dst_val[nnz_off + q] = src_val[q];
  }
}

}  // namespace

// ---------------------------------------------------------------------------------
BatchSolver::~BatchSolver() {
  if (exec_) cudaGraphExecDestroy(exec_);
  if (graph_) cudaGraphDestroy(graph_);
}

void BatchSolver::init(const std::vector<CsrView>& graphs, int64_t F, int64_t steps, cudaStream_t s) {
  SCL_REQUIRE(!graphs.empty(), kErrInvalidArgument, "a batch needs at least one graph");
  SCL_REQUIRE(F > 0 && steps >= 1, kErrInvalidArgument, "Dimensions must be positive");
  F_ = F;
  steps_ = steps;
  n_graphs_ = (int64_t)graphs.size();
  row_off_.assign(n_graphs_ + 1, 0);
  nnz_off_.assign(n_graphs_ + 1, 0);
  for (int64_t b = 0; b < n_graphs_; ++b) {
    const CsrView& g = graphs[b];
    SCL_REQUIRE(g.vtype == kF32, kErrTypeMismatch, "batched diffusion needs f32 graphs");
    SCL_REQUIRE(g.n_rows == g.n_cols, kErrDimensionMismatch, "batched diffusion needs square graphs");
    row_off_[b + 1] = row_off_[b] + g.n_rows;
    nnz_off_[b + 1] = nnz_off_[b] + g.nnz;
  }
  n_total_ = row_off_.back();
  nnz_total_ = nnz_off_.back();
  SCL_REQUIRE(n_total_ < (1ll << 31) && nnz_total_ < (1ll << 40), kErrInvalidArgument,
              "batch exceeds the int32 row range");
  indptr_ = DevBuf((n_total_ + 1) * 8, s);
  indices_ = DevBuf(std::max<int64_t>(nnz_total_, 1) * 4, s);
  values_ = DevBuf(std::max<int64_t>(nnz_total_, 1) * 4, s);
  for (int64_t b = 0; b < n_graphs_; ++b) {
    const CsrView& g = graphs[b];
    const int64_t work = std::max<int64_t>(g.n_rows + 1, g.nnz);
    const unsigned blocks = (unsigned)std::min<int64_t>(std::max<int64_t>(1, (work + 255) / 256), 148 * 8);
    k_concat_structure<<<blocks, 256, 0, s>>>(g.indptr, g.indices, static_cast<const float*>(g.values), g.n_rows,
                                              row_off_[b], nnz_off_[b], indptr_.as<int64_t>(),
                                              indices_.as<int32_t>(), values_.as<float>());
    SCL_CUDA(cudaGetLastError());
  }
  // host copy of the concatenated offsets for tiling
  h_indptr_.resize(n_total_ + 1);
  SCL_CUDA(cudaMemcpyAsync(h_indptr_.data(), indptr_.p, (n_total_ + 1) * 8, cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  scratch_ = DevBuf(std::max<int64_t>(n_total_ * F_, 1) * 4, s);
  counters_ = DevBuf((n_graphs_ + 4) * 4, s);
  status_ = DevBuf(4 * 4, s);
  SCL_CUDA(cudaMemsetAsync(status_.p, 0, 16, s));
  // lane mapping: 16-byte chunks when the row allows, else 8, else 4
  vec_ = (F_ % 4 == 0) ? 4 : ((F_ % 2 == 0) ? 2 : 1);
  int g = 1;
  while (g < 32 && (int64_t)g * vec_ < F_) g <<= 1;
  group_ = g;
  set_schedule(4096, 8, 0, s);
}

void BatchSolver::build_tiles(int64_t tile_nnz, cudaStream_t s) {
  // tiles of consecutive rows within each graph with about tile_nnz entries
  // (at least one row, at most 4096 rows); graphs in decreasing size order so
  // the largest graphs' tiles of each step are claimed first
  std::vector<int64_t> order(n_graphs_);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return (nnz_off_[a + 1] - nnz_off_[a]) > (nnz_off_[b + 1] - nnz_off_[b]);
  });
  std::vector<int64_t> trow;
  std::vector<int32_t> tgraph;
  std::vector<uint32_t> gtiles(n_graphs_, 0);
  // tiles are stored in schedule order; tile_row holds pairs (first row, end row)
  std::vector<int64_t> tend;
  for (int64_t gi : order) {
    int64_t r = row_off_[gi];
    const int64_t rend = row_off_[gi + 1];
    while (r < rend) {
      int64_t e = r + 1;
      while (e < rend && (h_indptr_[e + 1] - h_indptr_[r]) <= tile_nnz && (e - r) < 4096) ++e;
      trow.push_back(r);
      tend.push_back(e);
      tgraph.push_back((int32_t)gi);
      ++gtiles[gi];
      r = e;
    }
  }
  n_tiles_ = (int64_t)trow.size();
  // each tile's rows by decreasing length (stable), for balanced lane groups
  std::vector<int32_t> rord(n_total_);
  std::iota(rord.begin(), rord.end(), 0);
  for (size_t t = 0; t < trow.size(); ++t) {
    std::stable_sort(rord.begin() + trow[t], rord.begin() + tend[t], [&](int32_t a, int32_t b) {
      return (h_indptr_[a + 1] - h_indptr_[a]) > (h_indptr_[b + 1] - h_indptr_[b]);
    });
  }
  row_order_ = DevBuf(std::max<int64_t>(n_total_, 1) * 4, s);
  if (n_total_ > 0)
    SCL_CUDA(cudaMemcpyAsync(row_order_.p, rord.data(), n_total_ * 4, cudaMemcpyHostToDevice, s));
  // tile_row layout for the kernel: [t] = first row, [t+1] = end row is only
  // valid when tiles are contiguous in row space, which schedule order breaks;
  // store (first, end) interleaved as two arrays instead
  std::vector<int64_t> packed(2 * n_tiles_ + 2);
  for (int64_t t = 0; t < n_tiles_; ++t) {
    packed[t] = trow[t];
    packed[n_tiles_ + 1 + t] = tend[t];
  }
  tiles_ = DevBuf((2 * n_tiles_ + 2) * 8, s);
  tile_graph_ = DevBuf(std::max<int64_t>(n_tiles_, 1) * 4, s);
  graph_tiles_ = DevBuf(std::max<int64_t>(n_graphs_, 1) * 4, s);
  SCL_CUDA(cudaMemcpyAsync(tiles_.p, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaMemcpyAsync(tile_graph_.p, tgraph.data(), tgraph.size() * 4, cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaMemcpyAsync(graph_tiles_.p, gtiles.data(), gtiles.size() * 4, cudaMemcpyHostToDevice, s));
  SCL_CUDA(cudaStreamSynchronize(s));
}

void BatchSolver::set_schedule(int64_t tile_nnz, int unroll, int blocks_per_sm, cudaStream_t s) {
  SCL_REQUIRE(tile_nnz >= 1, kErrInvalidArgument, "tile size must be positive");
  SCL_REQUIRE(unroll == 4 || unroll == 8, kErrInvalidArgument, "batch unroll must be 4 or 8");
  SCL_REQUIRE(blocks_per_sm >= 0 && blocks_per_sm <= 8, kErrInvalidArgument, "blocks per SM must be in [0, 8]");
  tile_nnz_ = tile_nnz;
  unroll_ = unroll;
  build_tiles(tile_nnz, s);
  void* kern = nullptr;
  BatchParams dummy{};
  launch_batch(group_, vec_, unroll_, dummy, 0, s, &kern);
  int dev = 0, per_sm = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads, 0));
  const int bps = blocks_per_sm > 0 ? std::min(blocks_per_sm, std::max(per_sm, 1)) : std::max(per_sm, 1);
  blocks_per_sm_ = bps;
  grid_ = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)bps * sm_count(dev), n_tiles_ * steps_));
  invalidate_graph();
}

void BatchSolver::invalidate_graph() {
  if (exec_) cudaGraphExecDestroy(exec_);
  if (graph_) cudaGraphDestroy(graph_);
  exec_ = nullptr;
  graph_ = nullptr;
  knode_ = nullptr;
  cap_x0_ = nullptr;
  cap_y_ = nullptr;
}

void* BatchSolver::params_for(const float* X0, float* Y, void* storage) const {
  BatchParams* p = static_cast<BatchParams*>(storage);
  *p = BatchParams{};
  p->indptr = indptr_.as<int64_t>();
  p->indices = indices_.as<int32_t>();
  p->values = values_.as<float>();
  p->tile_row = tiles_.as<int64_t>();
  p->tile_graph = tile_graph_.as<int32_t>();
  p->row_order = row_order_.as<int32_t>();
  p->graph_tiles = graph_tiles_.as<uint32_t>();
  p->done = counters_.as<unsigned>();
  p->claim = counters_.as<unsigned>() + n_graphs_;
  p->status = status_.as<int32_t>();
  p->X0 = X0;
  p->Y = Y;
  p->scratch = scratch_.as<float>();
  p->F = F_;
  p->n_tiles = n_tiles_;
  p->steps = steps_;
  p->stall_graph = stall_graph_;
  return p;
}

void BatchSolver::launch_direct(const float* X0, float* Y, cudaStream_t s) {
  SCL_CUDA(cudaMemsetAsync(counters_.p, 0, (n_graphs_ + 1) * 4, s));
  BatchParams prm;
  params_for(X0, Y, &prm);
  launch_batch(group_, vec_, unroll_, prm, grid_, s, nullptr);
}

void BatchSolver::inject_stall(int graph) {
  SCL_REQUIRE(graph >= -1 && graph < n_graphs_, kErrInvalidArgument, "stall graph out of range");
  stall_graph_ = graph;
  invalidate_graph();
}

void BatchSolver::solve(const float* X0, float* Y, cudaStream_t s) {
  SCL_REQUIRE(X0 != Y, kErrInvalidArgument, "batched diffusion needs distinct input and output blocks");
  if (!exec_) {
    // capture memset + persistent kernel on a private stream, then instantiate
    cudaStream_t cs = nullptr;
    SCL_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      try {
        launch_direct(X0, Y, cs);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        throw;
      }
      e = cudaStreamEndCapture(cs, &graph_);
    }
    cudaStreamDestroy(cs);
    SCL_CUDA(e);
    SCL_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    size_t nn = 0;
    SCL_CUDA(cudaGraphGetNodes(graph_, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    SCL_CUDA(cudaGraphGetNodes(graph_, nodes.data(), &nn));
    for (auto nd : nodes) {
      cudaGraphNodeType ty;
      SCL_CUDA(cudaGraphNodeGetType(nd, &ty));
      if (ty == cudaGraphNodeTypeKernel) knode_ = nd;
    }
    SCL_REQUIRE(knode_ != nullptr, kErrInternal, "captured batch graph has no kernel node");
    cap_x0_ = X0;
    cap_y_ = Y;
  } else if (X0 != cap_x0_ || Y != cap_y_) {
    cudaKernelNodeParams kp{};
    SCL_CUDA(cudaGraphKernelNodeGetParams(knode_, &kp));
    BatchParams prm;
    params_for(X0, Y, &prm);
    void* args[1] = {&prm};
    kp.kernelParams = args;
    kp.extra = nullptr;
    SCL_CUDA(cudaGraphExecKernelNodeSetParams(exec_, knode_, &kp));
    cap_x0_ = X0;
    cap_y_ = Y;
  }
  SCL_CUDA(cudaGraphLaunch(exec_, s));
}

int32_t BatchSolver::status(cudaStream_t s, int32_t* item) {
  int32_t h[4] = {0, 0, 0, 0};
  SCL_CUDA(cudaMemcpyAsync(h, status_.p, 16, cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  if (item) *item = h[1];
  if (h[0] != 0) SCL_CUDA(cudaMemsetAsync(status_.p, 0, 16, s));
  return h[0];
}

double BatchSolver::time_solve(const float* X0, float* Y, int reps, cudaStream_t s) {
  cudaEvent_t a, b;
  SCL_CUDA(cudaEventCreate(&a));
  SCL_CUDA(cudaEventCreate(&b));
  launch_direct(X0, Y, s);  // warm-up
  SCL_CUDA(cudaEventRecord(a, s));
  for (int r = 0; r < reps; ++r) launch_direct(X0, Y, s);
  SCL_CUDA(cudaEventRecord(b, s));
  SCL_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  SCL_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return (double)ms / std::max(reps, 1);
}

void BatchSolver::autotune(const float* X0, float* Y, int reps, cudaStream_t s) {
  // candidate schedules: tile size x gathers in flight x resident CTAs per SM
  const int64_t tiles[] = {1024, 4096, 16384, 65536};
  const int unrolls[] = {4, 8};
  const int bps[] = {2, 4, 0};
  double best = 1e30;
  int64_t bt = tile_nnz_;
  int bu = unroll_, bb = 0;
  for (int64_t t : tiles)
    for (int u : unrolls)
      for (int b : bps) {
        set_schedule(t, u, b, s);
        const double ms = time_solve(X0, Y, reps, s);
        SCL_REQUIRE(status(s, nullptr) == 0, kErrInternal, "batched diffusion wait gave up during autotuning");
        if (ms < best) {
          best = ms;
          bt = t;
          bu = u;
          bb = b;
        }
      }
  set_schedule(bt, bu, bb, s);
  tuned_ms_ = best;
}

}  // namespace sclgpu
