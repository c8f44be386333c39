// Gather-throughput probe: the memory-system floor of one SpMM step.
//
// Every SpMM step gathers one X row per stored entry. This kernel performs
// exactly those gathers — the graph's column indices in the order the
// diffusion visits them, rows of the same pitch — and nothing else: no
// accumulation, no output rows, full occupancy (8 CTAs of 256 threads per
// SM), one 16-byte chunk per lane so a load instruction fetches several
// rows, U loads in flight per lane. Its time is the practical floor that an
// SpMM step on this graph cannot beat on this GPU; the benchmark reports the
// diffusion's achieved time against it beside the HBM roofline.
// No scl-core counterpart (a measurement aid).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine.hpp"

namespace sclgpu {
namespace {

template <int RB, int U>
__global__ void __launch_bounds__(256) k_gather_probe(const int32_t* __restrict__ idx, int64_t M,
                                                      const uint4* __restrict__ X, unsigned* __restrict__ out) {
  constexpr int L = RB / 16, Q = 32 / L;
  const int lane = threadIdx.x & 31, q = lane / L, lq = lane % L;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned acc = 0;
  for (int64_t base = warp * (Q * U); base < M; base += nw * (Q * U)) {
    uint4 r[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t e = base + u * Q + q;
      if (e < M) r[u] = __ldg(X + (int64_t)__ldcs(idx + e) * L + lq);
      else r[u] = make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) acc ^= r[u].x ^ r[u].y ^ r[u].z ^ r[u].w;
  }
  out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = acc;  // keeps the loads live
}

template <int RB>
void launch_probe(int U, const int32_t* idx, int64_t M, const void* X, unsigned* out, int blocks, cudaStream_t s) {
  if (U == 4) k_gather_probe<RB, 4><<<blocks, 256, 0, s>>>(idx, M, static_cast<const uint4*>(X), out);
  else k_gather_probe<RB, 8><<<blocks, 256, 0, s>>>(idx, M, static_cast<const uint4*>(X), out);
  SCL_CUDA(cudaGetLastError());
}

}  // namespace

double gather_floor_ms(const int32_t* idx, int64_t M, int64_t n_rows, int64_t row_bytes, int reps, cudaStream_t s) {
  SCL_REQUIRE(row_bytes == 128 || row_bytes == 256 || row_bytes == 512, kErrInvalidArgument,
              "the gather probe needs 128-, 256- or 512-byte rows");
  SCL_REQUIRE(reps >= 1, kErrInvalidArgument, "reps must be >= 1");
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  const int blocks = 8 * sm_count(dev);
  DevBuf X(std::max<int64_t>(n_rows, 1) * row_bytes, s);
  SCL_CUDA(cudaMemsetAsync(X.p, 0, X.bytes, s));
  DevBuf out((size_t)blocks * 256 * 4, s);
  DevBuf flush(256ull << 20, s);  // written between repetitions: larger than L2
  auto run = [&]() {
    const int U = 8;
    if (row_bytes == 128) launch_probe<128>(U, idx, M, X.p, out.as<unsigned>(), blocks, s);
    else if (row_bytes == 256) launch_probe<256>(U, idx, M, X.p, out.as<unsigned>(), blocks, s);
    else launch_probe<512>(U, idx, M, X.p, out.as<unsigned>(), blocks, s);
  };
  run();  // warm-up
  cudaEvent_t a, b;
  SCL_CUDA(cudaEventCreate(&a));
  SCL_CUDA(cudaEventCreate(&b));
  std::vector<float> t(reps);
  for (int r = 0; r < reps; ++r) {
    SCL_CUDA(cudaMemsetAsync(flush.p, r & 0xff, flush.bytes, s));
    SCL_CUDA(cudaEventRecord(a, s));
    run();
    SCL_CUDA(cudaEventRecord(b, s));
    SCL_CUDA(cudaEventSynchronize(b));
    SCL_CUDA(cudaEventElapsedTime(&t[r], a, b));
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::sort(t.begin(), t.end());
  return (double)t[reps / 2];
}

}  // namespace sclgpu
