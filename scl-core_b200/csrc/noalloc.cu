// Diffusion entry point that allocates no device memory.
//
// Some callers cannot allocate GPU memory while they run: a host framework
// that owns the whole device-memory budget through its own arena and forbids
// outside cudaMalloc, a serving loop that must neither block nor fail on an
// allocation after start-up, or code that must not let cudaMalloc/cudaFree
// implicitly synchronise the device. scl_gpu_diffuse_noalloc serves them: the
// caller passes the transition matrix, the input block and the output block
// (all device memory it owns), and the one intermediate iterate the power
// iteration needs lives in a fixed array compiled into this library.
//
// That array is a file-scope __device__ variable of kNoAllocMaxElems floats
// (32 MiB): every GPU on which the library is loaded holds it until the
// process exits. Host code must not pass the array's name to a kernel (on the
// host it is only a stand-in symbol); the device address is looked up with
// cudaGetSymbolAddress, with the device current, the first time a CUDA
// context calls in, and cached under that context's process-unique id
// (cuCtxGetId), so a caller that switches to another context on the same
// device, or resets the device, gets the address in the context it runs in.
//
// The kernel is a warp-per-row FP32 SpMM with the same per-element arithmetic
// as every other SpMM in this library: each output element is the sequential
// fma chain over its row's entries in stored order.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "abi_error.hpp"
#include "scl_gpu.h"

namespace {

constexpr int64_t kNoAllocMaxElems = 8388608;  // 32 MiB of float

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocMaxElems];

std::mutex g_noalloc_mu;
struct ScratchSlot {
  unsigned long long ctx_id;  // process-unique id of the context the address belongs to
  float* ptr;
};
ScratchSlot g_noalloc_slot[64] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

template <class Fn>
Fn driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return reinterpret_cast<Fn>(p);
}

// Id of the calling thread's current context (0 when it cannot be read).
unsigned long long current_context_id() {
  static const CtxGetCurrentFn get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
  static const CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array on `dev` (which must be current).
float* scratch_for(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  const unsigned long long ctx = current_context_id();
  ScratchSlot& slot = g_noalloc_slot[dev];
  if (slot.ptr == nullptr || ctx == 0 || slot.ctx_id != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      throw sclgpu::Error(SCL_ERROR_INTERNAL, "cudaGetSymbolAddress of the no-allocation scratch array failed");
    }
    slot.ptr = static_cast<float*>(p);
    slot.ctx_id = ctx;
  }
  return slot.ptr;
}

// True when the byte ranges [a, a + na) and [b, b + nb) share a byte.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + nb && y < x + na;
}

// One warp per row (grid-stride); lane l handles columns l, l+32, ...
__global__ void __launch_bounds__(256)
k_noalloc_spmm(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
               const float* __restrict__ values, const float* __restrict__ X, float* __restrict__ Y, int64_t n_rows,
               int64_t F) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n_rows; row += nw) {
    const int64_t start = indptr[row], end = indptr[row + 1];
    for (int64_t c0 = 0; c0 < F; c0 += 32) {
      const int64_t col = c0 + lane;
      float acc = 0.0f;
      for (int64_t base = start; base < end; base += 32) {
        const int64_t m = base + lane;
        int32_t j = 0;
        float v = 0.0f;
        if (m < end) {
          j = indices[m];
          v = values[m];
        }
        const int cnt = (int)((end - base) < 32 ? (end - base) : 32);
        for (int t = 0; t < cnt; ++t) {
          const int32_t jj = __shfl_sync(0xffffffffu, j, t);
          const float vv = __shfl_sync(0xffffffffu, v, t);
          if (col < F) acc = __fmaf_rn(vv, X[(int64_t)jj * F + col], acc);
        }
      }
      if (col < F) Y[row * F + col] = acc;
    }
  }
}

}  // namespace

extern "C" {

// Y = P^n_steps X for a device CSR transition matrix P (n_rows x n_rows), using
// only caller-owned memory plus this library's fixed scratch array.
SCL_EXPORT scl_error_t scl_gpu_diffuse_noalloc(const int64_t* indptr, const int32_t* indices, const float* values,
                                               int64_t n_rows, const float* X, float* Y, int64_t n_features,
                                               int64_t n_steps, void* stream) {
  SCL_API_CHECK_NULL(indptr, "Offset array pointer is null");
  SCL_API_CHECK_NULL(indices, "Indices array pointer is null");
  SCL_API_CHECK_NULL(values, "Data array pointer is null");
  SCL_API_CHECK_NULL(X, "Matrix X is null");
  SCL_API_CHECK_NULL(Y, "Matrix Y is null");
  SCL_API_CHECK(n_rows > 0 && n_features > 0 && n_steps >= 0, SCL_ERROR_INVALID_ARGUMENT,
                "Dimensions must be positive");
  SCL_API_CHECK(n_features <= kNoAllocMaxElems / n_rows, SCL_ERROR_INVALID_ARGUMENT,
                "n_rows * n_features exceeds the 8,388,608-element scratch array of the no-allocation entry point");
  const size_t block_bytes = (size_t)n_rows * (size_t)n_features * sizeof(float);
  SCL_API_CHECK(!overlaps(X, block_bytes, Y, block_bytes), SCL_ERROR_INVALID_ARGUMENT,
                "X and Y must not overlap");
  SCL_API_TRY
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  SCL_REQUIRE(dev >= 0 && dev < 64, SCL_ERROR_INTERNAL, "device ordinal out of range");
  float* scratch = scratch_for(dev);
  const size_t scratch_bytes = (size_t)kNoAllocMaxElems * sizeof(float);
  SCL_REQUIRE(!overlaps(X, block_bytes, scratch, scratch_bytes) && !overlaps(Y, block_bytes, scratch, scratch_bytes),
              SCL_ERROR_INVALID_ARGUMENT, "X and Y must not lie in the library's no-allocation scratch array");
  const int64_t n = n_rows, F = n_features;
  if (n_steps == 0) {
    SCL_CUDA(cudaMemcpyAsync(Y, X, n * F * sizeof(float), cudaMemcpyDeviceToDevice, s));
    SCL_API_RETURN_OK;
  }
  int sms = 0;
  SCL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t want = (n * 32 + 255) / 256;
  const unsigned grid = (unsigned)(want < (int64_t)sms * 8 ? want : (int64_t)sms * 8);
  // Ping-pong between the scratch array and Y so that the last step lands in
  // Y: step s writes Y when (n_steps - 1 - s) is even. Every element of each
  // step's output is written, so the scratch array needs no clearing.
  const float* src = X;
  for (int64_t st = 0; st < n_steps; ++st) {
    float* dst = ((n_steps - 1 - st) % 2 == 0) ? Y : scratch;
    k_noalloc_spmm<<<grid, 256, 0, s>>>(indptr, indices, values, src, dst, n, F);
    SCL_CUDA(cudaGetLastError());
    src = dst;
  }
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

}  // extern "C"
