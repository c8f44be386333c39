// Per-device runtime (stream + memory pool), error plumbing, dtype
// conversions, CSR validation and the scan / radix-sort building blocks.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdio>
#include <mutex>
#include <vector>

#include "engine.hpp"

namespace sclgpu {

void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  const int32_t code = (e == cudaErrorMemoryAllocation) ? kErrOutOfMemory
                       : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? kErrFeatureUnavailable
                                                                                        : kErrInternal;
  throw Error(code, buf);
}

size_t dtype_size(DType t) {
  switch (t) {
    case kF32: case kI32: return 4;
    case kF64: case kI64: return 8;
    case kBF16: case kF16: return 2;
  }
  throw Error(kErrInvalidArgument, "unknown dtype");
}

bool is_float_dtype(DType t) { return t == kF32 || t == kF64 || t == kBF16 || t == kF16; }

// ---------------------------------------------------------------------------
// Per-device state. Streams and pools live until process exit.
// ---------------------------------------------------------------------------
namespace {
struct DeviceState {
  bool init = false;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host<->device copies overlapped with work on `stream`
  cudaMemPool_t pool = nullptr;
  int sms = 0;
};
std::mutex g_mu;
DeviceState g_dev[64];

DeviceState& state(int dev) {
  SCL_REQUIRE(dev >= 0 && dev < 64, kErrInternal, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState& st = g_dev[dev];
  if (!st.init) {
    int prev = 0;
    SCL_CUDA(cudaGetDevice(&prev));
    SCL_CUDA(cudaSetDevice(dev));
    SCL_CUDA(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
    SCL_CUDA(cudaStreamCreateWithFlags(&st.copy_stream, cudaStreamNonBlocking));
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    SCL_CUDA(cudaMemPoolCreate(&st.pool, &props));
    // Keep up to 8 GiB cached between calls so repeated diffusions do not
    // return memory to the driver every time.
    uint64_t thresh = 8ull << 30;
    SCL_CUDA(cudaMemPoolSetAttribute(st.pool, cudaMemPoolAttrReleaseThreshold, &thresh));
    SCL_CUDA(cudaDeviceGetAttribute(&st.sms, cudaDevAttrMultiProcessorCount, dev));
    SCL_CUDA(cudaSetDevice(prev));
    st.init = true;
  }
  return st;
}
}  // namespace

int current_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    (void)cudaGetLastError();
    throw Error(kErrFeatureUnavailable, "no CUDA device available: the diffusion engine runs only on the GPU");
  }
  int dev = 0;
  SCL_CUDA(cudaGetDevice(&dev));
  return dev;
}

cudaStream_t library_stream(int dev) { return state(dev).stream; }
cudaStream_t library_copy_stream(int dev) { return state(dev).copy_stream; }

int sm_count(int dev) { return state(dev).sms; }

void* dev_alloc(size_t bytes, cudaStream_t s) {
  int dev = current_device();
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, state(dev).pool, s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    char buf[160];
    snprintf(buf, sizeof(buf), "device allocation of %zu bytes failed (%s)", bytes, cudaGetErrorString(e));
    throw Error(kErrOutOfMemory, buf);
  }
  return p;
}

void dev_free(void* p, cudaStream_t s) {
  if (p) (void)cudaFreeAsync(p, s);
}

// ---------------------------------------------------------------------------
// Status word
// ---------------------------------------------------------------------------
DevStatus::DevStatus(cudaStream_t s) : buf(2 * sizeof(int32_t), s) {
  SCL_CUDA(cudaMemsetAsync(buf.p, 0, 2 * sizeof(int32_t), s));
}

void DevStatus::check(cudaStream_t s, const char* what) {
  int32_t h[2] = {0, 0};
  SCL_CUDA(cudaMemcpyAsync(h, buf.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  SCL_CUDA(cudaStreamSynchronize(s));
  if (h[0] != 0) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s (at entry %d)", what, h[1]);
    throw Error(h[0], msg);
  }
}

// ---------------------------------------------------------------------------
// Conversions
// ---------------------------------------------------------------------------
namespace {
template <class S, class D>
__global__ void k_convert(const S* __restrict__ src, D* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = static_cast<D>(src[i]);
}

template <class T> __device__ __forceinline__ float to_f32(T v) { return static_cast<float>(v); }
template <> __device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }

template <class D> __device__ __forceinline__ D from_f64(double v);
template <> __device__ __forceinline__ float from_f64<float>(double v) { return static_cast<float>(v); }
template <> __device__ __forceinline__ double from_f64<double>(double v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_f64<__nv_bfloat16>(double v) { return __float2bfloat16_rn(static_cast<float>(v)); }
template <> __device__ __forceinline__ __half from_f64<__half>(double v) { return __float2half_rn(static_cast<float>(v)); }

template <class S> __device__ __forceinline__ double to_f64(S v) { return static_cast<double>(v); }
template <> __device__ __forceinline__ double to_f64<__nv_bfloat16>(__nv_bfloat16 v) { return (double)__bfloat162float(v); }
template <> __device__ __forceinline__ double to_f64<__half>(__half v) { return (double)__half2float(v); }

// Float conversions: f64 -> f32/bf16/f16 round once from the f64 value when
// the source is f64 is NOT what we want for bf16 (double rounding); for f32
// sources the path f32 -> bf16 is a single RNE rounding.
template <class S, class D>
__global__ void k_convert_float(const S* __restrict__ src, D* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (std::is_same<S, float>::value && std::is_same<D, __nv_bfloat16>::value) dst[i] = __float2bfloat16_rn(src[i]);
    else if constexpr (std::is_same<S, float>::value && std::is_same<D, __half>::value) dst[i] = __float2half_rn(src[i]);
    else if constexpr (std::is_same<S, double>::value && std::is_same<D, __nv_bfloat16>::value) dst[i] = __double2bfloat16(src[i]);
    else if constexpr (std::is_same<S, double>::value && std::is_same<D, __half>::value) dst[i] = __double2half(src[i]);
    else dst[i] = from_f64<D>(to_f64<S>(src[i]));
  }
}

inline int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

template <class S>
void convert_float_to(const S* src, void* dst, DType dst_t, int64_t n, cudaStream_t s) {
  const int g = grid_for(n);
  switch (dst_t) {
    case kF32: k_convert_float<S, float><<<g, 256, 0, s>>>(src, (float*)dst, n); break;
    case kF64: k_convert_float<S, double><<<g, 256, 0, s>>>(src, (double*)dst, n); break;
    case kBF16: k_convert_float<S, __nv_bfloat16><<<g, 256, 0, s>>>(src, (__nv_bfloat16*)dst, n); break;
    case kF16: k_convert_float<S, __half><<<g, 256, 0, s>>>(src, (__half*)dst, n); break;
    default: throw Error(kErrInvalidArgument, "convert_values: destination is not a float dtype");
  }
}
}  // namespace

void convert_indices(const void* src, DType src_t, int32_t* dst, int64_t count, cudaStream_t s) {
  if (count <= 0) return;
  if (src_t == kI32) {
    SCL_CUDA(cudaMemcpyAsync(dst, src, count * 4, cudaMemcpyDeviceToDevice, s));
  } else if (src_t == kI64) {
    k_convert<int64_t, int32_t><<<grid_for(count), 256, 0, s>>>((const int64_t*)src, dst, count);
  } else {
    throw Error(kErrTypeMismatch, "index arrays must be int32 or int64");
  }
  SCL_CUDA(cudaGetLastError());
}

void convert_offsets(const void* src, DType src_t, int64_t* dst, int64_t count, cudaStream_t s) {
  if (count <= 0) return;
  if (src_t == kI64) {
    SCL_CUDA(cudaMemcpyAsync(dst, src, count * 8, cudaMemcpyDeviceToDevice, s));
  } else if (src_t == kI32) {
    k_convert<int32_t, int64_t><<<grid_for(count), 256, 0, s>>>((const int32_t*)src, dst, count);
  } else {
    throw Error(kErrTypeMismatch, "offset arrays must be int32 or int64");
  }
  SCL_CUDA(cudaGetLastError());
}

void convert_values(const void* src, DType src_t, void* dst, DType dst_t, int64_t count, cudaStream_t s) {
  if (count <= 0) return;
  if (src_t == dst_t) {
    SCL_CUDA(cudaMemcpyAsync(dst, src, count * dtype_size(src_t), cudaMemcpyDeviceToDevice, s));
    return;
  }
  switch (src_t) {
    case kF32: convert_float_to<float>((const float*)src, dst, dst_t, count, s); break;
    case kF64: convert_float_to<double>((const double*)src, dst, dst_t, count, s); break;
    case kBF16: convert_float_to<__nv_bfloat16>((const __nv_bfloat16*)src, dst, dst_t, count, s); break;
    case kF16: convert_float_to<__half>((const __half*)src, dst, dst_t, count, s); break;
    default: throw Error(kErrTypeMismatch, "value arrays must be a float dtype");
  }
  SCL_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// CSR validation: records the first violation (atomicCAS on the code word).
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ void set_status(int32_t* st, int32_t code, int64_t where) {
  if (atomicCAS(st, 0, code) == 0) st[1] = (int32_t)where;
}

__global__ void k_validate_indptr(const int64_t* __restrict__ indptr, int64_t n, int64_t nnz, int32_t* st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = indptr[i];
    if (i == 0 && v != 0) set_status(st, kErrInvalidArgument, 0);
    if (i == n && v != nnz) set_status(st, kErrDimensionMismatch, n);
    if (i < n && indptr[i + 1] < v) set_status(st, kErrInvalidArgument, i);
  }
}

__global__ void k_validate_indices(const int32_t* __restrict__ idx, int64_t nnz, int64_t n_cols, int32_t* st) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t j = idx[i];
    if (j < 0 || (int64_t)j >= n_cols) set_status(st, kErrIndexOutOfBounds, i);
  }
}
}  // namespace

void validate_csr(const DeviceCSR& g, int32_t* status, cudaStream_t s) {
  k_validate_indptr<<<grid_for(g.n_rows + 1), 256, 0, s>>>(g.indptr.as<int64_t>(), g.n_rows, g.nnz, status);
  if (g.nnz > 0)
    k_validate_indices<<<grid_for(g.nnz), 256, 0, s>>>(g.indices.as<int32_t>(), g.nnz, g.n_cols, status);
  SCL_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Exclusive scan of int64: three-phase (tile sums, scan of tile sums, tile scan).
// ---------------------------------------------------------------------------
namespace {
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns (exclusive, total).
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* smem, int64_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t inc = warp_incl_scan(v);
  if (lane == 31) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int64_t w = (lane < nw) ? smem[lane] : 0;
    int64_t wi = warp_incl_scan(w);
    if (lane < nw) smem[lane] = wi - w;
    if (lane == nw - 1) smem[32] = wi;
  }
  __syncthreads();
  int64_t ex = inc - v + smem[warp];
  total = smem[32];
  __syncthreads();
  return ex;
}

__global__ void k_scan_tiles(const int64_t* __restrict__ in, int64_t* __restrict__ tile_sums, int64_t n) {
  __shared__ int64_t smem[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) s += in[i];
  }
  int64_t total;
  (void)block_excl_scan(s, smem, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_apply(const int64_t* __restrict__ in, int64_t* __restrict__ out,
                             const int64_t* __restrict__ tile_offsets, int64_t n) {
  __shared__ int64_t smem[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t loc[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    loc[k] = (i < n) ? in[i] : 0;
    s += loc[k];
  }
  int64_t total;
  int64_t ex = block_excl_scan(s, smem, total) + tile_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = ex;
    ex += loc[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = ex;
}
}  // namespace

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t count, cudaStream_t s) {
  // out has count + 1 entries; out[count] = total. `out` may alias `in`
  // only element-wise (each tile reads its inputs before writing them).
  if (count <= 0) {
    SCL_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    return;
  }
  const int64_t tiles = (count + kScanTile - 1) / kScanTile;
  DevBuf sums((tiles + 1) * sizeof(int64_t), s);
  k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, sums.as<int64_t>(), count);
  SCL_CUDA(cudaGetLastError());
  if (tiles > 1) exclusive_scan_i64(sums.as<int64_t>(), sums.as<int64_t>(), tiles, s);
  else SCL_CUDA(cudaMemsetAsync(sums.p, 0, sizeof(int64_t), s));
  k_scan_apply<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, sums.as<int64_t>(), count);
  SCL_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort, 8 bits per pass, 64-bit keys + 32-bit payload.
//   pass: (1) per-tile digit histogram -> hist[digit * tiles + tile]
//         (2) exclusive scan over hist (digit-major => global stable order)
//         (3) per-tile stable scatter: elements are ranked in tile order
//             round by round (one element per thread per round), using warp
//             match masks and per-warp digit counters in shared memory.
// ---------------------------------------------------------------------------
namespace {
constexpr int kRadixThreads = 256;
constexpr int kRadixRounds = 16;
constexpr int kRadixTile = kRadixThreads * kRadixRounds;  // elements per tile
constexpr int kRadixWarps = kRadixThreads / 32;

__global__ void k_radix_hist(const uint64_t* __restrict__ keys, int64_t n, int shift, int64_t* __restrict__ hist,
                             int64_t tiles) {
  __shared__ unsigned int h[256];
  for (int d = threadIdx.x; d < 256; d += blockDim.x) h[d] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    int64_t i = base + (int64_t)r * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(unsigned)((keys[i] >> shift) & 0xffu)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(int64_t)d * tiles + blockIdx.x] = h[d];
}

__global__ void k_radix_scatter(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t n,
                                int shift, const int64_t* __restrict__ offs, int64_t tiles,
                                uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
  __shared__ int64_t base_off[256];                 // next free global slot per digit for this tile
  __shared__ unsigned int wcnt[kRadixWarps][256];   // per-warp digit counts -> exclusive warp offsets
  __shared__ unsigned int rtot[256];                // per-digit total of the current round
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < 256; d += blockDim.x) base_off[d] = offs[(int64_t)d * tiles + blockIdx.x];
  const int64_t tbase = (int64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    for (int d = threadIdx.x; d < kRadixWarps * 256; d += blockDim.x) (&wcnt[0][0])[d] = 0u;
    __syncthreads();
    const int64_t i = tbase + (int64_t)r * kRadixThreads + threadIdx.x;
    const bool valid = i < n;
    const uint64_t k = valid ? keys[i] : 0ull;
    const uint32_t v = valid ? vals[i] : 0u;
    // Out-of-range lanes get a private pseudo-digit so they match no one.
    const unsigned dig = valid ? (unsigned)((k >> shift) & 0xffu) : 256u + (unsigned)lane;
    const unsigned peers = __match_any_sync(0xffffffffu, dig);
    const unsigned lower = peers & ((1u << lane) - 1u);
    if (valid && lower == 0u) wcnt[warp][dig] = (unsigned)__popc(peers);
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
      unsigned acc = 0u;
#pragma unroll
      for (int w = 0; w < kRadixWarps; ++w) {
        const unsigned c = wcnt[w][d];
        wcnt[w][d] = acc;
        acc += c;
      }
      rtot[d] = acc;
    }
    __syncthreads();
    if (valid) {
      const int64_t pos = base_off[dig] + (int64_t)wcnt[warp][dig] + (int64_t)__popc(lower);
      keys_out[pos] = k;
      vals_out[pos] = v;
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) base_off[d] += rtot[d];
    __syncthreads();
  }
}
}  // namespace

void radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_out, uint32_t* vals_out, int64_t count,
                      int key_bits, cudaStream_t s) {
  if (count <= 0) return;
  const int passes = (key_bits + 7) / 8;
  const int64_t tiles = (count + kRadixTile - 1) / kRadixTile;
  DevBuf hist((256 * tiles + 1) * sizeof(int64_t), s);
  uint64_t* kin = keys;
  uint32_t* vin = vals;
  uint64_t* kout = keys_out;
  uint32_t* vout = vals_out;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_radix_hist<<<(unsigned)tiles, kRadixThreads, 0, s>>>(kin, count, shift, hist.as<int64_t>(), tiles);
    SCL_CUDA(cudaGetLastError());
    exclusive_scan_i64(hist.as<int64_t>(), hist.as<int64_t>(), 256 * tiles, s);
    k_radix_scatter<<<(unsigned)tiles, kRadixThreads, 0, s>>>(kin, vin, count, shift, hist.as<int64_t>(), tiles,
                                                              kout, vout);
    SCL_CUDA(cudaGetLastError());
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  // After an odd number of passes the result is in keys_out; after an even
  // number it is back in keys — copy so the result always lands in *_out.
  if (kin != keys_out) {
    SCL_CUDA(cudaMemcpyAsync(keys_out, kin, count * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    SCL_CUDA(cudaMemcpyAsync(vals_out, vin, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
}

}  // namespace sclgpu
