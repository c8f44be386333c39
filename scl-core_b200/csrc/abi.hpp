// Internals shared by the C ABI translation units: thread-local error state,
// exception -> error-code mapping, the host sparse handle and its device mirror.
//
// Compiled once per library variant; SCL_USE_FLOAT32/64 and SCL_USE_INT32/64
// select scl_real_t / scl_index_t exactly as scl-core's core.h:79-111 does.
#pragma once

#include <memory>
#include <vector>

#include "abi_error.hpp"
#include "engine.hpp"
#include "scl_core.h"
#include "scl_sparse.h"

namespace sclabi {

using Real = scl_real_t;
using Index = scl_index_t;

constexpr sclgpu::DType kRealDType = sizeof(Real) == 8 ? sclgpu::kF64 : sclgpu::kF32;
constexpr sclgpu::DType kIndexDType = sizeof(Index) == 8 ? sclgpu::kI64 : sclgpu::kI32;

// ---- host sparse container ---------------------------------------------------
// Pointer-per-row storage (scl/core/sparse.hpp:152-170): row i of the primary
// dimension lives at data_ptrs[i] / index_ptrs[i] with lengths[i] entries.
// Blocks are allocated following scl/core/sparse.hpp:67-113 and 1761-1830.
struct BlockStrategyParams {
  Index min_block = 4096;
  Index max_block = 262144;
  bool force_contiguous = false;
};
BlockStrategyParams strategy_params(scl_block_strategy_t s);

struct DeviceMirror;  // defined in c_api_diffusion.cpp

}  // namespace sclabi

struct scl_sparse_matrix {
  bool is_csr = true;
  bool valid = false;
  sclabi::Index rows = 0, cols = 0, nnz = 0;
  std::vector<sclabi::Real*> data_ptrs;
  std::vector<sclabi::Index*> index_ptrs;
  std::vector<sclabi::Index> lengths;
  // storage owned by the handle (create / clone / transpose)
  std::vector<std::unique_ptr<sclabi::Real[]>> data_blocks;
  std::vector<std::unique_ptr<sclabi::Index[]>> index_blocks;
  // arrays handed over by scl_sparse_wrap_and_own (released with delete[])
  sclabi::Real* owned_data = nullptr;
  sclabi::Index* owned_indices = nullptr;
  // optional device copy kept by scl_diffusion_gpu_attach
  std::shared_ptr<sclabi::DeviceMirror> mirror;

  ~scl_sparse_matrix();
  sclabi::Index primary_dim() const { return is_csr ? rows : cols; }
  sclabi::Index secondary_dim() const { return is_csr ? cols : rows; }
  // scl/core/sparse.hpp:480-513
  bool is_contiguous() const;
  // scl/core/sparse.hpp:562-586 (nullptr unless contiguous with a nonempty row)
  sclabi::Real* contiguous_data() const;
  sclabi::Index* contiguous_indices() const;
};

namespace sclabi {
// Allocate block storage for the given row lengths (sparse.hpp:633-692).
void allocate_blocks(scl_sparse_matrix& m, const std::vector<Index>& lens, BlockStrategyParams st);
// Offsets (int64) of the traditional layout derived from lengths.
std::vector<int64_t> offsets_of(const scl_sparse_matrix& m);
}  // namespace sclabi

