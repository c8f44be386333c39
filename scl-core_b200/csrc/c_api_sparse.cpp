// Sparse-handle C ABI. Replaces scl/binding/c_api/core/sparse.cpp:51-560 (the
// subset the diffusion path uses) on top of the pointer-per-row container of
// scl/core/sparse.hpp. Validation rules and messages follow the reference.
#include <algorithm>
#include <cstring>
#include <thread>

#include "abi.hpp"

using sclabi::Index;
using sclabi::Real;

// ---- container ------------------------------------------------------------------
scl_sparse_matrix::~scl_sparse_matrix() {
  delete[] owned_data;
  delete[] owned_indices;
}

bool scl_sparse_matrix::is_contiguous() const {
  if (!valid || nnz == 0) return true;
  const Index pdim = primary_dim();
  Index first = -1;
  for (Index i = 0; i < pdim; ++i)
    if (lengths[i] > 0) { first = i; break; }
  if (first < 0) return true;
  const Real* ed = data_ptrs[first];
  const Index* ei = index_ptrs[first];
  for (Index i = first; i < pdim; ++i) {
    if (lengths[i] == 0) continue;
    if (data_ptrs[i] != ed || index_ptrs[i] != ei) return false;
    ed += lengths[i];
    ei += lengths[i];
  }
  return true;
}

Real* scl_sparse_matrix::contiguous_data() const {
  if (!valid || !is_contiguous()) return nullptr;
  for (Index i = 0; i < primary_dim(); ++i)
    if (lengths[i] > 0) return data_ptrs[i];
  return nullptr;
}

Index* scl_sparse_matrix::contiguous_indices() const {
  if (!valid || !is_contiguous()) return nullptr;
  for (Index i = 0; i < primary_dim(); ++i)
    if (lengths[i] > 0) return index_ptrs[i];
  return nullptr;
}

namespace sclabi {

BlockStrategyParams strategy_params(scl_block_strategy_t s) {
  // scl/core/sparse.hpp:85-99
  switch (s) {
    case SCL_BLOCK_STRATEGY_CONTIGUOUS: return {0, 0, true};
    case SCL_BLOCK_STRATEGY_SMALL: return {1024, 16384, false};
    case SCL_BLOCK_STRATEGY_LARGE: return {65536, 1048576, false};
    case SCL_BLOCK_STRATEGY_ADAPTIVE:
    default: return {4096, 262144, false};
  }
}

static Index block_size_for(Index total, BlockStrategyParams st) {
  // scl/core/sparse.hpp:102-113
  if (st.force_contiguous || total == 0) return total;
  Index target = std::max<Index>(4, (Index)std::thread::hardware_concurrency());
  Index ideal = (total + target - 1) / target;
  return std::clamp(ideal, st.min_block, st.max_block);
}

void allocate_blocks(scl_sparse_matrix& m, const std::vector<Index>& lens, BlockStrategyParams st) {
  const Index pdim = (Index)lens.size();
  m.lengths = lens;
  m.data_ptrs.assign(pdim, nullptr);
  m.index_ptrs.assign(pdim, nullptr);
  Index total = 0;
  for (Index v : lens) total += v;
  m.nnz = total;
  m.valid = true;
  if (total == 0) return;  // zeros(): all pointers null
  const Index bs = block_size_for(total, st);
  Index r0 = 0;
  while (r0 < pdim) {
    Index bnnz = 0, r1 = r0;
    while (r1 < pdim) {
      const Index len = lens[r1];
      if (bnnz > 0 && bnnz + len > bs) break;
      bnnz += len;
      ++r1;
    }
    if (bnnz > 0) {
      std::unique_ptr<Real[]> db(new Real[bnnz]());
      std::unique_ptr<Index[]> ib(new Index[bnnz]());
      Index off = 0;
      for (Index i = r0; i < r1; ++i) {
        if (lens[i] > 0) {
          m.data_ptrs[i] = db.get() + off;
          m.index_ptrs[i] = ib.get() + off;
        }
        off += lens[i];
      }
      m.data_blocks.push_back(std::move(db));
      m.index_blocks.push_back(std::move(ib));
    }
    r0 = r1;
  }
}

std::vector<int64_t> offsets_of(const scl_sparse_matrix& m) {
  const Index pdim = m.primary_dim();
  std::vector<int64_t> off(pdim + 1);
  off[0] = 0;
  for (Index i = 0; i < pdim; ++i) off[i + 1] = off[i] + (m.valid ? (int64_t)m.lengths[i] : 0);
  return off;
}

}  // namespace sclabi

namespace {

// Offsets must start at 0 and be non-decreasing (sparse.hpp:707-715).
void check_offsets(const Index* indptr, Index pdim) {
  SCL_REQUIRE(pdim == 0 || indptr[0] == 0, SCL_ERROR_INVALID_ARGUMENT, "offsets[0] must be 0");
  for (Index i = 0; i < pdim; ++i)
    SCL_REQUIRE(indptr[i + 1] >= indptr[i], SCL_ERROR_INVALID_ARGUMENT, "offsets must be non-decreasing");
}

scl_sparse_matrix* create_from_traditional(Index rows, Index cols, Index nnz, const Index* indptr,
                                           const Index* indices, const Real* data, bool is_csr,
                                           scl_block_strategy_t strategy) {
  const Index pdim = is_csr ? rows : cols;
  check_offsets(indptr, pdim);
  SCL_REQUIRE(indptr[pdim] <= nnz, SCL_ERROR_INVALID_ARGUMENT, "values/indices size mismatch");
  std::vector<Index> lens(pdim);
  for (Index i = 0; i < pdim; ++i) lens[i] = indptr[i + 1] - indptr[i];
  auto h = std::make_unique<scl_sparse_matrix>();
  h->is_csr = is_csr;
  h->rows = rows;
  h->cols = cols;
  sclabi::allocate_blocks(*h, lens, sclabi::strategy_params(strategy));
  for (Index i = 0; i < pdim; ++i) {
    if (lens[i] > 0) {
      std::memcpy(h->data_ptrs[i], data + indptr[i], sizeof(Real) * lens[i]);
      std::memcpy(h->index_ptrs[i], indices + indptr[i], sizeof(Index) * lens[i]);
    }
  }
  return h.release();
}

scl_sparse_matrix* wrap_traditional(Index rows, Index cols, Index* indptr, Index* indices, Real* data, bool is_csr) {
  const Index pdim = is_csr ? rows : cols;
  check_offsets(indptr, pdim);
  auto h = std::make_unique<scl_sparse_matrix>();
  h->is_csr = is_csr;
  h->rows = rows;
  h->cols = cols;
  h->valid = true;
  h->lengths.resize(pdim);
  h->data_ptrs.resize(pdim);
  h->index_ptrs.resize(pdim);
  for (Index i = 0; i < pdim; ++i) {
    const Index st = indptr[i];
    h->lengths[i] = indptr[i + 1] - st;
    h->data_ptrs[i] = h->lengths[i] > 0 ? data + st : nullptr;
    h->index_ptrs[i] = h->lengths[i] > 0 ? indices + st : nullptr;
  }
  h->nnz = indptr[pdim];
  return h.release();
}

// Copy of src with the given strategy (used by clone / to_contiguous / transpose).
scl_sparse_matrix* copy_with_strategy(const scl_sparse_matrix& src, scl_block_strategy_t strategy) {
  auto h = std::make_unique<scl_sparse_matrix>();
  h->is_csr = src.is_csr;
  h->rows = src.rows;
  h->cols = src.cols;
  sclabi::allocate_blocks(*h, src.lengths, sclabi::strategy_params(strategy));
  for (Index i = 0; i < src.primary_dim(); ++i) {
    if (src.lengths[i] > 0) {
      std::memcpy(h->data_ptrs[i], src.data_ptrs[i], sizeof(Real) * src.lengths[i]);
      std::memcpy(h->index_ptrs[i], src.index_ptrs[i], sizeof(Index) * src.lengths[i]);
    }
  }
  return h.release();
}

}  // namespace

extern "C" {

SCL_EXPORT scl_error_t scl_sparse_create(scl_sparse_t* out, scl_index_t rows, scl_index_t cols, scl_index_t nnz,
                                         const scl_index_t* indptr, const scl_index_t* indices,
                                         const scl_real_t* data, scl_bool_t is_csr) {
  return scl_sparse_create_with_strategy(out, rows, cols, nnz, indptr, indices, data, is_csr,
                                         SCL_BLOCK_STRATEGY_ADAPTIVE);
}

SCL_EXPORT scl_error_t scl_sparse_create_with_strategy(scl_sparse_t* out, scl_index_t rows, scl_index_t cols,
                                                       scl_index_t nnz, const scl_index_t* indptr,
                                                       const scl_index_t* indices, const scl_real_t* data,
                                                       scl_bool_t is_csr, scl_block_strategy_t strategy) {
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  SCL_API_CHECK_NULL(indptr, "Offset array pointer is null");
  SCL_API_CHECK_NULL(indices, "Index array pointer is null");
  SCL_API_CHECK_NULL(data, "Data array pointer is null");
  SCL_API_CHECK(rows > 0 && cols > 0, SCL_ERROR_INVALID_ARGUMENT, "Matrix dimensions must be positive");
  SCL_API_CHECK(nnz >= 0, SCL_ERROR_INVALID_ARGUMENT, "Number of non-zeros must be non-negative");
  SCL_API_TRY
  *out = create_from_traditional(rows, cols, nnz, indptr, indices, data, is_csr != SCL_FALSE, strategy);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_wrap(scl_sparse_t* out, scl_index_t rows, scl_index_t cols, scl_index_t nnz,
                                       scl_index_t* indptr, scl_index_t* indices, scl_real_t* data,
                                       scl_bool_t is_csr) {
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  SCL_API_CHECK_NULL(indptr, "Offset array pointer is null");
  SCL_API_CHECK_NULL(indices, "Index array pointer is null");
  SCL_API_CHECK_NULL(data, "Data array pointer is null");
  SCL_API_CHECK(rows > 0 && cols > 0, SCL_ERROR_INVALID_ARGUMENT, "Matrix dimensions must be positive");
  SCL_API_CHECK(nnz >= 0, SCL_ERROR_INVALID_ARGUMENT, "Number of non-zeros must be non-negative");
  SCL_API_TRY
  *out = wrap_traditional(rows, cols, indptr, indices, data, is_csr != SCL_FALSE);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_wrap_and_own(scl_sparse_t* out, scl_index_t rows, scl_index_t cols,
                                               scl_index_t nnz, scl_index_t* indptr, scl_index_t* indices,
                                               scl_real_t* data, scl_bool_t is_csr) {
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  SCL_API_CHECK_NULL(indptr, "Offset array pointer is null");
  SCL_API_CHECK_NULL(indices, "Index array pointer is null");
  SCL_API_CHECK_NULL(data, "Data array pointer is null");
  SCL_API_CHECK(rows > 0 && cols > 0, SCL_ERROR_INVALID_ARGUMENT, "Matrix dimensions must be positive");
  SCL_API_CHECK(nnz >= 0, SCL_ERROR_INVALID_ARGUMENT, "Number of non-zeros must be non-negative");
  SCL_API_TRY
  scl_sparse_matrix* h = wrap_traditional(rows, cols, indptr, indices, data, is_csr != SCL_FALSE);
  h->owned_data = data;
  h->owned_indices = indices;
  *out = h;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_clone(scl_sparse_t src, scl_sparse_t* out) {
  SCL_API_CHECK_NULL(src, "Source matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  SCL_API_TRY
  *out = copy_with_strategy(*src, src->is_contiguous() ? SCL_BLOCK_STRATEGY_CONTIGUOUS : SCL_BLOCK_STRATEGY_ADAPTIVE);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_destroy(scl_sparse_t* matrix) {
  if (matrix == nullptr || *matrix == nullptr) SCL_API_RETURN_OK;
  SCL_API_TRY
  delete *matrix;
  *matrix = nullptr;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_rows(scl_sparse_t m, scl_index_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->rows;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_cols(scl_sparse_t m, scl_index_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->cols;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_nnz(scl_sparse_t m, scl_index_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->nnz;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_is_csr(scl_sparse_t m, scl_bool_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->is_csr ? SCL_TRUE : SCL_FALSE;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_is_csc(scl_sparse_t m, scl_bool_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->is_csr ? SCL_FALSE : SCL_TRUE;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_is_valid(scl_sparse_t m, scl_bool_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->valid ? SCL_TRUE : SCL_FALSE;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_is_contiguous(scl_sparse_t m, scl_bool_t* out) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  *out = m->is_contiguous() ? SCL_TRUE : SCL_FALSE;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_layout_info(scl_sparse_t m, scl_sparse_layout_info_t* info) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(info, "Info pointer is null");
  SCL_API_TRY
  // count distinct blocks by pointer discontinuities in row order
  Index dblocks = 0;
  const Real* expect = nullptr;
  for (Index i = 0; i < m->primary_dim(); ++i) {
    if (m->lengths[i] == 0) continue;
    if (m->data_ptrs[i] != expect) ++dblocks;
    expect = m->data_ptrs[i] + m->lengths[i];
  }
  info->data_block_count = dblocks;
  info->index_block_count = dblocks;
  info->data_bytes = (scl_size_t)m->nnz * sizeof(Real);
  info->index_bytes = (scl_size_t)m->nnz * sizeof(Index);
  info->metadata_bytes = (scl_size_t)m->primary_dim() * (2 * sizeof(void*) + sizeof(Index));
  info->is_contiguous = m->is_contiguous() ? SCL_TRUE : SCL_FALSE;
  info->is_traditional_format = info->is_contiguous;
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_export(scl_sparse_t m, scl_index_t* indptr, scl_index_t* indices,
                                         scl_real_t* data) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(indptr, "Offset array pointer is null");
  SCL_API_CHECK_NULL(indices, "Index array pointer is null");
  SCL_API_CHECK_NULL(data, "Data array pointer is null");
  SCL_API_TRY
  const Index pdim = m->primary_dim();
  indptr[0] = 0;
  for (Index i = 0; i < pdim; ++i) {
    const Index len = m->valid ? m->lengths[i] : 0;
    const Index st = indptr[i];
    indptr[i + 1] = st + len;
    if (len > 0) {
      std::memcpy(indices + st, m->index_ptrs[i], sizeof(Index) * len);
      std::memcpy(data + st, m->data_ptrs[i], sizeof(Real) * len);
    }
  }
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_get_lengths(scl_sparse_t m, const scl_index_t** lengths,
                                              scl_size_t* lengths_size) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(lengths, "Output pointer is null");
  SCL_API_CHECK_NULL(lengths_size, "Size pointer is null");
  *lengths = m->lengths.data();
  *lengths_size = (scl_size_t)m->primary_dim();
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_get_indices(scl_sparse_t m, const scl_index_t** indices,
                                              scl_size_t* indices_size) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(indices, "Output pointer is null");
  SCL_API_CHECK_NULL(indices_size, "Size pointer is null");
  SCL_API_CHECK(m->is_contiguous(), SCL_ERROR_INVALID_ARGUMENT, "Matrix must be contiguous to get internal pointers");
  *indices = m->contiguous_indices();
  *indices_size = (scl_size_t)m->nnz;
  SCL_API_RETURN_OK;
}

SCL_EXPORT scl_error_t scl_sparse_get_data(scl_sparse_t m, const scl_real_t** data, scl_size_t* data_size) {
  SCL_API_CHECK_NULL(m, "Matrix is null");
  SCL_API_CHECK_NULL(data, "Output pointer is null");
  SCL_API_CHECK_NULL(data_size, "Size pointer is null");
  SCL_API_CHECK(m->is_contiguous(), SCL_ERROR_INVALID_ARGUMENT, "Matrix must be contiguous to get internal pointers");
  *data = m->contiguous_data();
  *data_size = (scl_size_t)m->nnz;
  SCL_API_RETURN_OK;
}

// scl/core/sparse.hpp:1141-1200: counting scatter over the original primary
// order, so each new primary list comes out sorted by its (old primary) index.
// The reference sizes the new primary dimension from the old one, which is only
// consistent for square matrices; rectangular inputs are rejected here.
SCL_EXPORT scl_error_t scl_sparse_transpose(scl_sparse_t src, scl_sparse_t* out) {
  SCL_API_CHECK_NULL(src, "Source matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  SCL_API_CHECK(src->rows == src->cols, SCL_ERROR_DIMENSION_MISMATCH, "transpose needs a square matrix");
  SCL_API_TRY
  const Index pdim = src->primary_dim();
  const Index new_pdim = src->secondary_dim();
  std::vector<Index> cnt(new_pdim, 0);
  for (Index i = 0; i < pdim; ++i)
    for (Index k = 0; k < src->lengths[i]; ++k) {
      const Index j = src->index_ptrs[i][k];
      SCL_REQUIRE(j >= 0 && j < new_pdim, SCL_ERROR_INDEX_OUT_OF_BOUNDS, "index out of range in transpose");
      ++cnt[j];
    }
  auto h = std::make_unique<scl_sparse_matrix>();
  h->is_csr = !src->is_csr;
  h->rows = src->rows;
  h->cols = src->cols;
  sclabi::allocate_blocks(*h, cnt, sclabi::strategy_params(SCL_BLOCK_STRATEGY_ADAPTIVE));
  std::vector<Index> pos(new_pdim, 0);
  for (Index i = 0; i < pdim; ++i)
    for (Index k = 0; k < src->lengths[i]; ++k) {
      const Index j = src->index_ptrs[i][k];
      const Index p = pos[j]++;
      h->data_ptrs[j][p] = src->data_ptrs[i][k];
      h->index_ptrs[j][p] = i;
    }
  *out = h.release();
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

SCL_EXPORT scl_error_t scl_sparse_to_contiguous(scl_sparse_t src, scl_sparse_t* out) {
  SCL_API_CHECK_NULL(src, "Source matrix is null");
  SCL_API_CHECK_NULL(out, "Output pointer is null");
  SCL_API_TRY
  *out = copy_with_strategy(*src, SCL_BLOCK_STRATEGY_CONTIGUOUS);
  SCL_API_RETURN_OK;
  SCL_API_CATCH
}

}  // extern "C"
