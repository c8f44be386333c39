// Chunk cursor for the cp.async-pipelined warp-per-row kernels.
//
// A warp owns rows row0, row0 + nw, row0 + 2nw, ... (persistent grid-stride).
// Their stored entries are cut into chunks of at most 32 entries that never
// span rows; an empty row yields one chunk of 0 entries so that its output row
// is still written. The cursor hands out the warp's chunks in order and keeps
// the bounds of the next two rows in flight, so moving to a new row costs no
// dependent load on the critical path. All fields are warp-uniform.
#pragma once

#include <cstdint>

namespace sclgpu {

struct Chunk {
  int64_t row = 0;   // row of the chunk (n when the stream is exhausted)
  int64_t pos = 0;   // first stored entry
  int cnt = 0;       // entries in the chunk (0..32)
  bool first = false;
  bool last = false;
  bool valid = false;
};

struct ChunkCursor {
  int64_t row, pos, end;  // current row, next entry, row end
  int64_t s1, e1, s2, e2; // bounds of row + nw and row + 2 nw
  int64_t n, nw;
  bool first;

  __device__ __forceinline__ void init(const int64_t* __restrict__ ptr, int64_t row0, int64_t n_rows,
                                       int64_t n_warps) {
    n = n_rows;
    nw = n_warps;
    row = row0;
    first = true;
    pos = end = s1 = e1 = s2 = e2 = 0;
    if (row < n) {
      pos = ptr[row];
      end = ptr[row + 1];
    }
    if (row + nw < n) {
      s1 = ptr[row + nw];
      e1 = ptr[row + nw + 1];
    }
    if (row + 2 * nw < n) {
      s2 = ptr[row + 2 * nw];
      e2 = ptr[row + 2 * nw + 1];
    }
  }

  // The chunk at the cursor; advances past it.
  __device__ __forceinline__ Chunk next(const int64_t* __restrict__ ptr) {
    Chunk c;
    c.valid = row < n;
    if (!c.valid) {
      c.row = n;
      return c;
    }
    c.row = row;
    c.pos = pos;
    c.first = first;
    const int64_t rem = end - pos;
    c.cnt = rem < 32 ? (int)rem : 32;
    c.last = rem <= 32;
    if (c.last) {
      row += nw;
      pos = s1;
      end = e1;
      s1 = s2;
      e1 = e2;
      s2 = e2 = 0;
      if (row + 2 * nw < n) {
        s2 = ptr[row + 2 * nw];
        e2 = ptr[row + 2 * nw + 1];
      }
      first = true;
    } else {
      pos += 32;
      first = false;
    }
    return c;
  }
};

__device__ __forceinline__ void cp_async16_ca(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace sclgpu
