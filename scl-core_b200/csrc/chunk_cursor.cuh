// Chunk cursor for the cp.async-pipelined warp-per-row kernels.
//
// A warp owns rows row0, row0 + nw, row0 + 2nw, ... (persistent grid-stride),
// or, given a schedule (warp_schedule with one row per group), the rows of its
// list sched[w] .. sched[w + 1] - 1, stored after the nw + 1 offsets. Their
// stored entries are cut into chunks of at most 32 entries that never span
// rows; an empty row yields one chunk of 0 entries so that its output row is
// still written. The cursor hands out the warp's chunks in order and keeps
// the bounds of the next two rows in flight (and, with a schedule, the id of
// the row after them), so moving to a new row costs no dependent load on the
// critical path. All fields are warp-uniform.
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
  int32_t r1, r2, r3;     // the next three rows (n: none; row ids are int32)
  int64_t s1, e1, s2, e2; // bounds of r1 and r2
  int64_t n, nw;
  const int32_t* list;    // schedule: this warp's rows are list[q .. q_end)
  int32_t q, q_end;
  bool first;

  // the warp's next row after the ones already taken (n when none is left)
  __device__ __forceinline__ int32_t take() {
    if (list == nullptr) {
      const int64_t r = (int64_t)r3 + nw;
      return (int32_t)(r < n ? r : n);
    }
    return q < q_end ? list[q++] : (int32_t)n;
  }

  __device__ __forceinline__ void init(const int64_t* __restrict__ ptr, int64_t row0, int64_t n_rows,
                                       int64_t n_warps, const int32_t* __restrict__ sched = nullptr) {
    n = n_rows;
    nw = n_warps;
    list = nullptr;
    q = q_end = 0;
    first = true;
    pos = end = s1 = e1 = s2 = e2 = 0;
    if (sched != nullptr) {
      list = sched + nw + 1;
      q = sched[row0];
      q_end = sched[row0 + 1];
      row = take();
    } else {
      row = row0;
      r3 = (int32_t)row0;
    }
    r1 = r3 = take();
    r2 = r3 = take();
    r3 = take();
    if (row < n) {
      pos = ptr[row];
      end = ptr[row + 1];
    }
    if (r1 < n) {
      s1 = ptr[r1];
      e1 = ptr[r1 + 1];
    }
    if (r2 < n) {
      s2 = ptr[r2];
      e2 = ptr[r2 + 1];
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
      row = r1;
      pos = s1;
      end = e1;
      r1 = r2;
      s1 = s2;
      e1 = e2;
      r2 = r3;
      s2 = e2 = 0;
      if (r2 < n) {
        s2 = ptr[r2];
        e2 = ptr[r2 + 1];
      }
      r3 = take();
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
