// Device workspace: a chunked bump allocator kept across calls.
//
// One partition call allocates its whole hierarchy (levels, cmaps, refinement
// scratch) from here. Chunks are cudaMalloc'd on first need and reused by later
// calls; rewind() frees nothing, it only resets the bump pointers.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace rmb {

// Optional cap on the device workspace all arenas of a process hold on one
// device (environment RMETIS_B200_ARENA_CAP, bytes; unset or 0 = none). An
// allocation that would pass it fails like a cudaMalloc out of memory. It
// emulates a smaller device, so that the out-of-memory handling of the worker
// pool can be exercised without driving a GPU out of memory.
size_t arena_cap_bytes();
// Reserves (or, with a negative delta, returns) bytes against the cap of a
// device; false when the reservation would pass the cap.
bool arena_cap_reserve(int device, long long delta);

class Arena {
 public:
  explicit Arena(size_t min_chunk = (size_t)256 << 20) : min_chunk_(min_chunk) {}
  ~Arena() { release(); }
  Arena(const Arena&) = delete;
  Arena& operator=(const Arena&) = delete;

  template <typename T>
  T* alloc(size_t count) {
    return static_cast<T*>(alloc_bytes(count * sizeof(T)));
  }

  void* alloc_bytes(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    if (bytes == 0) bytes = 256;
    while (cur_ < chunks_.size()) {
      Chunk& c = chunks_[cur_];
      if (c.top + bytes <= c.size) {
        void* p = c.base + c.top;
        c.top += bytes;
        return p;
      }
      ++cur_;
    }
    size_t sz = bytes > min_chunk_ ? bytes : min_chunk_;
    Chunk c;
    if (arena_cap_bytes()) {
      if (cudaGetDevice(&c.device) != cudaSuccess) throw Error(-4, "cudaGetDevice failed");
      if (!arena_cap_reserve(c.device, (long long)sz)) throw Error(-3, "device workspace cap reached");
    }
    cudaError_t e = cudaMalloc(&c.base, sz);
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (arena_cap_bytes()) arena_cap_reserve(c.device, -(long long)sz);
      throw Error(-3, "device workspace allocation failed");
    }
    c.size = sz;
    c.top = bytes;
    chunks_.push_back(c);
    cur_ = chunks_.size() - 1;
    return c.base;
  }

  // Marks let a caller drop the scratch of one phase while keeping older data.
  struct Mark {
    size_t chunk, top;
  };
  Mark mark() const {
    if (chunks_.empty()) return {0, 0};
    size_t c = cur_ < chunks_.size() ? cur_ : chunks_.size() - 1;
    return {c, chunks_[c].top};
  }
  void reset_to(const Mark& m) {
    for (size_t i = m.chunk + 1; i < chunks_.size(); ++i) chunks_[i].top = 0;
    if (m.chunk < chunks_.size()) chunks_[m.chunk].top = m.top;
    cur_ = m.chunk;
  }
  void rewind() {
    for (auto& c : chunks_) c.top = 0;
    cur_ = 0;
  }
  void release() {
    for (auto& c : chunks_) {
      cudaFree(c.base);
      if (arena_cap_bytes()) arena_cap_reserve(c.device, -(long long)c.size);
    }
    chunks_.clear();
    cur_ = 0;
  }
  size_t reserved() const {
    size_t s = 0;
    for (auto& c : chunks_) s += c.size;
    return s;
  }

 private:
  struct Chunk {
    char* base = nullptr;
    size_t size = 0, top = 0;
    int device = 0;
  };
  std::vector<Chunk> chunks_;
  size_t cur_ = 0;
  size_t min_chunk_;
};

}  // namespace rmb
