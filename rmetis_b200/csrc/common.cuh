// Shared device/host helpers for the rmetis B200 k-way engine.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

namespace rmb {

using idx_t = int32_t;

// Error carrying a METIS return code (-2 input, -3 memory, -4 other).
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define RMB_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e__ = (call);                                                               \
    if (e__ != cudaSuccess) {                                                               \
      int c__ = (e__ == cudaErrorMemoryAllocation) ? -3 : -4;                               \
      throw ::rmb::Error(c__, std::string(#call) + ": " + cudaGetErrorString(e__));        \
    }                                                                                       \
  } while (0)

// Every kernel launch is followed by RMB_LAUNCH_CHECK(), which also counts it.
std::atomic<long long>& launch_counter();
#define RMB_LAUNCH_CHECK()          \
  do {                              \
    RMB_CUDA(cudaGetLastError());   \
    ++::rmb::launch_counter();      \
  } while (0)

constexpr int kWarp = 32;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// splitmix64 finaliser: a bijective 64-bit mixer used for counter-based
// pseudo-random priorities (matching ties, seeds).
__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// Grid-stride loop helper.
// The loop set of a kernel body: every thread of the grid, or the threads of
// one block (a body run by a single block inside a fused kernel).
struct Lanes {
  int64_t first, stride;
};
__device__ inline Lanes grid_lanes() {
  return {(int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x};
}
__device__ inline Lanes block_lanes() { return {(int64_t)threadIdx.x, (int64_t)blockDim.x}; }
// The same over warps (a body that gives each item to one warp).
__device__ inline Lanes grid_warps() {
  return {(int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), (int64_t)gridDim.x * (blockDim.x >> 5)};
}
__device__ inline Lanes block_warps() { return {(int64_t)(threadIdx.x >> 5), (int64_t)(blockDim.x >> 5)}; }
#define RMB_FOR(i, n, L) for (int64_t i = (L).first; i < (int64_t)(n); i += (L).stride)

#define RMB_GRID_STRIDE(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)(n); i += (int64_t)gridDim.x * blockDim.x)

inline int grid_for(int64_t n, int threads, int max_blocks = 148 * 32) {
  int64_t b = ceil_div(n, threads);
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

__device__ inline unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Signed 64-bit atomic add through the unsigned overload (two's complement).
__device__ inline void atomic_add_i64(long long* a, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(a), static_cast<unsigned long long>(v));
}

template <typename T>
__device__ inline T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace rmb
