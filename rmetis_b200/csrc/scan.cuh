// Device-wide exclusive prefix sums (reduce-then-scan, three launches, no
// inter-block waiting). Used for cmap numbering, coarse CSR offsets and mover
// compaction.
#pragma once

#include "arena.h"
#include "common.cuh"

namespace rmb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ inline T block_exclusive_scan(T v, T* smem_warp, T* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < nw ? smem_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) smem_warp[lane] = w;  // inclusive per warp
  }
  __syncthreads();
  T warp_prefix = wid > 0 ? smem_warp[wid - 1] : T(0);
  if (total) *total = smem_warp[(blockDim.x >> 5) - 1];
  T r = warp_prefix + x - v;
  __syncthreads();
  return r;
}

// Phase 1: sum of each tile.
template <typename T, typename Load>
__global__ void k_tile_reduce(Load load, int64_t n, T* tile_sums) {
  __shared__ T sw[32];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t j = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (j < n) s += load(j);
  }
  T tot;
  block_exclusive_scan<T>(s, sw, &tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// Phase 2: exclusive scan of tile sums in one block; writes the grand total.
template <typename T>
__global__ void k_scan_tile_sums(T* tile_sums, int64_t ntiles, T* total_out) {
  __shared__ T sw[32];
  T carry = 0;
  for (int64_t base = 0; base < ntiles; base += (int64_t)blockDim.x * kScanItems) {
    T vals[kScanItems];
    T s = 0;
    int64_t my = base + (int64_t)threadIdx.x * kScanItems;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      vals[i] = (my + i < ntiles) ? tile_sums[my + i] : T(0);
      s += vals[i];
    }
    T tot;
    T ex = block_exclusive_scan<T>(s, sw, &tot);
    T run = carry + ex;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      if (my + i < ntiles) tile_sums[my + i] = run;
      run += vals[i];
    }
    carry += tot;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

// Phase 3: per-tile exclusive scan plus the tile offset; out[n] gets the total
// when `write_end` (so out can serve as a CSR offset array of length n+1).
template <typename T, typename Load, typename Store>
__global__ void k_tile_scan(Load load, Store store, int64_t n, const T* tile_offsets) {
  __shared__ T sw[32];
  __shared__ T tile[kScanTile];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t j = base + (int64_t)i * kScanThreads + threadIdx.x;
    tile[i * kScanThreads + threadIdx.x] = (j < n) ? load(j) : T(0);
  }
  __syncthreads();
  T vals[kScanItems];
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = tile[threadIdx.x * kScanItems + i];
    s += vals[i];
  }
  T ex = block_exclusive_scan<T>(s, sw, nullptr);
  T run = ex + tile_offsets[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    tile[threadIdx.x * kScanItems + i] = run;
    run += vals[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t j = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (j < n) store(j, tile[i * kScanThreads + threadIdx.x]);
  }
}

// Phases 2 and 3 in one launch for inputs of at most kScanFusedTiles tiles:
// each block sums the tile totals before it (a few thousand L2 reads) instead
// of waiting for a separate scan of the tile sums; the last block writes the
// grand total.
constexpr int64_t kScanFusedTiles = 4096;

template <typename T, typename Load, typename Store>
__global__ void k_tile_scan_fused(Load load, Store store, int64_t n, const T* tile_sums, int64_t ntiles,
                                  T* total_out) {
  __shared__ T sw[32];
  __shared__ T tile[kScanTile];
  T before = 0;
  for (int64_t i = threadIdx.x; i < (int64_t)blockIdx.x; i += blockDim.x) before += tile_sums[i];
  T offset;
  block_exclusive_scan<T>(before, sw, &offset);
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t j = base + (int64_t)i * kScanThreads + threadIdx.x;
    tile[i * kScanThreads + threadIdx.x] = (j < n) ? load(j) : T(0);
  }
  __syncthreads();
  T vals[kScanItems];
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = tile[threadIdx.x * kScanItems + i];
    s += vals[i];
  }
  T tile_total;
  T run = block_exclusive_scan<T>(s, sw, &tile_total) + offset;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    tile[threadIdx.x * kScanItems + i] = run;
    run += vals[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t j = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (j < n) store(j, tile[i * kScanThreads + threadIdx.x]);
  }
  if (threadIdx.x == 0 && total_out && (int64_t)blockIdx.x == ntiles - 1) *total_out = offset + tile_total;
}

// Small inputs: the whole scan in one block (tiles of 1024 x 8 items in
// order, with a running carry), one launch instead of three.
constexpr int kScanSmallThreads = 1024;
constexpr int kScanSmallTile = kScanSmallThreads * kScanItems;
constexpr int64_t kScanSmallMax = 2 * kScanSmallTile;

template <typename T, typename Load, typename Store>
__global__ void __launch_bounds__(kScanSmallThreads) k_scan_small(Load load, Store store, int64_t n, T* total_out) {
  __shared__ T sw[32];
  __shared__ T tile[kScanSmallTile];
  T carry = 0;
  for (int64_t base = 0; base < n; base += kScanSmallTile) {
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const int64_t j = base + (int64_t)i * kScanSmallThreads + threadIdx.x;
      tile[i * kScanSmallThreads + threadIdx.x] = (j < n) ? load(j) : T(0);
    }
    __syncthreads();
    T vals[kScanItems];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      vals[i] = tile[threadIdx.x * kScanItems + i];
      s += vals[i];
    }
    T tot;
    T run = carry + block_exclusive_scan<T>(s, sw, &tot);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      tile[threadIdx.x * kScanItems + i] = run;
      run += vals[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const int64_t j = base + (int64_t)i * kScanSmallThreads + threadIdx.x;
      if (j < n) store(j, tile[i * kScanSmallThreads + threadIdx.x]);
    }
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

// Exclusive scan of load(0..n-1) by one block (inside a fused kernel), in
// tiles of blockDim.x * 4 items: warp w takes the w-th run of 128 items of a
// tile, its lanes reading 32 consecutive items at a time (coalesced), and
// each item is loaded once. Every thread of the block must call it; sw holds
// 32 values of shared memory.
template <typename T, typename Load, typename Store>
__device__ void block_scan_n(Load load, Store store, int64_t n, T* total_out, T* sw) {
  constexpr int kIt = 4;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t tile = (int64_t)blockDim.x * kIt;
  T carry = 0;
  for (int64_t base = 0; base < n; base += tile) {
    const int64_t wbase = base + (int64_t)wid * 32 * kIt;
    T v[kIt];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kIt; ++i) {
      const int64_t idx = wbase + i * 32 + lane;
      v[i] = idx < n ? load(idx) : T(0);
      s += v[i];
    }
    s = warp_sum(s);
    T tile_total;
    // lane 0 of each warp stands for its run: the exclusive scan gives the run's offset
    const T wex = block_exclusive_scan<T>(lane == 0 ? s : T(0), sw, &tile_total);
    T off = carry + __shfl_sync(0xffffffffu, wex, 0);
#pragma unroll
    for (int i = 0; i < kIt; ++i) {
      T x = v[i];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      const int64_t idx = wbase + i * 32 + lane;
      if (idx < n) store(idx, off + x - v[i]);
      off += __shfl_sync(0xffffffffu, x, 31);
    }
    carry += tile_total;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

template <typename T>
struct LoadArr {
  const T* p;
  __device__ T operator()(int64_t i) const { return p[i]; }
};
struct LoadNonZero {
  const int32_t* f;
  __device__ int32_t operator()(int64_t i) const { return f[i] != 0 ? 1 : 0; }
};
// Compaction store: the index of every nonzero flag goes to its rank.
struct StoreCompact {
  const int32_t* f;
  int32_t* out;
  __device__ void operator()(int64_t i, int32_t pos) const {
    if (f[i] != 0) out[pos] = (int32_t)i;
  }
};

template <typename T>
struct StoreArr {
  T* p;
  __device__ void operator()(int64_t i, T v) const { p[i] = v; }
};

// Exclusive scan of `load(0..n-1)` into `store`; the total is written to
// device memory at `total_dev` (may be null). Scratch comes from the arena and
// is released on return.
template <typename T, typename Load, typename Store>
void exclusive_scan(Load load, Store store, int64_t n, T* total_dev, Arena& arena, cudaStream_t st) {
  if (n <= kScanSmallMax) {
    k_scan_small<T, Load, Store><<<1, kScanSmallThreads, 0, st>>>(load, store, n, total_dev);
    RMB_LAUNCH_CHECK();
    return;
  }
  Arena::Mark mk = arena.mark();
  int64_t ntiles = ceil_div(n, kScanTile);
  if (ntiles < 1) ntiles = 1;
  T* sums = arena.alloc<T>((size_t)ntiles);
  if (n > 0) {
    k_tile_reduce<T, Load><<<(unsigned)ntiles, kScanThreads, 0, st>>>(load, n, sums);
    RMB_LAUNCH_CHECK();
  } else {
    RMB_CUDA(cudaMemsetAsync(sums, 0, sizeof(T), st));
  }
  if (n > 0 && ntiles <= kScanFusedTiles) {
    k_tile_scan_fused<T, Load, Store><<<(unsigned)ntiles, kScanThreads, 0, st>>>(load, store, n, sums, ntiles,
                                                                                 total_dev);
    RMB_LAUNCH_CHECK();
    arena.reset_to(mk);
    return;
  }
  k_scan_tile_sums<T><<<1, 1024, 0, st>>>(sums, ntiles, total_dev);
  RMB_LAUNCH_CHECK();
  if (n > 0) {
    k_tile_scan<T, Load, Store><<<(unsigned)ntiles, kScanThreads, 0, st>>>(load, store, n, sums);
    RMB_LAUNCH_CHECK();
  }
  arena.reset_to(mk);
}

template <typename T>
void exclusive_scan_arr(const T* in, T* out, int64_t n, T* total_dev, Arena& arena, cudaStream_t st) {
  exclusive_scan<T>(LoadArr<T>{in}, StoreArr<T>{out}, n, total_dev, arena, st);
}

}  // namespace rmb
