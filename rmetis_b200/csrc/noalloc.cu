// Edge cut and partition weights with no allocation at all.
//
// Some callers cannot allocate device memory when they need these numbers:
// hosts that give a plugin a fixed memory budget or their own pool and forbid
// it to grow, and latency-sensitive loops where cudaMalloc/cudaFree would
// synchronise the device. This entry point serves them: the caller passes
// device inputs and outputs and a stream, and the only scratch (the 64-bit
// accumulators) is a file-scope __device__ array of fixed size, so the call
// never allocates.
//
// Limits and sharing: at most kNoAllocMaxParts accumulators (nparts * ncon),
// about 128 KiB that every GPU which loads the library keeps until exit. All
// calls on a device share the array; each call clears it first, so calls
// that overlap on the GPU (other streams, or other host threads) race and
// must be serialised by the caller. The first call on a device looks up the
// array's device address (cudaGetSymbolAddress), so that first call should
// come before any stream capture.
#include <cstdio>
#include <mutex>

#include "../../include/rmetis.h"
#include "common.cuh"

namespace rmb {
namespace {

constexpr int kNoAllocMaxParts = 16384;
constexpr int kNoAllocHeader = 32;  // [0] cut accumulator, [1] bad-input flag

// The scratch. In host code this name is only a host-side stand-in for the
// device variable; kernels get its device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocHeader + kNoAllocMaxParts];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does this set-up).
unsigned long long* noalloc_scratch_for_current_device(int* err) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *err = METIS_ERROR;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    unsigned long long* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "rmetis_b200: cudaGetSymbolAddress for the no-allocation scratch failed: %s\n",
                   cudaGetErrorString(e));
      *err = METIS_ERROR;
      return nullptr;
    }
    g_noalloc_ptr[dev] = p;
  }
  return g_noalloc_ptr[dev];
}

// Part weights of a block are summed in shared memory when nparts * ncon is
// at most this (one global atomic per part and block instead of one per
// vertex: with few parts, as in a bisection, per-vertex atomics would all hit
// the same few addresses).
constexpr int kNoAllocSmemParts = 4096;

// One pass: edge cut (sum of cross weights over both directions) and part
// weights, accumulated in the scratch. Every index is bounds-checked against
// n, nnz and nparts; an out-of-range entry is skipped and flagged.
__global__ void k_noalloc_cut_pw(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                                 const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ vwgt, int32_t n,
                                 int64_t nnz, int32_t ncon, const idx_t* __restrict__ part, int32_t nparts,
                                 unsigned long long* __restrict__ scratch) {
  __shared__ unsigned long long spw[kNoAllocSmemParts];
  const int32_t K = nparts * ncon;
  const bool local = K <= kNoAllocSmemParts;
  if (local)
    for (int32_t i = threadIdx.x; i < K; i += blockDim.x) spw[i] = 0;
  __syncthreads();
  unsigned long long acc = 0;
  int bad = 0;
  RMB_GRID_STRIDE(v, n) {
    const int32_t pv = part[v];
    if (pv < 0 || pv >= nparts) {
      bad = 1;
      continue;
    }
    for (int c = 0; c < ncon; ++c) {
      const long long w = vwgt ? vwgt[(int64_t)v * ncon + c] : 1;
      if (local) atomicAdd(&spw[(int64_t)pv * ncon + c], (unsigned long long)w);
      else atomicAdd(&scratch[kNoAllocHeader + (int64_t)pv * ncon + c], (unsigned long long)w);
    }
    int64_t s = xadj[v], e = xadj[v + 1];
    if (s < 0 || e > nnz || s > e) {
      bad = 1;
      continue;
    }
    for (int64_t j = s; j < e; ++j) {
      const int32_t u = adj[j];
      if (u < 0 || u >= n) {
        bad = 1;
        continue;
      }
      if (part[u] != pv) acc += (uint32_t)(adjwgt ? adjwgt[j] : 1);
    }
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&scratch[0], acc);
  if (bad) scratch[1] = 1;
  if (local) {
    __syncthreads();
    for (int32_t i = threadIdx.x; i < K; i += blockDim.x)
      if (spw[i]) atomicAdd(&scratch[kNoAllocHeader + i], spw[i]);
  }
}

// Outputs with the reference's i32 wrap-around: cut = (i32)sum / 2, pw as i32.
// A flagged bad input makes the cut -1 (the part weights then hold the sums
// of the well-formed entries only and mean nothing).
__global__ void k_noalloc_finish(const unsigned long long* __restrict__ scratch, int32_t K, idx_t* __restrict__ cut,
                                 idx_t* __restrict__ pw) {
  RMB_GRID_STRIDE(i, K) { pw[i] = (idx_t)(uint32_t)scratch[kNoAllocHeader + i]; }
  if (blockIdx.x == 0 && threadIdx.x == 0) *cut = scratch[1] ? -1 : (idx_t)(uint32_t)scratch[0] / 2;
}

}  // namespace
}  // namespace rmb

using namespace rmb;

extern "C" int RMETIS_GPU_EdgeCutWeightsNoAlloc(idx_t n, idx_t ncon, int64_t nnz, const idx_t* d_xadj,
                                                const idx_t* d_adjncy, const idx_t* d_adjwgt, const idx_t* d_vwgt,
                                                const idx_t* d_part, idx_t nparts, idx_t* d_cut, idx_t* d_pw,
                                                void* stream) {
  if (n <= 0 || ncon <= 0 || nparts <= 0 || nnz < 0 || !d_xadj || (nnz > 0 && !d_adjncy) || !d_part || !d_cut ||
      !d_pw)
    return METIS_ERROR_INPUT;
  const int64_t K = (int64_t)nparts * ncon;
  if (K > kNoAllocMaxParts) {
    std::fprintf(stderr,
                 "rmetis_b200: RMETIS_GPU_EdgeCutWeightsNoAlloc: nparts*ncon = %lld exceeds the fixed scratch "
                 "limit of %d\n",
                 (long long)K, kNoAllocMaxParts);
    return METIS_ERROR_INPUT;
  }
  int err = METIS_OK;
  unsigned long long* scratch = noalloc_scratch_for_current_device(&err);
  if (!scratch) return err;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // The array keeps the previous call's sums: clear the header and K sums.
  if (cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * (size_t)(kNoAllocHeader + K), st) != cudaSuccess)
    return METIS_ERROR;
  const int blocks = grid_for(n, 256, 148 * 8);
  k_noalloc_cut_pw<<<blocks, 256, 0, st>>>(d_xadj, d_adjncy, d_adjwgt, d_vwgt, n, nnz, ncon, d_part, nparts, scratch);
  if (cudaGetLastError() != cudaSuccess) return METIS_ERROR;
  k_noalloc_finish<<<grid_for(K, 256, 64), 256, 0, st>>>(scratch, (int32_t)K, d_cut, d_pw);
  if (cudaGetLastError() != cudaSuccess) return METIS_ERROR;
  return METIS_OK;
}
