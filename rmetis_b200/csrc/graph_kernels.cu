// Whole-graph kernels: validation, edge cut + partition weights, totals,
// projection, boundary flags, flag compaction.
#include "kernels.h"
#include "prof.h"
#include "scan.cuh"

namespace rmb {

// A warp owns 32 consecutive vertices and strides over their (contiguous)
// edge range in lane order, so CSR reads are coalesced whatever the degree
// mix. The source vertex of edge position p is found by binary search over
// the 33 row offsets held in shared memory.
template <typename F>
__device__ inline void warp_edge_tile(const idx_t* __restrict__ xadj, int32_t n, int32_t v0,
                                      int32_t* xs, F f) {
  const int lane = threadIdx.x & 31;
  const int32_t vend = min(v0 + 32, n);
  const int cnt = vend - v0;
  if (lane < cnt) xs[lane] = xadj[v0 + lane];
  if (lane == 0) xs[cnt] = xadj[vend];
  __syncwarp();
  const int32_t e0 = xs[0], e1 = xs[cnt];
  for (int32_t p = e0 + lane; p < e1; p += 32) {
    int lo = 0, hi = cnt;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (xs[mid] <= p) lo = mid; else hi = mid;
    }
    f(v0 + lo, p);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Validation (src/graph/validate.rs:16-142)
// ---------------------------------------------------------------------------
__global__ void k_val_xadj(const idx_t* __restrict__ xadj, int32_t n, int32_t* flags) {
  RMB_GRID_STRIDE(i, n) {
    if (xadj[i] > xadj[i + 1]) atomicOr(flags, 2);
  }
}

__global__ void k_val_adj(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj, int32_t n,
                          int32_t* degcheck, int32_t* flags) {
  __shared__ int32_t xs_all[8][33];
  int32_t* xs = xs_all[threadIdx.x >> 5];
  const int32_t nwarps_total = gridDim.x * (blockDim.x >> 5);
  for (int32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); (int64_t)w * 32 < n;
       w += nwarps_total) {
    warp_edge_tile(xadj, n, w * 32, xs, [&](int32_t v, int32_t p) {
      idx_t u = adj[p];
      if (u < 0 || u >= n) {
        atomicOr(flags, 4);
      } else if (u == v) {
        atomicOr(flags, 8);
      } else {
        atomicAdd(&degcheck[u], 1);
      }
    });
  }
}

__global__ void k_val_deg(const idx_t* __restrict__ xadj, const int32_t* degcheck, int32_t n,
                          int32_t* flags) {
  RMB_GRID_STRIDE(v, n) {
    if (degcheck[v] != xadj[v + 1] - xadj[v]) atomicOr(flags, 16);
  }
}

__global__ void k_val_vwgt(const idx_t* __restrict__ vwgt, int64_t len, int32_t* flags) {
  RMB_GRID_STRIDE(i, len) {
    if (vwgt[i] <= 0) atomicOr(flags, 32);
  }
}

int validate_device(const DGraph& g, Arena& arena, cudaStream_t st, int32_t* h_scratch) {
  Arena::Mark mk = arena.mark();
  int32_t* flags = arena.alloc<int32_t>(1);
  int32_t* degcheck = arena.alloc<int32_t>((size_t)g.n);
  RMB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int32_t), st));
  RMB_CUDA(cudaMemsetAsync(degcheck, 0, sizeof(int32_t) * (size_t)g.n, st));
  k_val_xadj<<<grid_for(g.n, 256), 256, 0, st>>>(g.xadj, g.n, flags);
  RMB_LAUNCH_CHECK();
  RMB_CUDA(cudaMemcpyAsync(h_scratch, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  int32_t f = h_scratch[0];
  if (f == 0) {  // row ranges are only meaningful once xadj is monotone
    k_val_adj<<<grid_for(ceil_div(g.n, 32), 8), 256, 0, st>>>(g.xadj, g.adjncy, g.n, degcheck, flags);
    RMB_LAUNCH_CHECK();
    k_val_deg<<<grid_for(g.n, 256), 256, 0, st>>>(g.xadj, degcheck, g.n, flags);
    RMB_LAUNCH_CHECK();
    if (g.vwgt) {
      k_val_vwgt<<<grid_for((int64_t)g.n * g.ncon, 256), 256, 0, st>>>(g.vwgt, (int64_t)g.n * g.ncon, flags);
      RMB_LAUNCH_CHECK();
    }
    RMB_CUDA(cudaMemcpyAsync(h_scratch, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    f = h_scratch[0];
  }
  arena.reset_to(mk);
  return f;
}

// ---------------------------------------------------------------------------
// Edge cut + partition weights (src/graph/mod.rs:123-149)
// ---------------------------------------------------------------------------
constexpr int kSmemPw = 4096;  // [k][ncon] entries kept in shared memory

template <bool HAS_W>
__global__ void k_cut(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                      const idx_t* __restrict__ adjwgt, int32_t n, const idx_t* __restrict__ part,
                      unsigned long long* cut_acc) {
  __shared__ int32_t xs_all[8][33];
  int32_t* xs = xs_all[threadIdx.x >> 5];
  unsigned long long acc = 0;
  const int32_t nwarps_total = gridDim.x * (blockDim.x >> 5);
  for (int32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); (int64_t)w * 32 < n;
       w += nwarps_total) {
    warp_edge_tile(xadj, n, w * 32, xs, [&](int32_t v, int32_t p) {
      if (part[v] != part[adj[p]]) acc += (uint32_t)(HAS_W ? adjwgt[p] : 1);
    });
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(cut_acc, acc);
}

// Edge cut (both directions, signed weights) of ntrials partitions of one
// graph at once: blockIdx.y is the trial, parts[trial][n], cuts[trial].
template <bool HAS_W>
__global__ void k_cut_trials(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                             const idx_t* __restrict__ adjwgt, int32_t n, const idx_t* __restrict__ parts,
                             long long* __restrict__ cuts) {
  __shared__ int32_t xs_all[8][33];
  int32_t* xs = xs_all[threadIdx.x >> 5];
  const idx_t* part = parts + (int64_t)blockIdx.y * n;
  unsigned long long acc = 0;
  const int32_t nwarps_total = gridDim.x * (blockDim.x >> 5);
  for (int32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); (int64_t)w * 32 < n;
       w += nwarps_total) {
    warp_edge_tile(xadj, n, w * 32, xs, [&](int32_t v, int32_t p) {
      if (part[v] != part[adj[p]]) acc += (unsigned long long)(long long)(HAS_W ? adjwgt[p] : 1);
    });
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(reinterpret_cast<unsigned long long*>(&cuts[blockIdx.y]), acc);
}

void trial_cuts(const DGraph& g, const idx_t* parts, int ntrials, long long* cuts, cudaStream_t st) {
  RMB_CUDA(cudaMemsetAsync(cuts, 0, sizeof(long long) * (size_t)ntrials, st));
  const dim3 grid((unsigned)grid_for(ceil_div(g.n, 32), 8, 148 * 8), (unsigned)ntrials);
  if (g.adjwgt) k_cut_trials<true><<<grid, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, parts, cuts);
  else k_cut_trials<false><<<grid, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, parts, cuts);
  RMB_LAUNCH_CHECK();
}

template <bool HAS_VW>
__global__ void k_pw(const idx_t* __restrict__ vwgt, int32_t n, int32_t ncon, const idx_t* __restrict__ part,
                     int32_t K, long long* pw) {
  __shared__ long long sh[kSmemPw];
  const bool use_sh = K <= kSmemPw;
  if (use_sh)
    for (int i = threadIdx.x; i < K; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  RMB_GRID_STRIDE(v, n) {
    int32_t p = part[v];
    for (int c = 0; c < ncon; ++c) {
      long long w = HAS_VW ? vwgt[(int64_t)v * ncon + c] : 1;
      if (use_sh) atomic_add_i64(&sh[p * ncon + c], w);
      else atomic_add_i64(&pw[p * ncon + c], w);
    }
  }
  __syncthreads();
  if (use_sh)
    for (int i = threadIdx.x; i < K; i += blockDim.x)
      if (sh[i]) atomic_add_i64(&pw[i], sh[i]);
}

void partition_weights_only(const DGraph& g, const idx_t* part, int k, long long* pw, cudaStream_t st) {
  int32_t K = k * g.ncon;
  RMB_CUDA(cudaMemsetAsync(pw, 0, sizeof(long long) * (size_t)K, st));
  int blocks = grid_for(g.n, 256, 148 * 4);
  if (g.vwgt) k_pw<true><<<blocks, 256, 0, st>>>(g.vwgt, g.n, g.ncon, part, K, pw);
  else k_pw<false><<<blocks, 256, 0, st>>>(g.vwgt, g.n, g.ncon, part, K, pw);
  RMB_LAUNCH_CHECK();
}

void cut_and_weights(const DGraph& g, const idx_t* part, int k, unsigned long long* cut_acc, long long* pw,
                     cudaStream_t st) {
  if (cut_acc) {
    RMB_CUDA(cudaMemsetAsync(cut_acc, 0, sizeof(unsigned long long), st));
    int blocks = grid_for(ceil_div(g.n, 32), 8, 148 * 8);
    const int ph = profiler().begin(kProfCut, st);
    if (g.adjwgt) k_cut<true><<<blocks, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, part, cut_acc);
    else k_cut<false><<<blocks, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, part, cut_acc);
    RMB_LAUNCH_CHECK();
    profiler().end(ph, st, 8.0 * g.n + (g.adjwgt ? 12.0 : 8.0) * (double)g.m);
  }
  if (pw) partition_weights_only(g, part, k, pw, st);
}

__global__ void k_total(const idx_t* __restrict__ vwgt, int32_t n, int32_t ncon, long long* tot) {
  long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int c0 = 0; c0 < ncon; c0 += 8) {
    for (int c = 0; c < 8; ++c) acc[c] = 0;
    RMB_GRID_STRIDE(v, n) {
      for (int c = c0; c < min(ncon, c0 + 8); ++c) acc[c - c0] += vwgt ? vwgt[(int64_t)v * ncon + c] : 1;
    }
    for (int c = c0; c < min(ncon, c0 + 8); ++c) {
      long long s = warp_sum(acc[c - c0]);
      if ((threadIdx.x & 31) == 0) atomic_add_i64(&tot[c], s);
    }
  }
}

void total_weight(const DGraph& g, long long* tot, cudaStream_t st) {
  RMB_CUDA(cudaMemsetAsync(tot, 0, sizeof(long long) * (size_t)g.ncon, st));
  k_total<<<grid_for(g.n, 256, 148 * 4), 256, 0, st>>>(g.vwgt, g.n, g.ncon, tot);
  RMB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Projection (src/partition/kway.rs:81-84)
// ---------------------------------------------------------------------------
__global__ void k_project(int32_t n, const idx_t* __restrict__ cmap, const idx_t* __restrict__ cpart,
                          idx_t* __restrict__ fpart) {
  RMB_GRID_STRIDE(v, n) { fpart[v] = cpart[cmap[v]]; }
}

void project(int32_t n_fine, const idx_t* cmap, const idx_t* coarse_part, idx_t* fine_part, cudaStream_t st) {
  k_project<<<grid_for(n_fine, 256), 256, 0, st>>>(n_fine, cmap, coarse_part, fine_part);
  RMB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Boundary flags (src/graph/mod.rs:164-171)
// ---------------------------------------------------------------------------
__global__ void k_boundary(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj, int32_t n,
                           const idx_t* __restrict__ part, idx_t* flag) {
  __shared__ int32_t xs_all[8][33];
  int32_t* xs = xs_all[threadIdx.x >> 5];
  const int32_t nwarps_total = gridDim.x * (blockDim.x >> 5);
  for (int32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); (int64_t)w * 32 < n;
       w += nwarps_total) {
    warp_edge_tile(xadj, n, w * 32, xs, [&](int32_t v, int32_t p) {
      if (part[v] != part[adj[p]]) flag[v] = 1;
    });
  }
}

void boundary_flags(const DGraph& g, const idx_t* part, idx_t* flag, cudaStream_t st) {
  RMB_CUDA(cudaMemsetAsync(flag, 0, sizeof(idx_t) * (size_t)g.n, st));
  k_boundary<<<grid_for(ceil_div(g.n, 32), 8, 148 * 8), 256, 0, st>>>(g.xadj, g.adjncy, g.n, part, flag);
  RMB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Flag compaction
// ---------------------------------------------------------------------------

void compact_flags(const idx_t* flag, int32_t n, idx_t* out, idx_t* count_dev, Arena& arena, cudaStream_t st) {
  exclusive_scan<idx_t>(LoadNonZero{flag}, StoreCompact{flag, out}, n, count_dev, arena, st);
}

}  // namespace rmb
