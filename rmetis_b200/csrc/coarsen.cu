// Coarsening: parallel matching (locally dominant edges) and contraction.
#include <cooperative_groups.h>

#include "kernels.h"
#include "prof.h"
#include "scan.cuh"

namespace rmb {

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// Matching
//
// The reference visits vertices one at a time, light (low degree) first, and
// each takes its heaviest still-free neighbour (shem.rs:13-56; rm.rs:13-43
// takes the first free neighbour in random order). The parallel form keeps
// both ingredients:
//   handshake rounds: every free vertex proposes to its best free neighbour
//     (heaviest edge, ties by a seeded edge hash; RM: the hash alone); a pair
//     that proposed to each other matches; otherwise a vertex that received
//     no proposal ("pure" proposer) competes for its target, and the target
//     takes the competitor that comes first in the reference's visit order
//     (lowest degree, then a seeded vertex hash);
//   finishing rounds: mutual proposals under the edge hash alone, a strict
//     total order, so each round matches at least one pair.
// Choosing partners by heaviest edge alone (locally dominant edges) lets
// large coarse vertices absorb each other level after level, which leaves
// star-like graphs that stop coarsening; the visit-order competition avoids it.
// ---------------------------------------------------------------------------
__device__ inline uint32_t edge_hash(uint64_t seed, int32_t a, int32_t b) {
  int32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return (uint32_t)(mix64(seed ^ (((uint64_t)(uint32_t)lo << 32) | (uint32_t)hi)) >> 32);
}

struct EdgeKey {
  int32_t w;
  uint32_t h;
  int32_t u;
  __device__ bool better(const EdgeKey& o) const {
    if (w != o.w) return w > o.w;
    if (h != o.h) return h > o.h;
    return u > o.u;
  }
};

// The bodies below run over a lane set (common.cuh): every thread of a grid
// kernel, or the threads of the one block of the fused coarse-tail kernel.
// They take no __restrict__ because the fused kernel reads, within one launch,
// arrays that it wrote in an earlier phase.
template <bool HAS_W, int MODE>
__device__ __forceinline__ void propose_body(const idx_t* xadj, const idx_t* adj, const idx_t* adjwgt, int32_t n,
                                             const idx_t* match, idx_t* prop, uint64_t seed, Lanes L) {
  RMB_FOR(v, n, L) {
    if (match[v] >= 0) continue;
    const int32_t s = xadj[v], e = xadj[v + 1];
    if (e - s > kHeavyDegree) continue;
    EdgeKey best{INT32_MIN, 0u, -1};
    bool have = false;
    // Four entries at a time: their adjncy and match gathers are in flight
    // together; they are then taken in row order.
    for (int32_t j0 = s; j0 < e; j0 += 4) {
      int32_t uq[4], mq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) uq[q] = j0 + q < e ? adj[j0 + q] : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q) mq[q] = uq[q] >= 0 ? match[uq[q]] : 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (j0 + q >= e) break;
        const int32_t u = uq[q];
        if (mq[q] >= 0) continue;
        EdgeKey k{MODE == 1 ? (HAS_W ? adjwgt[j0 + q] : 1) : 0, edge_hash(seed, (int32_t)v, u), u};
        if (!have || k.better(best)) { best = k; have = true; }
      }
    }
    prop[v] = have ? best.u : -1;
  }
}

// Rows of degree > kHeavyDegree, one warp each (W runs over warps).
template <bool HAS_W, int MODE>
__device__ __forceinline__ void propose_heavy_body(const idx_t* xadj, const idx_t* adj, const idx_t* adjwgt,
                                                   const idx_t* heavy, int32_t nheavy, const idx_t* match,
                                                   idx_t* prop, uint64_t seed, Lanes W) {
  const int lane = threadIdx.x & 31;
  RMB_FOR(i, nheavy, W) {
    const int32_t v = heavy[i];
    if (match[v] >= 0) continue;  // warp-uniform
    EdgeKey best{INT32_MIN, 0u, -1};
    bool have = false;
    for (int32_t j = xadj[v] + lane; j < xadj[v + 1]; j += 32) {
      const int32_t u = adj[j];
      if (match[u] >= 0) continue;
      EdgeKey k{MODE == 1 ? (HAS_W ? adjwgt[j] : 1) : 0, edge_hash(seed, v, u), u};
      if (!have || k.better(best)) { best = k; have = true; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      EdgeKey other;
      other.w = __shfl_xor_sync(0xffffffffu, best.w, o);
      other.h = __shfl_xor_sync(0xffffffffu, best.h, o);
      other.u = __shfl_xor_sync(0xffffffffu, best.u, o);
      int oh = __shfl_xor_sync(0xffffffffu, (int)have, o);
      if (oh && (!have || other.better(best))) { best = other; have = true; }
    }
    if (lane == 0) prop[v] = have ? best.u : -1;
  }
}

// Marks every vertex that received a proposal this round (stamp = round + 1).
__device__ __forceinline__ void stamp_body(int32_t n, const idx_t* match, const idx_t* prop, int32_t* stamp,
                                           int32_t round, Lanes L) {
  RMB_FOR(v, n, L) {
    if (match[v] < 0) {
      const int32_t t = prop[v];
      if (t >= 0) stamp[t] = round + 1;
    }
  }
}

// Pure proposers compete for their target with their visit-order key.
__device__ __forceinline__ void compete_body(const idx_t* xadj, int32_t n, const idx_t* match, const idx_t* prop,
                                             const int32_t* stamp, int32_t round, unsigned long long* best,
                                             uint64_t vseed, int use_degree, Lanes L) {
  RMB_FOR(v, n, L) {
    if (match[v] >= 0) continue;
    const int32_t t = prop[v];
    if (t < 0 || stamp[v] == round + 1 || prop[t] == (int32_t)v) continue;
    const uint32_t deg = (uint32_t)min(xadj[v + 1] - xadj[v], 0x7FFF);
    const uint32_t h = (uint32_t)(mix64(vseed ^ (uint64_t)v) >> 48);
    const uint32_t pri = use_degree ? (((0x7FFFu - deg) << 16) | h) : h;
    const unsigned long long key = (1ULL << 63) | ((unsigned long long)pri << 32) | (uint32_t)v;
    atomicMax(&best[t], key);
  }
}

// Mutual pairs match; a target that is not in a mutual pair takes its winning
// competitor. Only the target writes the pair, the winner (a pure proposer,
// which nobody proposed to and so has no competitor) writes nothing this
// round. Every thread of each warp must call it (warp sum of the count).
__device__ __forceinline__ void resolve_body(int32_t n, const idx_t* prop, idx_t* match, unsigned long long* best,
                                             int32_t* newly, Lanes L) {
  int32_t cnt = 0;
  RMB_FOR(u, n, L) {
    if (match[u] >= 0) continue;
    const int32_t t = prop[u];
    const unsigned long long b = best[u];
    if (b) best[u] = 0;
    if (t >= 0 && prop[t] == (int32_t)u) {
      match[u] = t;
      ++cnt;
    } else if (b) {
      const int32_t v = (int32_t)(uint32_t)(b & 0xffffffffULL);
      match[u] = v;
      match[v] = (idx_t)u;
      cnt += 2;
    }
  }
  cnt = warp_sum(cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(newly, cnt);
}

// Finishing rounds: mutual proposals only.
__device__ __forceinline__ void accept_body(int32_t n, const idx_t* prop, idx_t* match, int32_t* newly, Lanes L) {
  int32_t cnt = 0;
  RMB_FOR(v, n, L) {
    if (match[v] < 0) {
      const int32_t u = prop[v];
      if (u >= 0 && prop[u] == (int32_t)v) {
        match[v] = u;
        ++cnt;
      }
    }
  }
  cnt = warp_sum(cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(newly, cnt);
}

template <bool HAS_W, int MODE>
__global__ void k_match_propose(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                                const idx_t* __restrict__ adjwgt, int32_t n, const idx_t* __restrict__ match,
                                idx_t* __restrict__ prop, uint64_t seed) {
  propose_body<HAS_W, MODE>(xadj, adj, adjwgt, n, match, prop, seed, grid_lanes());
}

template <bool HAS_W, int MODE>
__global__ void k_match_propose_heavy(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                                      const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ heavy,
                                      int32_t nheavy, const idx_t* __restrict__ match, idx_t* __restrict__ prop,
                                      uint64_t seed) {
  propose_heavy_body<HAS_W, MODE>(xadj, adj, adjwgt, heavy, nheavy, match, prop, seed, grid_warps());
}

__global__ void k_match_init(int32_t n, idx_t* match) {
  RMB_GRID_STRIDE(v, n) { match[v] = -1; }
}

__global__ void k_match_stamp(int32_t n, const idx_t* __restrict__ match, const idx_t* __restrict__ prop,
                              int32_t* __restrict__ stamp, int32_t round) {
  stamp_body(n, match, prop, stamp, round, grid_lanes());
}

__global__ void k_match_compete(const idx_t* __restrict__ xadj, int32_t n, const idx_t* __restrict__ match,
                                const idx_t* __restrict__ prop, const int32_t* __restrict__ stamp, int32_t round,
                                unsigned long long* __restrict__ best, uint64_t vseed, int use_degree) {
  compete_body(xadj, n, match, prop, stamp, round, best, vseed, use_degree, grid_lanes());
}

__global__ void k_match_resolve(int32_t n, const idx_t* __restrict__ prop, idx_t* __restrict__ match,
                                unsigned long long* __restrict__ best, int32_t* __restrict__ newly) {
  resolve_body(n, prop, match, best, newly, grid_lanes());
}

__global__ void k_match_accept(int32_t n, const idx_t* __restrict__ prop, idx_t* __restrict__ match,
                               int32_t* __restrict__ newly) {
  accept_body(n, prop, match, newly, grid_lanes());
}

__global__ void k_match_finalize(int32_t n, idx_t* match) {
  RMB_GRID_STRIDE(v, n) {
    if (match[v] < 0) match[v] = (idx_t)v;
  }
}

// 1 (default): match_parallel runs its rounds in one cooperative launch.
int& coop_matching() {
  static int on = 1;
  return on;
}

// Every round of match_parallel in one cooperative launch: the phases of a
// round are separated by grid-wide barriers instead of launches, and the
// progress checks of the host loop below (every other round, the pairs the
// last two rounds matched) are made by every thread from the same counters,
// so the rounds, phases and result are the host loop's. The grid is at most
// the blocks that fit on the device at once (the launch fails otherwise).
struct MatchCoop {
  const idx_t* xadj;
  const idx_t* adj;
  const idx_t* adjwgt;
  const idx_t* heavy;
  int32_t n, nheavy, mode, rounds;
  idx_t* match;
  idx_t* prop;
  int32_t* stamp;
  unsigned long long* best;
  int32_t* newly;  // [rounds + 1], zero on entry
  uint64_t seed, vseed;
};

template <bool HAS_W>
__global__ void __launch_bounds__(256) k_match_coop(MatchCoop a) {
  cg::grid_group grid = cg::this_grid();
  const Lanes L = grid_lanes(), W = grid_warps();
  RMB_FOR(v, a.n, L) a.match[v] = -1;
  grid.sync();
  bool handshake = true;
  int phase_start = 0;
  for (int r = 0; r < a.rounds; ++r) {
    if (handshake && a.mode == 1) {
      propose_body<HAS_W, 1>(a.xadj, a.adj, a.adjwgt, a.n, a.match, a.prop, a.seed, L);
      propose_heavy_body<HAS_W, 1>(a.xadj, a.adj, a.adjwgt, a.heavy, a.nheavy, a.match, a.prop, a.seed, W);
    } else {
      propose_body<false, 0>(a.xadj, a.adj, a.adjwgt, a.n, a.match, a.prop, a.seed, L);
      propose_heavy_body<false, 0>(a.xadj, a.adj, a.adjwgt, a.heavy, a.nheavy, a.match, a.prop, a.seed, W);
    }
    grid.sync();
    if (handshake) {
      stamp_body(a.n, a.match, a.prop, a.stamp, r, L);
      grid.sync();
      compete_body(a.xadj, a.n, a.match, a.prop, a.stamp, r, a.best, a.vseed, a.mode == 1 ? 1 : 0, L);
      grid.sync();
      resolve_body(a.n, a.prop, a.match, a.best, a.newly + r, L);
    } else {
      accept_body(a.n, a.prop, a.match, a.newly + r, L);
    }
    grid.sync();
    if (r - phase_start >= 1 && ((r - phase_start) & 1) == 1) {
      const int64_t last2 = (int64_t)__ldcg(a.newly + r - 1) + __ldcg(a.newly + r);
      if (last2 * 1000 < (int64_t)a.n) {
        if (!handshake) break;  // the same decision in every thread
        handshake = false;
        phase_start = r + 1;
      }
    }
  }
  RMB_FOR(v, a.n, L) {
    if (a.match[v] < 0) a.match[v] = (idx_t)v;
  }
}

// Blocks of k_match_coop<HAS_W> that fit on the current device at once.
template <bool HAS_W>
static int coop_blocks() {
  static int blocks[64] = {0};
  int dev = 0;
  RMB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return 0;
  if (blocks[dev] == 0) {
    int per_sm = 0, sms = 0, coop = 0;
    RMB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    RMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_match_coop<HAS_W>, 256, 0));
    blocks[dev] = coop ? std::max(per_sm * sms, -1) : -1;
  }
  return blocks[dev];
}

void match_parallel(const DGraph& g, int mode, uint64_t seed, int rounds, idx_t* match, const idx_t* heavy,
                    int32_t nheavy, Arena& arena, cudaStream_t st, int32_t* h_scratch, bool coop) {
  Arena::Mark mk = arena.mark();
  idx_t* prop = arena.alloc<idx_t>((size_t)g.n);
  int32_t* stamp = arena.alloc<int32_t>((size_t)g.n);
  unsigned long long* best = arena.alloc<unsigned long long>((size_t)g.n);
  int32_t* newly = arena.alloc<int32_t>((size_t)rounds + 1);
  RMB_CUDA(cudaMemsetAsync(newly, 0, sizeof(int32_t) * ((size_t)rounds + 1), st));
  RMB_CUDA(cudaMemsetAsync(stamp, 0, sizeof(int32_t) * (size_t)g.n, st));
  RMB_CUDA(cudaMemsetAsync(best, 0, sizeof(unsigned long long) * (size_t)g.n, st));
  const int blocks = grid_for(g.n, 256);
  const bool w = g.adjwgt != nullptr;
  const uint64_t vseed = mix64(seed ^ 0x7669736974ULL);
  if (coop && coop_matching()) {
    const int cb = w ? coop_blocks<true>() : coop_blocks<false>();
    if (cb > 0) {
      MatchCoop a;
      a.xadj = g.xadj;
      a.adj = g.adjncy;
      a.adjwgt = g.adjwgt;
      a.heavy = heavy;
      a.n = g.n;
      a.nheavy = nheavy;
      a.mode = mode;
      a.rounds = rounds;
      a.match = match;
      a.prop = prop;
      a.stamp = stamp;
      a.best = best;
      a.newly = newly;
      a.seed = seed;
      a.vseed = vseed;
      void* args[] = {&a};
      const int ph = profiler().begin(kProfPropose, st);
      const cudaError_t e = cudaLaunchCooperativeKernel(w ? (const void*)k_match_coop<true>
                                                          : (const void*)k_match_coop<false>,
                                                        std::min(blocks, cb), 256, args, 0, st);
      profiler().end(ph, st, 12.0 * g.n + (w && mode == 1 ? 12.0 : 8.0) * (double)g.m);
      if (e == cudaSuccess) {
        launch_counter().fetch_add(1);
        arena.reset_to(mk);
        return;
      }
      cudaGetLastError();  // not launched: the launch-per-phase loop below
    }
  }
  k_match_init<<<blocks, 256, 0, st>>>(g.n, match);
  RMB_LAUNCH_CHECK();
  bool handshake = true;  // first phase; the finishing phase follows when it stalls
  int phase_start = 0;
  for (int r = 0; r < rounds; ++r) {
    const bool by_weight = handshake && mode == 1;
    // Round 0 reads every row: xadj, match (own + gathers), adjncy, adjwgt, prop.
    const int ph = r == 0 ? profiler().begin(kProfPropose, st) : -1;
#define RMB_PROP(HW, MD)                                                                                  \
  k_match_propose<HW, MD><<<blocks, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, match, prop, seed);   \
  if (nheavy > 0)                                                                                         \
    k_match_propose_heavy<HW, MD><<<grid_for(nheavy, 8, 148 * 8), 256, 0, st>>>(                         \
        g.xadj, g.adjncy, g.adjwgt, heavy, nheavy, match, prop, seed);
    if (by_weight) {
      if (w) { RMB_PROP(true, 1) } else { RMB_PROP(false, 1) }
    } else {
      RMB_PROP(false, 0)
    }
#undef RMB_PROP
    RMB_LAUNCH_CHECK();
    profiler().end(ph, st, 12.0 * g.n + (w && by_weight ? 12.0 : 8.0) * (double)g.m);
    if (handshake) {
      k_match_stamp<<<blocks, 256, 0, st>>>(g.n, match, prop, stamp, r);
      RMB_LAUNCH_CHECK();
      k_match_compete<<<blocks, 256, 0, st>>>(g.xadj, g.n, match, prop, stamp, r, best, vseed, mode == 1 ? 1 : 0);
      RMB_LAUNCH_CHECK();
      k_match_resolve<<<blocks, 256, 0, st>>>(g.n, prop, match, best, newly + r);
    } else {
      k_match_accept<<<blocks, 256, 0, st>>>(g.n, prop, match, newly + r);
    }
    RMB_LAUNCH_CHECK();
    // Every other round, look at the progress of the last two rounds.
    if (r - phase_start >= 1 && ((r - phase_start) & 1) == 1) {
      RMB_CUDA(cudaMemcpyAsync(h_scratch, newly + r - 1, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      RMB_CUDA(cudaStreamSynchronize(st));
      const int64_t last2 = (int64_t)h_scratch[0] + h_scratch[1];
      if (last2 * 1000 < (int64_t)g.n) {
        if (!handshake) break;
        handshake = false;
        phase_start = r + 1;
      }
    }
  }
  k_match_finalize<<<blocks, 256, 0, st>>>(g.n, match);
  RMB_LAUNCH_CHECK();
  arena.reset_to(mk);
}

// ---------------------------------------------------------------------------
// Contraction (src/graph/mod.rs:284-384)
// ---------------------------------------------------------------------------
struct LoadLeader {
  const idx_t* match;
  __device__ idx_t operator()(int64_t v) const { return match[v] >= (idx_t)v ? 1 : 0; }
};

// cmap numbering identical to the reference's ascending scan (mod.rs:286-297):
// the coarse id of a pair is the number of leaders (min endpoint) before it.
__device__ __forceinline__ void build_cmap_body(const idx_t* xadj, int32_t n, const idx_t* match, const idx_t* cidx,
                                                idx_t* cmap, idx_t* mem0, idx_t* mem1, idx_t* ub, Lanes L) {
  RMB_FOR(v, n, L) {
    const int32_t m = match[v];
    if (m >= (int32_t)v) {
      const int32_t c = cidx[v];
      cmap[v] = c;
      mem0[c] = (idx_t)v;
      const bool pair = m != (int32_t)v;
      mem1[c] = pair ? m : -1;
      ub[c] = (xadj[v + 1] - xadj[v]) + (pair ? (xadj[m + 1] - xadj[m]) : 0);
    } else {
      cmap[v] = cidx[m];
    }
  }
}

__device__ __forceinline__ void coarse_vwgt_body(int32_t cn, int32_t ncon, const idx_t* mem0, const idx_t* mem1,
                                                 const idx_t* vwgt, idx_t* cvwgt, Lanes L) {
  RMB_FOR(i, (int64_t)cn * ncon, L) {
    const int64_t c = i / ncon;
    const int cc = (int)(i - c * ncon);
    const int32_t a = mem0[c], b = mem1[c];
    idx_t w = vwgt ? vwgt[(int64_t)a * ncon + cc] : 1;
    if (b >= 0) w += vwgt ? vwgt[(int64_t)b * ncon + cc] : 1;
    cvwgt[i] = w;
  }
}

// Merge of one coarse row in registers (bound <= T). The
// row of the first member is scanned before the second, each in CSR order,
// and a neighbour is appended at its first appearance (mod.rs:323-341).
// Longer rows are listed in hlist for the warp merge.
template <bool HAS_W, int T>
__device__ __forceinline__ void contract_thread_body(const idx_t* xadj, const idx_t* adj, const idx_t* adjwgt,
                                                     const idx_t* cmap, int32_t cn, const idx_t* mem0,
                                                     const idx_t* mem1, const idx_t* ub, const idx_t* ub_off,
                                                     idx_t* tmp_adj, idx_t* tmp_w, idx_t* cdeg, idx_t* hlist,
                                                     int32_t* hcount, Lanes L) {
  RMB_FOR(c, cn, L) {
    if (ub[c] > T) {
      hlist[atomicAdd(hcount, 1)] = (idx_t)c;
      continue;
    }
    int32_t keys[T];
    int32_t wts[T];
#pragma unroll
    for (int i = 0; i < T; ++i) { keys[i] = -1; wts[i] = 0; }
    int cnt = 0;
#pragma unroll
    for (int mbr = 0; mbr < 2; ++mbr) {
      const int32_t src = mbr == 0 ? mem0[c] : mem1[c];
      if (src < 0) continue;
      const int32_t s = xadj[src], e = xadj[src + 1];
      for (int32_t j0 = s; j0 < e; j0 += 4) {
        int32_t cq[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) cq[q] = j0 + q < e ? adj[j0 + q] : -1;
#pragma unroll
        for (int q = 0; q < 4; ++q) cq[q] = cq[q] >= 0 ? cmap[cq[q]] : -1;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (j0 + q >= e) break;
          const int32_t cu = cq[q];
          if (cu == (int32_t)c) continue;
          const int32_t w = HAS_W ? adjwgt[j0 + q] : 1;
          bool found = false;
#pragma unroll
          for (int i = 0; i < T; ++i) {
            if (i < cnt && keys[i] == cu) { wts[i] += w; found = true; }
          }
          if (!found) {
#pragma unroll
            for (int i = 0; i < T; ++i) {
              if (i == cnt) { keys[i] = cu; wts[i] = w; }
            }
            ++cnt;
          }
        }
      }
    }
    const int32_t off = ub_off[c];
#pragma unroll
    for (int i = 0; i < T; ++i) {
      if (i < cnt) { tmp_adj[off + i] = keys[i]; tmp_w[off + i] = wts[i]; }
    }
    cdeg[c] = cnt;
  }
}

constexpr int kWarpTable = 1024;  // shared hash slots per warp

// Merge of a long coarse row by one warp, 32 entries at a time, with an
// open-addressing table (this warp's shared table when it is given and the
// row fits, else global scratch at twice the row's scratch offset). New keys
// of a chunk get slots in lane order, which keeps first-appearance order; each
// key's weights are summed by the lowest lane holding it. lanew: 32 shared
// ints of this warp. W runs over warps.
template <bool HAS_W>
__device__ __forceinline__ void contract_warp_body(const idx_t* xadj, const idx_t* adj, const idx_t* adjwgt,
                                                   const idx_t* cmap, const idx_t* mem0, const idx_t* mem1,
                                                   const idx_t* ub, const idx_t* ub_off, const idx_t* hlist,
                                                   int32_t nh, idx_t* tmp_adj, idx_t* tmp_w, idx_t* cdeg,
                                                   int32_t* gkey, int32_t* gslot, int32_t* skey, int32_t* sslot,
                                                   int32_t* lanew, Lanes W) {
  const int lane = threadIdx.x & 31;
  RMB_FOR(hi, nh, W) {
    const int32_t c = hlist[hi];
    const int32_t ubc = ub[c];
    const int32_t off = ub_off[c];
    const int32_t tsize = 2 * ubc;
    int32_t *tkey, *tslot;
    if (skey && tsize <= kWarpTable) {
      tkey = skey;
      tslot = sslot;
    } else {
      tkey = gkey + 2 * (int64_t)off;
      tslot = gslot + 2 * (int64_t)off;
    }
    for (int32_t i = lane; i < tsize; i += 32) tkey[i] = -1;
    __syncwarp();
    int32_t U = 0;
    // The two members' rows as one sequence (member 0's row first, each in
    // CSR order): first appearances keep their order whatever the chunking.
    // Four chunks are loaded at once so that their adjncy and cmap gathers
    // overlap instead of forming one dependent chain per chunk.
    const int32_t a0 = mem0[c], a1 = mem1[c];
    const int32_t s0 = xadj[a0], len0 = xadj[a0 + 1] - s0;
    const int32_t s1 = a1 >= 0 ? xadj[a1] : 0, len1 = a1 >= 0 ? xadj[a1 + 1] - s1 : 0;
    const int32_t total = len0 + len1;
    constexpr int kPre = 4;
    for (int32_t base = 0; base < total; base += 32 * kPre) {
      int32_t uu[kPre], ww[kPre];
#pragma unroll
      for (int q = 0; q < kPre; ++q) {
        const int32_t idx = base + q * 32 + lane;
        const int32_t j = idx < len0 ? s0 + idx : s1 + (idx - len0);
        const bool in = idx < total;
        uu[q] = in ? adj[j] : -1;
        ww[q] = in ? (HAS_W ? adjwgt[j] : 1) : 0;
      }
#pragma unroll
      for (int q = 0; q < kPre; ++q) uu[q] = uu[q] >= 0 ? cmap[uu[q]] : -1;
#pragma unroll
      for (int q = 0; q < kPre; ++q) {
        if (base + q * 32 >= total) break;  // warp-uniform
        const int32_t cu = uu[q];
        const int32_t w = ww[q];
        const bool valid = cu >= 0 && cu != c;
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? cu : -(lane + 2));
        const bool leader = valid && (__ffs(peers) - 1) == lane;
        lanew[lane] = valid ? w : 0;
        __syncwarp();
        int32_t gsum = 0;
        if (leader) {
          unsigned m = peers;
          while (m) {
            const int bb = __ffs(m) - 1;
            gsum += lanew[bb];
            m &= m - 1;
          }
        }
        int32_t slot = -1, hpos = -1;
        bool isnew = false;
        if (leader) {
          int32_t h = (int32_t)(((uint32_t)cu * 0x9E3779B1u) % (uint32_t)tsize);
          for (int32_t probe = 0; probe < tsize; ++probe) {
            const int32_t k0 = atomicCAS(&tkey[h], -1, cu);
            if (k0 == -1) { isnew = true; hpos = h; break; }
            if (k0 == cu) { slot = tslot[h]; break; }
            h = (h + 1 == tsize) ? 0 : h + 1;
          }
        }
        const unsigned newmask = __ballot_sync(0xffffffffu, isnew);
        if (isnew) {
          slot = U + __popc(newmask & lanemask_lt());
          tslot[hpos] = slot;
          tmp_adj[off + slot] = cu;
          tmp_w[off + slot] = gsum;
        } else if (leader && slot >= 0) {
          tmp_w[off + slot] += gsum;
        }
        U += __popc(newmask);
        __syncwarp();
      }
    }
    if (lane == 0) cdeg[c] = U;
    __syncwarp();
  }
}

// Gather the merged rows into the final coarse CSR: a warp takes 32 coarse
// vertices and strides over their contiguous scratch range. xs: 33 shared
// ints of this warp. W runs over warps. With VEC, each lane reads four
// scratch entries per 16-byte load (int4, both scratch arrays 16-byte aligned,
// checked here; the grid path allocates them with three entries of slack so
// that the last group of a range stays inside its allocation) and locates
// their rows with one binary search per group.
template <bool VEC>
__device__ __forceinline__ void compact_body(int32_t cn, const idx_t* ub_off, const idx_t* cdeg, const idx_t* cxadj,
                                             const idx_t* tmp_adj, const idx_t* tmp_w, idx_t* cadj, idx_t* cw,
                                             int32_t* xs, Lanes W) {
  const int lane = threadIdx.x & 31;
  const bool vec =
      VEC && ((reinterpret_cast<uintptr_t>(tmp_adj) | reinterpret_cast<uintptr_t>(tmp_w)) & 15) == 0;
  RMB_FOR(w, ceil_div(cn, 32), W) {
    const int32_t v0 = (int32_t)w * 32;
    const int32_t vend = min(v0 + 32, cn);
    const int cnt = vend - v0;
    if (lane < cnt) xs[lane] = ub_off[v0 + lane];
    if (lane == 0) xs[cnt] = ub_off[vend];
    __syncwarp();
    const int32_t e0 = xs[0], e1 = xs[cnt];
    if (vec) {
      for (int32_t q = (e0 & ~3) + 4 * lane; q < e1; q += 128) {
        const int4 a4 = *reinterpret_cast<const int4*>(tmp_adj + q);
        const int4 w4 = *reinterpret_cast<const int4*>(tmp_w + q);
        const int32_t av[4] = {a4.x, a4.y, a4.z, a4.w};
        const int32_t wv[4] = {w4.x, w4.y, w4.z, w4.w};
        const int32_t p0 = max(q, e0);
        int lo = 0, hi = cnt;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (xs[mid] <= p0) lo = mid; else hi = mid;
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int32_t p = q + t;
          if (p < e0 || p >= e1) continue;
          while (lo + 1 < cnt && xs[lo + 1] <= p) ++lo;
          const int32_t c = v0 + lo;
          const int32_t i = p - xs[lo];
          if (i < cdeg[c]) {
            const int32_t dst = cxadj[c] + i;
            cadj[dst] = av[t];
            cw[dst] = wv[t];
          }
        }
      }
    } else {
      for (int32_t p = e0 + lane; p < e1; p += 32) {
        int lo = 0, hi = cnt;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (xs[mid] <= p) lo = mid; else hi = mid;
        }
        const int32_t c = v0 + lo;
        const int32_t i = p - xs[lo];
        if (i < cdeg[c]) {
          const int32_t dst = cxadj[c] + i;
          cadj[dst] = tmp_adj[p];
          cw[dst] = tmp_w[p];
        }
      }
    }
    __syncwarp();
  }
}

__global__ void k_build_cmap(const idx_t* __restrict__ xadj, int32_t n, const idx_t* __restrict__ match,
                             const idx_t* __restrict__ cidx, idx_t* __restrict__ cmap, idx_t* __restrict__ mem0,
                             idx_t* __restrict__ mem1, idx_t* __restrict__ ub) {
  build_cmap_body(xadj, n, match, cidx, cmap, mem0, mem1, ub, grid_lanes());
}

__global__ void k_coarse_vwgt(int32_t cn, int32_t ncon, const idx_t* __restrict__ mem0,
                              const idx_t* __restrict__ mem1, const idx_t* __restrict__ vwgt,
                              idx_t* __restrict__ cvwgt) {
  coarse_vwgt_body(cn, ncon, mem0, mem1, vwgt, cvwgt, grid_lanes());
}

template <bool HAS_W, int T>
__global__ void k_contract_thread(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                                  const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ cmap, int32_t cn,
                                  const idx_t* __restrict__ mem0, const idx_t* __restrict__ mem1,
                                  const idx_t* __restrict__ ub, const idx_t* __restrict__ ub_off,
                                  idx_t* __restrict__ tmp_adj, idx_t* __restrict__ tmp_w, idx_t* __restrict__ cdeg,
                                  idx_t* __restrict__ hlist, int32_t* __restrict__ hcount) {
  contract_thread_body<HAS_W, T>(xadj, adj, adjwgt, cmap, cn, mem0, mem1, ub, ub_off, tmp_adj, tmp_w, cdeg, hlist,
                              hcount, grid_lanes());
}

template <bool HAS_W>
__global__ void k_contract_warp(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                                const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ cmap,
                                const idx_t* __restrict__ mem0, const idx_t* __restrict__ mem1,
                                const idx_t* __restrict__ ub, const idx_t* __restrict__ ub_off,
                                const idx_t* __restrict__ hlist, const int32_t* __restrict__ hcount,
                                idx_t* __restrict__ tmp_adj, idx_t* __restrict__ tmp_w, idx_t* __restrict__ cdeg,
                                int32_t* __restrict__ gkey, int32_t* __restrict__ gslot) {
  __shared__ int32_t skey_all[4][kWarpTable];
  __shared__ int32_t sslot_all[4][kWarpTable];
  __shared__ int32_t lanew_all[4][32];
  const int wib = threadIdx.x >> 5;
  contract_warp_body<HAS_W>(xadj, adj, adjwgt, cmap, mem0, mem1, ub, ub_off, hlist, *hcount, tmp_adj, tmp_w, cdeg,
                            gkey, gslot, skey_all[wib], sslot_all[wib], lanew_all[wib], grid_warps());
}

__global__ void k_contract_compact(int32_t cn, const idx_t* __restrict__ ub_off, const idx_t* __restrict__ cdeg,
                                   const idx_t* __restrict__ cxadj, const idx_t* __restrict__ tmp_adj,
                                   const idx_t* __restrict__ tmp_w, idx_t* __restrict__ cadj,
                                   idx_t* __restrict__ cw) {
  __shared__ int32_t xs_all[8][33];
  compact_body<true>(cn, ub_off, cdeg, cxadj, tmp_adj, tmp_w, cadj, cw, xs_all[threadIdx.x >> 5], grid_warps());
}

struct LoadHeavy {
  const idx_t* xadj;
  __device__ idx_t operator()(int64_t v) const { return (xadj[v + 1] - xadj[v]) > kHeavyDegree ? 1 : 0; }
};
struct StoreHeavy {
  const idx_t* xadj;
  idx_t* out;
  __device__ void operator()(int64_t v, idx_t pos) const {
    if ((xadj[v + 1] - xadj[v]) > kHeavyDegree) out[pos] = (idx_t)v;
  }
};

int32_t heavy_list(const DGraph& g, idx_t* out, Arena& arena, cudaStream_t st, int32_t* h_scratch) {
  Arena::Mark mk = arena.mark();
  idx_t* cnt = arena.alloc<idx_t>(1);
  exclusive_scan<idx_t>(LoadHeavy{g.xadj}, StoreHeavy{g.xadj, out}, g.n, cnt, arena, st);
  RMB_CUDA(cudaMemcpyAsync(h_scratch, cnt, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  arena.reset_to(mk);
  return h_scratch[0];
}

CoarseResult contract(const DGraph& g, const idx_t* match, int coarse_vwgt, Arena& arena, cudaStream_t st,
                      int32_t* h_scratch, int thread_max) {
  CoarseResult r;
  const int32_t n = g.n;
  // The coarse level is allocated first at upper-bound sizes (cn <= n,
  // cm <= m) so that all scratch below the mark is released on return.
  idx_t* cmap = arena.alloc<idx_t>((size_t)n);
  idx_t* counts = arena.alloc<idx_t>(4);  // [0] = cn, [1] = heavy rows
  idx_t* cxadj = arena.alloc<idx_t>((size_t)n + 1);
  idx_t* cadj = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* cw = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* cvwgt = coarse_vwgt ? arena.alloc<idx_t>((size_t)n * g.ncon) : nullptr;
  Arena::Mark mk = arena.mark();
  idx_t* cidx = arena.alloc<idx_t>((size_t)n);
  exclusive_scan<idx_t>(LoadLeader{match}, StoreArr<idx_t>{cidx}, n, counts, arena, st);
  // cn sizes the coarse level; one readback per level.
  RMB_CUDA(cudaMemcpyAsync(h_scratch, counts, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  const int32_t cn = h_scratch[0];
  idx_t* mem0 = arena.alloc<idx_t>((size_t)cn);
  idx_t* mem1 = arena.alloc<idx_t>((size_t)cn);
  idx_t* ub = arena.alloc<idx_t>((size_t)cn);
  idx_t* ub_off = arena.alloc<idx_t>((size_t)cn + 1);
  idx_t* cdeg = arena.alloc<idx_t>((size_t)cn);
  idx_t* hlist = arena.alloc<idx_t>((size_t)cn);
  // Three entries of slack: the compaction reads its ranges in aligned
  // groups of four, whose last one may reach up to three entries past the
  // range's end (at most g.m).
  idx_t* tmp_adj = arena.alloc<idx_t>((size_t)g.m + 4);
  idx_t* tmp_w = arena.alloc<idx_t>((size_t)g.m + 4);
  k_build_cmap<<<grid_for(n, 256), 256, 0, st>>>(g.xadj, n, match, cidx, cmap, mem0, mem1, ub);
  RMB_LAUNCH_CHECK();
  exclusive_scan_arr<idx_t>(ub, ub_off, cn, ub_off + cn, arena, st);
  RMB_CUDA(cudaMemsetAsync(counts + 1, 0, sizeof(idx_t), st));
  // members, bounds, offsets (20 B per coarse vertex), member row offsets,
  // adjncy + cmap gathers (+ adjwgt), merged rows written (8 B per entry).
  const int ph = profiler().begin(kProfContract, st);
#define RMB_CONTRACT_THREAD(HW, TT)                                                                           \
  k_contract_thread<HW, TT><<<grid_for(cn, 128), 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, cmap, cn, mem0, mem1, ub, \
                                                               ub_off, tmp_adj, tmp_w, cdeg, hlist, counts + 1)
  if (thread_max >= kContractThreadMaxGrid) {
    if (g.adjwgt) RMB_CONTRACT_THREAD(true, kContractThreadMaxGrid);
    else RMB_CONTRACT_THREAD(false, kContractThreadMaxGrid);
  } else {
    if (g.adjwgt) RMB_CONTRACT_THREAD(true, kContractThreadMax);
    else RMB_CONTRACT_THREAD(false, kContractThreadMax);
  }
#undef RMB_CONTRACT_THREAD
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 20.0 * cn + 8.0 * n + (g.adjwgt ? 12.0 : 8.0) * (double)g.m + 8.0 * (double)g.m);
  RMB_CUDA(cudaMemcpyAsync(h_scratch + 1, counts + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  const int32_t nheavy = h_scratch[1];
  if (nheavy > 0) {
    int32_t* gkey = arena.alloc<int32_t>(2 * (size_t)g.m + 2);
    int32_t* gslot = arena.alloc<int32_t>(2 * (size_t)g.m + 2);
    const int blocks = grid_for(nheavy, 4, 148 * 8);
    if (g.adjwgt)
      k_contract_warp<true><<<blocks, 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, cmap, mem0, mem1, ub, ub_off, hlist,
                                                     counts + 1, tmp_adj, tmp_w, cdeg, gkey, gslot);
    else
      k_contract_warp<false><<<blocks, 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, cmap, mem0, mem1, ub, ub_off, hlist,
                                                      counts + 1, tmp_adj, tmp_w, cdeg, gkey, gslot);
    RMB_LAUNCH_CHECK();
  }
  exclusive_scan_arr<idx_t>(cdeg, cxadj, cn, cxadj + cn, arena, st);
  k_contract_compact<<<grid_for(ceil_div(cn, 32), 8, 148 * 8), 256, 0, st>>>(cn, ub_off, cdeg, cxadj, tmp_adj,
                                                                            tmp_w, cadj, cw);
  RMB_LAUNCH_CHECK();
  if (coarse_vwgt) {
    k_coarse_vwgt<<<grid_for((int64_t)cn * g.ncon, 256), 256, 0, st>>>(cn, g.ncon, mem0, mem1, g.vwgt, cvwgt);
    RMB_LAUNCH_CHECK();
  }
  RMB_CUDA(cudaMemcpyAsync(h_scratch + 2, cxadj + cn, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  const int32_t cm = h_scratch[2];
  arena.reset_to(mk);
  r.cmap = cmap;
  r.xadj = cxadj;
  r.adjncy = cadj;
  r.adjwgt = cw;
  r.vwgt = cvwgt;
  r.g.n = cn;
  r.g.m = cm;
  r.g.ncon = g.ncon;
  r.g.xadj = cxadj;
  r.g.adjncy = cadj;
  r.g.adjwgt = cw;
  r.g.vwgt = cvwgt;
  return r;
}

// ---------------------------------------------------------------------------
// Coarse tail: every remaining coarsening level of a small graph in one
// single-block launch. The level loop of the host (heavy list, matching
// rounds with their progress checks, contraction, the stop rule of
// coarsen/mod.rs:43-66) runs inside the block with the same bodies as the
// grid kernels above, so it yields exactly the levels the host loop would;
// the host reads the level table back once instead of about six scalars per
// level. Small levels stay in the SM's L1, and the block needs no launch or
// host round trip between phases.
// ---------------------------------------------------------------------------
constexpr int kTailThreads = 1024;


__device__ __forceinline__ long long tail_round(long long b) { return (b + 255) & ~255LL; }

__device__ void tail_body(const TailArgs& a) {
  __shared__ idx_t sw[32];
  __shared__ int32_t lanew_all[kTailThreads / 32][32];
  __shared__ int32_t xs_all[kTailThreads / 32][33];
  const Lanes L = block_lanes(), W = block_warps();
  const int wib = threadIdx.x >> 5;
  TailOut* out = reinterpret_cast<TailOut*>(a.ws);
  if ((a.ws_bytes & 255) != 0) {  // offsets from the top would lose their alignment: leave it to the host loop
    if (threadIdx.x == 0) {
      out->levels = 0;
      out->ncoarse = 0;
      out->finished = 0;
    }
    return;
  }
  // Level data is taken from the bottom of the workspace and kept; the
  // scratch of one level is taken from the top and dropped after it. Every
  // thread computes the same offsets from block-uniform sizes.
  long long lo = tail_round(sizeof(TailOut));
  DGraph cur = a.g;
  int has_vw = a.has_vw;
  int nh_lv = 0, nc = 0, finished = 0;
  for (int lvl = a.lvl0; nh_lv < kTailMaxLevels - 1; ++lvl) {
    const int32_t n = cur.n;
    const bool w = cur.adjwgt != nullptr;
    const long long lvl_lo = lo;
    long long hi = a.ws_bytes;
    auto take_lo = [&](long long b) {
      const long long o = lo;
      lo += tail_round(b);
      return a.ws + o;
    };
    auto take_hi = [&](long long b) {
      hi -= tail_round(b);
      return a.ws + hi;
    };
    idx_t* hl = (idx_t*)take_lo(4LL * n);
    idx_t* match = (idx_t*)take_lo(4LL * n);
    idx_t* prop = (idx_t*)take_hi(4LL * n);
    int32_t* stamp = (int32_t*)take_hi(4LL * n);
    unsigned long long* best = (unsigned long long*)take_hi(8LL * n);
    idx_t* cidx = (idx_t*)take_hi(4LL * n);
    int32_t* newly = (int32_t*)take_hi(4LL * (a.rounds + 1));
    idx_t* cnt = (idx_t*)take_hi(64);  // [0] heavy rows, [1] cn, [2] long coarse rows
    if (lo > hi) {
      lo = lvl_lo;
      break;
    }
    // ---- heavy list and matching (match_parallel) ----
    block_scan_n<idx_t>(LoadHeavy{cur.xadj}, StoreHeavy{cur.xadj, hl}, n, cnt, sw);
    RMB_FOR(v, n, L) {
      match[v] = -1;
      stamp[v] = 0;
      best[v] = 0;
    }
    RMB_FOR(i, a.rounds + 1, L) newly[i] = 0;
    if (threadIdx.x == 0) cnt[2] = 0;
    __syncthreads();
    const int32_t nheavy = cnt[0];
    const uint64_t lseed = mix64(a.seed64 * 0x100000001b3ULL + (uint64_t)lvl + 1);
    const uint64_t vseed = mix64(lseed ^ 0x7669736974ULL);
    bool handshake = true;
    int phase_start = 0;
    for (int r = 0; r < a.rounds; ++r) {
      if (handshake && a.mode == 1) {
        if (w) {
          propose_body<true, 1>(cur.xadj, cur.adjncy, cur.adjwgt, n, match, prop, lseed, L);
          propose_heavy_body<true, 1>(cur.xadj, cur.adjncy, cur.adjwgt, hl, nheavy, match, prop, lseed, W);
        } else {
          propose_body<false, 1>(cur.xadj, cur.adjncy, cur.adjwgt, n, match, prop, lseed, L);
          propose_heavy_body<false, 1>(cur.xadj, cur.adjncy, cur.adjwgt, hl, nheavy, match, prop, lseed, W);
        }
      } else {
        propose_body<false, 0>(cur.xadj, cur.adjncy, cur.adjwgt, n, match, prop, lseed, L);
        propose_heavy_body<false, 0>(cur.xadj, cur.adjncy, cur.adjwgt, hl, nheavy, match, prop, lseed, W);
      }
      __syncthreads();
      if (handshake) {
        stamp_body(n, match, prop, stamp, r, L);
        __syncthreads();
        compete_body(cur.xadj, n, match, prop, stamp, r, best, vseed, a.mode == 1 ? 1 : 0, L);
        __syncthreads();
        resolve_body(n, prop, match, best, newly + r, L);
      } else {
        accept_body(n, prop, match, newly + r, L);
      }
      __syncthreads();
      if (r - phase_start >= 1 && ((r - phase_start) & 1) == 1) {
        const int64_t last2 = (int64_t)newly[r - 1] + newly[r];
        if (last2 * 1000 < (int64_t)n) {
          if (!handshake) break;
          handshake = false;
          phase_start = r + 1;
        }
      }
    }
    RMB_FOR(v, n, L) {
      if (match[v] < 0) match[v] = (idx_t)v;
    }
    __syncthreads();
    // ---- contraction (contract) ----
    block_scan_n<idx_t>(LoadLeader{match}, StoreArr<idx_t>{cidx}, n, cnt + 1, sw);
    __syncthreads();
    const int32_t cn = cnt[1];
    const int coarse_vw = (has_vw || a.summed_unit) ? 1 : 0;
    const long long coarse_lo = lo;
    idx_t* cmap = (idx_t*)take_lo(4LL * n);
    idx_t* cxadj = (idx_t*)take_lo(4LL * (cn + 1));
    idx_t* cvwgt = coarse_vw ? (idx_t*)take_lo(4LL * cn * cur.ncon) : nullptr;
    idx_t* mem0 = (idx_t*)take_hi(4LL * cn);
    idx_t* mem1 = (idx_t*)take_hi(4LL * cn);
    idx_t* ub = (idx_t*)take_hi(4LL * cn);
    idx_t* ub_off = (idx_t*)take_hi(4LL * (cn + 1));
    idx_t* cdeg = (idx_t*)take_hi(4LL * cn);
    idx_t* hlist = (idx_t*)take_hi(4LL * cn);
    if (lo > hi) {
      lo = lvl_lo;
      break;
    }
    build_cmap_body(cur.xadj, n, match, cidx, cmap, mem0, mem1, ub, L);
    __syncthreads();
    block_scan_n<idx_t>(LoadArr<idx_t>{ub}, StoreArr<idx_t>{ub_off}, cn, ub_off + cn, sw);
    __syncthreads();
    const int32_t mb = ub_off[cn];
    idx_t* tmp_adj = (idx_t*)take_hi(4LL * mb + 4);
    idx_t* tmp_w = (idx_t*)take_hi(4LL * mb + 4);
    int32_t* gkey = (int32_t*)take_hi(8LL * mb + 8);
    int32_t* gslot = (int32_t*)take_hi(8LL * mb + 8);
    if (lo > hi) {
      lo = lvl_lo;
      break;
    }
    if (w)
      contract_thread_body<true, kContractThreadMax>(cur.xadj, cur.adjncy, cur.adjwgt, cmap, cn, mem0, mem1, ub, ub_off, tmp_adj, tmp_w,
                                 cdeg, hlist, cnt + 2, L);
    else
      contract_thread_body<false, kContractThreadMax>(cur.xadj, cur.adjncy, cur.adjwgt, cmap, cn, mem0, mem1, ub, ub_off, tmp_adj,
                                  tmp_w, cdeg, hlist, cnt + 2, L);
    __syncthreads();
    const int32_t nlong = cnt[2];
    if (w)
      contract_warp_body<true>(cur.xadj, cur.adjncy, cur.adjwgt, cmap, mem0, mem1, ub, ub_off, hlist, nlong, tmp_adj,
                               tmp_w, cdeg, gkey, gslot, nullptr, nullptr, lanew_all[wib], W);
    else
      contract_warp_body<false>(cur.xadj, cur.adjncy, cur.adjwgt, cmap, mem0, mem1, ub, ub_off, hlist, nlong, tmp_adj,
                                tmp_w, cdeg, gkey, gslot, nullptr, nullptr, lanew_all[wib], W);
    __syncthreads();
    block_scan_n<idx_t>(LoadArr<idx_t>{cdeg}, StoreArr<idx_t>{cxadj}, cn, cxadj + cn, sw);
    __syncthreads();
    const int32_t cm = cxadj[cn];
    idx_t* cadj = (idx_t*)take_lo(4LL * cm);
    idx_t* cw = (idx_t*)take_lo(4LL * cm);
    if (lo > hi) {
      lo = lvl_lo;
      break;
    }
    compact_body<false>(cn, ub_off, cdeg, cxadj, tmp_adj, tmp_w, cadj, cw, xs_all[wib], W);
    if (coarse_vw) coarse_vwgt_body(cn, cur.ncon, mem0, mem1, cur.vwgt, cvwgt, L);
    __syncthreads();
    // ---- the level is complete: record it and apply the stop rule ----
    if (threadIdx.x == 0) {
      out->heavy[nh_lv] = (long long)hl;
      out->nheavy[nh_lv] = nheavy;
      out->match[nh_lv] = (long long)match;
    }
    ++nh_lv;
    if (cn < a.k) {  // too few vertices to seed k parts: keep the finer level
      lo = coarse_lo;
      finished = 1;
      break;
    }
    if (threadIdx.x == 0) {
      out->cmap[nc] = (long long)cmap;
      out->xadj[nc] = (long long)cxadj;
      out->adj[nc] = (long long)cadj;
      out->adjw[nc] = (long long)cw;
      out->vwgt[nc] = (long long)cvwgt;
      out->cn[nc] = cn;
      out->cm[nc] = cm;
      out->coarse_vw[nc] = coarse_vw;
    }
    ++nc;
    const float ratio = (float)cn / (float)n;
    cur.n = cn;
    cur.m = cm;
    cur.xadj = cxadj;
    cur.adjncy = cadj;
    cur.adjwgt = cw;
    cur.vwgt = cvwgt;
    has_vw = coarse_vw;
    if ((long long)cn <= a.limit || ratio > 0.95f) {
      finished = 1;
      // heavy list of the coarsest level (its refinement reads it)
      idx_t* hl2 = (idx_t*)take_lo(4LL * cn);
      idx_t* c2 = (idx_t*)(a.ws + a.ws_bytes - 256);
      if (lo <= a.ws_bytes - 256) {
        block_scan_n<idx_t>(LoadHeavy{cur.xadj}, StoreHeavy{cur.xadj, hl2}, cn, c2, sw);
        __syncthreads();
        if (threadIdx.x == 0) {
          out->heavy[nh_lv] = (long long)hl2;
          out->nheavy[nh_lv] = c2[0];
          out->match[nh_lv] = 0;
        }
        ++nh_lv;
      }
      break;
    }
    __syncthreads();  // the next level reuses this level's scratch
  }
  if (threadIdx.x == 0) {
    out->levels = nh_lv;
    out->ncoarse = nc;
    out->finished = finished;
  }
}

__global__ void __launch_bounds__(kTailThreads, 1) k_coarsen_tail(TailArgs a) { tail_body(a); }

// The coarsening of a batch of graphs: block b coarsens graph order[b]
// (largest first, so the longest jobs start first); a graph flagged in bad
// (failed validation) gets an empty level table.
__global__ void __launch_bounds__(kTailThreads, 1) k_batch_coarsen(const TailArgs* __restrict__ args,
                                                                   const int32_t* __restrict__ order,
                                                                   const int32_t* __restrict__ bad) {
  const int32_t gi = order[blockIdx.x];
  const TailArgs a = args[gi];
  if (bad[gi]) {
    if (threadIdx.x == 0) {
      TailOut* out = reinterpret_cast<TailOut*>(a.ws);
      out->levels = 0;
      out->ncoarse = 0;
      out->finished = 0;
    }
    return;
  }
  tail_body(a);
}

void coarsen_tail_batch(const TailArgs* d_args, const int32_t* d_order, const int32_t* d_bad, int ngraphs,
                        cudaStream_t st) {
  if (ngraphs <= 0) return;
  const int ph = profiler().begin(kProfTail, st);
  k_batch_coarsen<<<ngraphs, kTailThreads, 0, st>>>(d_args, d_order, d_bad);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 0.0);
}

int64_t tail_workspace_bytes(const DGraph& g, int rounds) {
  const int64_t n = g.n, m = g.m, ncon = g.ncon;
  // kept data of all levels (geometric shrinking, with margin) + one
  // level's scratch + allocation rounding
  const int64_t b = (int64_t)sizeof(TailOut) + 3 * (20 * n + 4 * n * ncon + 8 * m) + (44 * n + 24 * m) +
                    4 * (rounds + 1) + (int64_t)kTailMaxLevels * 16 * 256 + 4096;
  return (b + 255) & ~(int64_t)255;  // scratch is taken from the top: keep every offset 256-aligned
}

void coarsen_tail(const DGraph& g, int has_vw, int summed_unit, int mode, uint64_t seed64, int lvl0, int k,
                  int64_t limit, int rounds, Arena& arena, cudaStream_t st, TailOut* h_out) {
  const int64_t bytes = tail_workspace_bytes(g, rounds);
  char* ws = arena.alloc<char>((size_t)bytes);
  TailArgs a;
  a.g = g;
  a.has_vw = has_vw;
  a.summed_unit = summed_unit;
  a.mode = mode;
  a.lvl0 = lvl0;
  a.k = k;
  a.rounds = rounds;
  a.seed64 = seed64;
  a.limit = (long long)limit;
  a.ws = ws;
  a.ws_bytes = (long long)bytes;
  const int ph = profiler().begin(kProfTail, st);
  k_coarsen_tail<<<1, kTailThreads, 0, st>>>(a);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 0.0);
  RMB_CUDA(cudaMemcpyAsync(h_out, ws, sizeof(TailOut), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  if (ph >= 0) {
    // algorithmic bytes as the grid kernels count them: matching round 0 and
    // the contraction of every matched level
    double bytes = 0.0;
    int64_t n = g.n, m = g.m;
    bool w = g.adjwgt != nullptr;
    for (int j = 0; j < h_out->levels && h_out->match[j]; ++j) {
      const int64_t cn = j < h_out->ncoarse ? h_out->cn[j] : n;
      bytes += 12.0 * n + (w && mode == 1 ? 12.0 : 8.0) * m + 20.0 * cn + 8.0 * n + (w ? 20.0 : 16.0) * m;
      if (j < h_out->ncoarse) {
        n = h_out->cn[j];
        m = h_out->cm[j];
        w = true;
      }
    }
    profiler().set_bytes(ph, bytes);
  }
}

}  // namespace rmb
