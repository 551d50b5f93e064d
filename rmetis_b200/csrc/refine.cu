// Greedy boundary refinement, bit-identical to the sequential reference pass.
//
// Reference (src/refine/greedy.rs:36-193, one rank): every pass takes the
// boundary vertices in ascending id, and for each picks the feasible target
// part with the best gain (ties: lowest part id), where gains use the part
// vector of the start of the pass but the part weights `pw` are updated
// after every accepted move; the moves are applied together at the end.
//
// Gains and candidate orders depend only on the start-of-pass part vector, so
// they are computed for all vertices at once (k_gain). The only sequential
// dependency is `pw`. Movers (vertices that may move) are split into blocks of
// kDecideBlock in ascending id. Given the exact part weights at the start of a
// block, a block finds its exact decisions by iterating "decide every mover
// against the weights implied by the decisions of the movers before it" to a
// fixed point (mover t is final after t iterations). Blocks run in parallel
// against the prefix implied by the previous round's decisions of the blocks
// before them (a per-block delta table and its column scan), and rounds
// repeat until no decision changes, at which point every block saw the exact
// prefix. Block b is exact after b+1 rounds at the latest, so the loop always
// ends, and the result equals the sequential pass.
#include <climits>

#include "kernels.h"
#include "prof.h"
#include "scan.cuh"

namespace rmb {

constexpr int kMaxCon = 8;  // constraints supported by the refinement kernels
enum { kRepair = 0, kCut = 1, kTable = 2 };

__device__ inline bool cand_better(int32_t ga, int32_t pa, int32_t gb, int32_t pb) {
  return ga > gb || (ga == gb && pa < pb);
}

// ---------------------------------------------------------------------------
// Gain table: per vertex w_from, boundary flag, explicit candidates E = parts
// p != part[v] with nonzero connection weight w_to[p], stored at
// cand[xadj[v]..] sorted by (gain desc, part asc), gain = w_to - w_from (i32,
// wrapping like the reference's compute_move_gain). Parts outside E (not
// adjacent) all have gain -w_from.
//   kRepair: mover = boundary and source part overweight at pass start
//   kCut:    mover = boundary and some candidate gain > 0
//   kTable:  mover = boundary (used by the gain-table entry point)
// ---------------------------------------------------------------------------
template <bool HAS_W, int MODE>
__global__ void k_gain(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                       const idx_t* __restrict__ adjwgt, int32_t n, int32_t ncon, const idx_t* __restrict__ part,
                       int32_t k, const long long* __restrict__ pw0, const long long* __restrict__ over_thr,
                       idx_t* __restrict__ mover, idx_t* __restrict__ ncand, idx_t* __restrict__ wfrom,
                       idx_t* __restrict__ cand_p, idx_t* __restrict__ cand_g) {
  RMB_GRID_STRIDE(v, n) {
    const int32_t s = xadj[v], e = xadj[v + 1];
    if (e - s > kHeavyDegree) continue;  // warp path
    const int32_t pv = part[v];
    if (MODE == kRepair) {
      bool over = false;
      for (int c = 0; c < ncon; ++c)
        if (pw0[(int64_t)pv * ncon + c] > over_thr[(int64_t)pv * ncon + c]) over = true;
      if (!over) { mover[v] = 0; continue; }
    }
    uint32_t wf = 0;
    int cnt = 0;
    bool boundary = false;
    for (int32_t j = s; j < e; ++j) {
      const int32_t pu = part[adj[j]];
      const uint32_t w = (uint32_t)(HAS_W ? adjwgt[j] : 1);
      if (pu == pv) {
        wf += w;
      } else {
        boundary = true;
        int i = 0;
        for (; i < cnt; ++i)
          if (cand_p[s + i] == pu) break;
        if (i < cnt) {
          cand_g[s + i] = (int32_t)((uint32_t)cand_g[s + i] + w);
        } else {
          cand_p[s + cnt] = pu;
          cand_g[s + cnt] = (int32_t)w;
          ++cnt;
        }
      }
    }
    if (!boundary) { mover[v] = 0; continue; }
    int ne = 0;
    for (int i = 0; i < cnt; ++i) {
      const int32_t wt = cand_g[s + i];
      if (wt != 0) {
        cand_p[s + ne] = cand_p[s + i];
        cand_g[s + ne] = (int32_t)((uint32_t)wt - wf);
        ++ne;
      }
    }
    for (int i = 1; i < ne; ++i) {  // insertion sort, (gain desc, part asc)
      const int32_t g = cand_g[s + i], p = cand_p[s + i];
      int j = i - 1;
      while (j >= 0 && cand_better(g, p, cand_g[s + j], cand_p[s + j])) {
        cand_g[s + j + 1] = cand_g[s + j];
        cand_p[s + j + 1] = cand_p[s + j];
        --j;
      }
      cand_g[s + j + 1] = g;
      cand_p[s + j + 1] = p;
    }
    ncand[v] = ne;
    wfrom[v] = (int32_t)wf;
    int32_t is_mover = 1;
    if (MODE == kCut) {
      const int32_t ig = (int32_t)(0u - wf);
      is_mover = (ne > 0 && cand_g[s] > 0) || (ig > 0 && (k - 1 - ne) > 0);
    }
    mover[v] = is_mover;
  }
}

constexpr int kGainHist = 2048;  // dense per-warp part histogram in shared memory

// Warp-per-vertex gain table for vertices of degree > kHeavyDegree. The part
// histogram is dense over k (shared memory when k <= kGainHist, else the
// global scratch `ghist` of k entries per warp). Each explicit candidate is
// written straight to its sorted position, its rank being the number of
// better candidates.
template <bool HAS_W, int MODE>
__global__ void k_gain_heavy(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                             const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ heavy, int32_t nheavy,
                             int32_t ncon, const idx_t* __restrict__ part, int32_t k,
                             const long long* __restrict__ pw0, const long long* __restrict__ over_thr,
                             idx_t* __restrict__ mover, idx_t* __restrict__ ncand, idx_t* __restrict__ wfrom,
                             idx_t* __restrict__ cand_p, idx_t* __restrict__ cand_g, int32_t* __restrict__ ghist) {
  __shared__ int32_t sh_all[4][kGainHist];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int32_t gw = blockIdx.x * (blockDim.x >> 5) + wib;
  const int32_t nw = gridDim.x * (blockDim.x >> 5);
  int32_t* hist = (k <= kGainHist) ? sh_all[wib] : ghist + (int64_t)gw * k;
  for (int32_t hi = gw; hi < nheavy; hi += nw) {
    const int32_t v = heavy[hi];
    const int32_t s = xadj[v], e = xadj[v + 1];
    const int32_t pv = part[v];
    if (MODE == kRepair) {
      bool over = false;
      for (int c = 0; c < ncon; ++c)
        if (pw0[(int64_t)pv * ncon + c] > over_thr[(int64_t)pv * ncon + c]) over = true;
      if (!over) {
        if (lane == 0) mover[v] = 0;
        continue;
      }
    }
    for (int32_t p = lane; p < k; p += 32) hist[p] = 0;
    __syncwarp();
    uint32_t wf = 0;
    int bnd = 0;
    for (int32_t j = s + lane; j < e; j += 32) {
      const int32_t pu = part[adj[j]];
      const uint32_t w = (uint32_t)(HAS_W ? adjwgt[j] : 1);
      if (pu == pv) wf += w;
      else { bnd = 1; atomicAdd(reinterpret_cast<unsigned*>(&hist[pu]), w); }
    }
    wf = warp_sum(wf);
    const bool boundary = __any_sync(FULL, bnd);
    __syncwarp();
    if (!boundary) {
      if (lane == 0) mover[v] = 0;
      continue;
    }
    int32_t ne_lane = 0;
    for (int32_t p = lane; p < k; p += 32) {
      const int32_t wt = (p != pv) ? hist[p] : 0;
      if (wt == 0) continue;
      ++ne_lane;
      const int32_t g = (int32_t)((uint32_t)wt - wf);
      int32_t r = 0;
      for (int32_t q = 0; q < k; ++q) {
        const int32_t wq = (q != pv) ? hist[q] : 0;
        if (wq == 0) continue;
        if (cand_better((int32_t)((uint32_t)wq - wf), q, g, p)) ++r;
      }
      cand_p[s + r] = p;
      cand_g[s + r] = g;
    }
    const int32_t ne = warp_sum(ne_lane);
    if (lane == 0) {
      ncand[v] = ne;
      wfrom[v] = (int32_t)wf;
      int32_t is_mover = 1;
      if (MODE == kCut) {
        const int32_t ig = (int32_t)(0u - wf);
        is_mover = (ne > 0 && cand_g[s] > 0) || (ig > 0 && (k - 1 - ne) > 0);
      }
      mover[v] = is_mover;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Decision kernel. One block = kDecideBlock consecutive movers.
// ---------------------------------------------------------------------------
struct DecideArgs {
  int32_t nm;
  const idx_t* movers;
  const idx_t* part;
  const idx_t* vwgt;
  int32_t ncon;
  int32_t k;
  const idx_t* xadj;
  const idx_t* ncand;
  const idx_t* wfrom;
  const idx_t* cand_p;
  const idx_t* cand_g;
  const long long* pw0;
  const long long* feas_max;
  const long long* over_thr;
};

struct BlockShared {
  int32_t d[kDecideBlock];
  int32_t pv[kDecideBlock];
  int32_t vw[kDecideBlock * kMaxCon];
};

// Part weights seen by mover t of the block: base (exact weights at the start
// of the block) plus the moves of movers 0..t-1 of the block.
__device__ inline void pw_at(const DecideArgs& a, const BlockShared& sh, const long long* base, int t, int32_t p,
                             long long* out) {
  const int ncon = a.ncon;
  for (int c = 0; c < ncon; ++c) out[c] = base[(int64_t)p * ncon + c];
  for (int t2 = 0; t2 < t; ++t2) {
    const int32_t d2 = sh.d[t2];
    if (d2 < 0) continue;
    if (d2 == p)
      for (int c = 0; c < ncon; ++c) out[c] += sh.vw[t2 * kMaxCon + c];
    if (sh.pv[t2] == p)
      for (int c = 0; c < ncon; ++c) out[c] -= sh.vw[t2 * kMaxCon + c];
  }
}

__device__ inline bool feasible(const DecideArgs& a, const BlockShared& sh, const long long* base, int t,
                                int32_t p) {
  long long w[kMaxCon];
  pw_at(a, sh, base, t, p, w);
  for (int c = 0; c < a.ncon; ++c)
    if (w[c] + sh.vw[t * kMaxCon + c] > a.feas_max[(int64_t)p * a.ncon + c]) return false;
  return true;
}

// The reference's choice for mover t (greedy.rs:64-107 repair, :131-164 cut):
// candidates in (gain desc, part asc) order = explicit ones with gain above
// the non-adjacent gain, then non-adjacent parts by id, then the explicit ones
// below; the first feasible candidate with gain above the pass threshold.
template <int MODE>
__device__ int32_t decide_one(const DecideArgs& a, const BlockShared& sh, const long long* base, int t, int32_t v) {
  const int32_t pv = sh.pv[t];
  if (MODE == kRepair) {
    long long w[kMaxCon];
    pw_at(a, sh, base, t, pv, w);
    bool over = false;
    for (int c = 0; c < a.ncon; ++c)
      if (w[c] > a.over_thr[(int64_t)pv * a.ncon + c]) over = true;
    if (!over) return -1;
  }
  const int32_t thr = (MODE == kRepair) ? INT_MIN : 0;
  const int32_t s = a.xadj[v];
  const int32_t ne = a.ncand[v];
  const int32_t ig = (int32_t)(0u - (uint32_t)a.wfrom[v]);
  int32_t i = 0;
  for (; i < ne; ++i) {
    const int32_t g = a.cand_g[s + i];
    if (g <= ig) break;
    if (g <= thr) return -1;
    const int32_t p = a.cand_p[s + i];
    if (feasible(a, sh, base, t, p)) return p;
  }
  if (ig > thr) {
    for (int32_t p = 0; p < a.k; ++p) {
      if (p == pv) continue;
      bool in_e = false;
      for (int32_t q = 0; q < ne; ++q)
        if (a.cand_p[s + q] == p) { in_e = true; break; }
      if (in_e) continue;
      if (feasible(a, sh, base, t, p)) return p;
    }
  }
  for (; i < ne; ++i) {
    const int32_t g = a.cand_g[s + i];
    if (g <= thr) return -1;
    const int32_t p = a.cand_p[s + i];
    if (feasible(a, sh, base, t, p)) return p;
  }
  return -1;
}

// Exact decisions of one block given `base` (weights before its first mover).
template <int MODE>
__device__ int32_t block_fixpoint(const DecideArgs& a, BlockShared& sh, const long long* base, int32_t j0,
                                  int32_t d_init) {
  const int t = threadIdx.x;
  const int32_t j = j0 + t;
  const bool valid = j < a.nm;
  const int32_t v = valid ? a.movers[j] : -1;
  if (valid) {
    sh.pv[t] = a.part[v];
    for (int c = 0; c < a.ncon; ++c) sh.vw[t * kMaxCon + c] = a.vwgt ? a.vwgt[(int64_t)v * a.ncon + c] : 1;
  } else {
    sh.pv[t] = -1;
  }
  int32_t d = valid ? d_init : -1;
  for (int it = 0; it <= kDecideBlock; ++it) {
    sh.d[t] = d;
    __syncthreads();
    const int32_t nd = valid ? decide_one<MODE>(a, sh, base, t, v) : -1;
    const int changed = __syncthreads_or(nd != d);
    d = nd;
    if (!changed) break;
  }
  sh.d[t] = d;
  __syncthreads();
  return d;
}

// Parallel round: block b decides against pw0 + PD[b] (PD == nullptr: zero
// prefix), writes its decisions, its delta row D[b] and counts a change
// against d_prev.
template <int MODE>
__global__ void __launch_bounds__(kDecideBlock) k_decide(DecideArgs a, const long long* __restrict__ PD,
                                                        const idx_t* __restrict__ d_prev, idx_t* __restrict__ d_out,
                                                        int32_t* __restrict__ D, long long* __restrict__ base_scratch,
                                                        int32_t* __restrict__ changed) {
  __shared__ BlockShared sh;
  const int32_t b = blockIdx.x;
  const int32_t K = a.k * a.ncon;
  long long* base = base_scratch + (int64_t)b * K;
  for (int32_t x = threadIdx.x; x < K; x += blockDim.x) base[x] = a.pw0[x] + (PD ? PD[(int64_t)b * K + x] : 0);
  __syncthreads();
  const int32_t j0 = b * kDecideBlock;
  const int32_t j = j0 + threadIdx.x;
  const int32_t dinit = (d_prev && j < a.nm) ? d_prev[j] : -1;
  const int32_t d = block_fixpoint<MODE>(a, sh, base, j0, dinit);
  int ch = 0;
  if (j < a.nm) {
    d_out[j] = d;
    ch = d_prev ? (d != d_prev[j]) : 1;
  }
  if (__syncthreads_or(ch) && threadIdx.x == 0) atomicAdd(changed, 1);
  int32_t* row = D + (int64_t)b * K;
  for (int32_t x = threadIdx.x; x < K; x += blockDim.x) row[x] = 0;
  __syncthreads();
  if (d >= 0) {
    const int t = threadIdx.x;
    for (int c = 0; c < a.ncon; ++c) {
      atomicAdd(&row[d * a.ncon + c], sh.vw[t * kMaxCon + c]);
      atomicAdd(&row[sh.pv[t] * a.ncon + c], -sh.vw[t * kMaxCon + c]);
    }
  }
}

// Sequential variant: one block walks all mover blocks in order, carrying
// the exact running weights in `run` (K entries, initialised to pw0).
template <int MODE>
__global__ void __launch_bounds__(kDecideBlock) k_decide_seq(DecideArgs a, idx_t* __restrict__ d_out,
                                                            long long* __restrict__ run) {
  __shared__ BlockShared sh;
  const int32_t K = a.k * a.ncon;
  for (int32_t x = threadIdx.x; x < K; x += blockDim.x) run[x] = a.pw0[x];
  __syncthreads();
  for (int32_t j0 = 0; j0 < a.nm; j0 += kDecideBlock) {
    const int32_t d = block_fixpoint<MODE>(a, sh, run, j0, -1);
    const int32_t j = j0 + threadIdx.x;
    if (j < a.nm) d_out[j] = d;
    __syncthreads();  // every thread has finished reading `run`
    if (d >= 0) {
      const int t = threadIdx.x;
      for (int c = 0; c < a.ncon; ++c) {
        atomic_add_i64(&run[(int64_t)d * a.ncon + c], sh.vw[t * kMaxCon + c]);
        atomic_add_i64(&run[(int64_t)sh.pv[t] * a.ncon + c], -(long long)sh.vw[t * kMaxCon + c]);
      }
    }
    __syncthreads();
  }
}

// PD[b][x] = sum over b' < b of D[b'][x].
__global__ void k_prefix_blocks(const int32_t* __restrict__ D, int32_t nb, int32_t K, long long* __restrict__ PD) {
  RMB_GRID_STRIDE(x, K) {
    long long run = 0;
    for (int32_t b = 0; b < nb; ++b) {
      PD[(int64_t)b * K + x] = run;
      run += D[(int64_t)b * K + x];
    }
  }
}

// Apply the pass's moves together (greedy.rs:111-119, :168-181) and keep the
// part weights current.
__global__ void k_apply(int32_t nm, const idx_t* __restrict__ movers, const idx_t* __restrict__ d,
                        idx_t* __restrict__ part, const idx_t* __restrict__ vwgt, int32_t ncon,
                        long long* __restrict__ pw, int32_t* __restrict__ nmoves) {
  int32_t cnt = 0;
  RMB_GRID_STRIDE(j, nm) {
    const int32_t dd = d[j];
    if (dd >= 0) {
      const int32_t v = movers[j];
      const int32_t pv = part[v];
      part[v] = dd;
      for (int c = 0; c < ncon; ++c) {
        const long long w = vwgt ? vwgt[(int64_t)v * ncon + c] : 1;
        atomic_add_i64(&pw[(int64_t)dd * ncon + c], w);
        atomic_add_i64(&pw[(int64_t)pv * ncon + c], -w);
      }
      ++cnt;
    }
  }
  cnt = warp_sum(cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nmoves, cnt);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <int MODE>
static void launch_gain(const DGraph& g, const idx_t* part, int k, const long long* pw0, const long long* over_thr,
                        idx_t* mover, idx_t* ncand, idx_t* wfrom, idx_t* cand_p, idx_t* cand_g, const idx_t* heavy,
                        int32_t nheavy, int32_t* ghist, cudaStream_t st) {
  const int blocks = grid_for(g.n, 256);
  // Algorithmic bytes of a full pass: xadj, part (own + neighbour gathers),
  // adjncy, adjwgt, mover flag.
  const double bytes = 12.0 * g.n + (g.adjwgt ? 12.0 : 8.0) * (double)g.m;
  const int ph = MODE == kCut ? profiler().begin(kProfGain, st) : -1;
  if (g.adjwgt)
    k_gain<true, MODE><<<blocks, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, g.ncon, part, k, pw0, over_thr,
                                                mover, ncand, wfrom, cand_p, cand_g);
  else
    k_gain<false, MODE><<<blocks, 256, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, g.ncon, part, k, pw0, over_thr,
                                                 mover, ncand, wfrom, cand_p, cand_g);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, bytes);
  if (nheavy > 0) {
    const int hb = grid_for(nheavy, 4, 256);
    if (g.adjwgt)
      k_gain_heavy<true, MODE><<<hb, 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, heavy, nheavy, g.ncon, part, k, pw0,
                                                    over_thr, mover, ncand, wfrom, cand_p, cand_g, ghist);
    else
      k_gain_heavy<false, MODE><<<hb, 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, heavy, nheavy, g.ncon, part, k, pw0,
                                                     over_thr, mover, ncand, wfrom, cand_p, cand_g, ghist);
    RMB_LAUNCH_CHECK();
  }
}

void gain_table(const DGraph& g, const idx_t* part, int k, idx_t* boundary, idx_t* ncand, idx_t* wfrom,
                idx_t* cand_p, idx_t* cand_g, const idx_t* heavy, int32_t nheavy, cudaStream_t st) {
  int32_t* ghist = nullptr;
  if (nheavy > 0 && k > kGainHist) {
    RMB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ghist), sizeof(int32_t) * (size_t)k * 256 * 4, st));
  }
  launch_gain<kTable>(g, part, k, nullptr, nullptr, boundary, ncand, wfrom, cand_p, cand_g, heavy, nheavy, ghist, st);
  if (ghist) RMB_CUDA(cudaFreeAsync(ghist, st));
}

RefineStats greedy_refine(const DGraph& g, idx_t* part, const RefineParams& rp, const idx_t* heavy, int32_t nheavy,
                          Arena& arena, cudaStream_t st, int32_t* h_scratch) {
  if (g.ncon > kMaxCon) throw Error(-2, "ncon above the supported maximum of 8");
  RefineStats stats;
  const int k = rp.k;
  const int32_t K = k * g.ncon;
  Arena::Mark mk = arena.mark();
  long long* pw = arena.alloc<long long>((size_t)K);
  idx_t* mover = arena.alloc<idx_t>((size_t)g.n);
  idx_t* ncand = arena.alloc<idx_t>((size_t)g.n);
  idx_t* wfrom = arena.alloc<idx_t>((size_t)g.n);
  idx_t* cand_p = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* cand_g = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* movers = arena.alloc<idx_t>((size_t)g.n);
  idx_t* d_a = arena.alloc<idx_t>((size_t)g.n);
  idx_t* d_b = arena.alloc<idx_t>((size_t)g.n);
  int32_t* counters = arena.alloc<int32_t>(8);  // [0] nm, [1] changed, [2] moves
  int32_t* ghist = (nheavy > 0 && k > kGainHist) ? arena.alloc<int32_t>((size_t)k * 256 * 4) : nullptr;
  partition_weights_only(g, part, k, pw, st);

  DecideArgs a;
  a.movers = movers;
  a.part = part;
  a.vwgt = g.vwgt;
  a.ncon = g.ncon;
  a.k = k;
  a.xadj = g.xadj;
  a.ncand = ncand;
  a.wfrom = wfrom;
  a.cand_p = cand_p;
  a.cand_g = cand_g;
  a.pw0 = pw;
  a.feas_max = rp.feas_max;
  a.over_thr = rp.over_thr;

  for (int pass = 0; pass <= rp.niter; ++pass) {
    const int mode = pass == 0 ? kRepair : kCut;
    if (mode == kRepair)
      launch_gain<kRepair>(g, part, k, pw, rp.over_thr, mover, ncand, wfrom, cand_p, cand_g, heavy, nheavy, ghist, st);
    else
      launch_gain<kCut>(g, part, k, pw, rp.over_thr, mover, ncand, wfrom, cand_p, cand_g, heavy, nheavy, ghist, st);
    compact_flags(mover, g.n, movers, counters, arena, st);
    RMB_CUDA(cudaMemcpyAsync(h_scratch, counters, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    const int32_t nm = h_scratch[0];
    stats.passes += 1;
    stats.movers += nm;
    if (nm == 0) {
      if (mode == kCut) break;
      continue;
    }
    a.nm = nm;
    const int32_t nb = (int32_t)ceil_div(nm, kDecideBlock);
    idx_t* dfinal = nullptr;
    Arena::Mark pm = arena.mark();
    if (nb <= 4 || (int64_t)nb * K > ((int64_t)1 << 24)) {
      long long* run = arena.alloc<long long>((size_t)K);
      const int ph = profiler().begin(kProfDecide, st);
      if (mode == kRepair) k_decide_seq<kRepair><<<1, kDecideBlock, 0, st>>>(a, d_a, run);
      else k_decide_seq<kCut><<<1, kDecideBlock, 0, st>>>(a, d_a, run);
      RMB_LAUNCH_CHECK();
      profiler().end(ph, st, 0.0);
      dfinal = d_a;
      stats.decide_iters += 1;
    } else {
      int32_t* D = arena.alloc<int32_t>((size_t)nb * K);
      long long* PD = arena.alloc<long long>((size_t)nb * K);
      long long* base = arena.alloc<long long>((size_t)nb * K);
      idx_t* prev = nullptr;
      idx_t* cur = d_a;
      const long long* pd_in = nullptr;
      for (int round = 0; round <= nb; ++round) {
        RMB_CUDA(cudaMemsetAsync(counters + 1, 0, sizeof(int32_t), st));
        const int ph = profiler().begin(kProfDecide, st);
        if (mode == kRepair)
          k_decide<kRepair><<<nb, kDecideBlock, 0, st>>>(a, pd_in, prev, cur, D, base, counters + 1);
        else
          k_decide<kCut><<<nb, kDecideBlock, 0, st>>>(a, pd_in, prev, cur, D, base, counters + 1);
        RMB_LAUNCH_CHECK();
        profiler().end(ph, st, 0.0);
        stats.decide_iters += 1;
        k_prefix_blocks<<<grid_for(K, 128), 128, 0, st>>>(D, nb, K, PD);
        RMB_LAUNCH_CHECK();
        pd_in = PD;
        if (round >= 1) {
          RMB_CUDA(cudaMemcpyAsync(h_scratch + 1, counters + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
          RMB_CUDA(cudaStreamSynchronize(st));
          if (h_scratch[1] == 0) {
            dfinal = cur;
            break;
          }
        }
        prev = cur;
        cur = (cur == d_a) ? d_b : d_a;
      }
      if (!dfinal) throw Error(-4, "refinement decisions did not settle");
    }
    RMB_CUDA(cudaMemsetAsync(counters + 2, 0, sizeof(int32_t), st));
    k_apply<<<grid_for(nm, 256), 256, 0, st>>>(nm, movers, dfinal, part, g.vwgt, g.ncon, pw, counters + 2);
    RMB_LAUNCH_CHECK();
    RMB_CUDA(cudaMemcpyAsync(h_scratch + 2, counters + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    arena.reset_to(pm);
    stats.moves += h_scratch[2];
    if (mode == kCut && h_scratch[2] == 0) break;
  }
  arena.reset_to(mk);
  return stats;
}

}  // namespace rmb
