// 2-way FM refinement of a bisection (src/refine/fm.rs:12-127) in parallel
// rounds with a rollback to the best round.
//
// Reference: a pass computes every vertex's gain (weight to the other side
// minus weight to its own), queues the boundary vertices by gain, and pops
// them one at a time: a popped vertex moves when the other side stays
// feasible ((pw + vw) as f64 <= t * ub), is locked for the pass, and its
// unlocked neighbours get new gains (and enter the queue when they reach the
// boundary). Moves with negative gains are made too; after the queue runs
// empty, the moves after the point of the lowest cut are undone. Passes
// repeat while a pass improves the cut (at most niter).
//
// Here a pass runs in rounds that follow the queue's order by gain level:
// a round takes the largest gain among the free boundary vertices and
// selects every free boundary vertex with that gain whose (gain, lower id)
// beats that of each such neighbour, on either side: no two selected vertices
// are adjacent, so the cut changes by exactly minus the sum of the moved
// vertices' gains. Positive moves thus come first, then the least harmful
// negative ones, as the queue pops them. The selected moves go
// through the parallel admission (admit.cu, one candidate each, whatever its
// gain): each side admits the longest prefix of its incoming moves, in vertex
// order, that fits its limit given the moves out of it. Admitted vertices
// move and are locked; the others are dropped until a neighbour moves. Gains
// are recomputed for the vertices next to the round's changes only. The pass
// ends at a round that selects nothing, kFm2Patience rounds after its lowest
// cut, or after kFm2MaxRounds; the host then finds the round with the lowest
// cut (the earliest on ties, as the reference's strict <) and the vertices
// moved after it go back.
#include <climits>
#include <vector>

#include "kernels.h"
#include "prof.h"

namespace rmb {

namespace {

constexpr int kFree = 0, kLocked = 1, kDropped = 2;
constexpr int kFm2MaxRounds = 4096;  // bound on the rounds of one pass
constexpr int kFm2RoundsPerCheck = 8;
// A pass also ends once this many rounds have passed since its lowest cut:
// the moves after that point are undone anyway, and the queue's tail of ever
// more negative moves rarely leads back below it.
constexpr int kFm2Patience = 32;

// Gain, boundary and the single candidate (the other side) of every vertex in
// `only` (all when null; the flags are cleared as they are read). ncand = 1
// for a free boundary vertex.
template <bool HAS_W>
__global__ void k_fm2_gain(int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                           const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ part,
                           const int32_t* __restrict__ state, idx_t* __restrict__ only,
                           idx_t* __restrict__ ncand, idx_t* __restrict__ cand_p, idx_t* __restrict__ cand_g) {
  RMB_GRID_STRIDE(v, n) {
    if (only) {
      if (!only[v]) continue;
      only[v] = 0;
    }
    const int32_t s = xadj[v], e = xadj[v + 1];
    const int32_t pv = part[v];
    uint32_t wf = 0, wt = 0;
    bool bnd = false;
    for (int32_t j0 = s; j0 < e; j0 += 4) {
      int32_t pq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) pq[q] = j0 + q < e ? adj[j0 + q] : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q) pq[q] = pq[q] >= 0 ? part[pq[q]] : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (j0 + q >= e) break;
        const uint32_t w = (uint32_t)(HAS_W ? adjwgt[j0 + q] : 1);
        if (pq[q] == pv) wf += w;
        else {
          wt += w;
          bnd = true;
        }
      }
    }
    const bool cand = bnd && state[v] == kFree;
    ncand[v] = cand ? 1 : 0;
    if (cand) {  // a boundary vertex has an edge, so slot s is its own
      cand_p[s] = 1 - pv;
      cand_g[s] = (int32_t)(wt - wf);
    }
  }
}

// Largest gain among the free boundary vertices (INT_MIN when none).
__global__ void k_fm2_max(int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ ncand,
                          const idx_t* __restrict__ cand_g, int32_t* __restrict__ gmax) {
  int32_t m = INT_MIN;
  RMB_GRID_STRIDE(v, n) {
    if (ncand[v]) m = max(m, (int32_t)cand_g[xadj[v]]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m != INT_MIN) atomicMax(gmax, m);
}

// sel[v] = 1 for a free boundary vertex of gain *gmax whose (gain, lower id)
// beats that of every such neighbour.
__global__ void k_fm2_select(int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                             const idx_t* __restrict__ ncand, const idx_t* __restrict__ cand_g,
                             const int32_t* __restrict__ gmax_p, idx_t* __restrict__ sel) {
  const int32_t gmax = *gmax_p;
  RMB_GRID_STRIDE(v, n) {
    int32_t out = 0;
    if (ncand[v] && cand_g[xadj[v]] >= gmax) {
      const int32_t s = xadj[v], e = xadj[v + 1];
      const int32_t gv = cand_g[s];
      out = 1;
      for (int32_t j = s; j < e; ++j) {
        const int32_t u = adj[j];
        if (!ncand[u]) continue;
        const int32_t gu = cand_g[xadj[u]];
        if (gu < gmax) continue;
        if (gu > gv || (gu == gv && u < (int32_t)v)) {
          out = 0;
          break;
        }
      }
    }
    sel[v] = out;
  }
}

// Admitted movers move, are locked and record their round; their gains sum
// into the round's cut change (no two movers are adjacent). The others are
// dropped. changed (zero on entry): movers and the neighbours of moved ones,
// the vertices whose gain or state the round changed.
__global__ void k_fm2_apply(const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                            const int32_t* __restrict__ tgt, const int32_t* __restrict__ rank,
                            const int32_t* __restrict__ cut, const idx_t* __restrict__ xadj,
                            const idx_t* __restrict__ adj, const idx_t* __restrict__ cand_g,
                            const idx_t* __restrict__ sel, idx_t* __restrict__ part, int32_t* __restrict__ state,
                            int32_t* __restrict__ move_round, int32_t round, long long* __restrict__ gain_sum,
                            idx_t* __restrict__ changed) {
  const int32_t nm = *nm_dev;
  long long g = 0;
  RMB_GRID_STRIDE(i, nm) {
    const int32_t v = movers[i];
    const int32_t t = tgt[i];
    changed[v] = 1;
    if (t >= 0 && rank[i] < cut[t]) {
      part[v] = t;
      state[v] = kLocked;
      move_round[v] = round;
      g += cand_g[xadj[v]];
      for (int32_t j = xadj[v]; j < xadj[v + 1]; ++j) {
        const int32_t u = adj[j];
        changed[u] = 1;
        if (!sel[u] && state[u] == kDropped) state[u] = kFree;
      }
    } else {
      state[v] = kDropped;
    }
  }
  g = warp_sum(g);
  if ((threadIdx.x & 31) == 0 && g) atomic_add_i64(&gain_sum[round], g);
}

// Undo the moves of the rounds after `best` (move_round > best); clears the
// round records.
__global__ void k_fm2_rollback(int32_t n, int32_t* __restrict__ move_round, int32_t best,
                               idx_t* __restrict__ part) {
  RMB_GRID_STRIDE(v, n) {
    const int32_t r = move_round[v];
    if (r < 0) continue;
    if (r > best) part[v] = 1 - part[v];
    move_round[v] = -1;
  }
}

__global__ void k_fill_i32(int32_t* __restrict__ a, int32_t n, int32_t v) {
  RMB_GRID_STRIDE(i, n) a[i] = v;
}

}  // namespace

RefineStats fm2_refine(const DGraph& g, idx_t* part, const RefineParams& rp, Arena& arena, cudaStream_t st,
                       int32_t* h_scratch) {
  if (rp.k != 2) throw Error(-4, "fm2_refine refines bisections only");
  if (g.ncon > 8) throw Error(-2, "ncon above the supported maximum of 8");
  (void)h_scratch;
  RefineStats stats;
  const int32_t n = g.n;
  const int32_t K = 2 * g.ncon;
  Arena::Mark mk = arena.mark();
  long long* pw = arena.alloc<long long>((size_t)K);
  idx_t* ncand = arena.alloc<idx_t>((size_t)n);
  idx_t* zero = arena.alloc<idx_t>((size_t)n);
  idx_t* sel = arena.alloc<idx_t>((size_t)n);
  idx_t* movers = arena.alloc<idx_t>((size_t)n);
  int32_t* state = arena.alloc<int32_t>((size_t)n);
  int32_t* move_round = arena.alloc<int32_t>((size_t)n);
  idx_t* cand_p = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* cand_g = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* chg[2];  // vertices whose gain the last round changed, alternating
  for (int b = 0; b < 2; ++b) chg[b] = arena.alloc<idx_t>((size_t)n);
  int32_t* gmax = arena.alloc<int32_t>((size_t)kFm2MaxRounds);
  int32_t* counters = arena.alloc<int32_t>(2 * (size_t)kFm2MaxRounds);
  long long* gsum = arena.alloc<long long>((size_t)kFm2MaxRounds);
  AdmitScratch as;
  as.tgt = arena.alloc<int32_t>((size_t)n);
  as.src = arena.alloc<int32_t>((size_t)n);
  as.w = arena.alloc<int32_t>((size_t)n * g.ncon);
  as.rank = arena.alloc<int32_t>((size_t)n);
  as.pref = arena.alloc<long long>((size_t)n * g.ncon);
  as.gsrc = arena.alloc<int32_t>((size_t)n);
  as.out = arena.alloc<long long>((size_t)K);
  as.cut = arena.alloc<int32_t>(2);
  RMB_CUDA(cudaMemsetAsync(as.out, 0, sizeof(long long) * (size_t)K, st));
  RMB_CUDA(cudaMemsetAsync(zero, 0, sizeof(idx_t) * (size_t)n, st));
  const int nb = grid_for(n, 256);
  k_fill_i32<<<nb, 256, 0, st>>>(move_round, n, -1);
  RMB_LAUNCH_CHECK();
  partition_weights_only(g, part, 2, pw, st);
  std::vector<int32_t> hc(2 * (size_t)kFm2MaxRounds);
  std::vector<long long> hg(kFm2MaxRounds);
  for (int pass = 0; pass < rp.niter; ++pass) {  // fm.rs:22-27
    RMB_CUDA(cudaMemsetAsync(state, 0, sizeof(int32_t) * (size_t)n, st));
    RMB_CUDA(cudaMemsetAsync(counters, 0, sizeof(int32_t) * 2 * (size_t)kFm2MaxRounds, st));
    RMB_CUDA(cudaMemsetAsync(gsum, 0, sizeof(long long) * (size_t)kFm2MaxRounds, st));
    for (int b = 0; b < 2; ++b) RMB_CUDA(cudaMemsetAsync(chg[b], 0, sizeof(idx_t) * (size_t)n, st));
    k_fill_i32<<<grid_for(kFm2MaxRounds, 256), 256, 0, st>>>(gmax, kFm2MaxRounds, INT_MIN);
    RMB_LAUNCH_CHECK();
    int rounds = 0;
    bool done = false;
    long long run_cum = 0, run_best = 0;
    int run_best_q = -1;
    while (!done && rounds < kFm2MaxRounds) {
      const int r0 = rounds;
      for (int q = 0; q < kFm2RoundsPerCheck && rounds < kFm2MaxRounds; ++q, ++rounds) {
        int32_t* nm_dev = counters + 2 * rounds;
        idx_t* cur = rounds > 0 ? chg[rounds & 1] : nullptr;
        // Gains of the vertices the last round changed, after the first round.
        if (g.adjwgt)
          k_fm2_gain<true><<<nb, 256, 0, st>>>(n, g.xadj, g.adjncy, g.adjwgt, part, state, cur, ncand, cand_p,
                                               cand_g);
        else
          k_fm2_gain<false><<<nb, 256, 0, st>>>(n, g.xadj, g.adjncy, g.adjwgt, part, state, cur, ncand, cand_p,
                                                cand_g);
        RMB_LAUNCH_CHECK();
        k_fm2_max<<<grid_for(n, 256, 148 * 4), 256, 0, st>>>(n, g.xadj, ncand, cand_g, gmax + rounds);
        RMB_LAUNCH_CHECK();
        k_fm2_select<<<nb, 256, 0, st>>>(n, g.xadj, g.adjncy, ncand, cand_g, gmax + rounds, sel);
        RMB_LAUNCH_CHECK();
        compact_flags(sel, n, movers, nm_dev, arena, st);
        admit_cut_pass(g, 2, n, nm_dev, movers, sel, zero, cand_p, cand_g, part, pw, rp.feas_max, nm_dev + 1,
                       nullptr, as, st, /*apply=*/false, nullptr, /*any_gain=*/true);
        k_fm2_apply<<<grid_for(n, 256, 148 * 4), 256, 0, st>>>(nm_dev, movers, as.tgt, as.rank, as.cut, g.xadj,
                                                               g.adjncy, cand_g, sel, part, state, move_round,
                                                               rounds, gsum, chg[(rounds + 1) & 1]);
        RMB_LAUNCH_CHECK();
      }
      RMB_CUDA(cudaMemcpyAsync(hc.data() + 2 * r0, counters + 2 * r0, sizeof(int32_t) * 2 * (rounds - r0),
                               cudaMemcpyDeviceToHost, st));
      RMB_CUDA(cudaMemcpyAsync(hg.data() + r0, gsum + r0, sizeof(long long) * (rounds - r0), cudaMemcpyDeviceToHost,
                               st));
      RMB_CUDA(cudaStreamSynchronize(st));
      for (int q = r0; q < rounds && !done; ++q) {
        if (hc[2 * q] == 0) {
          done = true;
          break;
        }
        run_cum += hg[q];
        if (run_cum > run_best) {
          run_best = run_cum;
          run_best_q = q;
        }
        if (q - run_best_q > kFm2Patience) done = true;
      }
    }
    // The cut after each round falls by the round's gain sum; keep the
    // rounds up to the lowest cut (the first one on ties, fm.rs:100-103).
    long long cum = 0, best_cum = 0;
    int best = -1;
    int64_t kept = 0;
    for (int q = 0; q < rounds; ++q) {
      if (hc[2 * q] == 0) break;
      stats.movers += hc[2 * q];
      stats.decide_iters += 1;
      cum += hg[q];
      if (cum > best_cum) {
        best_cum = cum;
        best = q;
      }
    }
    for (int q = 0; q <= best; ++q) kept += hc[2 * q + 1];
    // Another pass follows one that lowered the cut. (fm.rs:116-118 also
    // asks that the moves after the lowest cut raised it again, comparing the
    // lowest cut with the cut before the rollback; a pass of rounds that ends
    // at its lowest cut, its candidates used up, would then stop the
    // refinement although it improved.)
    const bool improved = best >= 0 && best_cum > 0;
    k_fm2_rollback<<<nb, 256, 0, st>>>(n, move_round, best, part);
    RMB_LAUNCH_CHECK();
    // The part weights after the rollback (the admission kept pw for the
    // moves it made, including the ones undone).
    partition_weights_only(g, part, 2, pw, st);
    stats.passes += 1;
    stats.moves += kept;
    if (!improved) break;
  }
  RMB_CUDA(cudaStreamSynchronize(st));
  arena.reset_to(mk);
  return stats;
}

}  // namespace rmb
