// Initial partition of the coarsest graph: graph growing, one warp per trial.
#include <climits>

#include "kernels.h"
#include "prof.h"

namespace rmb {

// grow_partition (src/initial/grow.rs:12-103) given its k seed vertices.
//
// The reference's round-robin order is kept exactly: parts are visited in
// ascending order each round; a part below target pops queue vertices until
// one of them claims at least one unassigned neighbour (claiming all of them,
// in CSR order, and appending them to its queue in that order). The warp
// scans the popped vertex's row 32 entries at a time; a neighbour listed twice
// in a row is claimed once, by its first occurrence. Leftover vertices go,
// in ascending order, to the part with the smallest weight on constraint 0
// (first minimum).
//
// Per-trial state lives in global scratch: part[n], queue links next[n],
// part weights pw[k][ncon] (i64), queue head/tail[k].
template <bool HAS_VW>
__global__ void k_grow(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                       const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ vwgt, int32_t n, int32_t ncon,
                       int32_t k, int32_t ntrials, const idx_t* __restrict__ seeds,
                       const long long* __restrict__ grow_tgt, idx_t* __restrict__ parts, idx_t* __restrict__ nexts,
                       long long* __restrict__ pws, idx_t* __restrict__ heads, idx_t* __restrict__ tails,
                       long long* __restrict__ cuts) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int trial = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (trial >= ntrials) return;  // whole warp
  idx_t* part = parts + (int64_t)trial * n;
  idx_t* next = nexts + (int64_t)trial * n;
  long long* pw = pws + (int64_t)trial * k * ncon;
  idx_t* head = heads + (int64_t)trial * k;
  idx_t* tail = tails + (int64_t)trial * k;
  const idx_t* sd = seeds + (int64_t)trial * k;

  for (int32_t v = lane; v < n; v += 32) part[v] = -1;
  __syncwarp();
  for (int32_t p = lane; p < k; p += 32) {
    const int32_t s = sd[p];
    part[s] = p;
    head[p] = s;
    tail[p] = s;
    next[s] = -1;
    for (int c = 0; c < ncon; ++c) pw[(int64_t)p * ncon + c] = HAS_VW ? vwgt[(int64_t)s * ncon + c] : 1;
  }
  __syncwarp();

  int32_t active = k;
  while (active > 0) {
    active = 0;
    for (int32_t p = 0; p < k; ++p) {
      bool at_target = true;
      for (int c = 0; c < ncon; ++c)
        if (!(pw[(int64_t)p * ncon + c] >= grow_tgt[(int64_t)p * ncon + c])) { at_target = false; break; }
      if (at_target) continue;
      bool grew = false;
      int32_t qh = head[p], qt = tail[p];
      while (qh != -1) {
        const int32_t v = qh;
        qh = next[v];
        const int32_t e = xadj[v + 1];
        for (int32_t b = xadj[v]; b < e; b += 32) {
          const int32_t j = b + lane;
          int32_t u = -1;
          bool cand = false;
          if (j < e) {
            u = adj[j];
            cand = part[u] == -1;
          }
          const unsigned peers = __match_any_sync(FULL, cand ? u : -(lane + 2));
          const bool first = cand && (__ffs(peers) - 1) == lane;
          const unsigned fm = __ballot_sync(FULL, first);
          if (fm) {
            grew = true;
            if (first) part[u] = p;
            for (int c = 0; c < ncon; ++c) {
              long long w = first ? (long long)(HAS_VW ? vwgt[(int64_t)u * ncon + c] : 1) : 0;
              w = warp_sum(w);
              if (lane == 0) pw[(int64_t)p * ncon + c] += w;
            }
            // Link the claimed vertices in lane order and append them.
            const unsigned above = fm & ~((2u << lane) - 1u);
            const int nl = above ? (__ffs(above) - 1) : lane;
            const int32_t unext = __shfl_sync(FULL, u, nl);
            if (first) next[u] = above ? unext : -1;
            const int32_t ufirst = __shfl_sync(FULL, u, __ffs(fm) - 1);
            const int32_t ulast = __shfl_sync(FULL, u, 31 - __clz(fm));
            if (qh == -1) {
              qh = ufirst;
            } else if (lane == 0) {
              next[qt] = ufirst;
            }
            qt = ulast;
          }
          __syncwarp();
        }
        if (grew) break;
      }
      if (lane == 0) {
        head[p] = qh;
        tail[p] = qt;
      }
      __syncwarp();
      if (grew) ++active;
    }
  }

  // Leftovers (disconnected or unreachable): lightest part on constraint 0.
  for (int32_t b = 0; b < n; b += 32) {
    const int32_t v = b + lane;
    unsigned un = __ballot_sync(FULL, v < n && part[v] == -1);
    while (un) {
      const int i = __ffs(un) - 1;
      un &= un - 1;
      const int32_t vv = b + i;
      long long best = LLONG_MAX;
      int32_t bp = INT32_MAX;
      for (int32_t p = lane; p < k; p += 32) {
        const long long x = pw[(int64_t)p * ncon];
        if (x < best) { best = x; bp = p; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const long long ob = __shfl_xor_sync(FULL, best, o);
        const int32_t op = __shfl_xor_sync(FULL, bp, o);
        if (ob < best || (ob == best && op < bp)) { best = ob; bp = op; }
      }
      if (lane == 0) {
        part[vv] = bp;
        for (int c = 0; c < ncon; ++c) pw[(int64_t)bp * ncon + c] += HAS_VW ? vwgt[(int64_t)vv * ncon + c] : 1;
      }
      __syncwarp();
    }
  }
  __syncwarp();

  // Edge cut of this trial (sum over both directions).
  long long acc = 0;
  for (int32_t v = lane; v < n; v += 32) {
    const int32_t pv = part[v];
    for (int32_t j = xadj[v]; j < xadj[v + 1]; ++j)
      if (part[adj[j]] != pv) acc += adjwgt ? adjwgt[j] : 1;
  }
  acc = warp_sum(acc);
  if (lane == 0) cuts[trial] = acc;
}

void grow_trials(const DGraph& g, int k, int ntrials, const idx_t* seeds, const long long* grow_tgt, idx_t* parts,
                 long long* cuts, Arena& arena, cudaStream_t st) {
  Arena::Mark mk = arena.mark();
  idx_t* nexts = arena.alloc<idx_t>((size_t)ntrials * g.n);
  long long* pws = arena.alloc<long long>((size_t)ntrials * k * g.ncon);
  idx_t* heads = arena.alloc<idx_t>((size_t)ntrials * k);
  idx_t* tails = arena.alloc<idx_t>((size_t)ntrials * k);
  const int wpb = 4;
  const int blocks = (int)ceil_div(ntrials, wpb);
  const int ph = profiler().begin(kProfGrow, st);
  if (g.vwgt)
    k_grow<true><<<blocks, 32 * wpb, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.vwgt, g.n, g.ncon, k, ntrials, seeds,
                                              grow_tgt, parts, nexts, pws, heads, tails, cuts);
  else
    k_grow<false><<<blocks, 32 * wpb, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.vwgt, g.n, g.ncon, k, ntrials, seeds,
                                               grow_tgt, parts, nexts, pws, heads, tails, cuts);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, (double)ntrials * (16.0 * g.n + 8.0 * (double)g.m));
  arena.reset_to(mk);
}

}  // namespace rmb
