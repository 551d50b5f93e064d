// Gain tables of the greedy and FM passes (device bodies shared by the
// refinement kernels of refine.cu and the batched admission of admit.cu).
#pragma once

#include "kernels.h"

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
__device__ void gain_body(Lanes L, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                          const idx_t* __restrict__ adjwgt, int32_t n, int32_t ncon, const idx_t* __restrict__ part,
                          int32_t k, const long long* __restrict__ pw0, const long long* __restrict__ over_thr,
                          idx_t* __restrict__ mover, idx_t* __restrict__ ncand, idx_t* __restrict__ wfrom,
                          idx_t* __restrict__ cand_p, idx_t* __restrict__ cand_g,
                          const idx_t* __restrict__ only = nullptr, bool clear_only = false) {
  RMB_FOR(v, n, L) {
    if (only && !only[v]) continue;  // entries of vertices outside `only` stay as they are
    const int32_t s = xadj[v], e = xadj[v + 1];
    if (e - s > kHeavyDegree) continue;  // warp path
    if (clear_only) const_cast<idx_t*>(only)[v] = 0;  // consumed: the flag set is empty again after the pass
    const int32_t pv = part[v];
    if (MODE == kRepair) {
      bool over = false;
      for (int c = 0; c < ncon; ++c)
        if (pw0[(int64_t)pv * ncon + c] > over_thr[(int64_t)pv * ncon + c]) over = true;
      if (!over) { mover[v] = 0; continue; }
    }
    // Connection weight per neighbouring part, in first-appearance order:
    // up to kRegParts parts accumulate in registers (compile-time slots, so
    // no local memory) and are written out once; a vertex next to more parts
    // runs the accumulation again in its global candidate slots.
    constexpr int kRegParts = 8;
    uint32_t wf = 0;
    int cnt = 0;
    bool boundary = false, spill = false;
    int32_t rp[kRegParts];
    uint32_t rw[kRegParts];
#pragma unroll
    for (int i = 0; i < kRegParts; ++i) {
      rp[i] = -1;
      rw[i] = 0;
    }
    // Four entries at a time: their adjncy and part gathers are in flight
    // together; they are then taken in row order.
    for (int32_t j0 = s; j0 < e; j0 += 4) {
      int32_t pq[4];
      uint32_t wq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        pq[q] = j0 + q < e ? adj[j0 + q] : -1;
        wq[q] = j0 + q < e ? (uint32_t)(HAS_W ? adjwgt[j0 + q] : 1) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) pq[q] = pq[q] >= 0 ? part[pq[q]] : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (j0 + q >= e) break;
        const int32_t pu = pq[q];
        const uint32_t w = wq[q];
        if (pu == pv) {
          wf += w;
        } else {
          boundary = true;
          bool found = false;
#pragma unroll
          for (int i = 0; i < kRegParts; ++i)
            if (rp[i] == pu) {
              rw[i] += w;
              found = true;
            }
          if (!found) {
            if (cnt < kRegParts) {
#pragma unroll
              for (int i = 0; i < kRegParts; ++i)
                if (i == cnt) {
                  rp[i] = pu;
                  rw[i] = w;
                }
              ++cnt;
            } else {
              spill = true;
            }
          }
        }
      }
    }
    if (!boundary) { mover[v] = 0; continue; }
    if (!spill) {
#pragma unroll
      for (int i = 0; i < kRegParts; ++i)
        if (i < cnt) {
          cand_p[s + i] = rp[i];
          cand_g[s + i] = (int32_t)rw[i];
        }
    } else {
      cnt = 0;
      for (int32_t j = s; j < e; ++j) {
        const int32_t pu = part[adj[j]];
        if (pu == pv) continue;
        const uint32_t w = (uint32_t)(HAS_W ? adjwgt[j] : 1);
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
// Warps gw, gw + nw, ... take the heavy vertices; hist: k entries of this
// warp's own.
template <bool HAS_W, int MODE>
__device__ void gain_heavy_body(int32_t gw, int32_t nw, int32_t* hist, const idx_t* __restrict__ xadj,
                                const idx_t* __restrict__ adj, const idx_t* __restrict__ adjwgt,
                                const idx_t* __restrict__ heavy, int32_t nheavy, int32_t ncon,
                                const idx_t* __restrict__ part, int32_t k, const long long* __restrict__ pw0,
                                const long long* __restrict__ over_thr, idx_t* __restrict__ mover,
                                idx_t* __restrict__ ncand, idx_t* __restrict__ wfrom, idx_t* __restrict__ cand_p,
                                idx_t* __restrict__ cand_g, const idx_t* __restrict__ only = nullptr,
                                bool clear_only = false) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  for (int32_t hi = gw; hi < nheavy; hi += nw) {
    const int32_t v = heavy[hi];
    if (only && !only[v]) continue;  // warp-uniform: every lane reads the same flag
    __syncwarp();
    if (clear_only && lane == 0) const_cast<idx_t*>(only)[v] = 0;
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
    // Eight entries per lane at a time: their adjncy and part gathers are in
    // flight together (a hub's row is otherwise one long dependent chain).
    constexpr int kIlp = 8;
    for (int32_t j0 = s; j0 < e; j0 += 32 * kIlp) {
      int32_t uu[kIlp];
      uint32_t ww[kIlp];
#pragma unroll
      for (int q = 0; q < kIlp; ++q) {
        const int32_t j = j0 + q * 32 + lane;
        uu[q] = j < e ? adj[j] : -1;
        ww[q] = j < e ? (uint32_t)(HAS_W ? adjwgt[j] : 1) : 0u;
      }
#pragma unroll
      for (int q = 0; q < kIlp; ++q) uu[q] = uu[q] >= 0 ? part[uu[q]] : -1;
#pragma unroll
      for (int q = 0; q < kIlp; ++q) {
        const int32_t pu = uu[q];
        if (pu < 0) continue;
        if (pu == pv) wf += ww[q];
        else { bnd = 1; atomicAdd(reinterpret_cast<unsigned*>(&hist[pu]), ww[q]); }
      }
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

}  // namespace rmb
