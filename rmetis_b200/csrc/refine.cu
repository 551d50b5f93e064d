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
// dependency is `pw`: near the balance limit a move into a part is feasible
// only because earlier moves left it, which chains decisions together. The
// decisions are therefore made in mover order by a walker (k_walk: one
// block, part weights in shared memory, mover records streamed through
// shared memory while the walking warp works). Before the walk, a parallel
// pass resolves every mover whose decision cannot depend on the order: a
// candidate part that stays feasible even if every potential move into it
// happens first, or that stays infeasible even if every potential move out
// of it happens first (k_walk_classify). The walker only evaluates the rest.
#include <chrono>
#include <vector>
#include <climits>
#include <mutex>
#include <set>
#include <cstdio>
#include <cstdlib>

#include "kernels.h"
#include "prof.h"
#include "scan.cuh"
#include "gain.cuh"

namespace rmb {


template <bool HAS_W, int MODE>
__global__ void k_gain(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                       const idx_t* __restrict__ adjwgt, int32_t n, int32_t ncon, const idx_t* __restrict__ part,
                       int32_t k, const long long* __restrict__ pw0, const long long* __restrict__ over_thr,
                       idx_t* __restrict__ mover, idx_t* __restrict__ ncand, idx_t* __restrict__ wfrom,
                       idx_t* __restrict__ cand_p, idx_t* __restrict__ cand_g, const int32_t* __restrict__ stop,
                       const idx_t* __restrict__ only, bool clear_only) {
  // stop: moves of the previous cut pass. None means this pass would find the
  // same movers and make no move either (the reference stops there): no movers.
  if (stop && *stop == 0) {
    RMB_GRID_STRIDE(v, n) mover[v] = 0;
    return;
  }
  gain_body<HAS_W, MODE>(grid_lanes(), xadj, adj, adjwgt, n, ncon, part, k, pw0, over_thr, mover, ncand, wfrom,
                         cand_p, cand_g, only, clear_only);
}

template <bool HAS_W, int MODE>
__global__ void k_gain_heavy(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                             const idx_t* __restrict__ adjwgt, const idx_t* __restrict__ heavy, int32_t nheavy,
                             int32_t ncon, const idx_t* __restrict__ part, int32_t k,
                             const long long* __restrict__ pw0, const long long* __restrict__ over_thr,
                             idx_t* __restrict__ mover, idx_t* __restrict__ ncand, idx_t* __restrict__ wfrom,
                             idx_t* __restrict__ cand_p, idx_t* __restrict__ cand_g, int32_t* __restrict__ ghist,
                             const int32_t* __restrict__ stop, const idx_t* __restrict__ only,
                             bool clear_only) {
  if (stop && *stop == 0) return;  // k_gain has cleared every mover flag
  __shared__ int32_t sh_all[4][kGainHist];
  const int wib = threadIdx.x >> 5;
  const int32_t gw = blockIdx.x * (blockDim.x >> 5) + wib;
  const int32_t nw = gridDim.x * (blockDim.x >> 5);
  int32_t* hist = (k <= kGainHist) ? sh_all[wib] : ghist + (int64_t)gw * k;
  gain_heavy_body<HAS_W, MODE>(gw, nw, hist, xadj, adj, adjwgt, heavy, nheavy, ncon, part, k, pw0, over_thr, mover,
                               ncand, wfrom, cand_p, cand_g, only, clear_only);
}


// ---------------------------------------------------------------------------
// Mover records and the walk
// ---------------------------------------------------------------------------
constexpr int kInline = 4;          // candidates kept inline in a mover record
static_assert(kInline == kRecInline, "batched jobs size the records with kRecInline");
constexpr int kWalkChunk = 256;     // mover records per shared-memory chunk
constexpr int kWalkThreads = 256;   // warp 0 walks, the other warps stream records
constexpr int32_t kContended = -2;  // decision not known before the walk (general path)
constexpr int32_t kFast = -3;       // not known; at most two candidates, cut pass
constexpr int32_t kLong = -4;       // not known; cut pass, more candidates than the inline slots
constexpr int kWalkSmemParts = 4096;  // [k][ncon] entries kept in shared memory

// What the walk writes: each mover's new part straight into part (the moves
// of a pass apply together after its decisions, greedy.rs:111-119,
// :168-181; the walk itself reads only the records), and the cleared
// in/out bounds that the next pass's prep accumulates into.
struct WalkOut {
  const idx_t* movers;  // [nm] vertex of each mover record
  idx_t* part;
  long long* in_max;    // [k][ncon]
  long long* out_max;   // [k][ncon]
  int32_t K;            // k * ncon
};

struct MoverRecs {  // structure of arrays, nm entries each
  int32_t* pv;
  int32_t* ne;
  int32_t* wf;
  int32_t* coff;   // xadj[v]: start of the vertex's candidate slots
  int32_t* known;  // decision fixed before the walk, or kContended
  int32_t* cp;     // [nm][kInline] candidate parts
  int32_t* cg;     // [nm][kInline] candidate gains
  int32_t* vw;     // [nm][ncon]
  int32_t* np;     // kLong movers with -w_from <= 0: number of positive-gain candidates, else -1
};

// Positive-gain candidates of kLong movers, gathered into shared memory by the
// loader warps (dynamic shared memory after the walk's static buffers): per
// buffer, 32 slots per mover and the count (-1: not gathered).
constexpr int kPoolSlots = 32;
constexpr size_t kPoolBytes = sizeof(int32_t) * 2 * ((size_t)kWalkChunk * kPoolSlots + kWalkChunk);
__device__ __forceinline__ int32_t* pool_cand(int32_t* dyn, int buf) { return dyn + buf * kWalkChunk * kPoolSlots; }
__device__ __forceinline__ int32_t* pool_np(int32_t* dyn, int buf) {
  return dyn + 2 * kWalkChunk * kPoolSlots + buf * kWalkChunk;
}

// One thread per mover: copy its data into a record and add its weight to
// the bounds: in_max[p] over every part it may move to, out_max[pv].
template <int MODE>
__device__ void prep_body(Lanes L, const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                          const idx_t* __restrict__ part, const idx_t* __restrict__ vwgt, int32_t ncon,
                          const idx_t* __restrict__ xadj, const idx_t* __restrict__ ncand,
                          const idx_t* __restrict__ wfrom, const idx_t* __restrict__ cand_p,
                          const idx_t* __restrict__ cand_g, const MoverRecs& r, long long* __restrict__ in_max,
                          long long* __restrict__ out_max, int32_t* __restrict__ long_flag) {
  const int32_t nm = *nm_dev;
  RMB_FOR(j, nm, L) {
    const int32_t v = movers[j];
    const int32_t pv = part[v];
    const int32_t s = xadj[v];
    const int32_t ne = ncand[v];
    r.pv[j] = pv;
    if (MODE != kCut) {
      r.known[j] = kContended;
      // Count the movers with long candidate lists (one atomic per warp).
      const unsigned lm = __ballot_sync(__activemask(), ne > kInline);
      if (lm && (threadIdx.x & 31) == __ffs(lm) - 1) atomicAdd(long_flag, __popc(lm));
    }
    r.ne[j] = ne;
    r.wf[j] = wfrom[v];
    r.coff[j] = s;
    for (int i = 0; i < kInline; ++i) {
      r.cp[j * kInline + i] = i < ne ? cand_p[s + i] : -1;
      r.cg[j * kInline + i] = i < ne ? cand_g[s + i] : 0;
    }
    for (int c = 0; c < ncon; ++c) {
      const int32_t w = vwgt ? vwgt[(int64_t)v * ncon + c] : 1;
      r.vw[(int64_t)j * ncon + c] = w;
      if (MODE == kCut) {
        atomic_add_i64(&out_max[(int64_t)pv * ncon + c], w);
        for (int i = 0; i < ne; ++i) {
          if (cand_g[s + i] <= 0) break;  // sorted: the rest never qualify
          atomic_add_i64(&in_max[(int64_t)cand_p[s + i] * ncon + c], w);
        }
      }
    }
  }
}

template <int MODE>
__global__ void k_walk_prep(const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                            const idx_t* __restrict__ part, const idx_t* __restrict__ vwgt, int32_t ncon,
                            const idx_t* __restrict__ xadj, const idx_t* __restrict__ ncand,
                            const idx_t* __restrict__ wfrom, const idx_t* __restrict__ cand_p,
                            const idx_t* __restrict__ cand_g, MoverRecs r, long long* __restrict__ in_max,
                            long long* __restrict__ out_max, int32_t* __restrict__ long_flag) {
  prep_body<MODE>(grid_lanes(), nm_dev, movers, part, vwgt, ncon, xadj, ncand, wfrom, cand_p, cand_g, r, in_max,
                  out_max, long_flag);
}

// Cut passes: fix the decision of every mover whose walk through its
// candidates meets only parts that are infeasible whatever happens before it,
// and then a part that is feasible whatever happens before it (or runs out).
__device__ void classify_body(Lanes L, const int32_t* __restrict__ nm_dev, int32_t ncon,
                              const idx_t* __restrict__ cand_p, const idx_t* __restrict__ cand_g, const MoverRecs& r,
                              const long long* __restrict__ pw0, const long long* __restrict__ feas,
                              const long long* __restrict__ in_max, const long long* __restrict__ out_max,
                              int32_t* __restrict__ long_flag) {
  const int32_t nm = *nm_dev;
  RMB_FOR(j, nm, L) {
    const int32_t ne = r.ne[j];
    const int32_t ig = (int32_t)(0u - (uint32_t)r.wf[j]);
    int32_t known = -1;
    if (ig > 0) {
      known = kContended;  // non-adjacent parts have positive gain (negative weights)
    } else {
      const int32_t s = r.coff[j];
      for (int32_t i = 0; i < ne; ++i) {
        const int32_t g = i < kInline ? r.cg[j * kInline + i] : cand_g[s + i];
        if (g <= 0) break;
        const int32_t p = i < kInline ? r.cp[j * kInline + i] : cand_p[s + i];
        bool always = true, never = false;
        for (int c = 0; c < ncon; ++c) {
          const int64_t x = (int64_t)p * ncon + c;
          if (pw0[x] + in_max[x] > feas[x]) always = false;
          if (pw0[x] - out_max[x] + r.vw[(int64_t)j * ncon + c] > feas[x]) never = true;
        }
        if (always) { known = p; break; }
        if (never) continue;
        known = kContended;
        break;
      }
      if (known == kContended) {
        // Fast path: every candidate with positive gain is among the first two
        // inline slots (cut pass, no non-adjacent candidate since ig <= 0).
        int32_t npos = 0;
        for (int32_t i = 0; i < ne && i < 3; ++i) {
          const int32_t g = i < kInline ? r.cg[j * kInline + i] : cand_g[s + i];
          if (g > 0) ++npos;
        }
        if (npos <= 2) known = kFast;
      }
    }
    if (known == kContended && ne > kInline) known = kLong;
    int32_t npos = -1;
    if (known == kLong && ig <= 0) {
      // The decision of such a mover is the first feasible part among its
      // positive-gain candidates (the scan ends at the first gain <= 0).
      const int32_t s0 = r.coff[j];
      npos = 0;
      while (npos < ne && (npos < kInline ? r.cg[j * kInline + npos] : cand_g[s0 + npos]) > 0) ++npos;
    }
    r.np[j] = npos;
    // Count the kLong movers (one atomic per warp).
    const unsigned lm = __ballot_sync(__activemask(), known == kLong);
    if (lm && (threadIdx.x & 31) == __ffs(lm) - 1) atomicAdd(long_flag, __popc(lm));
    r.known[j] = known;
  }
}

__global__ void k_walk_classify(const int32_t* __restrict__ nm_dev, int32_t ncon, const idx_t* __restrict__ cand_p,
                                const idx_t* __restrict__ cand_g, MoverRecs r, const long long* __restrict__ pw0,
                                const long long* __restrict__ feas, const long long* __restrict__ in_max,
                                const long long* __restrict__ out_max, int32_t* __restrict__ long_flag) {
  classify_body(grid_lanes(), nm_dev, ncon, cand_p, cand_g, r, pw0, feas, in_max, out_max, long_flag);
}

struct WalkBuf {
  int32_t pv[kWalkChunk];
  int32_t ne[kWalkChunk];
  int32_t wf[kWalkChunk];
  int32_t coff[kWalkChunk];
  int32_t known[kWalkChunk];
  int32_t cp[kWalkChunk * kInline];
  int32_t cg[kWalkChunk * kInline];
  int32_t vw[kWalkChunk * kMaxCon];
};

__device__ inline void walk_load(WalkBuf& b, const MoverRecs& r, int32_t j0, int32_t nm, int32_t ncon, int tid,
                                 int nthreads) {
  for (int i = tid; i < kWalkChunk; i += nthreads) {
    const int32_t j = j0 + i;
    if (j < nm) {
      b.pv[i] = r.pv[j];
      b.ne[i] = r.ne[j];
      b.wf[i] = r.wf[j];
      b.coff[i] = r.coff[j];
      b.known[i] = r.known[j];
    }
  }
  for (int i = tid; i < kWalkChunk * kInline; i += nthreads) {
    const int64_t j = (int64_t)j0 * kInline + i;
    if (j < (int64_t)nm * kInline) {
      b.cp[i] = r.cp[j];
      b.cg[i] = r.cg[j];
    }
  }
  for (int i = tid; i < kWalkChunk * ncon; i += nthreads) {
    const int64_t j = (int64_t)j0 * ncon + i;
    if (j < (int64_t)nm * ncon) b.vw[(i / ncon) * kMaxCon + (i % ncon)] = r.vw[j];
  }
}

// Loader warps: the positive-gain candidates of the chunk's kLong movers
// (at most kPoolSlots each). A warp takes 32 movers at a time: one coalesced
// read of their kind, count and offset, then their candidate rows, eight
// movers per step so that eight loads are in flight before any store.
__device__ inline void walk_pool_load(int32_t* pc, int32_t* pn, const MoverRecs& r, const idx_t* __restrict__ cand_p,
                                      int32_t j0, int32_t nm, int tid, int nthreads) {
  const unsigned FULL = 0xffffffffu;
  const int lw = tid >> 5, nlw = nthreads >> 5, lane = tid & 31;
  for (int g0 = lw * 32; g0 < kWalkChunk; g0 += nlw * 32) {
    const int32_t j = j0 + g0 + lane;
    int32_t npv = -1, coff = 0;
    if (j < nm && r.known[j] == kLong) {
      npv = r.np[j];
      coff = r.coff[j];
    }
    pn[g0 + lane] = npv;
    unsigned todo = __ballot_sync(FULL, npv > 0);
    while (todo) {
      constexpr int kB = 8;
      int li[kB], cnt[kB], co[kB];
#pragma unroll
      for (int q = 0; q < kB; ++q) {
        li[q] = -1;
        cnt[q] = 0;
        co[q] = 0;
        if (todo) {  // uniform
          const int l = __ffs(todo) - 1;
          todo &= todo - 1;
          const int32_t c = __shfl_sync(FULL, npv, l);
          li[q] = l;
          cnt[q] = c < kPoolSlots ? c : kPoolSlots;
          co[q] = __shfl_sync(FULL, coff, l);
        }
      }
      int32_t val[kB];
#pragma unroll
      for (int q = 0; q < kB; ++q) val[q] = lane < cnt[q] ? __ldg(&cand_p[co[q] + lane]) : 0;
#pragma unroll
      for (int q = 0; q < kB; ++q)
        if (lane < cnt[q]) pc[(g0 + li[q]) * kPoolSlots + lane] = val[q];
    }
  }
}

// The decision of one mover (greedy.rs:64-107 repair, :131-164 cut) given
// the part weights `pwf(p, c)`: candidates in (gain desc, part asc) order =
// explicit ones with gain above the non-adjacent gain -w_from, then the
// non-adjacent parts by id, then the explicit ones below it; the first
// feasible candidate with gain above the pass threshold, or -1.
template <int MODE, typename PW>
__device__ __forceinline__ int32_t walk_decide(const WalkBuf& b, int i, int32_t ncon, int32_t k,
                                               const idx_t* __restrict__ cand_p, const idx_t* __restrict__ cand_g,
                                               const long long* feas, const long long* over, PW pwf) {
  const int32_t pv = b.pv[i];
  const int32_t* vw = &b.vw[i * kMaxCon];
  if (MODE == kRepair) {
    bool is_over = false;
    for (int c = 0; c < ncon; ++c)
      if (pwf(pv, c) > over[pv * ncon + c]) is_over = true;
    if (!is_over) return -1;
  }
  const int32_t thr = (MODE == kRepair) ? INT_MIN : 0;
  const int32_t ne = b.ne[i];
  const int32_t s = b.coff[i];
  const int32_t ig = (int32_t)(0u - (uint32_t)b.wf[i]);
  auto cpart = [&](int32_t q) { return q < kInline ? b.cp[i * kInline + q] : cand_p[s + q]; };
  auto cgain = [&](int32_t q) { return q < kInline ? b.cg[i * kInline + q] : cand_g[s + q]; };
  auto feasible = [&](int32_t p) {
    for (int c = 0; c < ncon; ++c)
      if (pwf(p, c) + vw[c] > feas[p * ncon + c]) return false;
    return true;
  };
  int32_t q = 0;
  for (; q < ne; ++q) {
    const int32_t g = cgain(q);
    if (g <= ig) break;
    if (g <= thr) return -1;
    const int32_t p = cpart(q);
    if (feasible(p)) return p;
  }
  if (ig > thr) {
    for (int32_t p = 0; p < k; ++p) {
      if (p == pv) continue;
      bool in_e = false;
      for (int32_t e = 0; e < ne; ++e)
        if (cpart(e) == p) { in_e = true; break; }
      if (!in_e && feasible(p)) return p;
    }
  }
  for (; q < ne; ++q) {
    const int32_t g = cgain(q);
    if (g <= thr) return -1;
    const int32_t p = cpart(q);
    if (feasible(p)) return p;
  }
  return -1;
}

// The walk. Warp 0 takes the movers of a chunk in windows of 32, one per
// lane, and iterates each window to its fixed point: every lane decides
// against the weights at the window start plus the moves the lanes before it
// made in the previous round. Lane t is final after t rounds (lane 0 sees the
// exact weights from the start), so at most 32 rounds, and the fixed point is
// the sequential result; independent decisions settle in the same round. The
// window then applies its moves and the next one starts. Warps 1.. stream the
// next chunk of mover records meanwhile. SMEM: [k][ncon] part weights and
// thresholds fit in shared memory (else they stay in global memory).
template <int MODE, bool SMEM>
__global__ void __launch_bounds__(kWalkThreads) k_walk(const int32_t* __restrict__ nm_dev, MoverRecs r,
                                                       int32_t ncon, int32_t k, const idx_t* __restrict__ cand_p,
                                                       const idx_t* __restrict__ cand_g, long long* __restrict__ pw,
                                                       const long long* __restrict__ feas_g,
                                                       const long long* __restrict__ over_g,
                                                       WalkOut wo, int32_t* __restrict__ nmoves) {
  extern __shared__ long long sparts[];
  __shared__ WalkBuf buf[2];
  __shared__ int32_t win_d[32], win_pv[32], win_vw[32 * kMaxCon];
  const int32_t nm = *nm_dev;
  const int32_t K = k * ncon;
  long long* spw = SMEM ? sparts : pw;
  const long long* sfeas = SMEM ? sparts + K : feas_g;
  const long long* sover = SMEM ? sparts + 2 * K : over_g;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (SMEM) {
    for (int32_t x = tid; x < K; x += blockDim.x) {
      sparts[x] = pw[x];
      sparts[K + x] = feas_g[x];
      sparts[2 * K + x] = over_g[x];
    }
  }
  if (nm > 0) walk_load(buf[0], r, 0, nm, ncon, tid, blockDim.x);
  __syncthreads();
  int32_t moves = 0;
  const int32_t nchunks = (int32_t)ceil_div(nm, kWalkChunk);
  for (int32_t ch = 0; ch < nchunks; ++ch) {
    if (warp == 0) {
      const WalkBuf& b = buf[ch & 1];
      const int32_t j0 = ch * kWalkChunk;
      const int32_t cnt = min(kWalkChunk, nm - j0);
      auto pw_start = [&](int32_t p, int c) { return spw[p * ncon + c]; };
      for (int32_t i0 = 0; i0 < cnt; i0 += 32) {
        const int i = i0 + lane;
        const bool valid = i < cnt;
        const int32_t known = valid ? b.known[i] : -1;
        const bool open = valid && (known == kContended || known == kFast || known == kLong);
        const int32_t pv = valid ? b.pv[i] : -1;
        for (int c = 0; c < ncon; ++c) win_vw[lane * kMaxCon + c] = valid ? b.vw[i * kMaxCon + c] : 0;
        win_pv[lane] = pv;
        int32_t d = open ? walk_decide<MODE>(b, i, ncon, k, cand_p, cand_g, sfeas, sover, pw_start) : known;
        for (int round = 0; round < 32; ++round) {
          win_d[lane] = d;
          __syncwarp();
          int32_t nd = d;
          if (open && lane > 0) {
            auto pw_prefix = [&](int32_t p, int c) {
              long long x = spw[p * ncon + c];
              for (int l = 0; l < lane; ++l) {
                const int32_t dl = win_d[l];
                if (dl < 0) continue;
                if (dl == p) x += win_vw[l * kMaxCon + c];
                if (win_pv[l] == p) x -= win_vw[l * kMaxCon + c];
              }
              return x;
            };
            nd = walk_decide<MODE>(b, i, ncon, k, cand_p, cand_g, sfeas, sover, pw_prefix);
          }
          const bool changed = __any_sync(0xffffffffu, nd != d);
          d = nd;
          __syncwarp();
          if (!changed) break;
        }
        if (valid) {
          if (d >= 0) wo.part[wo.movers[j0 + i]] = d;
          if (d >= 0) {
            for (int c = 0; c < ncon; ++c) {
              const long long w = win_vw[lane * kMaxCon + c];
              atomicAdd(reinterpret_cast<unsigned long long*>(&spw[pv * ncon + c]), (unsigned long long)(-w));
              atomicAdd(reinterpret_cast<unsigned long long*>(&spw[d * ncon + c]), (unsigned long long)w);
            }
          }
        }
        moves += __popc(__ballot_sync(0xffffffffu, valid && d >= 0));
        __syncwarp();
      }
    } else if (ch + 1 < nchunks) {
      walk_load(buf[(ch + 1) & 1], r, (ch + 1) * kWalkChunk, nm, ncon, tid - 32, blockDim.x - 32);
    }
    __syncthreads();
  }
  if (SMEM)
    for (int32_t x = tid; x < K; x += blockDim.x) pw[x] = sparts[x];
  // The next cut pass's prep accumulates into cleared bounds.
  for (int32_t x = tid; x < wo.K; x += blockDim.x) {
    wo.in_max[x] = 0;
    wo.out_max[x] = 0;
  }
  if (tid == 0) *nmoves = moves;
}

// Register-resident walk for k <= 32*R parts and NC <= 2 constraints. Only
// warp 0 walks: lane l holds, for parts l, l+32, ..., l+32*(R-1), the slack
// to the feasibility threshold (feas - pw) and to the overweight threshold
// (over - pw) in registers. Every lane reads the same mover record, so control
// flow stays uniform: a move into p is feasible iff w <= slack[p] in p's lane
// (one compare and one vote), the source is overweight iff its over-slack is
// negative. Cut-pass movers with at most two positive-gain candidates take a
// branch-free path (both tests and votes at once, then a select). The other
// warps stream mover records.
template <typename S, int R, int NC>
struct PartRegs {
  S sl[R][NC];  // feas - pw
  S ov[R][NC];  // over - pw
};

template <typename S, int R, int NC>
__device__ __forceinline__ bool lane_fits(const PartRegs<S, R, NC>& s, int lane, int32_t p, const int32_t* w) {
  bool ok = p >= 0 && (p & 31) == lane;
  const int slot = p >> 5;
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int c = 0; c < NC; ++c) ok = ok && (r != slot || (S)w[c] <= s.sl[r][c]);
  return ok;
}

// First 32 candidates of a mover (lane q holds candidate q, or p = -1 past
// the end): from the shared-memory record for q < kInline, else from the
// global candidate arrays.
struct CandChunk {
  int32_t g, p;
};
__device__ __forceinline__ CandChunk first_chunk(const WalkBuf& b, int i, int lane, const idx_t* __restrict__ cand_p,
                                                 const idx_t* __restrict__ cand_g) {
  CandChunk c{0, -1};
  const int32_t ne = b.ne[i];
  if (lane < ne) {
    if (lane < kInline) {
      c.g = b.cg[i * kInline + lane];
      c.p = b.cp[i * kInline + lane];
    } else {
      const int32_t st = b.coff[i];
      c.g = __ldg(&cand_g[st + lane]);
      c.p = __ldg(&cand_p[st + lane]);
    }
  }
  return c;
}

// Explicit candidates q0.. of one mover, 32 at a time: lane t takes
// candidate q0 + t, tests it against the shared copy of the part slacks, and
// the first lane in candidate order whose candidate ends the scan decides.
// The scan ends at a candidate whose gain is <= stop_gain (returns -2 - q:
// the caller goes on elsewhere from q), at one whose gain is <= thr (returns
// -1), or at a feasible one (returns its part); running out returns -2 - ne.
// `pre` holds candidates 0..31 already loaded (used when q0 == 0).
template <typename S, int NC>
__device__ __forceinline__ int32_t coop_scan(const S* sslack, int lane, const WalkBuf& b, int i, int32_t q0,
                                             int32_t ne, int32_t stop_gain, int32_t thr,
                                             const idx_t* __restrict__ cand_p, const idx_t* __restrict__ cand_g,
                                             const int32_t* w, const CandChunk& pre) {
  const int32_t st = b.coff[i];
  for (int32_t base = q0; base < ne; base += 32) {
    const int32_t q = base + lane;
    const bool valid = q < ne;
    int32_t g = 0, p = -1;
    if (base == 0) {
      g = pre.g;
      p = pre.p;
    } else if (valid) {
      g = q < kInline ? b.cg[i * kInline + q] : __ldg(&cand_g[st + q]);
      p = q < kInline ? b.cp[i * kInline + q] : __ldg(&cand_p[st + q]);
    }
    const bool stop = valid && g <= stop_gain;
    const bool below = valid && g <= thr;
    bool fits = valid;
#pragma unroll
    for (int c = 0; c < NC; ++c) fits = fits && (S)w[c] <= sslack[(valid ? p : 0) * NC + c];
    const unsigned m = __ballot_sync(0xffffffffu, stop || below || fits);
    if (m) {
      const int l = __ffs(m) - 1;
      const bool l_stop = __shfl_sync(0xffffffffu, stop, l);
      const bool l_below = __shfl_sync(0xffffffffu, below, l);
      const int32_t l_p = __shfl_sync(0xffffffffu, p, l);
      if (l_stop) return -2 - (base + l);
      if (l_below) return -1;
      return l_p;
    }
  }
  return -2 - ne;
}

// The decision of one mover in the register walk (greedy.rs:64-107 repair,
// :131-164 cut), in the reference's candidate order: explicit candidates with
// gain above the non-adjacent gain ig = -w_from, then the non-adjacent parts
// by id, then the explicit ones at or below ig; the first feasible one with
// gain above the pass threshold, or -1. Explicit candidates are tested 32 at
// a time against the shared slack copy `sslack`; membership in the candidate
// list for the non-adjacent step comes from the inline slots, or for longer
// lists from a shared bitmap `ebits` (R words, zero between calls).
// The decision of one mover when no mover of the pass has more candidates
// than the inline slots (the same order as reg_decide; a longer list, which
// the walk's flag rules out, would still be read correctly from global
// memory one candidate at a time).
template <int MODE, typename S, int R, int NC>
__device__ __forceinline__ int32_t lean_decide(const PartRegs<S, R, NC>& s, int lane, const WalkBuf& b, int i,
                                               int32_t k, const idx_t* __restrict__ cand_p,
                                              const idx_t* __restrict__ cand_g, const int32_t* w) {
  const int32_t pv = b.pv[i];
  if (MODE == kRepair) {
    bool over = false;
    if ((pv & 31) == lane) {
      const int slot = pv >> 5;
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int c = 0; c < NC; ++c)
          if (r == slot && s.ov[r][c] < 0) over = true;
    }
    if (!__any_sync(0xffffffffu, over)) return -1;
  }
  const int32_t thr = (MODE == kRepair) ? INT_MIN : 0;
  const int32_t ne = b.ne[i];
  const int32_t st = b.coff[i];
  const int32_t ig = (int32_t)(0u - (uint32_t)b.wf[i]);
  auto cpart = [&](int32_t q) { return q < kInline ? b.cp[i * kInline + q] : cand_p[st + q]; };
  auto cgain = [&](int32_t q) { return q < kInline ? b.cg[i * kInline + q] : cand_g[st + q]; };
  int32_t q = 0;
  for (; q < ne; ++q) {
    const int32_t g = cgain(q);
    if (g <= ig) break;
    if (g <= thr) return -1;
    const int32_t p = cpart(q);
    if (__any_sync(0xffffffffu, lane_fits(s, lane, p, w))) return p;
  }
  if (ig > thr) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int32_t p = r * 32 + lane;
      bool ok = p < k && p != pv;
      if (ok)
        for (int32_t e = 0; e < ne; ++e)
          if (cpart(e) == p) { ok = false; break; }
#pragma unroll
      for (int c = 0; c < NC; ++c) ok = ok && (S)w[c] <= s.sl[r][c];
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (m) return r * 32 + __ffs(m) - 1;
    }
  }
  for (; q < ne; ++q) {
    const int32_t g = cgain(q);
    if (g <= thr) return -1;
    const int32_t p = cpart(q);
    if (__any_sync(0xffffffffu, lane_fits(s, lane, p, w))) return p;
  }
  return -1;
}

template <int MODE, typename S, int R, int NC>
__device__ __forceinline__ int32_t reg_decide(const PartRegs<S, R, NC>& s, int lane,
                                              const WalkBuf& b, int i, int32_t k, const idx_t* __restrict__ cand_p,
                                              const idx_t* __restrict__ cand_g, const int32_t* w, unsigned* ebits,
                                              const CandChunk* pre, S* sslack, bool& dirty) {
  const int32_t pv = b.pv[i];
  if (MODE == kRepair) {
    bool over = false;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if (pv == r * 32 + lane && s.ov[r][c] < 0) over = true;
    if (!__any_sync(0xffffffffu, over)) return -1;
  }
  const int32_t thr = (MODE == kRepair) ? INT_MIN : 0;
  const int32_t ne = b.ne[i];
  const int32_t st = b.coff[i];
  const int32_t ig = (int32_t)(0u - (uint32_t)b.wf[i]);
  if (ne <= kInline) {
    // Short list, all in the shared-memory record: one candidate at a time
    // against the owner lane's register slack.
    int32_t q = 0;
    for (; q < ne; ++q) {
      const int32_t g = b.cg[i * kInline + q];
      if (g <= ig) break;
      if (g <= thr) return -1;
      const int32_t p = b.cp[i * kInline + q];
      if (__any_sync(0xffffffffu, lane_fits(s, lane, p, w))) return p;
    }
    if (ig > thr) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int32_t p = r * 32 + lane;
        bool ok = p < k && p != pv;
        for (int32_t e = 0; e < ne; ++e)
          if (b.cp[i * kInline + e] == p) ok = false;
#pragma unroll
        for (int c = 0; c < NC; ++c) ok = ok && (S)w[c] <= s.sl[r][c];
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (m) return r * 32 + __ffs(m) - 1;
      }
    }
    for (; q < ne; ++q) {
      const int32_t g = b.cg[i * kInline + q];
      if (g <= thr) return -1;
      const int32_t p = b.cp[i * kInline + q];
      if (__any_sync(0xffffffffu, lane_fits(s, lane, p, w))) return p;
    }
    return -1;
  }
  // Long list: 32 candidates per step against the shared slack copy, brought
  // up to date first if a move happened since it was last written. kLong
  // movers of the cut pass come with their first 32 candidates prefetched.
  const CandChunk pc = pre ? *pre : first_chunk(b, i, lane, cand_p, cand_g);
  if (dirty) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c < NC; ++c) sslack[(r * 32 + lane) * NC + c] = s.sl[r][c];
    __syncwarp();
    dirty = false;
  }
  int32_t q;
  {
    const int32_t r1 = coop_scan<S, NC>(sslack, lane, b, i, 0, ne, ig, thr, cand_p, cand_g, w, pc);
    if (r1 >= -1) return r1;
    q = -2 - r1;
  }
  if (ig > thr) {
    {
      for (int32_t base = 0; base < ne; base += 32) {
        const int32_t e = base + lane;
        if (e < ne) {
          const int32_t p = e < kInline ? b.cp[i * kInline + e] : __ldg(&cand_p[st + e]);
          atomicOr(&ebits[p >> 5], 1u << (p & 31));
        }
      }
      __syncwarp();
      int32_t found = -1;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int32_t p = r * 32 + lane;
        bool ok = found < 0 && p < k && p != pv && !((ebits[r] >> lane) & 1u);
#pragma unroll
        for (int c = 0; c < NC; ++c) ok = ok && (S)w[c] <= s.sl[r][c];
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (m && found < 0) found = r * 32 + __ffs(m) - 1;
      }
      __syncwarp();
      if (lane < R) ebits[lane] = 0u;
      __syncwarp();
      if (found >= 0) return found;
    }
  } else if (q < ne) {
    // The candidate at q has gain <= ig <= thr, and the rest are lower.
    return -1;
  }
  if (q >= ne) return -1;
  const int32_t r3 = coop_scan<S, NC>(sslack, lane, b, i, q, ne, INT_MIN, thr, cand_p, cand_g, w, pc);
  return r3 >= -1 ? r3 : -1;
}


// The chunk loop of k_walk_reg. LONG: many movers of the pass have more
// candidates than the inline slots, so the long-list decision (shared slack
// copy, candidates 32 at a time, prefetch) is compiled in; without it every
// mover takes the short decision, which reads long lists one candidate at a
// time. Both give the same decisions.
template <int MODE, typename S, int R, int NC, bool LONG>
__device__ __forceinline__ void walk_chunks(int32_t nm, const MoverRecs& r, int32_t k,
                                            const idx_t* __restrict__ cand_p, const idx_t* __restrict__ cand_g,
                                            const WalkOut& wo, WalkBuf* buf, int32_t* dbuf, unsigned* ebits,
                                            S* sslack, PartRegs<S, R, NC>& s, int32_t& moves, int tid, int lane,
                                            int warp, int32_t* dyn) {
  bool dirty = false;  // a move since sslack was last written
  constexpr bool POOL = LONG && MODE == kCut;  // kLong candidates gathered by the loaders
  // With 4+ part slots per lane the register test of a candidate costs a
  // compare per slot plus a vote; two-candidate movers then read the shared
  // slack copy instead (k > 128; moves are rare there, so the copy is rarely
  // rewritten). With fewer slots they stay on registers and go in pairs.
  constexpr bool kSharedFast = R >= 4;
  const int32_t nchunks = (int32_t)ceil_div(nm, kWalkChunk);
  for (int32_t ch = 0; ch < nchunks; ++ch) {
    const int32_t j0 = ch * kWalkChunk;
    const int32_t cnt = min(kWalkChunk, nm - j0);
    if (warp == 0) {
      const WalkBuf& b = buf[ch & 1];
      const int32_t* pc = POOL ? pool_cand(dyn, ch & 1) : nullptr;
      const int32_t* pn = POOL ? pool_np(dyn, ch & 1) : nullptr;
      auto c_of = [&](int i, int q) { return b.cg[i * kInline + q] > 0 ? b.cp[i * kInline + q] : -1; };
      // kContended and kLong movers take the general decision (in the repair
      // pass every mover is kContended, and most leave at the overweight
      // test); the first candidates of a kLong mover are loaded one mover
      // ahead.
      int32_t nk = b.known[0], npv = b.pv[0], nc1 = c_of(0, 0), nc2 = c_of(0, 1);
      int32_t nw[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) nw[c] = b.vw[c];
      CandChunk npre{0, -1};
      if (POOL && nk == kLong && pn[0] < 0) npre = first_chunk(b, 0, lane, cand_p, cand_g);
      // Moves a vertex of weight wv from part `from` to part `to` in the
      // register slacks.
      auto apply = [&](int32_t from, int32_t to, const int32_t* wv) {
#pragma unroll
        for (int rr = 0; rr < R; ++rr)
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const S dw = (S)wv[c];
            const int32_t p = rr * 32 + lane;
            const S delta = (from == p ? dw : (S)0) - (to == p ? dw : (S)0);
            s.sl[rr][c] += delta;
            s.ov[rr][c] += delta;
          }
      };
      auto load_next = [&](int32_t j) {
        nk = b.known[j];
        npv = b.pv[j];
        nc1 = c_of(j, 0);
        nc2 = c_of(j, 1);
#pragma unroll
        for (int c = 0; c < NC; ++c) nw[c] = b.vw[j * kMaxCon + c];
        if (POOL && nk == kLong && pn[j] < 0) npre = first_chunk(b, j, lane, cand_p, cand_g);
      };
      for (int32_t i = 0; i < cnt; ++i) {
        const int32_t kn = nk, pv = npv, c1 = nc1, c2 = nc2;
        int32_t w[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) w[c] = nw[c];
        CandChunk pre = npre;
        if (i + 1 < cnt) load_next(i + 1);
        int32_t d = kn;
        if (!kSharedFast && MODE == kCut && kn == kFast && nk == kFast && i + 1 < cnt) {
          // Two two-candidate movers in a row, decided together against the
          // same slacks. The second one's decision depends only on the slacks
          // of its own two candidates, which the first one's move changes
          // only if one of them is that move's source or target; then it is
          // decided again after the move.
          const bool f1 = __any_sync(0xffffffffu, lane_fits(s, lane, c1, w));
          const bool f2 = __any_sync(0xffffffffu, lane_fits(s, lane, c2, w));
          const bool g1 = __any_sync(0xffffffffu, lane_fits(s, lane, nc1, nw));
          const bool g2 = __any_sync(0xffffffffu, lane_fits(s, lane, nc2, nw));
          d = f1 ? c1 : (f2 ? c2 : -1);
          int32_t d2 = g1 ? nc1 : (g2 ? nc2 : -1);
          if (d >= 0) {
            apply(pv, d, w);
            dirty = true;
            ++moves;
            if (nc1 == pv || nc1 == d || nc2 == pv || nc2 == d) {
              const bool h1 = __any_sync(0xffffffffu, lane_fits(s, lane, nc1, nw));
              const bool h2 = __any_sync(0xffffffffu, lane_fits(s, lane, nc2, nw));
              d2 = h1 ? nc1 : (h2 ? nc2 : -1);
            }
          }
          if (lane == 0) {
            dbuf[i] = d;
            dbuf[i + 1] = d2;
          }
          if (d2 >= 0) {
            apply(npv, d2, nw);
            dirty = true;
            ++moves;
          }
          ++i;
          if (i + 1 < cnt) load_next(i + 1);
          continue;
        }
        if (MODE == kCut && kn == kFast && kSharedFast) {
          // Many part slots per lane: test the two candidates against the
          // shared slack copy (one broadcast read each), rewritten only after
          // a move.
          if (dirty) {
#pragma unroll
            for (int rr = 0; rr < R; ++rr)
#pragma unroll
              for (int c = 0; c < NC; ++c) sslack[(rr * 32 + lane) * NC + c] = s.sl[rr][c];
            __syncwarp();
            dirty = false;
          }
          bool f1 = c1 >= 0, f2 = c2 >= 0;
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            f1 = f1 && (S)w[c] <= sslack[(c1 >= 0 ? c1 : 0) * NC + c];
            f2 = f2 && (S)w[c] <= sslack[(c2 >= 0 ? c2 : 0) * NC + c];
          }
          d = f1 ? c1 : (f2 ? c2 : -1);
        } else if (MODE == kCut && kn == kFast) {
          const bool f1 = __any_sync(0xffffffffu, lane_fits(s, lane, c1, w));
          const bool f2 = __any_sync(0xffffffffu, lane_fits(s, lane, c2, w));
          d = f1 ? c1 : (f2 ? c2 : -1);
        } else if (kn <= kContended && kn != kFast) {  // kContended or kLong (this form keeps the
                                                        // common kFast path short)
          if (POOL && kn == kLong && pn[i] >= 0) {
            // Gathered positive-gain candidates: the first feasible one, in
            // order, against the shared slack copy.
            if (dirty) {
#pragma unroll
              for (int rr = 0; rr < R; ++rr)
#pragma unroll
                for (int c = 0; c < NC; ++c) sslack[(rr * 32 + lane) * NC + c] = s.sl[rr][c];
              __syncwarp();
              dirty = false;
            }
            const int32_t npos = pn[i];
            const int32_t cp = npos < kPoolSlots ? npos : kPoolSlots;
            const int32_t p = lane < cp ? pc[i * kPoolSlots + lane] : -1;
            bool fits = p >= 0;
#pragma unroll
            for (int c = 0; c < NC; ++c) fits = fits && (S)w[c] <= sslack[(p >= 0 ? p : 0) * NC + c];
            const unsigned m = __ballot_sync(0xffffffffu, fits);
            if (m) {
              d = __shfl_sync(0xffffffffu, p, __ffs(m) - 1);
            } else if (npos > kPoolSlots) {
              const int32_t ig = (int32_t)(0u - (uint32_t)b.wf[i]);
              const int32_t rs = coop_scan<S, NC>(sslack, lane, b, i, kPoolSlots, b.ne[i], ig, 0, cand_p, cand_g, w,
                                                  CandChunk{0, -1});
              d = rs >= -1 ? rs : -1;
            } else {
              d = -1;
            }
          } else if (LONG)
            d = reg_decide<MODE, S, R, NC>(s, lane, b, i, k, cand_p, cand_g, w, ebits,
                                           MODE == kCut && kn == kLong ? &pre : nullptr, sslack, dirty);
          else
            d = lean_decide<MODE, S, R, NC>(s, lane, b, i, k, cand_p, cand_g, w);
        }
        if (lane == 0) dbuf[i] = d;
        if (d >= 0) {
          apply(pv, d, w);
          dirty = true;
          ++moves;
        }
      }
      __syncwarp();
      for (int32_t i = lane; i < cnt; i += 32)
        if (dbuf[i] >= 0) wo.part[wo.movers[j0 + i]] = dbuf[i];
    } else if (ch + 1 < nchunks) {
      walk_load(buf[(ch + 1) & 1], r, (ch + 1) * kWalkChunk, nm, NC, tid - 32, blockDim.x - 32);
      if (POOL)
        walk_pool_load(pool_cand(dyn, (ch + 1) & 1), pool_np(dyn, (ch + 1) & 1), r, cand_p, (ch + 1) * kWalkChunk,
                       nm, tid - 32, blockDim.x - 32);
    }
    __syncthreads();
  }
}

// Register-resident walk for k <= 32*R parts and NC <= 2 constraints. Only
// warp 0 walks: lane l holds, for parts l, l+32, ..., l+32*(R-1), the slack
// to the feasibility threshold (feas - pw) and to the overweight threshold
// (over - pw) in registers, as S (int32 when the host has checked that every
// weight and threshold fits with margin, else int64). Every lane reads the
// same mover record, so control flow stays uniform: a move into p is feasible
// iff w <= slack[p] in p's lane (one compare and one vote), the source is
// overweight iff its over-slack is negative. Cut-pass movers with at most two
// positive-gain candidates take a branch-free path (both tests and votes at
// once, then a select) and their record is fetched one mover ahead. The other
// warps stream mover records.
// Shared memory of the register walk.
template <typename S, int R, int NC>
struct WalkShared {
  WalkBuf buf[2];
  int32_t dbuf[kWalkChunk];
  unsigned ebits[R];
  S sslack[32 * R * NC];  // copy of the feasibility slacks for the long-list scans
};

template <int MODE, typename S, int R, int NC>
__device__ __forceinline__ void walk_reg_body(WalkShared<S, R, NC>& sh, const int32_t* __restrict__ nm_dev,
                                              const MoverRecs& r, int32_t k, const idx_t* __restrict__ cand_p,
                                              const idx_t* __restrict__ cand_g, long long* __restrict__ pw,
                                              const long long* __restrict__ feas_g,
                                              const long long* __restrict__ over_g, const WalkOut& wo,
                                              int32_t* __restrict__ nmoves, int32_t* __restrict__ long_flag,
                                              int32_t* dyn) {
  WalkBuf* buf = sh.buf;
  int32_t* dbuf = sh.dbuf;
  unsigned* ebits = sh.ebits;
  S* sslack = sh.sslack;
  const int32_t nm = *nm_dev;
  // The long-list version of the loop pays off when long lists are common
  // (count from k_walk_prep / k_walk_classify); both versions decide alike.
  const bool any_long = (long long)*long_flag * 16 > (long long)nm;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < R) ebits[tid] = 0u;
  PartRegs<S, R, NC> s;
  if (warp == 0) {
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const int32_t p = rr * 32 + lane;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const bool in = p < k;
        const long long x = in ? pw[p * NC + c] : 0;
        // Parts beyond k are never feasible and never overweight.
        s.sl[rr][c] = in ? (S)(feas_g[p * NC + c] - x) : (S)(-(1 << 30));
        s.ov[rr][c] = in ? (S)(over_g[p * NC + c] - x) : (S)(1 << 30);
        sslack[p * NC + c] = s.sl[rr][c];
      }
    }
  }
  if (nm > 0) {
    walk_load(buf[0], r, 0, nm, NC, tid, blockDim.x);
    if (MODE == kCut && any_long) walk_pool_load(pool_cand(dyn, 0), pool_np(dyn, 0), r, cand_p, 0, nm, tid, blockDim.x);
  }
  __syncthreads();
  int32_t moves = 0;
  if (any_long)
    walk_chunks<MODE, S, R, NC, true>(nm, r, k, cand_p, cand_g, wo, buf, dbuf, ebits, sslack, s, moves, tid, lane,
                                      warp, dyn);
  else
    walk_chunks<MODE, S, R, NC, false>(nm, r, k, cand_p, cand_g, wo, buf, dbuf, ebits, sslack, s, moves, tid,
                                       lane, warp, dyn);
  if (warp == 0) {
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const int32_t p = rr * 32 + lane;
      if (p < k)
#pragma unroll
        for (int c = 0; c < NC; ++c) pw[p * NC + c] = feas_g[p * NC + c] - (long long)s.sl[rr][c];
    }
  }
  // The next cut pass's prep accumulates into cleared bounds.
  for (int32_t x = tid; x < wo.K; x += blockDim.x) {
    wo.in_max[x] = 0;
    wo.out_max[x] = 0;
  }
  if (tid == 0) {
    *nmoves = moves;
    *long_flag = 0;  // every thread read it before the first barrier
  }
}

template <int MODE, typename S, int R, int NC>
__global__ void __launch_bounds__(kWalkThreads) k_walk_reg(const int32_t* __restrict__ nm_dev, MoverRecs r,
                                                           int32_t k, const idx_t* __restrict__ cand_p,
                                                           const idx_t* __restrict__ cand_g,
                                                           long long* __restrict__ pw,
                                                           const long long* __restrict__ feas_g,
                                                           const long long* __restrict__ over_g,
                                                           WalkOut wo, int32_t* __restrict__ nmoves,
                                                           int32_t* __restrict__ long_flag) {
  __shared__ WalkShared<S, R, NC> sh;
  extern __shared__ __align__(16) int32_t wdyn[];  // kPoolBytes
  walk_reg_body<MODE, S, R, NC>(sh, nm_dev, r, k, cand_p, cand_g, pw, feas_g, over_g, wo, nmoves, long_flag, wdyn);
}


// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <int MODE>
static int launch_gain(const DGraph& g, const idx_t* part, int k, const long long* pw0, const long long* over_thr,
                       idx_t* mover, idx_t* ncand, idx_t* wfrom, idx_t* cand_p, idx_t* cand_g, const idx_t* heavy,
                       int32_t nheavy, int32_t* ghist, cudaStream_t st, const int32_t* stop = nullptr,
                       const idx_t* only = nullptr, int block = 256, bool clear_only = false) {
  const int blocks = grid_for(g.n, block, 148 * 32 * 256 / block);
  // Algorithmic bytes of a full pass: xadj, part (own + neighbour gathers),
  // adjncy, adjwgt, mover flag.
  // (A launch limited to the vertices of `only` counts only its flag scan.)
  const double bytes = only ? 4.0 * g.n : 12.0 * g.n + (g.adjwgt ? 12.0 : 8.0) * (double)g.m;
  const int ph = MODE == kCut ? profiler().begin(kProfGain, st) : -1;
  if (g.adjwgt)
    k_gain<true, MODE><<<blocks, block, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, g.ncon, part, k, pw0, over_thr,
                                                mover, ncand, wfrom, cand_p, cand_g, stop, only, clear_only);
  else
    k_gain<false, MODE><<<blocks, block, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, g.n, g.ncon, part, k, pw0, over_thr,
                                                 mover, ncand, wfrom, cand_p, cand_g, stop, only, clear_only);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, bytes);
  if (nheavy > 0) {
    const int hb = grid_for(nheavy, 4, 256);
    if (g.adjwgt)
      k_gain_heavy<true, MODE><<<hb, 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, heavy, nheavy, g.ncon, part, k, pw0,
                                                    over_thr, mover, ncand, wfrom, cand_p, cand_g, ghist, stop,
                                                    only, clear_only);
    else
      k_gain_heavy<false, MODE><<<hb, 128, 0, st>>>(g.xadj, g.adjncy, g.adjwgt, heavy, nheavy, g.ncon, part, k, pw0,
                                                     over_thr, mover, ncand, wfrom, cand_p, cand_g, ghist, stop,
                                                     only, clear_only);
    RMB_LAUNCH_CHECK();
  }
  return ph;
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

void allow_dyn_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  RMB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.insert({kernel, dev}).second)
    RMB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

template <int MODE>
static int launch_walk(int32_t nmax, const int32_t* nm_dev, const idx_t* movers, const DGraph& g, const idx_t* part,
                        int k, const idx_t* ncand, const idx_t* wfrom, const idx_t* cand_p, const idx_t* cand_g,
                        const MoverRecs& r, long long* pw, const long long* feas, const long long* over,
                        long long* in_max, long long* out_max, int32_t* nmoves, bool small_weights,
                        int32_t* long_flag, cudaStream_t st) {
  const int32_t K = k * g.ncon;
  const int blocks = grid_for(nmax, 256);
  // in_max/out_max are zero here: cleared once per level and by every walk.
  WalkOut wo{movers, const_cast<idx_t*>(part), in_max, out_max, K};
  k_walk_prep<MODE><<<blocks, 256, 0, st>>>(nm_dev, movers, part, g.vwgt, g.ncon, g.xadj, ncand, wfrom, cand_p,
                                            cand_g, r, in_max, out_max, long_flag);
  RMB_LAUNCH_CHECK();
  if (MODE == kCut) {
    k_walk_classify<<<blocks, 256, 0, st>>>(nm_dev, g.ncon, cand_p, cand_g, r, pw, feas, in_max, out_max,
                                            long_flag);
    RMB_LAUNCH_CHECK();
  }
  const int ph = profiler().begin(kProfDecide, st);
  const int ncon = g.ncon;
#define RMB_WALK_REG(ST, RR, NCC)                                                                         \
  do {                                                                                                    \
    allow_dyn_smem((const void*)k_walk_reg<MODE, ST, RR, NCC>, kPoolBytes);                               \
    k_walk_reg<MODE, ST, RR, NCC><<<1, kWalkThreads, kPoolBytes, st>>>(nm_dev, r, k, cand_p, cand_g, pw, feas, \
                                                                       over, wo, nmoves, long_flag);       \
  } while (0)
#define RMB_WALK_REG_R(ST, NCC)                       \
  do {                                                \
    if (rr == 1) RMB_WALK_REG(ST, 1, NCC);            \
    else if (rr == 2) RMB_WALK_REG(ST, 2, NCC);       \
    else if (rr == 4) RMB_WALK_REG(ST, 4, NCC);       \
    else RMB_WALK_REG(ST, 8, NCC);                    \
  } while (0)
  if (ncon <= 2 && k <= 256) {
    const int rr = k <= 32 ? 1 : k <= 64 ? 2 : k <= 128 ? 4 : 8;
    if (small_weights) {
      if (ncon == 1) RMB_WALK_REG_R(int32_t, 1); else RMB_WALK_REG_R(int32_t, 2);
    } else {
      if (ncon == 1) RMB_WALK_REG_R(long long, 1); else RMB_WALK_REG_R(long long, 2);
    }
#undef RMB_WALK_REG_R
#undef RMB_WALK_REG
  } else if (K <= kWalkSmemParts) {
    static thread_local int attr_device = -1;  // attribute set on this device already
    int dev = 0;
    RMB_CUDA(cudaGetDevice(&dev));
    if (attr_device != dev) {
      RMB_CUDA(cudaFuncSetAttribute(k_walk<kRepair, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(sizeof(long long) * 3 * kWalkSmemParts)));
      RMB_CUDA(cudaFuncSetAttribute(k_walk<kCut, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(sizeof(long long) * 3 * kWalkSmemParts)));
      attr_device = dev;
    }
    k_walk<MODE, true><<<1, kWalkThreads, sizeof(long long) * 3 * (size_t)K, st>>>(
        nm_dev, r, g.ncon, k, cand_p, cand_g, pw, feas, over, wo, nmoves);
  } else {
    k_walk<MODE, false><<<1, kWalkThreads, 0, st>>>(nm_dev, r, g.ncon, k, cand_p, cand_g, pw, feas, over, wo,
                                                   nmoves);
  }
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 0.0);
  return ph;
}

// ---------------------------------------------------------------------------
// One level's refinement in one launch (small levels): a single block runs the
// start-of-level part weights and then, for every pass, the gain table, the
// mover compaction, the records, the classification and the walk, with block
// barriers between the steps instead of kernel boundaries. The bodies are the
// ones of the multi-kernel path, so every pass decides exactly as there.
// ---------------------------------------------------------------------------
constexpr int kFusedThreads = 512;

struct LevelRefine {
  const idx_t* xadj;
  const idx_t* adj;
  const idx_t* adjwgt;
  const idx_t* vwgt;
  int32_t n;
  int32_t k;
  int32_t niter;
  idx_t* part;
  long long* pw;
  long long* in_max;
  long long* out_max;
  const long long* feas;
  const long long* over;
  idx_t* mover;
  idx_t* ncand;
  idx_t* wfrom;
  idx_t* cand_p;
  idx_t* cand_g;
  idx_t* movers;
  MoverRecs r;
  const idx_t* heavy;
  int32_t nheavy;
  int32_t* ghist;     // [kFusedThreads / 32][k]
  int32_t* counters;  // [2 * (niter + 1)]: movers, moves per pass
  int32_t* long_flag;
};

template <bool HAS_W, int MODE, typename S, int R, int NC>
__device__ __forceinline__ void fused_pass(const LevelRefine& P, WalkShared<S, R, NC>& sh, int32_t* sw, int pass) {
  const Lanes L = block_lanes();
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  int32_t* nm_dev = P.counters + 2 * pass;
  gain_body<HAS_W, MODE>(L, P.xadj, P.adj, P.adjwgt, P.n, NC, P.part, P.k, P.pw, P.over, P.mover, P.ncand, P.wfrom,
                         P.cand_p, P.cand_g);
  if (P.nheavy > 0)
    gain_heavy_body<HAS_W, MODE>(warp, nwarps, P.ghist + (int64_t)warp * P.k, P.xadj, P.adj, P.adjwgt, P.heavy,
                                 P.nheavy, NC, P.part, P.k, P.pw, P.over, P.mover, P.ncand, P.wfrom, P.cand_p,
                                 P.cand_g);
  __syncthreads();
  block_scan_n<int32_t>(LoadNonZero{P.mover}, StoreCompact{P.mover, P.movers}, P.n, nm_dev, sw);
  __syncthreads();
  prep_body<MODE>(L, nm_dev, P.movers, P.part, P.vwgt, NC, P.xadj, P.ncand, P.wfrom, P.cand_p, P.cand_g, P.r,
                  P.in_max, P.out_max, P.long_flag);
  __syncthreads();
  if (MODE == kCut) {
    classify_body(L, nm_dev, NC, P.cand_p, P.cand_g, P.r, P.pw, P.feas, P.in_max, P.out_max, P.long_flag);
    __syncthreads();
  }
  const WalkOut wo{P.movers, P.part, P.in_max, P.out_max, P.k * NC};
  extern __shared__ __align__(16) int32_t wdyn[];  // kPoolBytes
  walk_reg_body<MODE, S, R, NC>(sh, nm_dev, P.r, P.k, P.cand_p, P.cand_g, P.pw, P.feas, P.over, wo, nm_dev + 1,
                                P.long_flag, wdyn);
  __syncthreads();
}

// A whole level in one block: part weights of the start partition, the
// repair pass and (cut_passes) the cut passes with the exact walk.
template <bool HAS_W, typename S, int R, int NC>
__device__ void level_body(const LevelRefine& P, WalkShared<S, R, NC>& sh, int32_t* sw, bool cut_passes) {
  const int32_t K = P.k * NC;
  for (int32_t x = threadIdx.x; x < K; x += blockDim.x) {
    P.pw[x] = 0;
    P.in_max[x] = 0;
    P.out_max[x] = 0;
  }
  if (threadIdx.x == 0) *P.long_flag = 0;
  __syncthreads();
  // Part weights of the start partition (src/graph/mod.rs:140-149).
  RMB_FOR(v, P.n, block_lanes()) {
    const int32_t p = P.part[v];
#pragma unroll
    for (int c = 0; c < NC; ++c) atomic_add_i64(&P.pw[p * NC + c], P.vwgt ? P.vwgt[v * NC + c] : 1);
  }
  __syncthreads();
  fused_pass<HAS_W, kRepair, S, R, NC>(P, sh, sw, 0);
  if (!cut_passes) return;
  for (int pass = 1; pass <= P.niter; ++pass) {
    // A cut pass without a move ends the level (greedy.rs:184-186); the
    // count is read by every thread after the pass's last barrier.
    if (pass >= 2 && P.counters[2 * (pass - 1) + 1] == 0) break;
    fused_pass<HAS_W, kCut, S, R, NC>(P, sh, sw, pass);
  }
}

template <bool HAS_W, typename S, int R, int NC>
__global__ void __launch_bounds__(kFusedThreads) k_refine_level(LevelRefine P) {
  __shared__ WalkShared<S, R, NC> sh;
  __shared__ int32_t sw[32];
  level_body<HAS_W, S, R, NC>(P, sh, sw, true);
}

// A step of the batched refinement: block b takes the level of jobs[b]. Its
// start partition is the best grow trial (the coarsest level: the first
// lowest cut, as the single call keeps it) or the projection of the coarser
// level's partition; then the level is refined as k_refine_level does (the
// cut passes of an admission level follow in k_batch_admit).
template <bool HAS_W, typename S, int R, int NC>
__global__ void __launch_bounds__(kFusedThreads) k_batch_level(const LevelJob* __restrict__ jobs) {
  __shared__ WalkShared<S, R, NC> sh;
  __shared__ int32_t sw[32];
  __shared__ int32_t best_trial;
  const LevelJob& J = jobs[blockIdx.x];
  if (J.trial_parts) {
    if (threadIdx.x == 0) {
      int32_t bt = 0;
      for (int32_t t = 1; t < J.trials; ++t)
        if (J.trial_cuts[t] < J.trial_cuts[bt]) bt = t;
      best_trial = bt;
    }
    __syncthreads();
    const idx_t* src = J.trial_parts + (int64_t)best_trial * J.n;
    RMB_FOR(v, J.n, block_lanes()) J.part[v] = src[v];
  } else {
    RMB_FOR(v, J.n, block_lanes()) J.part[v] = J.cpart[J.cmap[v]];
  }
  __syncthreads();
  LevelRefine P;
  P.xadj = J.xadj;
  P.adj = J.adjncy;
  P.adjwgt = J.adjwgt;
  P.vwgt = J.vwgt;
  P.n = J.n;
  P.k = J.k;
  P.niter = J.niter;
  P.part = J.part;
  P.pw = J.pw;
  P.in_max = J.in_max;
  P.out_max = J.out_max;
  P.feas = J.feas;
  P.over = J.over;
  P.mover = J.mover;
  P.ncand = J.ncand;
  P.wfrom = J.wfrom;
  P.cand_p = J.cand_p;
  P.cand_g = J.cand_g;
  P.movers = J.movers;
  P.r.pv = J.rec_pv;
  P.r.ne = J.rec_ne;
  P.r.wf = J.rec_wf;
  P.r.coff = J.rec_coff;
  P.r.known = J.rec_known;
  P.r.cp = J.rec_cp;
  P.r.cg = J.rec_cg;
  P.r.vw = J.rec_vw;
  P.r.np = J.rec_np;
  P.heavy = J.heavy;
  P.nheavy = J.nheavy;
  P.ghist = J.ghist;
  P.counters = J.counters;
  P.long_flag = J.long_flag;
  level_body<HAS_W, S, R, NC>(P, sh, sw, J.admit == 0);
}

template <bool HAS_W, typename S, int NC>
static void launch_fused_r(const LevelRefine& P, cudaStream_t st) {
  const int k = P.k;
  auto kern = k <= 32 ? k_refine_level<HAS_W, S, 1, NC>
              : k <= 64 ? k_refine_level<HAS_W, S, 2, NC>
              : k <= 128 ? k_refine_level<HAS_W, S, 4, NC> : k_refine_level<HAS_W, S, 8, NC>;
  allow_dyn_smem((const void*)kern, kPoolBytes);
  kern<<<1, kFusedThreads, kPoolBytes, st>>>(P);
}

template <bool HAS_W>
static void launch_fused(const LevelRefine& P, int ncon, bool small_weights, cudaStream_t st) {
  if (small_weights) {
    if (ncon == 1) launch_fused_r<HAS_W, int32_t, 1>(P, st); else launch_fused_r<HAS_W, int32_t, 2>(P, st);
  } else {
    if (ncon == 1) launch_fused_r<HAS_W, long long, 1>(P, st); else launch_fused_r<HAS_W, long long, 2>(P, st);
  }
}

template <bool HAS_W, typename S, int NC>
static void launch_batch_r(const LevelJob* d_jobs, int njobs, int k, cudaStream_t st) {
  auto kern = k <= 32 ? k_batch_level<HAS_W, S, 1, NC>
              : k <= 64 ? k_batch_level<HAS_W, S, 2, NC>
              : k <= 128 ? k_batch_level<HAS_W, S, 4, NC> : k_batch_level<HAS_W, S, 8, NC>;
  allow_dyn_smem((const void*)kern, kPoolBytes);
  kern<<<njobs, kFusedThreads, kPoolBytes, st>>>(d_jobs);
}

void batch_level_launch(const LevelJob* d_jobs, int njobs, bool has_w, bool small_weights, int k, int ncon,
                        cudaStream_t st) {
  if (njobs <= 0) return;
  if (ncon < 1 || ncon > 2 || k > 256) throw Error(-4, "batched level refinement: ncon above 2 or k above 256");
  const int ph = profiler().begin(kProfLevel, st);
  if (has_w) {
    if (small_weights) {
      if (ncon == 1) launch_batch_r<true, int32_t, 1>(d_jobs, njobs, k, st);
      else launch_batch_r<true, int32_t, 2>(d_jobs, njobs, k, st);
    } else {
      if (ncon == 1) launch_batch_r<true, long long, 1>(d_jobs, njobs, k, st);
      else launch_batch_r<true, long long, 2>(d_jobs, njobs, k, st);
    }
  } else {
    if (small_weights) {
      if (ncon == 1) launch_batch_r<false, int32_t, 1>(d_jobs, njobs, k, st);
      else launch_batch_r<false, int32_t, 2>(d_jobs, njobs, k, st);
    } else {
      if (ncon == 1) launch_batch_r<false, long long, 1>(d_jobs, njobs, k, st);
      else launch_batch_r<false, long long, 2>(d_jobs, njobs, k, st);
    }
  }
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 0.0);
}

RefineStats greedy_refine(const DGraph& g, idx_t* part, const RefineParams& rp, const idx_t* heavy, int32_t nheavy,
                          Arena& arena, cudaStream_t st, int32_t* h_scratch) {
  if (g.ncon > kMaxCon) throw Error(-2, "ncon above the supported maximum of 8");
  RefineStats stats;
  const int k = rp.k;
  const int32_t K = k * g.ncon;
  Arena::Mark mk = arena.mark();
  long long* pw = arena.alloc<long long>((size_t)K);
  long long* in_max = arena.alloc<long long>((size_t)K);
  long long* out_max = arena.alloc<long long>((size_t)K);
  idx_t* mover = arena.alloc<idx_t>((size_t)g.n);
  idx_t* ncand = arena.alloc<idx_t>((size_t)g.n);
  idx_t* wfrom = arena.alloc<idx_t>((size_t)g.n);
  idx_t* cand_p = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* cand_g = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* movers = arena.alloc<idx_t>((size_t)g.n);
  // Per pass: [2*pass] movers, [2*pass+1] moves.
  int32_t* counters = arena.alloc<int32_t>(2 * ((size_t)rp.niter + 1));
  // Number of a pass's movers with more candidates than the inline slots,
  // counted by prep/classify; the register walk reads and clears it.
  int32_t* long_flag = arena.alloc<int32_t>(1);
  RMB_CUDA(cudaMemsetAsync(long_flag, 0, sizeof(int32_t), st));
  RMB_CUDA(cudaMemsetAsync(in_max, 0, sizeof(long long) * (size_t)K, st));
  RMB_CUDA(cudaMemsetAsync(out_max, 0, sizeof(long long) * (size_t)K, st));
  MoverRecs r;
  r.pv = arena.alloc<int32_t>((size_t)g.n);
  r.ne = arena.alloc<int32_t>((size_t)g.n);
  r.wf = arena.alloc<int32_t>((size_t)g.n);
  r.coff = arena.alloc<int32_t>((size_t)g.n);
  r.known = arena.alloc<int32_t>((size_t)g.n);
  r.cp = arena.alloc<int32_t>((size_t)g.n * kInline);
  r.cg = arena.alloc<int32_t>((size_t)g.n * kInline);
  r.vw = arena.alloc<int32_t>((size_t)g.n * g.ncon);
  r.np = arena.alloc<int32_t>((size_t)g.n);
  // One block refines a level well while its edges stay few; a denser level of
  // the same size does better spread over the device.
  const bool fused = rp.fused_max_n > 0 && g.n <= rp.fused_max_n &&
                     g.m <= (int64_t)rp.fused_edge_factor * rp.fused_max_n && k <= 256 &&
                     g.ncon <= 2;
  int32_t* ghist = nullptr;
  if (nheavy > 0 && (fused || k > kGainHist))
    ghist = arena.alloc<int32_t>((size_t)k * (fused ? kFusedThreads / 32 : 256 * 4));
  // Cut passes of large levels decide by parallel admission (admit.cu).
  const bool admit = !fused && g.n > rp.exact_max_n && admit_supported(k, g.ncon);
  AdmitScratch as;
  int32_t* rounds = nullptr;
  idx_t* touched[2] = {nullptr, nullptr};
  if (admit) {
    as.tgt = arena.alloc<int32_t>((size_t)g.n);
    as.src = arena.alloc<int32_t>((size_t)g.n);
    as.w = arena.alloc<int32_t>((size_t)g.n * g.ncon);
    as.rank = arena.alloc<int32_t>((size_t)g.n);
    as.pref = arena.alloc<long long>((size_t)g.n * g.ncon);
    as.gsrc = arena.alloc<int32_t>((size_t)g.n);
    as.out = arena.alloc<long long>((size_t)K);
    as.cut = arena.alloc<int32_t>((size_t)k);
    RMB_CUDA(cudaMemsetAsync(as.out, 0, sizeof(long long) * (size_t)K, st));
    rounds = arena.alloc<int32_t>((size_t)rp.niter + 1);
    // Incremental gain tables: after the first cut pass, a pass recomputes
    // only the vertices the previous pass moved and their neighbours (the
    // other entries are unchanged); each pass's moves flag the next pass's
    // set, alternating between two flag arrays.
    for (int b = 0; b < 2; ++b) {
      touched[b] = arena.alloc<idx_t>((size_t)g.n);
      RMB_CUDA(cudaMemsetAsync(touched[b], 0, sizeof(idx_t) * (size_t)g.n, st));
    }
  }
  std::vector<int> walk_handles, gain_handles;
  if (fused) {
    LevelRefine P;
    P.xadj = g.xadj;
    P.adj = g.adjncy;
    P.adjwgt = g.adjwgt;
    P.vwgt = g.vwgt;
    P.n = g.n;
    P.k = k;
    P.niter = rp.niter;
    P.part = part;
    P.pw = pw;
    P.in_max = in_max;
    P.out_max = out_max;
    P.feas = rp.feas_max;
    P.over = rp.over_thr;
    P.mover = mover;
    P.ncand = ncand;
    P.wfrom = wfrom;
    P.cand_p = cand_p;
    P.cand_g = cand_g;
    P.movers = movers;
    P.r = r;
    P.heavy = heavy;
    P.nheavy = nheavy;
    P.ghist = ghist;
    P.counters = counters;
    P.long_flag = long_flag;
    const int ph = profiler().begin(kProfLevel, st);
    if (g.adjwgt) launch_fused<true>(P, g.ncon, rp.small_weights, st);
    else launch_fused<false>(P, g.ncon, rp.small_weights, st);
    RMB_LAUNCH_CHECK();
    profiler().end(ph, st, (rp.niter + 1) * (12.0 * g.n + (g.adjwgt ? 12.0 : 8.0) * (double)g.m));
  } else {
  partition_weights_only(g, part, k, pw, st);

  // The reference stops the cut passes at the first pass without a move
  // (greedy.rs:184-186). Such a pass leaves part and pw unchanged, so every
  // later pass would again find the same movers and make no move: running all
  // niter passes gives the same result, and the whole level is queued without
  // waiting for the host.
  for (int pass = 0; pass <= rp.niter; ++pass) {
    const int mode = pass == 0 ? kRepair : kCut;
    int32_t* nm_dev = counters + 2 * pass;
    // From the second cut pass on, a previous cut pass without a move makes
    // this one empty on the device (same result as the reference's break).
    const int32_t* stop = pass >= 2 ? counters + 2 * (pass - 1) + 1 : nullptr;
    if (mode == kRepair)
      launch_gain<kRepair>(g, part, k, pw, rp.over_thr, mover, ncand, wfrom, cand_p, cand_g, heavy, nheavy, ghist, st);
    else
      gain_handles.push_back(launch_gain<kCut>(g, part, k, pw, rp.over_thr, mover, ncand, wfrom, cand_p, cand_g,
                                               heavy, nheavy, ghist, st, stop,
                                               admit && pass >= 2 ? touched[(pass - 1) & 1] : nullptr,
                                               rp.gain_block, admit && pass >= 2));
    compact_flags(mover, g.n, movers, nm_dev, arena, st);
    if (mode == kRepair)
      walk_handles.push_back(launch_walk<kRepair>(g.n, nm_dev, movers, g, part, k, ncand, wfrom, cand_p, cand_g, r,
                                                  pw, rp.feas_max, rp.over_thr, in_max, out_max, nm_dev + 1,
                                                  rp.small_weights, long_flag, st));
    else if (admit)
      walk_handles.push_back(admit_cut_pass(g, k, g.n, nm_dev, movers, ncand, wfrom, cand_p, cand_g, part, pw,
                                            rp.feas_max, nm_dev + 1, rounds + pass, as, st, true,
                                            pass + 1 <= rp.niter ? touched[pass & 1] : nullptr));
    else
      walk_handles.push_back(launch_walk<kCut>(g.n, nm_dev, movers, g, part, k, ncand, wfrom, cand_p, cand_g, r, pw,
                                               rp.feas_max, rp.over_thr, in_max, out_max, nm_dev + 1,
                                               rp.small_weights, long_flag, st));
  }
  }
  static const bool trace = std::getenv("RMETIS_B200_TRACE") != nullptr;
  if (profiler().on && !fused) {
    // The walk reads one record per mover (pv, ne, w_from, offset, known,
    // 4 inline candidates and gains, ncon weights) and writes its decision.
    RMB_CUDA(cudaMemcpyAsync(h_scratch, counters, sizeof(int32_t) * 2 * ((size_t)rp.niter + 1),
                             cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    const double rec_bytes = 4.0 * (5 + 2 * kInline + g.ncon) + 4.0;
    // An admission pass reads per mover its id, part, row offset, candidate
    // count, w_from, its first candidate pair and weights, and writes its
    // target, rank, grouped slot and running sums.
    const double adm_bytes = 4.0 * (7 + g.ncon) + 4.0 * (4 + 2 * g.ncon);
    for (int pass = 0; pass <= rp.niter; ++pass)
      profiler().set_bytes(walk_handles[pass], (admit && pass > 0 ? adm_bytes : rec_bytes) * h_scratch[2 * pass]);
    // A cut pass emptied by the one before it only clears the mover flags.
    for (int pass = 2; pass <= rp.niter; ++pass)
      if (h_scratch[2 * (pass - 1) + 1] == 0) {
        profiler().set_bytes(gain_handles[pass - 1], 4.0 * g.n);
        for (int q = pass; q <= rp.niter; ++q) h_scratch[2 * q + 1] = 0;
      }
  }
  if (trace || rp.collect_stats) {
    RMB_CUDA(cudaMemcpyAsync(h_scratch, counters, sizeof(int32_t) * 2 * ((size_t)rp.niter + 1),
                             cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    for (int pass = 0; pass <= rp.niter; ++pass) {
      const int32_t nm = h_scratch[2 * pass], nmoves = h_scratch[2 * pass + 1];
      stats.passes += 1;
      stats.movers += nm;
      stats.moves += nmoves;
      stats.decide_iters += 1;
      if (trace) {
        int32_t rr = 0;
        if (admit && pass > 0) RMB_CUDA(cudaMemcpy(&rr, rounds + pass, sizeof(int32_t), cudaMemcpyDeviceToHost));
        std::fprintf(stderr, "refine n=%d m=%lld k=%d pass=%d mode=%d movers=%d moves=%d admit_rounds=%d\n", g.n,
                     (long long)g.m, k, pass, pass == 0 ? 0 : 1, nm, nmoves, rr);
      }
      if (pass > 0 && nmoves == 0) break;
    }
  }
  arena.reset_to(mk);
  return stats;
}

// ---------------------------------------------------------------------------
// k-way FM refinement (src/refine/fm_kway.rs:12-158).
//
// The reference pops boundary vertices from a priority queue keyed by the
// gain of their best move (the adjacent part with the largest positive gain,
// lowest id on ties), moves each one whose target stays feasible, locks it
// for the rest of the pass and re-evaluates its unlocked neighbours; a vertex
// whose move is infeasible leaves the queue until a neighbour moves. Every
// move has a positive exact gain, so the cut falls with each move and the
// reference's rollback to the best prefix never undoes one. Passes repeat
// while one moves something (at most niter).
//
// Here a pass runs in rounds. Each round brings the gain table up to date
// with the current partition (k_gain: every vertex's best move, exact; after
// the first round of a pass only for the vertices next to the last round's
// moves, the others' entries being unchanged), and selects
// every free vertex whose move beats the moves of all its free neighbours in
// the queue's order (gain, then lower id) among its neighbours in other
// parts: local maxima, so no two movers of a round in different parts are
// adjacent and the cut falls at least by the sum of the round's gains (two
// adjacent movers of one part can only do better than their gains say). The
// selected moves go through the greedy walk with
// one candidate each (k_walk_prep/classify/walk_reg, cut mode: the candidate
// if it stays feasible under the part weights of the moves before it, in
// vertex order), which applies them to part and pw. A selected vertex that
// moved is locked; one that did not is dropped until a neighbour moves. Only
// vertices within two hops of a round's moves and drops can change their
// selection in the next round, so later rounds select among those alone. The
// pass ends at a round that selects nothing. Cut monotonicity, the
// destination-only feasibility test and the fixed point at the end (no free
// vertex with a feasible positive-gain move) are the reference's; the order
// of moves among non-adjacent vertices differs, so partitions are compared
// by quality, not bit for bit.
// ---------------------------------------------------------------------------
constexpr int kFmFree = 0, kFmLocked = 1, kFmDropped = 2;
constexpr int kFmRoundsPerCheck = 4;   // rounds queued between two reads of the round counters
constexpr int kFmMaxRounds = 512;      // bound on the rounds of one pass

__device__ __forceinline__ int32_t fm_gain_of(int32_t v, const idx_t* __restrict__ xadj,
                                              const idx_t* __restrict__ mover, const idx_t* __restrict__ ncand,
                                              const idx_t* __restrict__ cand_g, const int32_t* __restrict__ state) {
  if (state[v] != kFmFree || !mover[v] || ncand[v] <= 0) return 0;
  const int32_t g = cand_g[xadj[v]];
  return g > 0 ? g : 0;
}

// sel[v] = 1 when v's best move has a positive gain above the move of every
// free neighbour in another part (equal gains: the lower id first). Two
// movers of the same part may move together: the edge between them was
// counted as a loss by both gains, and whatever parts they reach it costs at
// most that, so the cut falls at least by the sum of the gains. sel doubles
// as the candidate count the walk reads (the best move only).
// active (rounds after the first of a pass): only vertices within two hops
// of the last round's changes can change their selection; the others were
// not selected then and are not now.
__device__ void fm_select_body(Lanes L, int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                               const idx_t* __restrict__ part, const idx_t* __restrict__ mover,
                               const idx_t* __restrict__ ncand, const idx_t* __restrict__ cand_g,
                               const int32_t* __restrict__ state, const idx_t* __restrict__ active,
                               idx_t* __restrict__ sel) {
  RMB_FOR(v, n, L) {
    if (active && !active[v]) {
      sel[v] = 0;
      continue;
    }
    const int32_t gv = fm_gain_of((int32_t)v, xadj, mover, ncand, cand_g, state);
    int32_t out = 0;
    if (gv > 0) {
      out = 1;
      const int32_t pv = part[v];
      const int32_t s = xadj[v], e = xadj[v + 1];
      // Four neighbours at a time: their ids and parts are gathered together,
      // then compared in row order (the first better one ends the scan).
      for (int32_t j0 = s; j0 < e && out; j0 += 4) {
        int32_t uq[4], pq[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) uq[q] = j0 + q < e ? adj[j0 + q] : -1;
#pragma unroll
        for (int q = 0; q < 4; ++q) pq[q] = uq[q] >= 0 ? part[uq[q]] : pv;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int32_t u = uq[q];
          if (u < 0 || u == (int32_t)v || pq[q] == pv) continue;
          const int32_t gu = fm_gain_of(u, xadj, mover, ncand, cand_g, state);
          if (gu > gv || (gu == gv && u < (int32_t)v)) {
            out = 0;
            break;
          }
        }
      }
    }
    sel[v] = out;
  }
}

__global__ void k_fm_select(int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                            const idx_t* __restrict__ part, const idx_t* __restrict__ mover,
                            const idx_t* __restrict__ ncand, const idx_t* __restrict__ cand_g,
                            const int32_t* __restrict__ state, const idx_t* __restrict__ active,
                            idx_t* __restrict__ sel) {
  fm_select_body(grid_lanes(), n, xadj, adj, part, mover, ncand, cand_g, state, active, sel);
}

// After the walk: a selected vertex that took its move is locked and frees
// its dropped neighbours that were not selected this round (the reference
// re-queues the unlocked neighbours of a moved vertex); a selected vertex
// that did not move is dropped. Each selected vertex's state is written by
// its own thread only, so the result does not depend on thread order.
// changed (for the next round; zero on entry): every vertex whose best move
// may differ now (a moved vertex and its neighbours) or whose state changed
// (a dropped one).
__device__ void fm_after_body(Lanes L, const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                              const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                              const idx_t* __restrict__ part, const idx_t* __restrict__ cand_p,
                              const idx_t* __restrict__ sel, int32_t* __restrict__ state,
                              idx_t* __restrict__ changed) {
  const int32_t nm = *nm_dev;
  RMB_FOR(i, nm, L) {
    const int32_t v = movers[i];
    const int32_t s = xadj[v], e = xadj[v + 1];
    changed[v] = 1;
    if (part[v] == cand_p[s]) {
      state[v] = kFmLocked;
      for (int32_t j = s; j < e; ++j) {
        const int32_t u = adj[j];
        changed[u] = 1;
        if (!sel[u] && state[u] == kFmDropped) state[u] = kFmFree;
      }
    } else {
      state[v] = kFmDropped;
    }
  }
}

__global__ void k_fm_after(const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                           const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                           const idx_t* __restrict__ part, const idx_t* __restrict__ cand_p,
                           const idx_t* __restrict__ sel, int32_t* __restrict__ state,
                           idx_t* __restrict__ changed) {
  fm_after_body(grid_lanes(), nm_dev, movers, xadj, adj, part, cand_p, sel, state, changed);
}

// k_fm_after for a round decided by admission, with the moves applied here:
// an admitted mover moves and is locked, and frees its dropped unselected
// neighbours; a mover that was not admitted is dropped.
__global__ void k_fm_apply_after(const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                                 const int32_t* __restrict__ tgt, const int32_t* __restrict__ rank,
                                 const int32_t* __restrict__ cut, const idx_t* __restrict__ xadj,
                                 const idx_t* __restrict__ adj, idx_t* __restrict__ part, const idx_t* __restrict__ sel,
                                 int32_t* __restrict__ state, idx_t* __restrict__ changed) {
  const int32_t nm = *nm_dev;
  RMB_GRID_STRIDE(i, nm) {
    const int32_t v = movers[i];
    const int32_t t = tgt[i];
    changed[v] = 1;
    if (t >= 0 && rank[i] < cut[t]) {
      part[v] = t;
      state[v] = kFmLocked;
      for (int32_t j = xadj[v]; j < xadj[v + 1]; ++j) {
        const int32_t u = adj[j];
        changed[u] = 1;
        if (!sel[u] && state[u] == kFmDropped) state[u] = kFmFree;
      }
    } else {
      state[v] = kFmDropped;
    }
  }
}

// active_next = changed and their neighbours (zero on entry). Also clears the
// flags the round just used (changed_cur, active_cur) for the round after next.
__device__ void fm_spread_body(Lanes L, int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                               const idx_t* __restrict__ changed, idx_t* __restrict__ active_next,
                               idx_t* __restrict__ changed_cur, idx_t* __restrict__ active_cur) {
  RMB_FOR(v, n, L) {
    changed_cur[v] = 0;
    active_cur[v] = 0;
    if (!changed[v]) continue;
    active_next[v] = 1;
    for (int32_t j = xadj[v]; j < xadj[v + 1]; ++j) active_next[adj[j]] = 1;
  }
}

__global__ void k_fm_spread(int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                            const idx_t* __restrict__ changed, idx_t* __restrict__ active_next,
                            idx_t* __restrict__ changed_cur, idx_t* __restrict__ active_cur) {
  fm_spread_body(grid_lanes(), n, xadj, adj, changed, active_next, changed_cur, active_cur);
}

// A whole FM level in one block (levels of at most fused_max_n vertices): the
// passes and rounds of fm_refine below, with the same bodies and decisions,
// the host loop replaced by the block's own loop. Per pass it writes the
// number of rounds that selected movers, the movers and the moves to
// pass_stats[3 * pass ..].
struct FmLevel {
  LevelRefine P;        // gain tables, walk records and part weights
  idx_t* sel;
  idx_t* zero;
  int32_t* state;
  idx_t* flags[2][2];   // per round parity: [0] changed, [1] active
  int32_t* rcount;      // [2 * kFmMaxRounds]: selected movers and moves per round
  long long* pass_stats;  // [niter][3]
};

template <bool HAS_W, typename S, int R, int NC>
__global__ void __launch_bounds__(kFusedThreads) k_fm_level(FmLevel F) {
  __shared__ WalkShared<S, R, NC> sh;
  __shared__ int32_t sw[32];
  extern __shared__ __align__(16) int32_t wdyn[];  // kPoolBytes
  const LevelRefine& P = F.P;
  const Lanes L = block_lanes();
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int32_t K = P.k * NC;
  for (int32_t x = threadIdx.x; x < K; x += blockDim.x) {
    P.pw[x] = 0;
    P.in_max[x] = 0;
    P.out_max[x] = 0;
  }
  if (threadIdx.x == 0) *P.long_flag = 0;
  RMB_FOR(v, P.n, L) F.zero[v] = 0;
  __syncthreads();
  RMB_FOR(v, P.n, L) {
    const int32_t p = P.part[v];
#pragma unroll
    for (int c = 0; c < NC; ++c) atomic_add_i64(&P.pw[p * NC + c], P.vwgt ? P.vwgt[v * NC + c] : 1);
  }
  __syncthreads();
  const WalkOut wo{P.movers, P.part, P.in_max, P.out_max, P.k * NC};
  for (int pass = 0; pass < P.niter; ++pass) {  // fm_kway.rs:23-27
    RMB_FOR(v, P.n, L) {
      F.state[v] = kFmFree;
      F.flags[0][0][v] = 0;
      F.flags[0][1][v] = 0;
      F.flags[1][0][v] = 0;
      F.flags[1][1][v] = 0;
    }
    __syncthreads();
    long long moves = 0, movers = 0, rounds_used = 0;
    for (int r = 0; r < kFmMaxRounds; ++r) {
      idx_t* const* cur = F.flags[r & 1];
      idx_t* const* nxt = F.flags[(r + 1) & 1];
      int32_t* nm_dev = F.rcount + 2 * r;
      const idx_t* only = r > 0 ? cur[0] : nullptr;
      gain_body<HAS_W, kCut>(L, P.xadj, P.adj, P.adjwgt, P.n, NC, P.part, P.k, nullptr, nullptr, P.mover, P.ncand,
                             P.wfrom, P.cand_p, P.cand_g, only, false);
      if (P.nheavy > 0)
        gain_heavy_body<HAS_W, kCut>(warp, nwarps, P.ghist + (int64_t)warp * P.k, P.xadj, P.adj, P.adjwgt, P.heavy,
                                     P.nheavy, NC, P.part, P.k, nullptr, nullptr, P.mover, P.ncand, P.wfrom,
                                     P.cand_p, P.cand_g, only, false);
      __syncthreads();
      fm_select_body(L, P.n, P.xadj, P.adj, P.part, P.mover, P.ncand, P.cand_g, F.state, r > 0 ? cur[1] : nullptr,
                     F.sel);
      __syncthreads();
      block_scan_n<int32_t>(LoadNonZero{F.sel}, StoreCompact{F.sel, P.movers}, P.n, nm_dev, sw);
      __syncthreads();
      const int32_t nm = *nm_dev;
      if (nm == 0) break;  // nothing selected: the pass is over
      // The selected moves through the walk, one candidate each (sel is the
      // candidate count, w_from 0), as launch_walk<kCut> decides them.
      prep_body<kCut>(L, nm_dev, P.movers, P.part, P.vwgt, NC, P.xadj, F.sel, F.zero, P.cand_p, P.cand_g, P.r,
                      P.in_max, P.out_max, P.long_flag);
      __syncthreads();
      classify_body(L, nm_dev, NC, P.cand_p, P.cand_g, P.r, P.pw, P.feas, P.in_max, P.out_max, P.long_flag);
      __syncthreads();
      walk_reg_body<kCut, S, R, NC>(sh, nm_dev, P.r, P.k, P.cand_p, P.cand_g, P.pw, P.feas, P.over, wo, nm_dev + 1,
                                    P.long_flag, wdyn);
      __syncthreads();
      fm_after_body(L, nm_dev, P.movers, P.xadj, P.adj, P.part, P.cand_p, F.sel, F.state, nxt[0]);
      __syncthreads();
      fm_spread_body(L, P.n, P.xadj, P.adj, nxt[0], nxt[1], cur[0], cur[1]);
      __syncthreads();
      moves += nm_dev[1];
      movers += nm;
      rounds_used += 1;
    }
    if (threadIdx.x == 0) {
      F.pass_stats[3 * pass] = rounds_used;
      F.pass_stats[3 * pass + 1] = movers;
      F.pass_stats[3 * pass + 2] = moves;
    }
    __syncthreads();
    if (moves == 0) break;  // fm_kway_pass returned false
  }
}

template <bool HAS_W, typename S, int NC>
static void launch_fm_level_r(const FmLevel& F, cudaStream_t st) {
  const int k = F.P.k;
  auto kern = k <= 32 ? k_fm_level<HAS_W, S, 1, NC>
              : k <= 64 ? k_fm_level<HAS_W, S, 2, NC>
              : k <= 128 ? k_fm_level<HAS_W, S, 4, NC> : k_fm_level<HAS_W, S, 8, NC>;
  allow_dyn_smem((const void*)kern, kPoolBytes);
  kern<<<1, kFusedThreads, kPoolBytes, st>>>(F);
}

template <bool HAS_W>
static void launch_fm_level(const FmLevel& F, int ncon, bool small_weights, cudaStream_t st) {
  if (small_weights) {
    if (ncon == 1) launch_fm_level_r<HAS_W, int32_t, 1>(F, st); else launch_fm_level_r<HAS_W, int32_t, 2>(F, st);
  } else {
    if (ncon == 1) launch_fm_level_r<HAS_W, long long, 1>(F, st); else launch_fm_level_r<HAS_W, long long, 2>(F, st);
  }
}

RefineStats fm_refine(const DGraph& g, idx_t* part, const RefineParams& rp, const idx_t* heavy, int32_t nheavy,
                      Arena& arena, cudaStream_t st, int32_t* h_scratch) {
  if (g.ncon > kMaxCon) throw Error(-2, "ncon above the supported maximum of 8");
  RefineStats stats;
  const int k = rp.k;
  const int32_t K = k * g.ncon;
  Arena::Mark mk = arena.mark();
  long long* pw = arena.alloc<long long>((size_t)K);
  long long* in_max = arena.alloc<long long>((size_t)K);
  long long* out_max = arena.alloc<long long>((size_t)K);
  idx_t* mover = arena.alloc<idx_t>((size_t)g.n);
  idx_t* ncand = arena.alloc<idx_t>((size_t)g.n);
  idx_t* wfrom = arena.alloc<idx_t>((size_t)g.n);
  idx_t* zero = arena.alloc<idx_t>((size_t)g.n);
  idx_t* sel = arena.alloc<idx_t>((size_t)g.n);
  int32_t* state = arena.alloc<int32_t>((size_t)g.n);
  // Two sets of round flags, used alternately: [0] changed, [1] active.
  idx_t* flags[2][2];
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 2; ++f) flags[b][f] = arena.alloc<idx_t>((size_t)g.n);
  idx_t* cand_p = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* cand_g = arena.alloc<idx_t>((size_t)g.m + 1);
  idx_t* movers = arena.alloc<idx_t>((size_t)g.n);
  // Per round: [2*r] selected movers, [2*r+1] moves.
  int32_t* counters = arena.alloc<int32_t>(2 * (size_t)kFmMaxRounds);
  int32_t* long_flag = arena.alloc<int32_t>(1);
  MoverRecs r;
  r.pv = arena.alloc<int32_t>((size_t)g.n);
  r.ne = arena.alloc<int32_t>((size_t)g.n);
  r.wf = arena.alloc<int32_t>((size_t)g.n);
  r.coff = arena.alloc<int32_t>((size_t)g.n);
  r.known = arena.alloc<int32_t>((size_t)g.n);
  r.cp = arena.alloc<int32_t>((size_t)g.n * kInline);
  r.cg = arena.alloc<int32_t>((size_t)g.n * kInline);
  r.vw = arena.alloc<int32_t>((size_t)g.n * g.ncon);
  r.np = arena.alloc<int32_t>((size_t)g.n);
  int32_t* ghist = nullptr;
  if (nheavy > 0 && k > kGainHist) ghist = arena.alloc<int32_t>((size_t)k * 256 * 4);
  // The moves of a round on a large level are decided by parallel admission
  // (admit.cu) instead of the sequential walk: every selected vertex is a
  // local maximum whose move alone is feasible or not, and a part admits the
  // longest prefix of its selected in-moves that fits its limit given the
  // moves out of it.
  const bool admit = g.n > rp.exact_max_n && admit_supported(k, g.ncon);
  AdmitScratch as;
  if (admit) {
    as.tgt = arena.alloc<int32_t>((size_t)g.n);
    as.src = arena.alloc<int32_t>((size_t)g.n);
    as.w = arena.alloc<int32_t>((size_t)g.n * g.ncon);
    as.rank = arena.alloc<int32_t>((size_t)g.n);
    as.pref = arena.alloc<long long>((size_t)g.n * g.ncon);
    as.gsrc = arena.alloc<int32_t>((size_t)g.n);
    as.out = arena.alloc<long long>((size_t)K);
    as.cut = arena.alloc<int32_t>((size_t)k);
    RMB_CUDA(cudaMemsetAsync(as.out, 0, sizeof(long long) * (size_t)K, st));
  }
  // A small level runs all its passes and rounds in one single-block launch.
  // (A round of the multi-kernel form costs about ten launches whatever the
  // level's size, and a round's work is mostly the vertices next to its
  // moves, so dense levels qualify too.)
  const bool fused = rp.fm_fused_max_n > 0 && g.n <= rp.fm_fused_max_n && k <= 256 && g.ncon <= 2 && !admit;
  if (fused) {
    FmLevel F;
    F.P.xadj = g.xadj;
    F.P.adj = g.adjncy;
    F.P.adjwgt = g.adjwgt;
    F.P.vwgt = g.vwgt;
    F.P.n = g.n;
    F.P.k = k;
    F.P.niter = rp.niter;
    F.P.part = part;
    F.P.pw = pw;
    F.P.in_max = in_max;
    F.P.out_max = out_max;
    F.P.feas = rp.feas_max;
    F.P.over = rp.over_thr;
    F.P.mover = mover;
    F.P.ncand = ncand;
    F.P.wfrom = wfrom;
    F.P.cand_p = cand_p;
    F.P.cand_g = cand_g;
    F.P.movers = movers;
    F.P.r = r;
    F.P.heavy = heavy;
    F.P.nheavy = nheavy;
    F.P.ghist = nheavy > 0 ? arena.alloc<int32_t>((size_t)k * (kFusedThreads / 32)) : nullptr;
    F.P.counters = nullptr;
    F.P.long_flag = long_flag;
    F.sel = sel;
    F.zero = zero;
    F.state = state;
    for (int b = 0; b < 2; ++b)
      for (int f = 0; f < 2; ++f) F.flags[b][f] = flags[b][f];
    F.rcount = counters;
    F.pass_stats = arena.alloc<long long>(3 * (size_t)std::max(rp.niter, 1));
    RMB_CUDA(cudaMemsetAsync(F.pass_stats, 0, sizeof(long long) * 3 * (size_t)std::max(rp.niter, 1), st));
    const int ph = profiler().begin(kProfLevel, st);
    if (g.adjwgt) launch_fm_level<true>(F, g.ncon, rp.small_weights, st);
    else launch_fm_level<false>(F, g.ncon, rp.small_weights, st);
    RMB_LAUNCH_CHECK();
    profiler().end(ph, st, 0.0);
    if (rp.collect_stats) {
      std::vector<long long> ps(3 * (size_t)std::max(rp.niter, 1));
      RMB_CUDA(cudaMemcpyAsync(ps.data(), F.pass_stats, sizeof(long long) * ps.size(), cudaMemcpyDeviceToHost, st));
      RMB_CUDA(cudaStreamSynchronize(st));
      for (int pass = 0; pass < rp.niter; ++pass) {
        stats.passes += 1;
        stats.decide_iters += (int)ps[3 * pass];
        stats.movers += ps[3 * pass + 1];
        stats.moves += ps[3 * pass + 2];
        if (ps[3 * pass + 2] == 0) break;
      }
    }
    arena.reset_to(mk);
    return stats;
  }
  RMB_CUDA(cudaMemsetAsync(long_flag, 0, sizeof(int32_t), st));
  RMB_CUDA(cudaMemsetAsync(in_max, 0, sizeof(long long) * (size_t)K, st));
  RMB_CUDA(cudaMemsetAsync(out_max, 0, sizeof(long long) * (size_t)K, st));
  RMB_CUDA(cudaMemsetAsync(zero, 0, sizeof(idx_t) * (size_t)g.n, st));
  partition_weights_only(g, part, k, pw, st);
  const int nb = grid_for(g.n, 256);
  std::vector<int32_t> hc(2 * (size_t)kFmMaxRounds);
  for (int pass = 0; pass < rp.niter; ++pass) {  // fm_kway.rs:23-27
    RMB_CUDA(cudaMemsetAsync(state, 0, sizeof(int32_t) * (size_t)g.n, st));
    RMB_CUDA(cudaMemsetAsync(counters, 0, sizeof(int32_t) * 2 * (size_t)kFmMaxRounds, st));
    for (int b = 0; b < 2; ++b)
      for (int f = 0; f < 2; ++f) RMB_CUDA(cudaMemsetAsync(flags[b][f], 0, sizeof(idx_t) * (size_t)g.n, st));
    int64_t pass_moves = 0;
    int rounds = 0;
    bool done = false;
    while (!done && rounds < kFmMaxRounds) {
      const int r0 = rounds;
      for (int q = 0; q < kFmRoundsPerCheck && rounds < kFmMaxRounds; ++q, ++rounds) {
        int32_t* nm_dev = counters + 2 * rounds;
        // A round after one that selected nothing finds nothing either: the
        // gain kernel then only clears the mover flags.
        const int32_t* stop = rounds > 0 ? counters + 2 * (rounds - 1) : nullptr;
        // The first round of a pass evaluates every vertex; later rounds only
        // the ones the previous round's changes can reach.
        idx_t* const* cur = flags[rounds & 1];
        idx_t* const* nxt = flags[(rounds + 1) & 1];
        launch_gain<kCut>(g, part, k, nullptr, nullptr, mover, ncand, wfrom, cand_p, cand_g, heavy, nheavy, ghist,
                          st, stop, rounds > 0 ? cur[0] : nullptr, rp.gain_block);
        k_fm_select<<<nb, 256, 0, st>>>(g.n, g.xadj, g.adjncy, part, mover, ncand, cand_g, state,
                                        rounds > 0 ? cur[1] : nullptr, sel);
        RMB_LAUNCH_CHECK();
        compact_flags(sel, g.n, movers, nm_dev, arena, st);
        if (admit) {
          admit_cut_pass(g, k, g.n, nm_dev, movers, sel, zero, cand_p, cand_g, part, pw, rp.feas_max, nm_dev + 1,
                         nullptr, as, st, /*apply=*/false);
          k_fm_apply_after<<<grid_for(g.n, 256, 148 * 4), 256, 0, st>>>(nm_dev, movers, as.tgt, as.rank, as.cut,
                                                                        g.xadj, g.adjncy, part, sel, state, nxt[0]);
        } else {
          launch_walk<kCut>(g.n, nm_dev, movers, g, part, k, sel, zero, cand_p, cand_g, r, pw, rp.feas_max,
                            rp.over_thr, in_max, out_max, nm_dev + 1, rp.small_weights, long_flag, st);
          k_fm_after<<<nb, 256, 0, st>>>(nm_dev, movers, g.xadj, g.adjncy, part, cand_p, sel, state, nxt[0]);
        }
        RMB_LAUNCH_CHECK();
        k_fm_spread<<<nb, 256, 0, st>>>(g.n, g.xadj, g.adjncy, nxt[0], nxt[1], cur[0], cur[1]);
        RMB_LAUNCH_CHECK();
      }
      RMB_CUDA(cudaMemcpyAsync(hc.data() + 2 * r0, counters + 2 * r0, sizeof(int32_t) * 2 * (rounds - r0),
                               cudaMemcpyDeviceToHost, st));
      RMB_CUDA(cudaStreamSynchronize(st));
      for (int q = r0; q < rounds; ++q) {
        stats.movers += hc[2 * q];
        pass_moves += hc[2 * q + 1];
        if (hc[2 * q] > 0) stats.decide_iters += 1;
        if (hc[2 * q] == 0) done = true;
      }
    }
    stats.passes += 1;
    stats.moves += pass_moves;
    if (pass_moves == 0) break;  // fm_kway_pass returned false
  }
  arena.reset_to(mk);
  return stats;
}

}  // namespace rmb
