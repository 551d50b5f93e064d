// Parallel admission of a greedy cut pass: the production form of the
// reference's pass on large levels.
//
// Reference (src/refine/greedy.rs:126-190): boundary vertices in ascending id
// each take the feasible part with the best positive gain (gains from the
// start-of-pass part vector, feasibility pw[p] + vw <= t[p]*ub under the part
// weights left by the moves before it), and the moves apply together after
// the pass. Only the part weights chain the decisions together.
//
// Here a pass is decided in three launches:
//  1. pick (all movers in parallel): every mover takes the best positive-gain
//     candidate that is feasible under the start-of-pass weights (its move
//     alone);
//  then one block:
//  2. groups the picks by target part, in ascending vertex id (stable ranks),
//     and sums their weights along each part's in-list;
//  3. admission: a part keeps the longest prefix of its in-list whose weight
//     fits its budget feas - pw + (weight of its admitted out-moves). A part
//     that drops in-moves keeps their movers at home, which lowers the
//     out-credit of those movers' parts: repeat until no budget changes (the
//     admitted set only shrinks, so this ends). At the fixed point every part
//     that receives a move ends within its limit, as after the reference's
//     pass. Should the bound on the rounds be reached first, every part keeps
//     only what fits without any out-credit, which is within the limit
//     whatever else moves;
//  4. the new part weights (per part: + admitted in-moves - admitted
//     out-moves); then, in parallel again, the admitted moves are applied to
//     the part vector (k_admit_apply).
// Everything is integer and ordered by vertex id, so the result is the same
// on every run. The decisions differ from the reference's sequential ones
// (a part may take a vertex whose room appears only through moves of higher
// ids), so partitions built this way are compared by quality; the exact
// sequential walk (refine.cu) stays the path of small levels and of the
// checkers that replay a pass bit for bit.
#include "kernels.h"
#include "prof.h"
#include "scan.cuh"
#include "gain.cuh"

namespace rmb {

namespace {

constexpr int kAdmitThreads = 1024;
constexpr int kAdmitWarps = kAdmitThreads / 32;
constexpr int kAdmitMaxRounds = 64;

__device__ __forceinline__ int32_t vweight(const idx_t* vwgt, int32_t v, int32_t ncon, int c) {
  return vwgt ? vwgt[(int64_t)v * ncon + c] : 1;
}

// ---------------------------------------------------------------------------
// Picks (all movers at once): the best positive-gain part that the move alone
// keeps feasible under the start-of-pass weights, or -1 (greedy.rs:131-155).
// Writes per mover its target, source part and weights, so that the
// single-block admission reads them coalesced.
// ---------------------------------------------------------------------------
struct PickArgs {
  const int32_t* nm_dev;
  const idx_t* movers;
  const idx_t* xadj;
  const idx_t* ncand;
  const idx_t* wfrom;
  const idx_t* cand_p;
  const idx_t* cand_g;
  const idx_t* vwgt;
  const idx_t* part;
  const long long* pw;
  const long long* feas;
  int32_t ncon;
  int32_t k;
  int32_t* tgt;
  int32_t* src;
  int32_t* w;      // [nm][ncon]
  long long* out;  // [k][ncon], zero on entry: weight of the picks out of each part
  int any_gain;    // 1: the first feasible candidate is picked whatever its gain (2-way FM rounds)
};

__device__ void pick_body(const PickArgs& A, Lanes L) {
  const int32_t nm = *A.nm_dev;
  const int32_t ncon = A.ncon;
  RMB_FOR(j, nm, L) {
    const int32_t v = A.movers[j];
    const int32_t pv = A.part[v];
    const int32_t s = A.xadj[v];
    const int32_t ne = A.ncand[v];
    const int32_t ig = (int32_t)(0u - (uint32_t)A.wfrom[v]);
    int32_t vw[8];
    for (int c = 0; c < ncon; ++c) {
      vw[c] = vweight(A.vwgt, v, ncon, c);
      A.w[(int64_t)j * ncon + c] = vw[c];
    }
    auto feasible = [&](int32_t p) {
      for (int c = 0; c < ncon; ++c)
        if (A.pw[(int64_t)p * ncon + c] + vw[c] > A.feas[(int64_t)p * ncon + c]) return false;
      return true;
    };
    int32_t t = -1;
    if (ig <= 0) {
      // Candidates are sorted by (gain desc, part asc); parts outside the
      // list have gain ig <= 0 and never qualify.
      for (int32_t i = 0; i < ne; ++i) {
        if (A.cand_g[s + i] <= 0 && !A.any_gain) break;
        const int32_t p = A.cand_p[s + i];
        if (feasible(p)) {
          t = p;
          break;
        }
      }
    } else {
      // Negative edge weights: every part outside the list has the positive
      // gain ig. All parts in ascending order; strict > keeps the lowest.
      int32_t bestg = 0;
      for (int32_t p = 0; p < A.k; ++p) {
        if (p == pv) continue;
        int32_t gp = ig;
        for (int32_t i = 0; i < ne; ++i)
          if (A.cand_p[s + i] == p) {
            gp = A.cand_g[s + i];
            break;
          }
        if (gp > bestg && feasible(p)) {
          t = p;
          bestg = gp;
        }
      }
    }
    A.tgt[j] = t;
    A.src[j] = pv;
    if (t >= 0)
      for (int c = 0; c < ncon; ++c) atomic_add_i64(&A.out[(int64_t)pv * ncon + c], vw[c]);
  }
}

__global__ void k_admit_pick(PickArgs A) { pick_body(A, grid_lanes()); }

// The admitted moves of a pass, applied to the part vector: mover j moves to
// its target when its rank in the target's in-list is below the part's
// admitted prefix.
// With `touched`, every moved vertex and its neighbours are flagged there:
// the only vertices whose gain table the move changes.
__device__ void apply_body(Lanes L, const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                           const int32_t* __restrict__ tgt, const int32_t* __restrict__ rank,
                           const int32_t* __restrict__ cut, idx_t* __restrict__ part,
                           const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                           idx_t* __restrict__ touched) {
  const unsigned FULL = 0xffffffffu;
  const int32_t nm = *nm_dev;
  const int lane = threadIdx.x & 31;
  // Warp-uniform trips (the lanes of a warp hold consecutive movers); the
  // neighbours of a moved vertex with a long row are flagged by the whole
  // warp, so a hub's row is not one thread's loop.
  for (int64_t j0 = L.first - lane; j0 < nm; j0 += L.stride) {
    const int64_t j = j0 + lane;
    int32_t v = -1;
    if (j < nm) {
      const int32_t t = tgt[j];
      if (t >= 0 && rank[j] < cut[t]) {
        v = movers[j];
        part[v] = t;
      }
    }
    if (touched) {
      // Short rows by their own thread, rows above kHeavyDegree by the warp.
      bool long_row = false;
      if (v >= 0) {
        touched[v] = 1;
        const int32_t s0 = xadj[v], e0 = xadj[v + 1];
        long_row = e0 - s0 > kHeavyDegree;
        if (!long_row)
          for (int32_t x = s0; x < e0; ++x) touched[adj[x]] = 1;
      }
      unsigned mv = __ballot_sync(FULL, long_row);
      while (mv) {
        const int l = __ffs(mv) - 1;
        mv &= mv - 1;
        const int32_t u = __shfl_sync(FULL, v, l);
        const int32_t e = xadj[u + 1];
        for (int32_t x = xadj[u] + lane; x < e; x += 32) touched[adj[x]] = 1;
      }
    }
  }
}

__global__ void k_admit_apply(const int32_t* __restrict__ nm_dev, const idx_t* __restrict__ movers,
                              const int32_t* __restrict__ tgt, const int32_t* __restrict__ rank,
                              const int32_t* __restrict__ cut, idx_t* __restrict__ part,
                              const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                              idx_t* __restrict__ touched) {
  apply_body(grid_lanes(), nm_dev, movers, tgt, rank, cut, part, xadj, adj, touched);
}

// ---------------------------------------------------------------------------
// The admission of one pass in one block.
// ---------------------------------------------------------------------------
struct AdmitArgs {
  const int32_t* nm_dev;
  int32_t ncon;
  int32_t k;
  long long* pw;
  const long long* feas;
  int32_t* nmoves;
  int32_t* rounds_out;  // admission rounds used (diagnostics), may be null
  const int32_t* tgt;
  const int32_t* src;
  const int32_t* w;
  int32_t* rank;
  long long* out_g;     // [k][ncon] out-weights of the picks; read, then cleared for the next pass
  int32_t* cut_g;       // [k] admitted prefix per part, for the apply kernel
  long long* pref_g;    // [nm][ncon] running weight sums in grouped order (when shared memory is short)
  int32_t* src_g;       // [nm] source part in grouped order (same)
};

// Shared-memory layout (dynamic), in bytes; the staging area of the grouped
// order takes the rest of kAdmitMaxSmem.
struct AdmitSmem {
  size_t pw, feas, out, wcnt, run, off, cut, lo, hi, stage, total;
  int64_t cap;  // grouped positions that fit in shared memory
  __host__ __device__ AdmitSmem(int k, int ncon) {
    const size_t K = (size_t)k * ncon;
    size_t o = 0;
    pw = o;   o += 8 * K;
    feas = o; o += 8 * K;
    out = o;  o += 8 * K;
    wcnt = o; o += 4 * (size_t)kAdmitWarps * (k + 1);  // rows padded against bank conflicts
    run = o;  o += 4 * (size_t)k;
    off = o;  o += 4 * ((size_t)k + 1);
    cut = o;  o += 4 * (size_t)k;
    lo = o;   o += 4 * (size_t)k;
    hi = o;   o += 4 * (size_t)k;
    stage = (o + 15) & ~(size_t)15;
    total = stage;
    const size_t per = 8 * (size_t)ncon + 4;
    cap = stage < kAdmitMaxSmem ? (int64_t)((kAdmitMaxSmem - stage) / per) : 0;
  }
};

// Sum of the first i in-moves of part p on constraint c.
__device__ __forceinline__ long long inlist_sum(const long long* pref, int32_t ncon, int32_t off_p, int32_t i,
                                                int c) {
  if (i == 0) return 0;
  const long long hi = pref[(int64_t)(off_p + i - 1) * ncon + c];
  const long long lo = off_p > 0 ? pref[(int64_t)(off_p - 1) * ncon + c] : 0;
  return hi - lo;
}

// Largest i <= imax whose first i in-moves fit budget[c] on every
// constraint (the sums grow with i: vertex weights are positive). The search
// gallops down from imax: from one round to the next most prefixes stay or
// lose a few entries.
__device__ int32_t fit_prefix(const long long* pref, int32_t ncon, int32_t off_p, int32_t imax,
                              const long long* budget) {
  for (int c = 0; c < ncon; ++c)
    if (budget[c] < 0) return 0;
  auto fits = [&](int32_t i) {
    for (int c = 0; c < ncon; ++c)
      if (inlist_sum(pref, ncon, off_p, i, c) > budget[c]) return false;
    return true;
  };
  if (imax == 0 || fits(imax)) return imax;
  int32_t bad = imax, good = 0, step = 1;  // fits(good) holds, fits(bad) does not
  for (;;) {
    const int32_t probe = bad - step;
    if (probe <= 0) break;
    if (fits(probe)) {
      good = probe;
      break;
    }
    bad = probe;
    step <<= 1;
  }
  while (bad - good > 1) {
    const int32_t mid = good + (bad - good) / 2;
    if (fits(mid)) good = mid;
    else bad = mid;
  }
  return good;
}

// The admission of one pass by a block of kAdmitThreads threads; smem:
// kAdmitMaxSmem bytes of dynamic shared memory.
__device__ void admit_body(const AdmitArgs& A, unsigned char* smem) {
  const AdmitSmem L(A.k, A.ncon);
  long long* pw_s = reinterpret_cast<long long*>(smem + L.pw);
  long long* feas_s = reinterpret_cast<long long*>(smem + L.feas);
  long long* out_s = reinterpret_cast<long long*>(smem + L.out);
  int32_t* wcnt = reinterpret_cast<int32_t*>(smem + L.wcnt);  // [warp][k + 1]
  int32_t* run = reinterpret_cast<int32_t*>(smem + L.run);
  int32_t* off = reinterpret_cast<int32_t*>(smem + L.off);
  int32_t* cut = reinterpret_cast<int32_t*>(smem + L.cut);
  int32_t* rlo = reinterpret_cast<int32_t*>(smem + L.lo);
  int32_t* rhi = reinterpret_cast<int32_t*>(smem + L.hi);
  __shared__ long long wsum[kAdmitWarps][2];
  __shared__ int32_t flag[2];
  __shared__ int32_t warp_tot[kAdmitWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int32_t k = A.k, ncon = A.ncon;
  const int32_t K = k * ncon;
  const int32_t ks = k + 1;  // row stride of wcnt
  const int32_t nm = *A.nm_dev;
  for (int32_t i = tid; i < K; i += kAdmitThreads) {
    pw_s[i] = A.pw[i];
    feas_s[i] = A.feas[i];
    out_s[i] = A.out_g[i];
    A.out_g[i] = 0;  // the next pass's picks sum into it again
  }
  for (int32_t i = tid; i < kAdmitWarps * ks; i += kAdmitThreads) wcnt[i] = 0;
  for (int32_t i = tid; i < k; i += kAdmitThreads) run[i] = 0;
  if (tid < 2) flag[tid] = 0;
  __syncthreads();
  if (nm == 0) {
    if (tid == 0) {
      *A.nmoves = 0;
      if (A.rounds_out) *A.rounds_out = 0;
    }
    return;
  }

  // ---- stable ranks per target (ascending mover order), tile by tile; the
  // next tile's targets are loaded while this one is ranked ----
  int32_t t_next = tid < nm ? A.tgt[tid] : -1;
  for (int32_t base = 0; base < nm; base += kAdmitThreads) {
    const int32_t j = base + tid;
    const int32_t t = t_next;
    t_next = j + kAdmitThreads < nm ? A.tgt[j + kAdmitThreads] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, t);
    const unsigned before = peers & lanemask_lt();
    const int32_t rin = __popc(before);
    if (t >= 0 && before == 0) wcnt[warp * ks + t] = __popc(peers);
    __syncthreads();
    // Warp w scans targets w, w + 32, ...: lane l holds warp l's count, so a
    // shuffle scan gives every warp its base (entries without movers stay 0).
    for (int32_t p = warp; p < k; p += kAdmitWarps) {
      const int32_t c = wcnt[lane * ks + p];
      const int32_t base_p = run[p];
      int32_t x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (c) wcnt[lane * ks + p] = base_p + x - c;
      __syncwarp();
      if (lane == 31) run[p] = base_p + x;
    }
    __syncthreads();
    if (t >= 0) A.rank[j] = wcnt[warp * ks + t] + rin;
    __syncwarp();
    // Only this warp's leaders write its row again (next tile, after the
    // first barrier), so no barrier is needed here.
    if (t >= 0 && before == 0) wcnt[warp * ks + t] = 0;
  }
  __syncthreads();

  // ---- offsets of the in-lists: exclusive scan of the counts over parts ----
  {
    int32_t carry = 0;
    for (int32_t p0 = 0; p0 < k; p0 += kAdmitThreads) {
      const int32_t p = p0 + tid;
      const int32_t c = p < k ? run[p] : 0;
      int32_t x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) warp_tot[warp] = x;
      __syncthreads();
      if (warp == 0) {
        int32_t s = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t y = __shfl_up_sync(0xffffffffu, s, o);
          if (lane >= o) s += y;
        }
        warp_tot[lane] = s;  // inclusive over warps
      }
      __syncthreads();
      const int32_t wbase = warp > 0 ? warp_tot[warp - 1] : 0;
      if (p < k) {
        off[p] = carry + wbase + x - c;
        cut[p] = c;
      }
      const int32_t tile_total = warp_tot[kAdmitWarps - 1];
      __syncthreads();
      carry += tile_total;
    }
    if (tid == 0) off[k] = carry;
    __syncthreads();
  }
  const int32_t total = off[k];

  // ---- grouped order: source part and weights at each in-list position,
  // then running weight sums along it (shared memory when it fits) ----
  const bool in_smem = total <= L.cap;
  long long* pref = in_smem ? reinterpret_cast<long long*>(smem + L.stage) : A.pref_g;
  int32_t* gsrc = in_smem ? reinterpret_cast<int32_t*>(smem + L.stage + 8 * (size_t)ncon * (size_t)L.cap) : A.src_g;
  for (int32_t j = tid; j < nm; j += kAdmitThreads) {
    const int32_t t = A.tgt[j];
    if (t >= 0) {
      const int32_t pos = off[t] + A.rank[j];
      gsrc[pos] = A.src[j];
      for (int c = 0; c < ncon; ++c) pref[(int64_t)pos * ncon + c] = A.w[(int64_t)j * ncon + c];
    }
  }
  __syncthreads();
  for (int c = 0; c < ncon; ++c) {
    long long carry = 0;
    for (int32_t base = 0; base < total; base += kAdmitThreads) {
      const int32_t pos = base + tid;
      const long long w = pos < total ? pref[(int64_t)pos * ncon + c] : 0;
      long long x = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp][0] = x;
      __syncthreads();
      if (warp == 0) {
        long long s = wsum[lane][0];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const long long y = __shfl_up_sync(0xffffffffu, s, o);
          if (lane >= o) s += y;
        }
        wsum[lane][1] = s;
      }
      __syncthreads();
      const long long wbase = warp > 0 ? wsum[warp - 1][1] : 0;
      if (pos < total) pref[(int64_t)pos * ncon + c] = carry + wbase + x;
      const long long tile_total = wsum[kAdmitWarps - 1][1];
      __syncthreads();
      carry += tile_total;
    }
  }
  __syncthreads();

  // ---- admission rounds: new prefixes from the out-credit (barrier), then
  // the dropped moves return their credit (barrier) ----
  // A warp walks each part's dropped range [rlo, rhi).
  auto return_credit = [&]() {
    for (int32_t p = warp; p < k; p += kAdmitWarps) {
      const int32_t o = off[p];
      for (int32_t i = rlo[p] + lane; i < rhi[p]; i += 32) {
        const int32_t pos = o + i;
        const int32_t sp = gsrc[pos];
        for (int c = 0; c < ncon; ++c) {
          const long long wv = pref[(int64_t)pos * ncon + c] - (pos > 0 ? pref[(int64_t)(pos - 1) * ncon + c] : 0);
          atomic_add_i64(&out_s[sp * ncon + c], -wv);
        }
      }
    }
  };
  int rounds = 0;
  bool converged = false;
  while (rounds < kAdmitMaxRounds) {
    const int fb = rounds & 1;
    ++rounds;
    for (int32_t p = tid; p < k; p += kAdmitThreads) {
      long long budget[8];
      for (int c = 0; c < ncon; ++c) {
        const int32_t x = p * ncon + c;
        budget[c] = feas_s[x] - pw_s[x] + out_s[x];
      }
      const int32_t old = cut[p];
      const int32_t now = fit_prefix(pref, ncon, off[p], old, budget);
      rlo[p] = now;
      rhi[p] = old;
      if (now < old) {
        cut[p] = now;
        flag[fb] = 1;
      }
    }
    // The other flag was last read before the previous round's second
    // barrier; clear it for the next round.
    if (tid == 0) flag[fb ^ 1] = 0;
    __syncthreads();
    if (!flag[fb]) {
      converged = true;
      break;
    }
    return_credit();
    __syncthreads();
  }
  if (!converged) {
    // Keep only what fits with no out-credit at all, and return the credit
    // of what this drops, so that out_s holds the admitted out-weights.
    for (int32_t p = tid; p < k; p += kAdmitThreads) {
      long long budget[8];
      for (int c = 0; c < ncon; ++c) budget[c] = feas_s[p * ncon + c] - pw_s[p * ncon + c];
      const int32_t old = cut[p];
      const int32_t now = fit_prefix(pref, ncon, off[p], old, budget);
      rlo[p] = now;
      rhi[p] = old;
      cut[p] = now;
    }
    __syncthreads();
    return_credit();
    __syncthreads();
  }

  // ---- new part weights: + the admitted in-moves, - the admitted out-moves ----
  int32_t moved = 0;
  for (int32_t p = tid; p < k; p += kAdmitThreads) {
    for (int c = 0; c < ncon; ++c) {
      const int32_t x = p * ncon + c;
      A.pw[x] = pw_s[x] + inlist_sum(pref, ncon, off[p], cut[p], c) - out_s[x];
    }
    A.cut_g[p] = cut[p];
    moved += cut[p];
  }
  moved = warp_sum(moved);
  if (lane == 0) warp_tot[warp] = moved;
  __syncthreads();
  if (tid == 0) {
    int32_t s = 0;
    for (int w = 0; w < kAdmitWarps; ++w) s += warp_tot[w];
    *A.nmoves = s;
    if (A.rounds_out) *A.rounds_out = converged ? rounds : -rounds;
  }
}

__global__ void __launch_bounds__(kAdmitThreads, 1) k_admit(AdmitArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  admit_body(A, smem);
}

// The cut passes of admission levels of a batch: block b refines the level
// of jobs[b] (its part vector and part weights left by k_batch_level's repair
// pass). Each pass as greedy_refine runs it with admit_cut_pass: gain table
// (the first pass everywhere, later ones for the vertices the last pass
// moved and their neighbours), mover list in ascending id, picks, admission,
// moves; a pass without a move ends the level (greedy.rs:184-186).
template <bool HAS_W>
__global__ void __launch_bounds__(kAdmitThreads, 1) k_batch_admit(const LevelJob* __restrict__ jobs) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int32_t sw[32];
  const LevelJob& J = jobs[blockIdx.x];
  const Lanes L = block_lanes();
  const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int pass = 1; pass <= J.niter; ++pass) {
    if (pass >= 2 && J.counters[2 * (pass - 1) + 1] == 0) break;
    idx_t* only = pass >= 2 ? J.touched[(pass - 1) & 1] : nullptr;
    int32_t* nm_dev = J.counters + 2 * pass;
    gain_body<HAS_W, kCut>(L, J.xadj, J.adjncy, J.adjwgt, J.n, J.ncon, J.part, J.k, J.pw, J.over, J.mover, J.ncand,
                           J.wfrom, J.cand_p, J.cand_g, only, only != nullptr);
    if (J.nheavy > 0)
      gain_heavy_body<HAS_W, kCut>(warp, nwarps, J.ghist + (int64_t)warp * J.k, J.xadj, J.adjncy, J.adjwgt,
                                   J.heavy, J.nheavy, J.ncon, J.part, J.k, J.pw, J.over, J.mover, J.ncand, J.wfrom,
                                   J.cand_p, J.cand_g, only, only != nullptr);
    __syncthreads();
    block_scan_n<int32_t>(LoadNonZero{J.mover}, StoreCompact{J.mover, J.movers}, J.n, nm_dev, sw);
    __syncthreads();
    PickArgs P;
    P.nm_dev = nm_dev;
    P.movers = J.movers;
    P.xadj = J.xadj;
    P.ncand = J.ncand;
    P.wfrom = J.wfrom;
    P.cand_p = J.cand_p;
    P.cand_g = J.cand_g;
    P.vwgt = J.vwgt;
    P.part = J.part;
    P.pw = J.pw;
    P.feas = J.feas;
    P.ncon = J.ncon;
    P.k = J.k;
    P.tgt = J.a_tgt;
    P.src = J.a_src;
    P.w = J.a_w;
    P.out = J.a_out;
    P.any_gain = 0;
    pick_body(P, L);
    __syncthreads();
    AdmitArgs A;
    A.nm_dev = nm_dev;
    A.ncon = J.ncon;
    A.k = J.k;
    A.pw = J.pw;
    A.feas = J.feas;
    A.nmoves = nm_dev + 1;
    A.rounds_out = nullptr;
    A.tgt = J.a_tgt;
    A.src = J.a_src;
    A.w = J.a_w;
    A.rank = J.a_rank;
    A.out_g = J.a_out;
    A.cut_g = J.a_cut;
    A.pref_g = J.a_pref;
    A.src_g = J.a_gsrc;
    admit_body(A, smem);
    __syncthreads();
    apply_body(L, nm_dev, J.movers, J.a_tgt, J.a_rank, J.a_cut, J.part, J.xadj, J.adjncy,
               pass + 1 <= J.niter ? J.touched[pass & 1] : nullptr);
    __syncthreads();
  }
}

}  // namespace

size_t admit_smem_bytes(int k, int ncon) { return AdmitSmem(k, ncon).total; }

bool admit_supported(int k, int ncon) {
  return k >= 2 && ncon >= 1 && ncon <= 8 && admit_smem_bytes(k, ncon) <= kAdmitMaxSmem;
}

int admit_cut_pass(const DGraph& g, int k, int32_t nmax, const int32_t* nm_dev, const idx_t* movers,
                   const idx_t* ncand, const idx_t* wfrom, const idx_t* cand_p, const idx_t* cand_g, idx_t* part,
                   long long* pw, const long long* feas, int32_t* nmoves, int32_t* rounds_out,
                   const AdmitScratch& s, cudaStream_t st, bool apply, idx_t* touched, bool any_gain) {
  const int ph = profiler().begin(kProfAdmit, st);
  PickArgs P;
  P.nm_dev = nm_dev;
  P.movers = movers;
  P.xadj = g.xadj;
  P.ncand = ncand;
  P.wfrom = wfrom;
  P.cand_p = cand_p;
  P.cand_g = cand_g;
  P.vwgt = g.vwgt;
  P.part = part;
  P.pw = pw;
  P.feas = feas;
  P.ncon = g.ncon;
  P.k = k;
  P.tgt = s.tgt;
  P.src = s.src;
  P.w = s.w;
  P.out = s.out;
  P.any_gain = any_gain ? 1 : 0;
  const int blocks = grid_for(nmax, 256, 148 * 4);
  k_admit_pick<<<blocks, 256, 0, st>>>(P);
  RMB_LAUNCH_CHECK();
  AdmitArgs A;
  A.nm_dev = nm_dev;
  A.ncon = g.ncon;
  A.k = k;
  A.pw = pw;
  A.feas = feas;
  A.nmoves = nmoves;
  A.rounds_out = rounds_out;
  A.tgt = s.tgt;
  A.src = s.src;
  A.w = s.w;
  A.rank = s.rank;
  A.out_g = s.out;
  A.cut_g = s.cut;
  A.pref_g = s.pref;
  A.src_g = s.gsrc;
  allow_dyn_smem((const void*)k_admit, kAdmitMaxSmem);
  k_admit<<<1, kAdmitThreads, kAdmitMaxSmem, st>>>(A);
  RMB_LAUNCH_CHECK();
  if (apply) {
    k_admit_apply<<<blocks, 256, 0, st>>>(nm_dev, movers, s.tgt, s.rank, s.cut, part, g.xadj, g.adjncy, touched);
    RMB_LAUNCH_CHECK();
  }
  profiler().end(ph, st, 0.0);
  return ph;
}

void batch_admit_launch(const LevelJob* d_jobs, int njobs, bool has_w, cudaStream_t st) {
  if (njobs <= 0) return;
  const int ph = profiler().begin(kProfAdmit, st);
  auto kern = has_w ? k_batch_admit<true> : k_batch_admit<false>;
  allow_dyn_smem((const void*)kern, kAdmitMaxSmem);
  kern<<<njobs, kAdmitThreads, kAdmitMaxSmem, st>>>(d_jobs);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 0.0);
}

}  // namespace rmb
