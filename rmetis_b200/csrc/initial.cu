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
// One warp (one block) per trial. Its mutable state (part[n], queue links
// next[n], part weights pw[k][ncon] as i64, queue head/tail[k], and a bitmap
// of the parts below target in the current round) lives in shared memory when
// it fits, else in the trial's global scratch. A part's weight only changes
// during its own turn, so the parts that may grow in a round are known at the
// round's start.
// Row chunks of 32 whose neighbour ids and labels are loaded together (a
// hub's row is otherwise one long chain of dependent loads).
constexpr int kGrowGroup = 8;

template <bool HAS_VW>
__device__ void grow_body(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                          const idx_t* __restrict__ vwgt, int32_t n, int32_t ncon, int32_t k,
                          const idx_t* __restrict__ sd, const long long* __restrict__ grow_tgt,
                          idx_t* __restrict__ out, unsigned char* base) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  long long* pw = reinterpret_cast<long long*>(base);
  idx_t* part = reinterpret_cast<idx_t*>(pw + (size_t)k * ncon);
  idx_t* next = part + n;
  idx_t* head = next + n;
  idx_t* tail = head + k;
  unsigned* needy = reinterpret_cast<unsigned*>(tail + k);
  const int32_t nwords = (k + 31) >> 5;

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

  // A part whose queue has run empty can never grow again (its queue only
  // receives vertices it claims by popping), so it is dropped from the rounds:
  // lane w keeps the bits of parts 32w..32w+31 still holding a queue (k <=
  // 1024; above that every part stays in).
  const bool track = nwords <= 32;
  unsigned alive = ~0u;
  bool any_active = true;
  while (any_active) {
    // Parts below target on some constraint (grow.rs:54-58), as a bitmap.
    for (int32_t w0 = 0; w0 < nwords; ++w0) {
      const int32_t p = w0 * 32 + lane;
      bool needs = false;
      if (p < k) {
        for (int c = 0; c < ncon; ++c)
          if (!(pw[(int64_t)p * ncon + c] >= grow_tgt[(int64_t)p * ncon + c])) { needs = true; break; }
      }
      const unsigned m = __ballot_sync(FULL, needs);
      const unsigned al = track ? __shfl_sync(FULL, alive, w0) : ~0u;
      if (lane == 0) needy[w0] = m & al;
    }
    __syncwarp();
    int32_t active = 0;
    for (int32_t w0 = 0; w0 < nwords; ++w0) {
      unsigned bits = needy[w0];
      while (bits) {
        const int32_t p = w0 * 32 + __ffs(bits) - 1;
        bits &= bits - 1;
        bool grew = false;
        int32_t qh = head[p], qt = tail[p];
        while (qh != -1) {
          const int32_t v = qh;
          qh = next[v];
          const int32_t e = __ldg(&xadj[v + 1]);
          // The row is read kGrowGroup chunks of 32 at a time: neighbours and their
          // part labels are loaded together, then the chunks are claimed in
          // order. A claim earlier in the group may have taken a neighbour that
          // is listed again later in the row, so after one the later
          // candidates' labels are read again.
          for (int32_t b0 = __ldg(&xadj[v]); b0 < e; b0 += kGrowGroup * 32) {
            int32_t uu[kGrowGroup];
            bool cc[kGrowGroup];
#pragma unroll
            for (int q = 0; q < kGrowGroup; ++q) {
              const int32_t j = b0 + q * 32 + lane;
              uu[q] = j < e ? __ldg(&adj[j]) : -1;
            }
#pragma unroll
            for (int q = 0; q < kGrowGroup; ++q) cc[q] = uu[q] >= 0 && part[uu[q]] == -1;
            bool claimed = false;
#pragma unroll
            for (int q = 0; q < kGrowGroup; ++q) {
              if (b0 + q * 32 >= e) break;
              const int32_t u = uu[q];
              bool cand = cc[q];
              if (claimed && cand) cand = part[u] == -1;
              const unsigned peers = __match_any_sync(FULL, cand ? u : -(lane + 2));
              const bool first = cand && (__ffs(peers) - 1) == lane;
              const unsigned fm = __ballot_sync(FULL, first);
              if (fm) {
                grew = true;
                claimed = true;
                if (first) part[u] = p;
                for (int c = 0; c < ncon; ++c) {
                  long long w = first ? (long long)(HAS_VW ? __ldg(&vwgt[(int64_t)u * ncon + c]) : 1) : 0;
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
          }
          if (grew) break;
        }
        if (lane == 0) {
          head[p] = qh;
          tail[p] = qt;
        }
        if (track && qh == -1 && lane == (p >> 5)) alive &= ~(1u << (p & 31));
        __syncwarp();
        if (grew) ++active;
      }
    }
    any_active = active > 0;
  }

  // Leftovers (disconnected or unreachable): lightest part on constraint 0,
  // first minimum, in ascending vertex order.
  if (!HAS_VW && k <= 1024) {
    // Unit weights: the leftovers fill the parts level by level. At level L
    // the parts whose weight before this phase is <= L each take one leftover,
    // in id order, and then the level rises by one; parts join as L reaches
    // their weight. Lane l keeps the bitmap word of parts 32l..32l+31.
    long long L = LLONG_MAX;
    for (int32_t p = lane; p < k; p += 32) L = min(L, pw[(int64_t)p * ncon]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) L = min(L, __shfl_xor_sync(FULL, L, o));
    unsigned act = 0;
    long long nxt = LLONG_MAX;  // smallest weight of this lane's parts not yet active
    auto activate = [&]() {
      nxt = LLONG_MAX;
      for (int bb = 0; bb < 32; ++bb) {
        const int32_t p = lane * 32 + bb;
        if (p < k && !((act >> bb) & 1u)) {
          const long long x = pw[(int64_t)p * ncon];
          if (x <= L) act |= 1u << bb;
          else nxt = min(nxt, x);
        }
      }
    };
    activate();
    int32_t cursor = 0;  // parts below cursor have had their turn at level L
    for (int32_t b = 0; b < n; b += 32) {
      const int32_t v = b + lane;
      unsigned un = __ballot_sync(FULL, v < n && part[v] == -1);
      while (un) {
        const int i = __ffs(un) - 1;
        un &= un - 1;
        const int32_t w0 = lane * 32;
        unsigned mask = w0 + 31 < cursor ? 0u : (w0 >= cursor ? act : act & (~0u << (cursor & 31)));
        unsigned m = __ballot_sync(FULL, mask != 0u);
        if (m == 0u) {
          // Level L is done: every active part now weighs L + 1.
          ++L;
          cursor = 0;
          long long g = nxt;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) g = min(g, __shfl_xor_sync(FULL, g, o));
          if (g <= L) activate();
          mask = act;
          m = __ballot_sync(FULL, mask != 0u);
        }
        const int wl = __ffs(m) - 1;
        const unsigned word = __shfl_sync(FULL, mask, wl);
        const int32_t p = wl * 32 + __ffs(word) - 1;
        if (lane == 0) part[b + i] = p;
        cursor = p + 1;
      }
      __syncwarp();
    }
  } else {
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
  }
  __syncwarp();

  // Write the partition out; the trial cuts are computed edge-parallel for
  // all trials at once afterwards (trial_cuts).
  for (int32_t v = lane; v < n; v += 32) out[v] = part[v];
  __syncwarp();
}

template <bool HAS_VW>
__global__ void __launch_bounds__(32) k_grow(const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                                             const idx_t* __restrict__ vwgt, int32_t n, int32_t ncon, int32_t k,
                                             const idx_t* __restrict__ seeds,
                                             const long long* __restrict__ grow_tgt, idx_t* __restrict__ parts,
                                             unsigned char* __restrict__ gscratch, size_t scratch_bytes,
                                             int use_smem) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int trial = blockIdx.x;
  unsigned char* base = use_smem ? smem : gscratch + (size_t)trial * scratch_bytes;
  grow_body<HAS_VW>(xadj, adj, vwgt, n, ncon, k, seeds + (int64_t)trial * k, grow_tgt, parts + (int64_t)trial * n,
                    base);
}

// The grow trials of a batch of coarsest graphs: block b runs trial
// b - first_block of job block_job[b] and then sums its directed edge cut
// (the quantity trial_cuts computes) into the job's cuts.
__global__ void __launch_bounds__(32) k_batch_grow(const GrowJob* __restrict__ jobs,
                                                   const int32_t* __restrict__ block_job) {
  extern __shared__ __align__(16) unsigned char smem[];
  const GrowJob& J = jobs[block_job[blockIdx.x]];
  const int trial = blockIdx.x - J.first_block;
  unsigned char* base = J.use_smem ? smem : J.scratch + (size_t)trial * (size_t)J.scratch_bytes;
  idx_t* out = J.parts + (int64_t)trial * J.n;
  if (J.vwgt)
    grow_body<true>(J.xadj, J.adjncy, J.vwgt, J.n, J.ncon, J.k, J.seeds + (int64_t)trial * J.k, J.grow_tgt, out,
                    base);
  else
    grow_body<false>(J.xadj, J.adjncy, J.vwgt, J.n, J.ncon, J.k, J.seeds + (int64_t)trial * J.k, J.grow_tgt, out,
                     base);
  const int lane = threadIdx.x & 31;
  unsigned long long acc = 0;
  for (int32_t v = lane; v < J.n; v += 32) {
    const int32_t pv = out[v];
    for (int32_t j = J.xadj[v]; j < J.xadj[v + 1]; ++j)
      if (out[J.adjncy[j]] != pv) acc += (unsigned long long)(long long)(J.adjwgt ? J.adjwgt[j] : 1);
  }
  acc = warp_sum(acc);
  if (lane == 0) J.cuts[trial] = (long long)acc;
}

void grow_trials_batch(const GrowJob* d_jobs, const int32_t* d_block_job, int nblocks, size_t dyn_smem,
                       cudaStream_t st) {
  if (nblocks <= 0) return;
  RMB_CUDA(cudaFuncSetAttribute(k_batch_grow, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(200 * 1024)));
  const int ph = profiler().begin(kProfGrow, st);
  k_batch_grow<<<nblocks, 32, dyn_smem, st>>>(d_jobs, d_block_job);
  RMB_LAUNCH_CHECK();
  profiler().end(ph, st, 0.0);
}

size_t grow_scratch_bytes(int32_t n, int k, int ncon) {
  const size_t bytes = sizeof(long long) * (size_t)k * ncon + sizeof(idx_t) * (2 * (size_t)n + 2 * (size_t)k) +
                       sizeof(unsigned) * (((size_t)k + 31) / 32) + 16;
  return (bytes + 255) & ~(size_t)255;
}

void grow_trials(const DGraph& g, int k, int ntrials, const idx_t* seeds, const long long* grow_tgt, idx_t* parts,
                 long long* cuts, Arena& arena, cudaStream_t st) {
  Arena::Mark mk = arena.mark();
  const size_t bytes_al = grow_scratch_bytes(g.n, k, g.ncon);
  const size_t kSmemLimit = 200 * 1024;
  const int use_smem = bytes_al <= kSmemLimit ? 1 : 0;
  unsigned char* scratch = use_smem ? nullptr : arena.alloc<unsigned char>(bytes_al * (size_t)ntrials);
  const size_t dyn = use_smem ? bytes_al : 0;
  auto kern = g.vwgt ? k_grow<true> : k_grow<false>;
  RMB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit));
  const int ph = profiler().begin(kProfGrow, st);
  kern<<<ntrials, 32, dyn, st>>>(g.xadj, g.adjncy, g.vwgt, g.n, g.ncon, k, seeds, grow_tgt, parts, scratch, bytes_al,
                                 use_smem);
  RMB_LAUNCH_CHECK();
  trial_cuts(g, parts, ntrials, cuts, st);
  profiler().end(ph, st, (double)ntrials * (16.0 * g.n + 8.0 * (double)g.m));
  arena.reset_to(mk);
}

}  // namespace rmb
