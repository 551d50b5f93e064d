// Batched k-way partitioning (src/partition/kway.rs:20-162 for every graph of
// a batch): the whole batch goes through the multilevel pipeline in a handful
// of launches instead of one pipeline of launches per graph.
//
// Small graphs leave a GPU idle between their launches: a 40,000-vertex graph
// runs about a thousand short kernels, each on a fraction of the SMs, and the
// device spends its time on launch and synchronisation latency. Here every
// step of the pipeline is one launch over the batch, one block per graph,
// each block running the same single-block bodies that the single call uses
// for its small levels (the coarsening tail, the grow trials, the fused level
// refinement and the single-block admission):
//
//   1. validation of every graph and its total weights     (k_batch_validate)
//   2. the whole coarsening of every graph                 (k_batch_coarsen)
//   3. one read-back of every level table; the host derives each graph's
//      thresholds, grow seeds and refinement jobs and uploads them at once
//   4. every grow trial of every coarsest graph            (k_batch_grow)
//   5. step s = 0, 1, ...: level Lmax - s of every graph that has it (the
//      coarsest of a graph first), with its projection or best grow trial,
//      repair pass and exact cut passes                     (k_batch_level)
//      and the admission cut passes of its large levels     (k_batch_admit)
//   6. the cut of every result                              (k_batch_cut)
//
// The bodies decide exactly as the single call's kernels, so every result
// equals the single call's (the tests compare them graph by graph). The
// largest graphs are started first (blocks in descending size), which keeps
// the device busy while they finish.
#include <algorithm>
#include <climits>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "engine.h"
#include "hostrng.h"
#include "prof.h"

namespace rmb {

namespace {

// validate_device's checks for one graph per block: xadj monotone (bit 2);
// then neighbour ids in range (4), no self loop (8), every vertex listed as
// often as its degree (16, symmetric structure); vertex weights positive
// (32). Also the total weight per constraint.
__global__ void k_batch_validate(const ValJob* __restrict__ jobs) {
  __shared__ int32_t bits;
  __shared__ long long tot[8];
  const ValJob& J = jobs[blockIdx.x];
  const Lanes L = block_lanes();
  if (threadIdx.x == 0) bits = 0;
  if (threadIdx.x < 8) tot[threadIdx.x] = 0;
  __syncthreads();
  RMB_FOR(i, J.n, L) {
    if (J.xadj[i] > J.xadj[i + 1]) atomicOr(&bits, 2);
  }
  __syncthreads();
  if (bits == 0) {
    RMB_FOR(v, J.n, L) {
      for (int32_t p = J.xadj[v]; p < J.xadj[v + 1]; ++p) {
        const idx_t u = J.adjncy[p];
        if (u < 0 || u >= J.n) atomicOr(&bits, 4);
        else if (u == (idx_t)v) atomicOr(&bits, 8);
        else atomicAdd(&J.degcheck[u], 1);
      }
    }
    __syncthreads();
    RMB_FOR(v, J.n, L) {
      if (__ldcg(&J.degcheck[v]) != J.xadj[v + 1] - J.xadj[v]) atomicOr(&bits, 16);
    }
    if (J.vwgt) {
      long long s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      RMB_FOR(i, (int64_t)J.n * J.ncon, L) {
        const idx_t w = J.vwgt[i];
        if (w <= 0) atomicOr(&bits, 32);
        s[i % J.ncon] += w;
      }
      for (int c = 0; c < J.ncon; ++c) {
        const long long x = warp_sum(s[c]);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(reinterpret_cast<unsigned long long*>(&tot[c]),
                                                    (unsigned long long)x);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *J.flag = bits;
  if (threadIdx.x < J.ncon) J.total[threadIdx.x] = tot[threadIdx.x];
}

// Level tables of the batch into one contiguous array (one read-back).
__global__ void k_gather_tables(const TailArgs* __restrict__ args, int32_t ngraphs, TailOut* __restrict__ out) {
  constexpr int kWords = (int)(sizeof(TailOut) / sizeof(int32_t));
  static_assert(sizeof(TailOut) % sizeof(int32_t) == 0, "TailOut is copied in 4-byte words");
  for (int32_t g = blockIdx.x; g < ngraphs; g += gridDim.x) {
    const int32_t* src = reinterpret_cast<const int32_t*>(args[g].ws);
    int32_t* dst = reinterpret_cast<int32_t*>(out + g);
    for (int i = threadIdx.x; i < kWords; i += blockDim.x) dst[i] = src[i];
  }
}

struct CutJob {
  const idx_t* xadj;
  const idx_t* adjncy;
  const idx_t* adjwgt;
  const idx_t* part;
  int32_t n;
  unsigned long long* cut;  // zero on entry: directed cut as cut_and_weights sums it
};

__global__ void k_batch_cut(const CutJob* __restrict__ jobs) {
  const CutJob& J = jobs[blockIdx.x];
  unsigned long long acc = 0;
  RMB_FOR(v, J.n, block_lanes()) {
    const idx_t pv = J.part[v];
    for (int32_t p = J.xadj[v]; p < J.xadj[v + 1]; ++p)
      if (J.part[J.adjncy[p]] != pv) acc += (uint32_t)(J.adjwgt ? J.adjwgt[p] : 1);
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(J.cut, acc);
}

// The thresholds of every level of a graph (Engine::thresholds with uniform
// targets: t = total / k for every part, the same f64 expression) written on
// the device: [level][feas, over, grow][k][ncon]. tot: [level][ncon], the i32
// level totals.
struct ThrJob {
  long long* thr;
  const int32_t* tot;
  int32_t k, ncon, nlevels;
};

__device__ void threshold_values_dev(double t, double ub, long long* feas, long long* over, long long* grow) {
  const double lim = 9.0e18;
  const double x = t * ub;
  if (isnan(x)) {
    *feas = LLONG_MIN;
    *over = LLONG_MAX;
  } else if (x >= lim) {
    *feas = LLONG_MAX;
    *over = LLONG_MAX;
  } else if (x <= -lim) {
    *feas = LLONG_MIN;
    *over = LLONG_MIN;
  } else {
    const long long f = (long long)floor(x);
    *feas = f;
    *over = f;
  }
  if (isnan(t) || t >= lim) *grow = LLONG_MAX;
  else if (t <= -lim) *grow = LLONG_MIN;
  else *grow = (long long)ceil(t);
}

struct UbVec {
  double v[8];
};

__global__ void k_batch_thresholds(const ThrJob* __restrict__ jobs, UbVec ub) {
  const ThrJob& J = jobs[blockIdx.x];
  const int64_t K = (int64_t)J.k * J.ncon;
  const double inv = 1.0 / (double)J.k;
  for (int64_t idx = threadIdx.x; idx < (int64_t)J.nlevels * K; idx += blockDim.x) {
    const int64_t l = idx / K, i = idx - l * K;
    const int c = (int)(i % J.ncon);
    const double t = inv * (double)J.tot[l * J.ncon + c];
    long long* h = J.thr + 3 * K * l;
    threshold_values_dev(t, ub.v[c], &h[i], &h[K + i], &h[2 * K + i]);
  }
}

}  // namespace

bool batch_eligible(const KwayOptions& o, int32_t n, int k, int ncon) {
  return o.rtype == 1 && o.ncuts == 1 && o.iptype != 1 && !o.bisect_fm2 && ncon >= 1 && ncon <= 2 && k >= 2 &&
         k <= 256 && k <= n;
}

namespace {

// Bump carving of one device allocation, every piece 256-byte aligned.
struct Carver {
  char* base = nullptr;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
    off += (count * sizeof(T) + 255) & ~(size_t)255;
    return p;
  }
};

// Host staging of arrays uploaded together: pieces appended at 256-byte
// aligned offsets, then one copy to a device block of the same layout.
struct Staging {
  std::vector<char> host;
  template <typename T>
  size_t put(const T* src, size_t count) {
    const size_t off = host.size();
    const size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
    host.resize(off + bytes, 0);
    if (count) std::memcpy(host.data() + off, src, count * sizeof(T));
    return off;
  }
};

int r_bucket(int k) { return k <= 32 ? 0 : k <= 64 ? 1 : k <= 128 ? 2 : 3; }

// Per-graph state of the host side of the batch.
struct GraphPlan {
  int item = 0;
  int k = 2;
  uint64_t seed64 = 0;
  TailOut table{};
  std::vector<DGraph> levels;     // 0: the input graph, L: the coarsest
  std::vector<const idx_t*> cmaps;  // cmaps[l]: level l -> level l + 1
  std::vector<bool> has_vw;
  std::vector<const idx_t*> heavy;
  std::vector<int32_t> nheavy;
  std::vector<bool> small;
  std::vector<bool> admit;
  bool ok = false;
  // device pieces
  long long* thr = nullptr;  // [L + 1][3][k * ncon]
  idx_t* buf[2] = {nullptr, nullptr};
  idx_t* seeds = nullptr;
  idx_t* trial_parts = nullptr;
  long long* trial_cuts = nullptr;
  unsigned char* grow_scratch = nullptr;  // [trials][grow_scratch_bytes] when the state is not in shared memory
  LevelJob scratch{};  // the scratch pointers shared by the graph's jobs
};

}  // namespace

void Engine::partition_kway_batch(std::vector<BatchItem>& items, const float* ubvec, const KwayOptions& o) {
  cudaStream_t st = stream_;
  const int B = (int)items.size();
  if (B == 0) return;
  const int ncon = items[0].g.ncon;
  for (const BatchItem& it : items)
    if (it.g.ncon != ncon || !batch_eligible(o, it.g.n, it.k, ncon))
      throw Error(-4, "partition_kway_batch: an item is not eligible for the batched kernels");
  std::vector<double> ub(ncon);  // kway.rs:44-49
  for (int c = 0; c < ncon; ++c) ub[c] = ubvec ? (double)ubvec[c] : 1.0 + (double)o.ufactor / 1000.0;
  Arena::Mark call_mark = arena_.mark();
  struct Rewind {
    Arena& a;
    Arena::Mark m;
    ~Rewind() { a.reset_to(m); }
  } rewind{arena_, call_mark};

  using clock = std::chrono::steady_clock;
  const auto t_start = clock::now();
  std::random_device rd;
  std::vector<GraphPlan> plan(B);
  for (int b = 0; b < B; ++b) {
    plan[b].item = b;
    plan[b].k = items[b].k;
    // kway.rs:55-61, attempt 0
    const uint64_t sd = items[b].seed >= 0 ? (uint64_t)items[b].seed : o.seed;
    plan[b].seed64 = sd == 0 ? (((uint64_t)rd() << 32) ^ (uint64_t)rd()) : sd;
  }
  // Largest graphs first: blocks start in index order.
  std::vector<int32_t> order(B);
  for (int b = 0; b < B; ++b) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
    return items[x].g.m != items[y].g.m ? items[x].g.m > items[y].g.m : items[x].g.n > items[y].g.n;
  });

  // ---- 1-2: validation and coarsening ----
  nvtxRangePushA("batch coarsen");
  int64_t ntot = 0;
  for (const BatchItem& it : items) ntot += it.g.n;
  Carver z;  // zero on entry
  int32_t* degcheck = nullptr;
  {
    Carver probe;
    probe.take<int32_t>((size_t)ntot);
    probe.take<int32_t>((size_t)B);
    probe.take<long long>((size_t)B * ncon);
    probe.take<unsigned long long>((size_t)B);
    z.base = arena_.alloc<char>(probe.off);
    RMB_CUDA(cudaMemsetAsync(z.base, 0, probe.off, st));
  }
  degcheck = z.take<int32_t>((size_t)ntot);
  int32_t* d_flags = z.take<int32_t>((size_t)B);
  long long* d_totals = z.take<long long>((size_t)B * ncon);
  unsigned long long* d_cuts = z.take<unsigned long long>((size_t)B);
  const size_t limit_of = 20;  // coarsen/mod.rs:43: max(20 k, 20)
  std::vector<ValJob> vj(B);
  std::vector<TailArgs> ta(B);
  {
    int64_t off = 0;
    for (int b = 0; b < B; ++b) {
      const DGraph& g = items[b].g;
      vj[b].xadj = g.xadj;
      vj[b].adjncy = g.adjncy;
      vj[b].vwgt = g.vwgt;
      vj[b].n = g.n;
      vj[b].ncon = ncon;
      vj[b].degcheck = degcheck + off;
      vj[b].flag = d_flags + b;
      vj[b].total = d_totals + (size_t)b * ncon;
      off += g.n;
      TailArgs& a = ta[b];
      a.g = g;
      a.has_vw = g.vwgt ? 1 : 0;
      a.summed_unit = o.summed_unit_weights;
      a.mode = o.ctype == 0 ? 0 : 1;
      a.lvl0 = 0;
      a.k = items[b].k;
      a.rounds = o.match_rounds;
      a.seed64 = plan[b].seed64;
      a.limit = (long long)std::max<size_t>(limit_of * (size_t)items[b].k, limit_of);
      a.ws_bytes = tail_workspace_bytes(g, o.match_rounds);
      a.ws = arena_.alloc<char>((size_t)a.ws_bytes);
    }
  }
  Staging s1;
  const size_t o_vj = s1.put(vj.data(), vj.size());
  const size_t o_ta = s1.put(ta.data(), ta.size());
  const size_t o_ord = s1.put(order.data(), order.size());
  char* d_s1 = arena_.alloc<char>(s1.host.size());
  RMB_CUDA(cudaMemcpyAsync(d_s1, s1.host.data(), s1.host.size(), cudaMemcpyHostToDevice, st));
  const TailArgs* d_ta = reinterpret_cast<const TailArgs*>(d_s1 + o_ta);
  k_batch_validate<<<B, 512, 0, st>>>(reinterpret_cast<const ValJob*>(d_s1 + o_vj));
  RMB_LAUNCH_CHECK();
  coarsen_tail_batch(d_ta, reinterpret_cast<const int32_t*>(d_s1 + o_ord), d_flags, B, st);
  TailOut* d_tables = arena_.alloc<TailOut>((size_t)B);
  k_gather_tables<<<std::min(B, 148 * 4), 256, 0, st>>>(d_ta, B, d_tables);
  RMB_LAUNCH_CHECK();
  std::vector<TailOut> tables(B);
  std::vector<int32_t> flags(B);
  std::vector<long long> totals((size_t)B * ncon);
  RMB_CUDA(cudaMemcpyAsync(tables.data(), d_tables, sizeof(TailOut) * (size_t)B, cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaMemcpyAsync(flags.data(), d_flags, sizeof(int32_t) * (size_t)B, cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaMemcpyAsync(totals.data(), d_totals, sizeof(long long) * totals.size(), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  nvtxRangePop();
  const auto t_coarsened = clock::now();

  // ---- 3: the plan of every graph ----
  const int T = std::max(1, o.grow_trials);
  Staging s2;
  std::vector<size_t> o_thr(B), o_seed(B);
  size_t zero2 = 0;  // bytes of the second zeroed region (admission out-weights, touched flags)
  for (int b = 0; b < B; ++b) {
    GraphPlan& P = plan[b];
    BatchItem& it = items[b];
    if (flags[b] != 0) {
      it.status = -2;  // METIS_ERROR_INPUT, as validate_device reports it
      continue;
    }
    const TailOut& t = tables[b];
    P.table = t;
    if (!t.finished || t.levels != t.ncoarse + 1) continue;  // status 0: the caller runs it alone
    const int k = it.k;
    const size_t K = (size_t)k * ncon;
    P.levels.push_back(it.g);
    P.has_vw.push_back(it.g.vwgt != nullptr);
    for (int j = 0; j < t.ncoarse; ++j) {
      DGraph c;
      c.n = t.cn[j];
      c.m = t.cm[j];
      c.ncon = ncon;
      c.xadj = reinterpret_cast<const idx_t*>(t.xadj[j]);
      c.adjncy = reinterpret_cast<const idx_t*>(t.adj[j]);
      c.adjwgt = reinterpret_cast<const idx_t*>(t.adjw[j]);
      c.vwgt = t.coarse_vw[j] ? reinterpret_cast<const idx_t*>(t.vwgt[j]) : nullptr;
      P.levels.push_back(c);
      P.cmaps.push_back(reinterpret_cast<const idx_t*>(t.cmap[j]));
      P.has_vw.push_back(t.coarse_vw[j] != 0);
    }
    for (int j = 0; j < t.levels; ++j) {
      P.heavy.push_back(reinterpret_cast<const idx_t*>(t.heavy[j]));
      P.nheavy.push_back(t.nheavy[j]);
    }
    const int L = (int)P.levels.size() - 1;
    // Totals and thresholds of every level (Engine::thresholds, run_attempt's
    // level_total).
    std::vector<int32_t> total0(ncon, it.g.n);
    if (it.g.vwgt)
      for (int c = 0; c < ncon; ++c)
        total0[c] = (int32_t)(uint32_t)(unsigned long long)totals[(size_t)b * ncon + c];
    // The thresholds are filled on the device (k_batch_thresholds); here one
    // value per level and constraint decides the slack width (all parts have
    // the same target).
    std::vector<int32_t> ltot((size_t)(L + 1) * ncon);
    for (int l = 0; l <= L; ++l) {
      std::vector<long long> tot(ncon);
      for (int c = 0; c < ncon; ++c) {
        tot[c] = P.has_vw[l] ? total0[c] : (!it.g.vwgt && o.summed_unit_weights) ? it.g.n : P.levels[l].n;
        ltot[(size_t)l * ncon + c] = (int32_t)tot[c];
      }
      std::vector<long long> f1(ncon), o1(ncon), g1(ncon);
      for (int c = 0; c < ncon; ++c)
        threshold_values((1.0 / (double)k) * (double)(int32_t)tot[c], ub[c], &f1[c], &o1[c], &g1[c]);
      P.small.push_back(weights_fit_int32(tot.data(), ncon, f1.data(), o1.data(), (size_t)ncon));
      const DGraph& lg = P.levels[l];
      const bool fused = o.fused_max_n > 0 && lg.n <= o.fused_max_n &&
                         lg.m <= (int64_t)o.fused_edge_factor * o.fused_max_n;
      P.admit.push_back(!fused && lg.n > o.exact_max_n && admit_supported(k, ncon));
    }
    o_thr[b] = s2.put(ltot.data(), ltot.size());
    // Grow seeds of every trial (grow.rs:26-32, run_attempt's draws).
    const int32_t cn = P.levels[L].n;
    std::vector<int32_t> seeds((size_t)T * k);
    std::vector<char> used(cn);
    for (int tr = 0; tr < T; ++tr) {
      HostRng rng(mix64(P.seed64 ^ (0x9E3779B97F4A7C15ULL * (uint64_t)(tr + 1))));
      std::fill(used.begin(), used.end(), 0);
      for (int p = 0; p < k;) {
        const int32_t v = (int32_t)rng.below((uint64_t)cn);
        if (!used[v]) {
          used[v] = 1;
          seeds[(size_t)tr * k + p] = v;
          ++p;
        }
      }
    }
    o_seed[b] = s2.put(seeds.data(), seeds.size());
    bool any_admit = false;
    for (int l = 0; l <= L; ++l) any_admit = any_admit || P.admit[l];
    if (any_admit) {
      Carver c;
      c.take<long long>(K);
      c.take<idx_t>((size_t)it.g.n);
      c.take<idx_t>((size_t)it.g.n);
      zero2 += c.off;
    }
    P.ok = true;
  }
  char* d_s2 = s2.host.empty() ? nullptr : arena_.alloc<char>(s2.host.size());
  if (d_s2) RMB_CUDA(cudaMemcpyAsync(d_s2, s2.host.data(), s2.host.size(), cudaMemcpyHostToDevice, st));
  Carver z2;
  if (zero2) {
    z2.base = arena_.alloc<char>(zero2);
    RMB_CUDA(cudaMemsetAsync(z2.base, 0, zero2, st));
  }

  // Device scratch of every planned graph, carved from one allocation.
  constexpr size_t kGrowSmemCap = 48 * 1024;  // grow state kept in shared memory up to this size
  const int niter = o.niter;
  auto carve = [&](Carver& c, GraphPlan& P, const BatchItem& it, Carver* zc) {
    const int k = it.k;
    const size_t K = (size_t)k * ncon;
    const int L = (int)P.levels.size() - 1;
    const int32_t n0 = it.g.n;
    const int64_t m0 = it.g.m;
    const int32_t cn = P.levels[L].n;
    P.thr = c.take<long long>(3 * K * (size_t)(L + 1));
    P.trial_parts = c.take<idx_t>((size_t)T * cn);
    P.trial_cuts = c.take<long long>((size_t)T);
    const size_t gb = grow_scratch_bytes(cn, k, ncon);
    P.grow_scratch = gb > kGrowSmemCap ? c.take<unsigned char>(gb * (size_t)T) : nullptr;
    if (L >= 1) {
      P.buf[0] = c.take<idx_t>((size_t)P.levels[1].n);
      P.buf[1] = c.take<idx_t>((size_t)P.levels[1].n);
    }
    LevelJob& J = P.scratch;
    J.pw = c.take<long long>(K);
    J.in_max = c.take<long long>(K);
    J.out_max = c.take<long long>(K);
    J.mover = c.take<idx_t>((size_t)n0);
    J.ncand = c.take<idx_t>((size_t)n0);
    J.wfrom = c.take<idx_t>((size_t)n0);
    J.movers = c.take<idx_t>((size_t)n0);
    J.cand_p = c.take<idx_t>((size_t)m0 + 1);
    J.cand_g = c.take<idx_t>((size_t)m0 + 1);
    J.rec_pv = c.take<int32_t>((size_t)n0);
    J.rec_ne = c.take<int32_t>((size_t)n0);
    J.rec_wf = c.take<int32_t>((size_t)n0);
    J.rec_coff = c.take<int32_t>((size_t)n0);
    J.rec_known = c.take<int32_t>((size_t)n0);
    J.rec_np = c.take<int32_t>((size_t)n0);
    J.rec_cp = c.take<int32_t>((size_t)n0 * kRecInline);
    J.rec_cg = c.take<int32_t>((size_t)n0 * kRecInline);
    J.rec_vw = c.take<int32_t>((size_t)n0 * ncon);
    J.ghist = c.take<int32_t>((size_t)32 * k);
    J.counters = c.take<int32_t>(2 * ((size_t)niter + 1));
    J.long_flag = c.take<int32_t>(1);
    bool any_admit = false;
    for (int l = 0; l <= L; ++l) any_admit = any_admit || P.admit[l];
    if (any_admit) {
      J.a_tgt = c.take<int32_t>((size_t)n0);
      J.a_src = c.take<int32_t>((size_t)n0);
      J.a_rank = c.take<int32_t>((size_t)n0);
      J.a_gsrc = c.take<int32_t>((size_t)n0);
      J.a_w = c.take<int32_t>((size_t)n0 * ncon);
      J.a_pref = c.take<long long>((size_t)n0 * ncon);
      J.a_cut = c.take<int32_t>((size_t)k);
      if (zc) {
        J.a_out = zc->take<long long>(K);
        J.touched[0] = zc->take<idx_t>((size_t)n0);
        J.touched[1] = zc->take<idx_t>((size_t)n0);
      }
    }
    return gb;
  };
  Carver sc;
  {
    Carver probe;
    for (int b = 0; b < B; ++b)
      if (plan[b].ok) carve(probe, plan[b], items[b], nullptr);
    sc.base = probe.off ? arena_.alloc<char>(probe.off) : nullptr;
  }
  // ---- 4: grow trials ----
  std::vector<GrowJob> gj;
  std::vector<ThrJob> thr_jobs;
  std::vector<int32_t> block_job;
  size_t grow_dyn = 0;
  std::vector<int32_t> planned;  // planned graphs, largest first
  for (int32_t b : order)
    if (plan[b].ok) planned.push_back(b);
  for (int32_t b : planned) {
    GraphPlan& P = plan[b];
    const BatchItem& it = items[b];
    const size_t gb = carve(sc, P, it, &z2);
    const int L = (int)P.levels.size() - 1;
    const DGraph& cg = P.levels[L];
    GrowJob j{};
    j.xadj = cg.xadj;
    j.adjncy = cg.adjncy;
    j.adjwgt = cg.adjwgt;
    j.vwgt = cg.vwgt;
    j.n = cg.n;
    j.ncon = ncon;
    j.k = it.k;
    j.trials = T;
    j.seeds = reinterpret_cast<const idx_t*>(d_s2 + o_seed[b]);
    j.grow_tgt = P.thr + 3 * (size_t)it.k * ncon * L + 2 * (size_t)it.k * ncon;
    j.parts = P.trial_parts;
    j.cuts = P.trial_cuts;
    j.use_smem = gb <= kGrowSmemCap ? 1 : 0;
    j.scratch = P.grow_scratch;
    j.scratch_bytes = (long long)gb;
    j.first_block = (int32_t)block_job.size();
    if (j.use_smem) grow_dyn = std::max(grow_dyn, gb);
    for (int tr = 0; tr < T; ++tr) block_job.push_back((int32_t)gj.size());
    gj.push_back(j);
    ThrJob tj;
    tj.thr = P.thr;
    tj.tot = reinterpret_cast<const int32_t*>(d_s2 + o_thr[b]);
    tj.k = it.k;
    tj.ncon = ncon;
    tj.nlevels = L + 1;
    thr_jobs.push_back(tj);
  }

  // ---- 5: the refinement steps (coarsest levels first) ----
  struct Group {
    int step, kind;  // kind 0: k_batch_level, 1: k_batch_admit
    bool has_w, small;
    int rb, kmax;
    size_t first, count;  // range in `jobs`
  };
  std::vector<LevelJob> jobs;
  std::vector<Group> groups;
  int max_steps = 0;
  for (int32_t b : planned) max_steps = std::max(max_steps, (int)plan[b].levels.size());
  for (int s = 0; s < max_steps; ++s) {
    struct Entry {
      int32_t b;
      int l;
    };
    // Step s refines level index max_steps - 1 - s of every graph that has
    // it: the graphs with the most levels start first and every graph ends
    // with its input level in the last step. A step lasts as long as its
    // largest level, and the largest levels of a step are then the same
    // graph's (the largest graphs have the largest level at each index), so
    // the steps add up to about that graph's own refinement time.
    std::vector<Entry> es;
    const int l_step = max_steps - 1 - s;
    for (int32_t b : planned) {
      const int L = (int)plan[b].levels.size() - 1;
      if (l_step <= L) es.push_back({b, l_step});
    }
    auto make_job = [&](const Entry& e) {
      GraphPlan& P = plan[e.b];
      const BatchItem& it = items[e.b];
      const int L = (int)P.levels.size() - 1;
      const int l = e.l;
      const DGraph& lg = P.levels[l];
      const size_t K = (size_t)it.k * ncon;
      LevelJob J = P.scratch;
      J.xadj = lg.xadj;
      J.adjncy = lg.adjncy;
      J.adjwgt = lg.adjwgt;
      J.vwgt = lg.vwgt;
      J.n = lg.n;
      J.ncon = ncon;
      J.k = it.k;
      J.niter = niter;
      if (l == L) {
        J.trial_parts = P.trial_parts;
        J.trial_cuts = P.trial_cuts;
        J.trials = T;
        J.cmap = nullptr;
        J.cpart = nullptr;
      } else {
        J.trial_parts = nullptr;
        J.trial_cuts = nullptr;
        J.trials = 0;
        J.cmap = P.cmaps[l];
        J.cpart = P.buf[(l + 1) & 1];
      }
      J.part = l == 0 ? it.part_out : P.buf[l & 1];
      J.feas = P.thr + 3 * K * (size_t)l;
      J.over = P.thr + 3 * K * (size_t)l + K;
      J.heavy = P.heavy[l];
      J.nheavy = P.nheavy[l];
      J.admit = P.admit[l] ? 1 : 0;
      return J;
    };
    // k_batch_level groups by kernel variant, largest levels first
    std::stable_sort(es.begin(), es.end(), [&](const Entry& x, const Entry& y) {
      return plan[x.b].levels[x.l].m > plan[y.b].levels[y.l].m;
    });
    for (int kind = 0; kind < 2; ++kind) {
      for (int hw = 1; hw >= 0; --hw)
        for (int sm = 1; sm >= 0; --sm)
          for (int rb = 0; rb < 4; ++rb) {
            if (kind == 1 && (sm != 1 || rb != 0)) continue;  // admission groups: by edge weights only
            Group gr{s, kind, hw == 1, sm == 1, rb, 0, jobs.size(), 0};
            for (const Entry& e : es) {
              const GraphPlan& P = plan[e.b];
              const DGraph& lg = P.levels[e.l];
              if ((lg.adjwgt != nullptr) != (hw == 1)) continue;
              if (kind == 0 && ((bool)P.small[e.l] != (sm == 1) || r_bucket(items[e.b].k) != rb)) continue;
              if (kind == 1 && !P.admit[e.l]) continue;
              jobs.push_back(make_job(e));
              gr.kmax = std::max(gr.kmax, items[e.b].k);
              ++gr.count;
            }
            if (gr.count) groups.push_back(gr);
          }
    }
  }
  // ---- 6: cuts ----
  std::vector<CutJob> cj;
  for (int32_t b : planned) {
    const BatchItem& it = items[b];
    CutJob c{};
    c.xadj = it.g.xadj;
    c.adjncy = it.g.adjncy;
    c.adjwgt = it.g.adjwgt;
    c.part = it.part_out;
    c.n = it.g.n;
    c.cut = d_cuts + b;
    cj.push_back(c);
  }
  const auto t_planned = clock::now();
  Staging s3;
  const size_t o_gj = s3.put(gj.data(), gj.size());
  const size_t o_tj = s3.put(thr_jobs.data(), thr_jobs.size());
  const size_t o_bj = s3.put(block_job.data(), block_job.size());
  const size_t o_jobs = s3.put(jobs.data(), jobs.size());
  const size_t o_cj = s3.put(cj.data(), cj.size());
  char* d_s3 = s3.host.empty() ? nullptr : arena_.alloc<char>(s3.host.size());
  if (!planned.empty()) {
    RMB_CUDA(cudaMemcpyAsync(d_s3, s3.host.data(), s3.host.size(), cudaMemcpyHostToDevice, st));
    UbVec ubv{};
    for (int c = 0; c < ncon && c < 8; ++c) ubv.v[c] = ub[c];
    k_batch_thresholds<<<(int)thr_jobs.size(), 256, 0, st>>>(reinterpret_cast<const ThrJob*>(d_s3 + o_tj), ubv);
    RMB_LAUNCH_CHECK();
    nvtxRangePushA("batch grow");
    grow_trials_batch(reinterpret_cast<const GrowJob*>(d_s3 + o_gj), reinterpret_cast<const int32_t*>(d_s3 + o_bj),
                      (int)block_job.size(), grow_dyn, st);
    nvtxRangePop();
    nvtxRangePushA("batch refine");
    const LevelJob* d_jobs = reinterpret_cast<const LevelJob*>(d_s3 + o_jobs);
    const bool verbose = std::getenv("RMETIS_B200_VERBOSE") != nullptr;
    std::vector<cudaEvent_t> ev;
    if (verbose) {
      ev.resize(groups.size() + 1);
      for (auto& e : ev) RMB_CUDA(cudaEventCreate(&e));
      RMB_CUDA(cudaEventRecord(ev[0], st));
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      const Group& gr = groups[gi];
      if (gr.kind == 0)
        batch_level_launch(d_jobs + gr.first, (int)gr.count, gr.has_w, gr.small, gr.kmax, ncon, st);
      else
        batch_admit_launch(d_jobs + gr.first, (int)gr.count, gr.has_w, st);
      if (verbose) RMB_CUDA(cudaEventRecord(ev[gi + 1], st));
    }
    if (verbose) {
      RMB_CUDA(cudaEventSynchronize(ev.back()));
      for (size_t gi = 0; gi < groups.size(); ++gi) {
        float ms = 0.f;
        RMB_CUDA(cudaEventElapsedTime(&ms, ev[gi], ev[gi + 1]));
        const Group& gr = groups[gi];
        int32_t nmax = 0;
        for (size_t j = gr.first; j < gr.first + gr.count; ++j) nmax = std::max(nmax, jobs[j].n);
        std::fprintf(stderr, "rmetis_b200: batch step %d %s: %zu levels (largest %d vertices), %.2f ms\n", gr.step,
                     gr.kind == 0 ? "level" : "admission", gr.count, nmax, ms);
      }
      for (auto& e : ev) cudaEventDestroy(e);
    }
    nvtxRangePop();
    k_batch_cut<<<(int)cj.size(), 512, 0, st>>>(reinterpret_cast<const CutJob*>(d_s3 + o_cj));
    RMB_LAUNCH_CHECK();
  }
  std::vector<unsigned long long> cuts(B, 0);
  RMB_CUDA(cudaMemcpyAsync(cuts.data(), d_cuts, sizeof(unsigned long long) * (size_t)B, cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  for (int32_t b : planned) {
    items[b].objval = (int32_t)(uint32_t)cuts[b] / 2;  // kway.rs:94-98 as run_attempt reads it
    items[b].status = 1;
  }
  if (std::getenv("RMETIS_B200_VERBOSE")) {
    const auto t_end = clock::now();
    auto ms = [](clock::time_point a, clock::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    std::fprintf(stderr,
                 "rmetis_b200: batch of %d graphs: %zu through the batched kernels in %zu refinement launches; "
                 "validation and coarsening %.1f ms, planning %.1f ms, grow, refinement and cuts %.1f ms\n",
                 B, planned.size(), groups.size(), ms(t_start, t_coarsened), ms(t_coarsened, t_planned),
                 ms(t_planned, t_end));
  }
  if (profiler().on) profiler().collect();
}

}  // namespace rmb
