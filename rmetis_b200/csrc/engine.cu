// Host orchestration of the multilevel k-way pipeline
// (src/partition/kway.rs:20-162 and src/coarsen/mod.rs:36-71).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <sstream>

#include <nvtx3/nvToolsExt.h>

#include "engine.h"
#include "hostrng.h"
#include "prof.h"

namespace rmb {

// ---------------------------------------------------------------------------
// Profiler
// ---------------------------------------------------------------------------
Profiler& profiler() {
  static Profiler p;
  return p;
}

std::atomic<long long>& launch_counter() {
  static std::atomic<long long> c{0};
  return c;
}

cudaEvent_t Profiler::get() {
  if (!pool_.empty()) {
    cudaEvent_t e = pool_.back();
    pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  RMB_CUDA(cudaEventCreate(&e));
  return e;
}

int Profiler::begin(int id, cudaStream_t st) {
  if (!on) return -1;
  std::lock_guard<std::mutex> lk(mu_);
  Rec r{id, get(), get(), 0.0};
  RMB_CUDA(cudaEventRecord(r.a, st));
  recs_.push_back(r);
  return (int)recs_.size() - 1;
}

void Profiler::end(int h, cudaStream_t st, double bytes) {
  if (h < 0) return;
  std::lock_guard<std::mutex> lk(mu_);
  recs_[h].bytes = bytes;
  RMB_CUDA(cudaEventRecord(recs_[h].b, st));
}

void Profiler::collect() {
  std::lock_guard<std::mutex> lk(mu_);
  for (auto& r : recs_) {
    RMB_CUDA(cudaEventSynchronize(r.b));
    float ms = 0.f;
    RMB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    totals.launches[r.id] += 1;
    totals.ms[r.id] += ms;
    totals.bytes[r.id] += r.bytes;
    pool_.push_back(r.a);
    pool_.push_back(r.b);
  }
  recs_.clear();
}

void Profiler::reset() {
  collect();
  std::lock_guard<std::mutex> lk(mu_);
  totals = ProfTotals{};
}

// ---------------------------------------------------------------------------
// Thresholds
// ---------------------------------------------------------------------------
void threshold_values(double t, double ub, long long* feas, long long* over, long long* grow) {
  const double lim = 9.0e18;
  const double x = t * ub;
  if (std::isnan(x)) {
    *feas = LLONG_MIN;
    *over = LLONG_MAX;
  } else if (x >= lim) {
    *feas = LLONG_MAX;
    *over = LLONG_MAX;
  } else if (x <= -lim) {
    *feas = LLONG_MIN;
    *over = LLONG_MIN;
  } else {
    const long long f = (long long)std::floor(x);
    *feas = f;
    *over = f;
  }
  if (std::isnan(t) || t >= lim) *grow = LLONG_MAX;
  else if (t <= -lim) *grow = LLONG_MIN;
  else *grow = (long long)std::ceil(t);
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
Engine::Engine(bool is_worker) : is_worker_(is_worker) {
  RMB_CUDA(cudaGetDevice(&device_));
  RMB_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
  stream_ = own_stream_;
  RMB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_scratch_), 4096));
  RMB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_tail_), sizeof(TailOut)));
}

Engine::~Engine() {
  // Process teardown may already have unloaded the driver; ignore errors.
  arena_.release();
  if (h_thr_) cudaFreeHost(h_thr_);
  if (h_scratch_) cudaFreeHost(h_scratch_);
  if (h_tail_) cudaFreeHost(h_tail_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Engine::reset_stats() { profiler().reset(); }

void Engine::thresholds(const std::vector<std::vector<int32_t>>& totals, int k, int ncon, const float* tpwgts,
                        const std::vector<double>& ub, long long* d_thr) {
  const size_t K = (size_t)k * ncon;
  const size_t need = 3 * K * totals.size();
  // The staging buffer may still feed an earlier copy.
  RMB_CUDA(cudaStreamSynchronize(stream_));
  if (h_thr_cap_ < need) {
    if (h_thr_) cudaFreeHost(h_thr_);
    RMB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_thr_), sizeof(long long) * need));
    h_thr_cap_ = need;
  }
  for (size_t l = 0; l < totals.size(); ++l) {
    long long* h = h_thr_ + 3 * K * l;
    for (int p = 0; p < k; ++p)
      for (int c = 0; c < ncon; ++c) {
        // compute_target_weights (src/graph/mod.rs:392-410), f64
        const double f = tpwgts ? (double)tpwgts[(size_t)p * ncon + c] : 1.0 / (double)k;
        const double t = f * (double)totals[l][c];
        const size_t i = (size_t)p * ncon + c;
        threshold_values(t, ub[c], &h[i], &h[K + i], &h[2 * K + i]);
      }
  }
  RMB_CUDA(cudaMemcpyAsync(d_thr, h_thr_, sizeof(long long) * need, cudaMemcpyHostToDevice, stream_));
}

int Engine::partition_kway(const DGraph& g0, int nparts, const float* tpwgts, const float* ubvec,
                           const KwayOptions& o, idx_t* part_out, int32_t* objval, KwayTrace* trace) {
  cudaStream_t st = stream_;
  const int k = nparts;
  const int ncon = g0.ncon;
  if (k < 2 || k > g0.n) throw Error(-2, "nparts out of range");   // kway.rs:31-38
  if (ncon > 8) throw Error(-2, "ncon above the supported maximum of 8");
  std::vector<double> ub(ncon);                                     // kway.rs:44-49
  for (int c = 0; c < ncon; ++c) ub[c] = ubvec ? (double)ubvec[c] : 1.0 + (double)o.ufactor / 1000.0;

  Arena::Mark call_mark = arena_.mark();
  long long* d_tot = arena_.alloc<long long>((size_t)ncon);

  // Total weight of the input (i32 with wrap-around, like the reference).
  std::vector<int32_t> total0(ncon, g0.n);
  if (g0.vwgt) {
    total_weight(g0, d_tot, st);
    RMB_CUDA(cudaMemcpyAsync(h_scratch_ + 16, d_tot, sizeof(long long) * ncon, cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    for (int c = 0; c < ncon; ++c) {
      long long t;
      std::memcpy(&t, reinterpret_cast<char*>(h_scratch_ + 16) + sizeof(long long) * c, sizeof(long long));
      total0[c] = (int32_t)(uint32_t)(unsigned long long)t;
    }
  }

  std::random_device rd;
  std::vector<uint64_t> seeds(o.ncuts);
  for (int a = 0; a < o.ncuts; ++a)                                 // kway.rs:55-61
    seeds[a] = o.seed == 0 ? (((uint64_t)rd() << 32) ^ (uint64_t)rd()) : o.seed + (uint64_t)a;

  bool have_best = false;
  int32_t best_obj = 0;
  if (o.ncuts > 1 && o.parallel_attempts && !is_worker_ && !trace) {
    // Attempts are independent (the reference stripes them over MPI ranks,
    // kway.rs:54): run them on the worker pool, each into its own buffer, and
    // keep the first attempt with the lowest cut (strict <, kway.rs:96-98).
    WorkerPool& pool = pool_for_device(device_);
    std::vector<idx_t*> parts(o.ncuts);
    for (int a = 0; a < o.ncuts; ++a) parts[a] = arena_.alloc<idx_t>((size_t)g0.n);
    RMB_CUDA(cudaStreamSynchronize(st));  // the input is complete before other streams read it
    std::vector<int32_t> objs(o.ncuts, 0);
    std::vector<std::future<int>> fut;
    const size_t fp = footprint_bytes(g0.n, g0.m, k, ncon);
    for (int a = 0; a < o.ncuts; ++a) {
      fut.push_back(pool.submit(fp, [&, a](Engine& e) {
        e.run_attempt(g0, k, tpwgts, ub, total0, o, seeds[a], parts[a], &objs[a], nullptr);
        return 1;
      }));
    }
    int rc = 1;
    for (auto& f : fut) {
      const int r = f.get();
      if (r != 1 && rc == 1) rc = r;
    }
    if (rc != 1) {
      arena_.reset_to(call_mark);
      throw Error(rc, "an attempt failed");
    }
    int best = 0;
    for (int a = 1; a < o.ncuts; ++a)
      if (objs[a] < objs[best]) best = a;
    best_obj = objs[best];
    RMB_CUDA(cudaMemcpyAsync(part_out, parts[best], sizeof(idx_t) * g0.n, cudaMemcpyDeviceToDevice, st));
    RMB_CUDA(cudaStreamSynchronize(st));
  } else {
    for (int a = 0; a < o.ncuts; ++a) {                                 // kway.rs:54
      Arena::Mark att_mark = arena_.mark();
      idx_t* part = arena_.alloc<idx_t>((size_t)g0.n);
      KwayTrace local;
      int32_t obj = 0;
      run_attempt(g0, k, tpwgts, ub, total0, o, seeds[a], part, &obj, trace ? &local : nullptr);
      if (!have_best || obj < best_obj) {                               // kway.rs:96-98
        best_obj = obj;
        have_best = true;
        RMB_CUDA(cudaMemcpyAsync(part_out, part, sizeof(idx_t) * g0.n, cudaMemcpyDeviceToDevice, st));
        if (trace) *trace = std::move(local);
      }
      RMB_CUDA(cudaStreamSynchronize(st));
      arena_.reset_to(att_mark);
    }
  }
  arena_.reset_to(call_mark);
  if (objval) *objval = best_obj;
  if (profiler().on) profiler().collect();
  return 1;
}

void Engine::run_attempt(const DGraph& g0, int k, const float* tpwgts, const std::vector<double>& ub,
                         const std::vector<int32_t>& total0, const KwayOptions& o, uint64_t seed64, idx_t* part_out,
                         int32_t* objval, KwayTrace* trace) {
  cudaStream_t st = stream_;
  const int ncon = g0.ncon;
  const size_t K = (size_t)k * ncon;
  const size_t limit = std::max<size_t>((size_t)20 * k, 20);         // coarsen/mod.rs:43
  Arena::Mark att_mark = arena_.mark();
  unsigned long long* d_cut = arena_.alloc<unsigned long long>(1);
  KwayTrace local;
  const bool json = trace_json_path() != nullptr;
  struct LevelRec {
    int32_t n;
    int64_t m;
    int64_t passes = 0, moves = 0;
    cudaEvent_t a = nullptr, b = nullptr;
  };
  std::vector<LevelRec> recs;
  nvtxRangePushA("rmetis attempt");
  {
    // ---- coarsening (coarsen/mod.rs:36-71) ----
    nvtxRangePushA("coarsen");
    std::vector<DGraph> levels{g0};
    std::vector<idx_t*> cmaps;
    std::vector<idx_t*> heavy_lists;
    std::vector<int32_t> heavy_counts;
    std::vector<bool> has_vw{g0.vwgt != nullptr};
    bool tail_open = o.tail_max_n > 0;
    for (int lvl = 0;; ++lvl) {
      if (tail_open && levels.back().n <= o.tail_max_n && levels.back().m <= 64LL * o.tail_max_n) {
        // The remaining levels in one launch; a tail that ran out of room
        // hands back to this loop at the level after the last one it kept.
        tail_open = false;
        const DGraph from = levels.back();
        const size_t base = levels.size() - 1;
        coarsen_tail(from, has_vw.back() ? 1 : 0, o.summed_unit_weights, o.ctype == 0 ? 0 : 1, seed64, lvl, k,
                     (int64_t)limit, o.match_rounds, arena_, st, h_tail_);
        const TailOut& t = *h_tail_;
        for (int j = 0; j < t.ncoarse; ++j) {
          DGraph c;
          c.n = t.cn[j];
          c.m = t.cm[j];
          c.ncon = from.ncon;
          c.xadj = reinterpret_cast<const idx_t*>(t.xadj[j]);
          c.adjncy = reinterpret_cast<const idx_t*>(t.adj[j]);
          c.adjwgt = reinterpret_cast<const idx_t*>(t.adjw[j]);
          c.vwgt = t.coarse_vw[j] ? reinterpret_cast<const idx_t*>(t.vwgt[j]) : nullptr;
          levels.push_back(c);
          cmaps.push_back(reinterpret_cast<idx_t*>(t.cmap[j]));
          has_vw.push_back(t.coarse_vw[j] != 0);
        }
        for (int j = 0; j < t.levels; ++j) {
          heavy_lists.push_back(reinterpret_cast<idx_t*>(t.heavy[j]));
          heavy_counts.push_back(t.nheavy[j]);
          if (trace && t.match[j]) {
            std::vector<int32_t> hm(levels[base + j].n);
            RMB_CUDA(cudaMemcpyAsync(hm.data(), reinterpret_cast<const void*>(t.match[j]), sizeof(int32_t) * hm.size(),
                                     cudaMemcpyDeviceToHost, st));
            RMB_CUDA(cudaStreamSynchronize(st));
            local.matchings.push_back(std::move(hm));
          }
        }
        if (t.finished) break;
        if (t.ncoarse > 0) {
          lvl += t.ncoarse - 1;
          continue;
        }
      }
      const DGraph& cur = levels.back();
      idx_t* hl = arena_.alloc<idx_t>((size_t)cur.n);
      const int32_t nh = heavy_list(cur, hl, arena_, st, h_scratch_);
      heavy_lists.push_back(hl);
      heavy_counts.push_back(nh);
      Arena::Mark mm = arena_.mark();
      idx_t* match = arena_.alloc<idx_t>((size_t)cur.n);
      const uint64_t lseed = mix64(seed64 * 0x100000001b3ULL + (uint64_t)lvl + 1);
      // A cooperative launch waits until all its blocks fit on the device at
      // once, which stalls a worker whose jobs share the device with others:
      // workers match with one launch per phase.
      match_parallel(cur, o.ctype == 0 ? 0 : 1, lseed, o.match_rounds, match, hl, nh, arena_, st, h_scratch_,
                     !is_worker_);
      if (trace) {
        std::vector<int32_t> hm(cur.n);
        RMB_CUDA(cudaMemcpyAsync(hm.data(), match, sizeof(int32_t) * cur.n, cudaMemcpyDeviceToHost, st));
        RMB_CUDA(cudaStreamSynchronize(st));
        local.matchings.push_back(std::move(hm));
      }
      // Coarse vertex weights: the reference gives a coarse graph vwgt only
      // when the fine graph has it (graph/mod.rs:300).
      const bool coarse_vw = has_vw.back() || o.summed_unit_weights;
      CoarseResult cr = contract(cur, match, coarse_vw ? 1 : 0, arena_, st, h_scratch_, o.contract_thread_max);
      // The matching is scratch once contracted; keep the coarse level.
      (void)mm;
      const float ratio = (float)cr.g.n / (float)cur.n;
      if ((size_t)cr.g.n < (size_t)k) {
        // A coarsest graph with fewer vertices than parts cannot seed k parts
        // (the reference's seed draw would never end); keep the finer level.
        break;
      }
      levels.push_back(cr.g);
      cmaps.push_back(cr.cmap);
      has_vw.push_back(coarse_vw);
      if ((size_t)cr.g.n <= limit || ratio > 0.95f) break;
    }
    nvtxRangePop();  // coarsen
    const int L = (int)levels.size() - 1;  // number of coarse levels
    if (checks_enabled())
      for (int l = 0; l < L; ++l) check_contraction(levels[l], levels[l + 1], cmaps[l], arena_, st, h_scratch_);
    // heavy list of the coarsest level (the loop computed lists for 0..L-1)
    if ((int)heavy_lists.size() < (int)levels.size()) {
      idx_t* hl = arena_.alloc<idx_t>((size_t)levels.back().n);
      heavy_counts.push_back(heavy_list(levels.back(), hl, arena_, st, h_scratch_));
      heavy_lists.push_back(hl);
    }
    if (trace) {
      for (auto& lv : levels) {
        local.level_n.push_back(lv.n);
        local.level_m.push_back(lv.m);
      }
    }

    auto level_total = [&](int l) {
      if (has_vw[l]) return total0;
      if (!g0.vwgt && o.summed_unit_weights) return std::vector<int32_t>(ncon, g0.n);
      return std::vector<int32_t>(ncon, levels[l].n);
    };

    // Thresholds of every level (one upload): [l][feas, over, grow][k][ncon].
    long long* d_thr = arena_.alloc<long long>(3 * K * (size_t)(L + 1));
    {
      std::vector<std::vector<int32_t>> totals;
      for (int l = 0; l <= L; ++l) totals.push_back(level_total(l));
      thresholds(totals, k, ncon, tpwgts, ub, d_thr);
    }
    // Host copy of the thresholds (still in the staging buffer) decides
    // whether each level's walk can keep 32-bit slacks.
    std::vector<bool> small(L + 1);
    for (int l = 0; l <= L; ++l) {
      std::vector<long long> tot;
      for (int32_t t : level_total(l)) tot.push_back(t);
      small[l] = weights_fit_int32(tot.data(), ncon, h_thr_ + 3 * K * (size_t)l, h_thr_ + 3 * K * (size_t)l + K, K);
    }
    auto feas_of = [&](int l) { return d_thr + 3 * K * (size_t)l; };
    auto over_of = [&](int l) { return d_thr + 3 * K * (size_t)l + K; };
    long long* d_grow = d_thr + 3 * K * (size_t)L + 2 * K;

    // ---- initial partition of the coarsest graph (initial/mod.rs:11-22) ----
    nvtxRangePushA("initial partition");
    const DGraph& cg = levels.back();
    idx_t* part = arena_.alloc<idx_t>((size_t)cg.n);
    if (o.iptype == 1) {
      // random_partition (src/initial/random.rs:8-10): every vertex draws
      // gen_range(0..k), rand 0.8's widening-multiply sampler, from an
      // xoshiro256++ stream. Like the grown partitions, grow_trials draws are
      // made (one stream each) and the one with the lowest cut is kept.
      const int T = std::max(1, o.grow_trials);
      std::vector<int32_t> hp((size_t)T * cg.n);
      for (int t = 0; t < T; ++t) {
        HostRng rng(mix64(seed64 ^ 0x52414e44ULL ^ (0x9E3779B97F4A7C15ULL * (uint64_t)t)));
        for (int32_t v = 0; v < cg.n; ++v) hp[(size_t)t * cg.n + v] = (int32_t)rng.below((uint64_t)k);
      }
      Arena::Mark rm = arena_.mark();
      idx_t* d_parts = arena_.alloc<idx_t>(hp.size());
      long long* d_cuts = arena_.alloc<long long>((size_t)T);
      RMB_CUDA(cudaMemcpyAsync(d_parts, hp.data(), sizeof(int32_t) * hp.size(), cudaMemcpyHostToDevice, st));
      trial_cuts(cg, d_parts, T, d_cuts, st);
      std::vector<long long> cuts(T);
      RMB_CUDA(cudaMemcpyAsync(cuts.data(), d_cuts, sizeof(long long) * T, cudaMemcpyDeviceToHost, st));
      RMB_CUDA(cudaStreamSynchronize(st));
      int bt = 0;
      for (int t = 1; t < T; ++t)
        if (cuts[t] < cuts[bt]) bt = t;
      RMB_CUDA(cudaMemcpyAsync(part, d_parts + (size_t)bt * cg.n, sizeof(idx_t) * cg.n, cudaMemcpyDeviceToDevice,
                               st));
      (void)rm;
    } else {
      const int T = std::max(1, o.grow_trials);
      std::vector<int32_t> seeds((size_t)T * k);
      std::vector<char> used(cg.n);
      for (int t = 0; t < T; ++t) {
        HostRng rng(mix64(seed64 ^ (0x9E3779B97F4A7C15ULL * (uint64_t)(t + 1))));
        std::fill(used.begin(), used.end(), 0);
        for (int p = 0; p < k;) {                                     // grow.rs:26-32
          const int32_t v = (int32_t)rng.below((uint64_t)cg.n);
          if (!used[v]) {
            used[v] = 1;
            seeds[(size_t)t * k + p] = v;
            ++p;
          }
        }
      }
      Arena::Mark gm = arena_.mark();
      idx_t* d_seeds = arena_.alloc<idx_t>(seeds.size());
      idx_t* d_parts = arena_.alloc<idx_t>((size_t)T * cg.n);
      long long* d_cuts = arena_.alloc<long long>((size_t)T);
      RMB_CUDA(cudaMemcpyAsync(d_seeds, seeds.data(), sizeof(int32_t) * seeds.size(), cudaMemcpyHostToDevice, st));
      grow_trials(cg, k, T, d_seeds, d_grow, d_parts, d_cuts, arena_, st);
      std::vector<long long> cuts(T);
      RMB_CUDA(cudaMemcpyAsync(cuts.data(), d_cuts, sizeof(long long) * T, cudaMemcpyDeviceToHost, st));
      RMB_CUDA(cudaStreamSynchronize(st));
      int bt = 0;
      for (int t = 1; t < T; ++t)
        if (cuts[t] < cuts[bt]) bt = t;
      RMB_CUDA(cudaMemcpyAsync(part, d_parts + (size_t)bt * cg.n, sizeof(idx_t) * cg.n, cudaMemcpyDeviceToDevice,
                               st));
      if (trace) local.grow_seeds.assign(seeds.begin() + (size_t)bt * k, seeds.begin() + (size_t)(bt + 1) * k);
      (void)gm;
    }

    // ---- refinement at the coarsest level and on the way up (kway.rs:72-92) ----
    // refine_level (kway.rs:145-162): Greedy, or FM through refine_kway
    // (src/refine/mod.rs:26-38).
    nvtxRangePop();  // initial partition
    auto refine_level = [&](int rtype, const DGraph& lg, idx_t* lpart, const RefineParams& lrp, const idx_t* hl,
                            int32_t nh) {
      nvtxRangePushA(rtype == 1 ? "refine level (greedy)" : "refine level (fm)");
      LevelRec rec;
      rec.n = lg.n;
      rec.m = lg.m;
      if (json) {
        RMB_CUDA(cudaEventCreate(&rec.a));
        RMB_CUDA(cudaEventCreate(&rec.b));
        RMB_CUDA(cudaEventRecord(rec.a, st));
      }
      RefineStats rs = rtype == 1 ? greedy_refine(lg, lpart, lrp, hl, nh, arena_, st, h_scratch_)
                       : (k == 2 && o.bisect_fm2) ? fm2_refine(lg, lpart, lrp, arena_, st, h_scratch_)
                                                   : fm_refine(lg, lpart, lrp, hl, nh, arena_, st, h_scratch_);
      if (json) {
        RMB_CUDA(cudaEventRecord(rec.b, st));
        rec.passes = rs.passes;
        rec.moves = rs.moves;
        recs.push_back(rec);
      }
      if (checks_enabled()) check_refined(lg, lpart, k, arena_, st, h_scratch_);
      nvtxRangePop();
      return rs;
    };
    RefineParams rp;
    rp.k = k;
    rp.niter = o.niter;
    rp.feas_max = feas_of(L);
    rp.over_thr = over_of(L);
    rp.small_weights = small[L];
    rp.fused_max_n = o.fused_max_n;
    rp.fused_edge_factor = o.fused_edge_factor;
    rp.fm_fused_max_n = o.fm_fused_max_n;
    // A traced run replays bit for bit in the oracle: exact walks everywhere.
    rp.exact_max_n = trace ? INT32_MAX : o.exact_max_n;
    rp.gain_block = o.gain_block;
    rp.collect_stats = trace != nullptr || json;
    {
      RefineStats rs = refine_level(o.rtype, cg, part, rp, heavy_lists[L], heavy_counts[L]);
      local.refine_passes += rs.passes;
      local.refine_moves += rs.moves;
      local.decide_rounds += rs.decide_iters;
    }
    for (int i = L - 1; i >= 0; --i) {
      const DGraph& fg = levels[i];
      idx_t* fpart = arena_.alloc<idx_t>((size_t)fg.n);
      project(fg.n, cmaps[i], part, fpart, st);
      part = fpart;
      rp.feas_max = feas_of(i);
      rp.over_thr = over_of(i);
      rp.small_weights = small[i];
      RefineStats rs = refine_level(o.rtype, fg, part, rp, heavy_lists[i], heavy_counts[i]);
      local.refine_passes += rs.passes;
      local.refine_moves += rs.moves;
      local.decide_rounds += rs.decide_iters;
    }

    // ---- objective (kway.rs:94-98) ----
    cut_and_weights(g0, part, k, d_cut, nullptr, st);
    unsigned long long cut_raw = 0;
    RMB_CUDA(cudaMemcpyAsync(part_out, part, sizeof(idx_t) * g0.n, cudaMemcpyDeviceToDevice, st));
    RMB_CUDA(cudaMemcpyAsync(h_scratch_ + 32, d_cut, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    std::memcpy(&cut_raw, h_scratch_ + 32, sizeof(cut_raw));
    *objval = (int32_t)(uint32_t)cut_raw / 2;
    if (trace) *trace = std::move(local);
    if (json) {
      // One line per attempt: every refined level, coarsest first.
      std::ostringstream os;
      os << "{\"n\": " << g0.n << ", \"m\": " << g0.m << ", \"k\": " << k << ", \"ncon\": " << ncon
         << ", \"seed\": " << seed64 << ", \"rtype\": \"" << (o.rtype == 1 ? "greedy" : "fm")
         << "\", \"cut\": " << *objval << ", \"levels\": [";
      for (size_t i = 0; i < recs.size(); ++i) {
        float ms = 0.f;
        RMB_CUDA(cudaEventElapsedTime(&ms, recs[i].a, recs[i].b));
        const double bytes = (double)recs[i].passes * (12.0 * recs[i].n + 12.0 * (double)recs[i].m);
        os << (i ? ", " : "") << "{\"n\": " << recs[i].n << ", \"m\": " << recs[i].m << ", \"passes\": "
           << recs[i].passes << ", \"moves\": " << recs[i].moves << ", \"refine_ms\": " << ms
           << ", \"gain_gbps\": " << (ms > 0 ? bytes / (ms * 1e-3) / 1e9 : 0.0) << "}";
        cudaEventDestroy(recs[i].a);
        cudaEventDestroy(recs[i].b);
      }
      os << "]}";
      trace_json_write(os.str());
    }
  }
  nvtxRangePop();  // attempt
  arena_.reset_to(att_mark);
}

Engine& engine_for_current_device() {
  static std::mutex m;
  static std::vector<Engine*> engines;
  int dev = 0;
  RMB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(m);
  if ((int)engines.size() <= dev) engines.resize(dev + 1, nullptr);
  if (!engines[dev]) engines[dev] = new Engine();  // lives until process exit
  return *engines[dev];
}

}  // namespace rmb
