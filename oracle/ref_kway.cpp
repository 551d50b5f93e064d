// Oracle: CPU restatement of rmetis's multilevel k-way hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the CPU reference that the CUDA path in
// rmetis_b200/ is compared with. Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference legs load it; the product never links it.
//
// It restates, function by function and quirks included, the Rust reference
// (javagg/rmetis). Every function cites the reference file:line it follows.
// The reference itself cannot be built here (no Rust toolchain; the crate also
// needs a system MPI), so this restatement is pinned against the reference's
// own known-answer unit tests (tests/test_oracle.py).
//
// Third-party arithmetic: the reference draws random numbers from
// rand 0.8.5 / rand_core 0.6.4 (Cargo.lock:634-660), not vendored. SmallRng on
// 64-bit targets is xoshiro256++ (Blackman & Vigna); SmallRng::seed_from_u64 is
// rand_core's default PCG32-based seed expansion (O'Neill); uniform integers use
// rand 0.8's widening-multiply rejection sampler. They are restated below from
// those published algorithms. No reference test pins a seeded random stream or
// a seeded cut value, so the seeded RNG streams are "parity unpinned".
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <limits>
#include <random>
#include <set>
#include <vector>

namespace {

using Idx = int32_t;

// ---------------------------------------------------------------------------
// rand 0.8.5 SmallRng (xoshiro256++) + rand_core 0.6.4 seed_from_u64
// ---------------------------------------------------------------------------
struct SmallRng {
  uint64_t s[4];

  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

  // rand_core::SeedableRng::seed_from_u64 default: PCG32 output, 4 bytes at a
  // time, little-endian into the 32-byte seed.
  static SmallRng seed_from_u64(uint64_t state) {
    const uint64_t MUL = 6364136223846793005ULL;
    const uint64_t INC = 11634580027462260723ULL;
    uint8_t seed[32];
    for (int chunk = 0; chunk < 8; ++chunk) {
      state = state * MUL + INC;
      uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
      uint32_t rot = (uint32_t)(state >> 59);
      uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
      for (int b = 0; b < 4; ++b) seed[chunk * 4 + b] = (uint8_t)(x >> (8 * b));
    }
    return from_seed(seed);
  }

  // Xoshiro256PlusPlus::from_seed; an all-zero seed falls back to the
  // generator's own SplitMix64 seeding of 0.
  static SmallRng from_seed(const uint8_t seed[32]) {
    SmallRng r;
    bool all_zero = true;
    for (int i = 0; i < 32; ++i) all_zero &= (seed[i] == 0);
    if (all_zero) return splitmix_seed(0);
    for (int w = 0; w < 4; ++w) {
      uint64_t v = 0;
      for (int b = 0; b < 8; ++b) v |= (uint64_t)seed[w * 8 + b] << (8 * b);
      r.s[w] = v;
    }
    return r;
  }

  static SmallRng splitmix_seed(uint64_t state) {
    const uint64_t PHI = 0x9e3779b97f4a7c15ULL;
    uint8_t seed[32];
    for (int w = 0; w < 4; ++w) {
      state += PHI;
      uint64_t z = state;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      z = z ^ (z >> 31);
      for (int b = 0; b < 8; ++b) seed[w * 8 + b] = (uint8_t)(z >> (8 * b));
    }
    SmallRng r;
    for (int w = 0; w < 4; ++w) {
      uint64_t v = 0;
      for (int b = 0; b < 8; ++b) v |= (uint64_t)seed[w * 8 + b] << (8 * b);
      r.s[w] = v;
    }
    return r;
  }

  uint64_t next_u64() {
    uint64_t result = rotl(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  // xoshiro256++ in rand 0.8 returns the upper half for u32.
  uint32_t next_u32() { return (uint32_t)(next_u64() >> 32); }

  // rand 0.8.5 UniformInt<usize>::sample_single_inclusive (64-bit usize).
  uint64_t gen_range_inclusive(uint64_t low, uint64_t high) {
    uint64_t range = high - low + 1;
    if (range == 0) return next_u64();
    int lz = __builtin_clzll(range);
    uint64_t zone = (range << lz) - 1;
    for (;;) {
      uint64_t v = next_u64();
      unsigned __int128 m = (unsigned __int128)v * range;
      uint64_t hi = (uint64_t)(m >> 64), lo = (uint64_t)m;
      if (lo <= zone) return hi + low;
    }
  }
  // gen_range(low..high) == sample_single(low, high) == inclusive(low, high-1)
  uint64_t gen_range(uint64_t low, uint64_t high) { return gen_range_inclusive(low, high - 1); }
};

// ---------------------------------------------------------------------------
// Graph (src/graph/mod.rs:13-34)
// ---------------------------------------------------------------------------
struct Graph {
  size_t nvtxs = 0;
  size_t ncon = 1;
  std::vector<Idx> xadj, adjncy;
  bool has_vwgt = false, has_adjwgt = false, has_vsize = false;
  std::vector<Idx> vwgt, adjwgt, vsize;

  size_t degree(size_t v) const { return (size_t)(xadj[v + 1] - xadj[v]); }   // mod.rs:85-87
  Idx vwgt_at(size_t v, size_t c) const { return has_vwgt ? vwgt[v * ncon + c] : 1; }  // mod.rs:91-96
  Idx edge_weight_at(size_t pos) const { return has_adjwgt ? adjwgt[pos] : 1; }       // mod.rs:111-116

  // edge_cut (mod.rs:123-137): i32 accumulator (wrapping), counted twice, / 2.
  Idx edge_cut(const Idx* part) const {
    uint32_t cut = 0;
    for (size_t v = 0; v < nvtxs; ++v) {
      Idx pv = part[v];
      for (Idx j = xadj[v]; j < xadj[v + 1]; ++j) {
        size_t u = (size_t)adjncy[j];
        if (part[u] != pv) cut += (uint32_t)edge_weight_at(j);
      }
    }
    return (Idx)cut / 2;
  }

  // partition_weights (mod.rs:140-149): [nparts][ncon] i32.
  std::vector<Idx> partition_weights(const Idx* part, size_t nparts) const {
    std::vector<uint32_t> pw(nparts * ncon, 0);
    for (size_t v = 0; v < nvtxs; ++v) {
      size_t p = (size_t)part[v];
      for (size_t c = 0; c < ncon; ++c) pw[p * ncon + c] += (uint32_t)vwgt_at(v, c);
    }
    return std::vector<Idx>(pw.begin(), pw.end());
  }

  // total_weight (mod.rs:152-160)
  std::vector<Idx> total_weight() const {
    std::vector<uint32_t> tw(ncon, 0);
    for (size_t v = 0; v < nvtxs; ++v)
      for (size_t c = 0; c < ncon; ++c) tw[c] += (uint32_t)vwgt_at(v, c);
    return std::vector<Idx>(tw.begin(), tw.end());
  }

  // boundary_vertices (mod.rs:164-171): ascending.
  std::vector<size_t> boundary_vertices(const Idx* part) const {
    std::vector<size_t> b;
    for (size_t v = 0; v < nvtxs; ++v) {
      Idx pv = part[v];
      for (Idx j = xadj[v]; j < xadj[v + 1]; ++j)
        if (part[adjncy[j]] != pv) { b.push_back(v); break; }
    }
    return b;
  }

  // build_coarse_graph (mod.rs:284-384).
  Graph build_coarse_graph(const std::vector<size_t>& matching, std::vector<size_t>& cmap) const {
    const size_t UNSET = std::numeric_limits<size_t>::max();
    cmap.assign(nvtxs, UNSET);
    size_t cn = 0;
    for (size_t v = 0; v < nvtxs; ++v) {                    // mod.rs:288-297
      if (cmap[v] == UNSET) {
        cmap[v] = cn;
        size_t u = matching[v];
        if (u != v && cmap[u] == UNSET) cmap[u] = cn;
        ++cn;
      }
    }
    Graph cg;
    cg.nvtxs = cn;
    cg.ncon = ncon;
    cg.has_vwgt = has_vwgt;                                  // mod.rs:300
    cg.has_vsize = has_vsize;                                // mod.rs:301
    if (has_vwgt) cg.vwgt.assign(cn * ncon, 0);
    if (has_vsize) cg.vsize.assign(cn, 0);
    for (size_t v = 0; v < nvtxs; ++v) {                    // mod.rs:303-314
      size_t cv = cmap[v];
      if (has_vwgt)
        for (size_t c = 0; c < ncon; ++c) cg.vwgt[cv * ncon + c] += vwgt_at(v, c);
      if (has_vsize) cg.vsize[cv] += vsize[v];
    }
    // Merge multi-edges by first appearance, summing weights (mod.rs:321-341).
    std::vector<std::vector<std::pair<size_t, Idx>>> lists(cn);
    for (size_t v = 0; v < nvtxs; ++v) {
      size_t cv = cmap[v];
      for (Idx j = xadj[v]; j < xadj[v + 1]; ++j) {
        size_t cu = cmap[(size_t)adjncy[j]];
        if (cu == cv) continue;
        Idx ew = edge_weight_at(j);
        auto& L = lists[cv];
        bool found = false;
        for (auto& e : L)
          if (e.first == cu) { e.second += ew; found = true; break; }
        if (!found) L.emplace_back(cu, ew);
      }
    }
    cg.xadj.assign(cn + 1, 0);
    for (size_t cv = 0; cv < cn; ++cv) cg.xadj[cv + 1] = cg.xadj[cv] + (Idx)lists[cv].size();
    std::vector<Idx> cw;
    cw.reserve(cg.xadj[cn]);
    cg.adjncy.reserve(cg.xadj[cn]);
    for (size_t cv = 0; cv < cn; ++cv)
      for (auto& e : lists[cv]) { cg.adjncy.push_back((Idx)e.first); cw.push_back(e.second); }
    // cadjwgt kept if the input had weights or any merged weight != 1 (mod.rs:366-369)
    bool keep = has_adjwgt;
    if (!keep) for (Idx w : cw) if (w != 1) { keep = true; break; }
    cg.has_adjwgt = keep;
    if (keep) cg.adjwgt = std::move(cw);
    return cg;
  }

  // compute_target_weights (mod.rs:392-410), f64.
  std::vector<double> compute_target_weights(size_t nparts, const float* tpwgts) const {
    std::vector<Idx> total = total_weight();
    std::vector<double> t(nparts * ncon);
    for (size_t p = 0; p < nparts; ++p)
      for (size_t c = 0; c < ncon; ++c) {
        double f = tpwgts ? (double)tpwgts[p * ncon + c] : 1.0 / (double)nparts;
        t[p * ncon + c] = f * (double)total[c];
      }
    return t;
  }
};

// validate_csr (src/graph/validate.rs:16-142). Returns 0 when valid, else the
// number (1..8) of the failed check (nvtxs/ncon zero report 9/10).
int validate_csr(size_t nvtxs, size_t ncon, const Idx* xadj, size_t xadj_len, const Idx* adjncy,
                 size_t adjncy_len, const Idx* vwgt, size_t vwgt_len, const Idx* adjwgt,
                 size_t adjwgt_len) {
  if (nvtxs == 0) return 9;
  if (ncon == 0) return 10;
  if (xadj_len != nvtxs + 1) return 1;
  if (xadj[0] != 0) return 2;
  for (size_t i = 0; i < nvtxs; ++i)
    if (xadj[i] > xadj[i + 1]) return 2;
  size_t ne = (size_t)xadj[nvtxs];
  if (adjncy_len != ne) return 3;
  for (size_t v = 0; v < nvtxs; ++v)
    for (Idx j = xadj[v]; j < xadj[v + 1]; ++j) {
      Idx u = adjncy[j];
      if (u < 0 || (size_t)u >= nvtxs) return 4;
      if ((size_t)u == v) return 5;
    }
  std::vector<size_t> degree_check(nvtxs, 0);               // validate.rs:88-108
  for (size_t v = 0; v < nvtxs; ++v)
    for (Idx j = xadj[v]; j < xadj[v + 1]; ++j) degree_check[(size_t)adjncy[j]] += 1;
  for (size_t v = 0; v < nvtxs; ++v)
    if (degree_check[v] != (size_t)(xadj[v + 1] - xadj[v])) return 6;
  if (adjwgt && adjwgt_len != ne) return 7;
  if (vwgt) {
    if (vwgt_len != nvtxs * ncon) return 8;
    for (size_t i = 0; i < vwgt_len; ++i)
      if (vwgt[i] <= 0) return 8;
  }
  return 0;
}

// shem_matching (src/coarsen/shem.rs:13-56)
std::vector<size_t> shem_matching(const Graph& g, SmallRng& rng) {
  size_t n = g.nvtxs;
  std::vector<size_t> matching(n);
  for (size_t v = 0; v < n; ++v) matching[v] = v;
  std::vector<char> visited(n, 0);
  std::vector<size_t> perm(n);
  for (size_t v = 0; v < n; ++v) perm[v] = v;
  std::vector<uint32_t> tb(n);
  for (size_t v = 0; v < n; ++v) tb[v] = rng.next_u32() >> 16;   // shem.rs:22
  std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) {  // shem.rs:23
    size_t da = g.degree(a), db = g.degree(b);
    if (da != db) return da < db;
    return tb[a] < tb[b];
  });
  for (size_t v : perm) {
    if (visited[v]) continue;
    visited[v] = 1;
    size_t best_u = std::numeric_limits<size_t>::max();
    Idx best_w = std::numeric_limits<Idx>::min();
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
      size_t u = (size_t)g.adjncy[j];
      if (visited[u]) continue;
      Idx w = g.edge_weight_at(j);
      if (w > best_w) { best_w = w; best_u = u; }            // strict > (shem.rs:43)
    }
    if (best_u != std::numeric_limits<size_t>::max()) {
      matching[v] = best_u;
      matching[best_u] = v;
      visited[best_u] = 1;
    }
  }
  return matching;
}

// random_matching (src/coarsen/rm.rs:13-43)
std::vector<size_t> random_matching(const Graph& g, SmallRng& rng) {
  size_t n = g.nvtxs;
  std::vector<size_t> matching(n);
  for (size_t v = 0; v < n; ++v) matching[v] = v;
  std::vector<char> visited(n, 0);
  std::vector<size_t> perm(n);
  for (size_t v = 0; v < n; ++v) perm[v] = v;
  for (size_t i = n; i-- > 1;) {                              // rm.rs:21-24
    size_t j = (size_t)rng.gen_range_inclusive(0, i);
    std::swap(perm[i], perm[j]);
  }
  for (size_t v : perm) {
    if (visited[v]) continue;
    visited[v] = 1;
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
      size_t u = (size_t)g.adjncy[j];
      if (!visited[u]) {
        matching[v] = u;
        matching[u] = v;
        visited[u] = 1;
        break;
      }
    }
  }
  return matching;
}

// grow_partition (src/initial/grow.rs:12-103). When `fixed_seeds` is given,
// the k seed vertices are taken from it instead of the rejection loop
// (grow.rs:26-32); everything after the seed choice is unchanged.
std::vector<Idx> grow_partition(const Graph& g, size_t nparts, const double* tpwgts, SmallRng* rng,
                                const Idx* fixed_seeds, std::vector<Idx>* seeds_out) {
  size_t n = g.nvtxs, ncon = g.ncon;
  std::vector<Idx> part(n, -1);
  std::vector<int64_t> pw(nparts * ncon, 0);
  std::vector<size_t> seeds;
  if (fixed_seeds) {
    for (size_t p = 0; p < nparts; ++p) seeds.push_back((size_t)fixed_seeds[p]);
  } else {
    std::vector<char> used(n, 0);
    while (seeds.size() < nparts) {
      size_t v = (size_t)rng->gen_range(0, n);
      if (!used[v]) { used[v] = 1; seeds.push_back(v); }
    }
  }
  if (seeds_out) {
    seeds_out->clear();
    for (size_t s : seeds) seeds_out->push_back((Idx)s);
  }
  std::vector<std::deque<size_t>> queues(nparts);
  for (size_t p = 0; p < nparts; ++p) queues[p].push_back(seeds[p]);
  for (size_t p = 0; p < nparts; ++p) {
    size_t s = seeds[p];
    part[s] = (Idx)p;
    for (size_t c = 0; c < ncon; ++c) pw[p * ncon + c] += g.vwgt_at(s, c);
  }
  size_t active = nparts;
  while (active > 0) {                                        // grow.rs:51-86
    active = 0;
    for (size_t p = 0; p < nparts; ++p) {
      bool at_target = true;
      for (size_t c = 0; c < ncon; ++c)
        if (!((double)pw[p * ncon + c] >= tpwgts[p * ncon + c])) { at_target = false; break; }
      if (at_target) continue;
      bool grew = false;
      while (!queues[p].empty()) {
        size_t v = queues[p].front();
        queues[p].pop_front();
        for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
          size_t u = (size_t)g.adjncy[j];
          if (part[u] == -1) {
            part[u] = (Idx)p;
            for (size_t c = 0; c < ncon; ++c) pw[p * ncon + c] += g.vwgt_at(u, c);
            queues[p].push_back(u);
            grew = true;
          }
        }
        if (grew) break;
      }
      if (grew) active += 1;
    }
  }
  for (size_t v = 0; v < n; ++v) {                            // grow.rs:89-100
    if (part[v] == -1) {
      size_t best_p = 0;
      for (size_t p = 1; p < nparts; ++p)
        if (pw[p * ncon] < pw[best_p * ncon]) best_p = p;     // min_by_key: first min
      part[v] = (Idx)best_p;
      for (size_t c = 0; c < ncon; ++c) pw[best_p * ncon + c] += g.vwgt_at(v, c);
    }
  }
  return part;
}

// random_partition (src/initial/random.rs:8-10)
std::vector<Idx> random_partition(const Graph& g, size_t nparts, SmallRng& rng) {
  std::vector<Idx> part(g.nvtxs);
  for (size_t v = 0; v < g.nvtxs; ++v) part[v] = (Idx)rng.gen_range(0, nparts);
  return part;
}

// compute_move_gain (src/refine/greedy.rs:197-218)
Idx compute_move_gain(const Graph& g, size_t v, const Idx* part, Idx from, Idx to) {
  uint32_t gain = 0;
  for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
    Idx pu = part[g.adjncy[j]];
    uint32_t w = (uint32_t)g.edge_weight_at(j);
    if (pu == from) gain -= w;
    else if (pu == to) gain += w;
  }
  return (Idx)gain;
}

// greedy_refine_with_comm with SingleComm (src/refine/greedy.rs:36-193).
// Returns the pass statistics through `moves_per_pass` when given.
Idx greedy_refine(const Graph& g, std::vector<Idx>& part, size_t nparts, const double* tpwgts,
                  const double* ubvec, size_t niter, std::vector<int64_t>* moves_per_pass) {
  size_t ncon = g.ncon;
  std::vector<Idx> pw = g.partition_weights(part.data(), nparts);
  std::vector<Idx> vw(ncon);
  // Balance-repair pass (greedy.rs:60-123)
  {
    std::vector<size_t> boundary = g.boundary_vertices(part.data());
    std::vector<std::pair<size_t, size_t>> moves;
    for (size_t v : boundary) {
      size_t pv = (size_t)part[v];
      for (size_t c = 0; c < ncon; ++c) vw[c] = g.vwgt_at(v, c);
      bool over = false;
      for (size_t c = 0; c < ncon; ++c)
        if ((double)pw[pv * ncon + c] > tpwgts[pv * ncon + c] * ubvec[c]) { over = true; break; }
      if (!over) continue;
      Idx best_gain = std::numeric_limits<Idx>::min();
      size_t best_p = std::numeric_limits<size_t>::max();
      for (size_t p = 0; p < nparts; ++p) {
        if (p == pv) continue;
        bool feasible = true;
        for (size_t c = 0; c < ncon; ++c) {
          Idx new_w = (Idx)((uint32_t)pw[p * ncon + c] + (uint32_t)vw[c]);
          if (!((double)new_w <= tpwgts[p * ncon + c] * ubvec[c])) { feasible = false; break; }
        }
        if (!feasible) continue;
        Idx gain = compute_move_gain(g, v, part.data(), (Idx)pv, (Idx)p);
        if (gain > best_gain) { best_gain = gain; best_p = p; }
      }
      if (best_p != std::numeric_limits<size_t>::max()) {
        moves.emplace_back(v, best_p);
        for (size_t c = 0; c < ncon; ++c) {
          pw[pv * ncon + c] = (Idx)((uint32_t)pw[pv * ncon + c] - (uint32_t)vw[c]);
          pw[best_p * ncon + c] = (Idx)((uint32_t)pw[best_p * ncon + c] + (uint32_t)vw[c]);
        }
      }
    }
    for (auto& m : moves) part[m.first] = (Idx)m.second;     // greedy.rs:111-119
    if (moves_per_pass) moves_per_pass->push_back((int64_t)moves.size());
  }
  // Cut-optimisation passes (greedy.rs:126-190)
  for (size_t it = 0; it < niter; ++it) {
    std::vector<size_t> boundary = g.boundary_vertices(part.data());
    std::vector<std::pair<size_t, size_t>> moves;
    for (size_t v : boundary) {
      size_t pv = (size_t)part[v];
      for (size_t c = 0; c < ncon; ++c) vw[c] = g.vwgt_at(v, c);
      Idx best_gain = 0;
      size_t best_p = pv;
      for (size_t p = 0; p < nparts; ++p) {
        if (p == pv) continue;
        bool feasible = true;
        for (size_t c = 0; c < ncon; ++c) {
          Idx new_w = (Idx)((uint32_t)pw[p * ncon + c] + (uint32_t)vw[c]);
          if (!((double)new_w <= tpwgts[p * ncon + c] * ubvec[c])) { feasible = false; break; }
        }
        if (!feasible) continue;
        Idx gain = compute_move_gain(g, v, part.data(), (Idx)pv, (Idx)p);
        if (gain > best_gain) { best_gain = gain; best_p = p; }
      }
      if (best_p != pv) {
        moves.emplace_back(v, best_p);
        for (size_t c = 0; c < ncon; ++c) {
          pw[pv * ncon + c] = (Idx)((uint32_t)pw[pv * ncon + c] - (uint32_t)vw[c]);
          pw[best_p * ncon + c] = (Idx)((uint32_t)pw[best_p * ncon + c] + (uint32_t)vw[c]);
        }
      }
    }
    bool any_move = false;
    for (auto& m : moves) {
      if ((size_t)part[m.first] != m.second) { part[m.first] = (Idx)m.second; any_move = true; }
    }
    if (moves_per_pass) moves_per_pass->push_back((int64_t)moves.size());
    if (!any_move) break;
  }
  return g.edge_cut(part.data());
}

// fm_kway_refine (src/refine/fm_kway.rs:12-31) and fm_kway_pass (:34-158).
// The reference keeps its boundary vertices in a priority_queue 1.4.0
// PriorityQueue keyed by gain (Cargo.lock; not vendored). Among equal gains
// this restatement pops the lowest vertex id first; the crate's heap order
// among equal priorities is not restated (parity unpinned for that order).
// i32 sums wrap like the reference's release build.
struct FmStats {
  int64_t passes = 0;
  int64_t moves = 0;
};

// compute_best_move (fm_kway.rs:47-71): the adjacent part p != pv with the
// largest gain edge_to[p] - edge_to[pv] > 0 (strict >, so the lowest p on
// ties); false when there is none.
bool fm_best_move(const Graph& g, size_t v, const Idx* part, size_t nparts, std::vector<Idx>& edge_to,
                  size_t* best_p_out, Idx* best_g_out) {
  size_t pv = (size_t)part[v];
  std::fill(edge_to.begin(), edge_to.end(), 0);
  for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
    size_t pu = (size_t)part[g.adjncy[j]];
    edge_to[pu] = (Idx)((uint32_t)edge_to[pu] + (uint32_t)g.edge_weight_at(j));
  }
  size_t best_p = std::numeric_limits<size_t>::max();
  Idx best_g = 0;
  for (size_t p = 0; p < nparts; ++p) {
    if (p == pv) continue;
    if (edge_to[p] == 0) continue;
    Idx gain = (Idx)((uint32_t)edge_to[p] - (uint32_t)edge_to[pv]);
    if (gain > best_g) { best_g = gain; best_p = p; }
  }
  if (best_p == std::numeric_limits<size_t>::max()) return false;
  *best_p_out = best_p;
  *best_g_out = best_g;
  return true;
}

bool fm_kway_pass(const Graph& g, std::vector<Idx>& part, size_t nparts, std::vector<Idx>& pw,
                  const double* tpwgts, const double* ubvec, FmStats* st) {
  const size_t n = g.nvtxs, ncon = g.ncon;
  std::vector<Idx> edge_to(nparts);
  std::vector<size_t> bm_p(n);
  std::vector<Idx> bm_g(n);
  std::vector<char> has_bm(n, 0);
  // The queue: (gain desc, vertex asc), plus each queued vertex's key.
  auto cmp = [](const std::pair<Idx, size_t>& a, const std::pair<Idx, size_t>& b) {
    if (a.first != b.first) return a.first > b.first;
    return a.second < b.second;
  };
  std::set<std::pair<Idx, size_t>, decltype(cmp)> pq(cmp);
  std::vector<Idx> key(n);
  std::vector<char> queued(n, 0);
  auto push = [&](size_t v, Idx gain) {   // push, or change_priority when queued
    if (queued[v]) pq.erase({key[v], v});
    key[v] = gain;
    queued[v] = 1;
    pq.insert({gain, v});
  };
  auto remove = [&](size_t v) {
    if (queued[v]) { pq.erase({key[v], v}); queued[v] = 0; }
  };
  for (size_t v = 0; v < n; ++v) {                            // fm_kway.rs:74-85
    Idx pv = part[v];
    bool on_boundary = false;
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j)
      if (part[g.adjncy[j]] != pv) { on_boundary = true; break; }
    if (!on_boundary) continue;
    size_t tp;
    Idx gain;
    if (fm_best_move(g, v, part.data(), nparts, edge_to, &tp, &gain)) {
      bm_p[v] = tp; bm_g[v] = gain; has_bm[v] = 1;
      push(v, gain);
    }
  }
  std::vector<char> locked(n, 0);
  struct Move { size_t v; Idx from, to; };
  std::vector<Move> moves;
  Idx cut = g.edge_cut(part.data());
  Idx best_cut = cut;
  size_t best_len = 0;
  std::vector<Idx> vw(ncon);
  while (!pq.empty()) {                                       // fm_kway.rs:93-149
    auto top = *pq.begin();
    pq.erase(pq.begin());
    size_t v = top.second;
    Idx gain = top.first;
    queued[v] = 0;
    if (locked[v] || gain <= 0) break;
    if (!has_bm[v]) continue;
    size_t to = bm_p[v];
    size_t from = (size_t)part[v];
    for (size_t c = 0; c < ncon; ++c) vw[c] = g.vwgt_at(v, c);
    bool feasible = true;
    for (size_t c = 0; c < ncon; ++c) {
      Idx new_w = (Idx)((uint32_t)pw[to * ncon + c] + (uint32_t)vw[c]);
      if (!((double)new_w <= tpwgts[to * ncon + c] * ubvec[c])) { feasible = false; break; }
    }
    if (!feasible) continue;
    part[v] = (Idx)to;
    for (size_t c = 0; c < ncon; ++c) {
      pw[from * ncon + c] = (Idx)((uint32_t)pw[from * ncon + c] - (uint32_t)vw[c]);
      pw[to * ncon + c] = (Idx)((uint32_t)pw[to * ncon + c] + (uint32_t)vw[c]);
    }
    locked[v] = 1;
    moves.push_back({v, (Idx)from, (Idx)to});
    cut = (Idx)((uint32_t)cut - (uint32_t)gain);
    if (cut < best_cut) { best_cut = cut; best_len = moves.size(); }
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {         // fm_kway.rs:131-148
      size_t u = (size_t)g.adjncy[j];
      if (locked[u]) continue;
      size_t tp;
      Idx gu;
      if (fm_best_move(g, u, part.data(), nparts, edge_to, &tp, &gu)) {
        bm_p[u] = tp; bm_g[u] = gu; has_bm[u] = 1;
        push(u, gu);
      } else {
        remove(u);
        has_bm[u] = 0;
      }
    }
  }
  for (size_t i = moves.size(); i-- > best_len;) {            // fm_kway.rs:152-161 (rollback)
    const Move& m = moves[i];
    size_t cur = (size_t)part[m.v];
    for (size_t c = 0; c < ncon; ++c) {
      Idx w = g.vwgt_at(m.v, c);
      pw[cur * ncon + c] = (Idx)((uint32_t)pw[cur * ncon + c] - (uint32_t)w);
      pw[(size_t)m.from * ncon + c] = (Idx)((uint32_t)pw[(size_t)m.from * ncon + c] + (uint32_t)w);
    }
    part[m.v] = m.from;
  }
  if (st) st->moves += (int64_t)best_len;
  return best_len > 0 && best_cut < (Idx)((uint32_t)g.edge_cut(part.data()) + 1u);
}

Idx fm_kway_refine(const Graph& g, std::vector<Idx>& part, size_t nparts, const double* tpwgts,
                   const double* ubvec, size_t niter, FmStats* st) {
  std::vector<Idx> pw = g.partition_weights(part.data(), nparts);
  for (size_t it = 0; it < niter; ++it) {
    if (st) st->passes += 1;
    if (!fm_kway_pass(g, part, nparts, pw, tpwgts, ubvec, st)) break;
  }
  return g.edge_cut(part.data());
}

// Options (src/types.rs:52-95) with the C-ABI option codec (types.rs:190-245).
struct Options {
  int ctype = 1;      // 0 = Rm, 1 = Shem
  int iptype = 0;     // 0 = Grow, 1 = Random, 4 = MetisRb (== Grow for kway)
  int rtype = 0;      // 0 = Fm, 1 = Greedy
  int objtype = 0;
  int no2hop = 0;
  int64_t ncuts = 1;
  int64_t niter = 10;
  uint64_t seed = 0;
  int minconn = 0, contig = 0;
  uint32_t ufactor = 30;
  int numbering = 0;
  uint32_t dbglvl = 0;
};

constexpr int NOPT = 40;
enum { O_PTYPE = 0, O_OBJTYPE = 1, O_CTYPE = 2, O_IPTYPE = 3, O_RTYPE = 4, O_DBGLVL = 5, O_NITER = 6,
       O_NCUTS = 7, O_SEED = 8, O_NO2HOP = 9, O_MINCONN = 10, O_CONTIG = 11, O_UFACTOR = 16,
       O_NUMBERING = 17 };

Options from_raw(const Idx* a) {                               // types.rs:190-224
  Options o;
  if (a[O_CTYPE] == 0) o.ctype = 0;
  if (a[O_IPTYPE] == 1) o.iptype = 1; else if (a[O_IPTYPE] == 4) o.iptype = 4;
  if (a[O_RTYPE] == 1) o.rtype = 1;
  if (a[O_OBJTYPE] == 1) o.objtype = 1;
  if (a[O_NO2HOP] != 0) o.no2hop = 1;
  if (a[O_NCUTS] > 0) o.ncuts = a[O_NCUTS];
  if (a[O_NITER] > 0) o.niter = a[O_NITER];
  o.seed = (uint64_t)std::max<Idx>(a[O_SEED], 0);
  o.minconn = a[O_MINCONN] != 0;
  o.contig = a[O_CONTIG] != 0;
  if (a[O_UFACTOR] > 0) o.ufactor = (uint32_t)a[O_UFACTOR];
  o.numbering = (uint8_t)a[O_NUMBERING];
  o.dbglvl = (uint32_t)a[O_DBGLVL];
  return o;
}

void to_raw(const Options& o, Idx* a) {                        // types.rs:227-245
  for (int i = 0; i < NOPT; ++i) a[i] = -1;
  a[O_CTYPE] = o.ctype == 0 ? 0 : 1;
  a[O_IPTYPE] = o.iptype;
  a[O_RTYPE] = o.rtype == 1 ? 1 : 0;
  a[O_OBJTYPE] = o.objtype;
  a[O_NO2HOP] = o.no2hop;
  a[O_NCUTS] = (Idx)o.ncuts;
  a[O_NITER] = (Idx)o.niter;
  a[O_SEED] = (Idx)o.seed;
  a[O_MINCONN] = o.minconn;
  a[O_CONTIG] = o.contig;
  a[O_UFACTOR] = (Idx)o.ufactor;
  a[O_NUMBERING] = o.numbering;
  a[O_DBGLVL] = (Idx)o.dbglvl;
}

// A script replaces the random choices of partition_kway: per attempt, the
// matching of every coarsening level and the k grow seeds. It lets a caller
// replay, through this restatement, choices that another implementation made.
struct Script {
  const Idx* matchings = nullptr;       // concatenated matchings, level after level
  const int64_t* level_offsets = nullptr;  // start of each level's matching
  int64_t nlevels = 0;
  const Idx* grow_seeds = nullptr;      // nparts seed vertices
};

struct KwayStats {
  int64_t nlevels = 0;
  int64_t level_n[64];
  int64_t level_m[64];
};

// refine_level (src/partition/kway.rs:145-162): Greedy, or FM through
// refine_kway (src/refine/mod.rs:26-38).
void refine_level(const Graph& g, std::vector<Idx>& part, size_t nparts, const double* t, const double* ub,
                  const Options& opt) {
  if (opt.rtype == 1) greedy_refine(g, part, nparts, t, ub, (size_t)opt.niter, nullptr);
  else fm_kway_refine(g, part, nparts, t, ub, (size_t)opt.niter, nullptr);
}

// partition_kway (src/partition/kway.rs:20-141) with SingleComm.
// Returns 1 / -2 / -4 like the C ABI.
int partition_kway(const Graph& graph, size_t nparts, const float* tpwgts, const float* ubvec,
                   const Options& opt, std::vector<Idx>& best_part, Idx& best_obj,
                   const Script* script, KwayStats* stats) {
  if (nparts < 2) return -2;                                  // kway.rs:31-33
  if (nparts > graph.nvtxs) return -2;                        // kway.rs:34-38
  size_t ncon = graph.ncon;
  std::vector<double> ub(ncon);                               // kway.rs:44-49
  for (size_t c = 0; c < ncon; ++c)
    ub[c] = ubvec ? (double)ubvec[c] : 1.0 + (double)opt.ufactor / 1000.0;
  bool have_best = false;
  for (int64_t attempt = 0; attempt < opt.ncuts; ++attempt) {   // kway.rs:54
    uint64_t seed;
    if (opt.seed == 0) {
      std::random_device rd;
      seed = ((uint64_t)rd() << 32) ^ (uint64_t)rd();
    } else {
      seed = opt.seed + (uint64_t)attempt;
    }
    SmallRng rng = SmallRng::seed_from_u64(seed);
    // coarsen_with_comm (src/coarsen/mod.rs:36-71)
    size_t limit = std::max<size_t>(20 * nparts, 20);
    std::vector<Graph> levels;
    levels.reserve(128);
    std::vector<std::vector<size_t>> cmaps;
    const Graph* current = &graph;
    int64_t lvl = 0;
    for (;;) {
      std::vector<size_t> matching;
      if (script && script->matchings) {
        if (lvl >= script->nlevels) return -4;
        matching.resize(current->nvtxs);
        const Idx* m = script->matchings + script->level_offsets[lvl];
        for (size_t v = 0; v < current->nvtxs; ++v) matching[v] = (size_t)m[v];
      } else if (opt.ctype == 0) {
        matching = random_matching(*current, rng);
      } else {
        matching = shem_matching(*current, rng);
      }
      std::vector<size_t> cmap;
      Graph cg = current->build_coarse_graph(matching, cmap);
      float ratio = (float)cg.nvtxs / (float)current->nvtxs;
      levels.push_back(std::move(cg));
      cmaps.push_back(std::move(cmap));
      ++lvl;
      const Graph& last = levels.back();
      if (last.nvtxs <= limit || ratio > 0.95f) break;
      current = &levels.back();
    }
    if (stats) {
      stats->nlevels = (int64_t)levels.size();
      stats->level_n[0] = (int64_t)graph.nvtxs;
      stats->level_m[0] = (int64_t)graph.adjncy.size();
      for (size_t i = 0; i < levels.size() && i + 1 < 64; ++i) {
        stats->level_n[i + 1] = (int64_t)levels[i].nvtxs;
        stats->level_m[i + 1] = (int64_t)levels[i].adjncy.size();
      }
    }
    const Graph& coarsest = levels.empty() ? graph : levels.back();
    // With fewer coarse vertices than parts the reference's seed draw
    // (grow.rs:26-32) never ends; the restatement reports an error instead.
    if (coarsest.nvtxs < nparts && opt.iptype != 1) return -4;
    std::vector<double> coarse_t = coarsest.compute_target_weights(nparts, tpwgts);
    std::vector<Idx> part;
    if (opt.iptype == 1 && !(script && script->grow_seeds)) {
      part = random_partition(coarsest, nparts, rng);         // initial/mod.rs:20
    } else {
      part = grow_partition(coarsest, nparts, coarse_t.data(), &rng,
                            script ? script->grow_seeds : nullptr, nullptr);
    }
    refine_level(coarsest, part, nparts, coarse_t.data(), ub.data(), opt);  // kway.rs:72
    for (size_t i = levels.size(); i-- > 0;) {                // kway.rs:76-92
      const Graph& fine = (i == 0) ? graph : levels[i - 1];
      std::vector<Idx> fine_part(fine.nvtxs);
      for (size_t v = 0; v < fine.nvtxs; ++v) fine_part[v] = part[cmaps[i][v]];
      std::vector<double> t = fine.compute_target_weights(nparts, tpwgts);
      refine_level(fine, fine_part, nparts, t.data(), ub.data(), opt);
      part = std::move(fine_part);
    }
    Idx obj = graph.edge_cut(part.data());
    if (!have_best || obj < best_obj) {                       // kway.rs:96-98 (strict <)
      best_obj = obj;
      best_part = part;
      have_best = true;
    }
  }
  return 1;
}

// ---------------------------------------------------------------------------
// Recursive bisection (src/partition/recursive.rs:12-187) with its 2-way
// refinement (src/refine/mod.rs:12-23: Greedy, or FM of src/refine/fm.rs).
// ---------------------------------------------------------------------------

// Graph::extract_subgraph (src/graph/mod.rs:209-273): the vertices of
// `target` in ascending id, their edges inside it in CSR order.
Graph extract_subgraph(const Graph& g, const Idx* part, Idx target, std::vector<size_t>& new_to_old) {
  new_to_old.clear();
  for (size_t v = 0; v < g.nvtxs; ++v)
    if (part[v] == target) new_to_old.push_back(v);
  const size_t sn = new_to_old.size();
  std::vector<size_t> old_to_new(g.nvtxs, std::numeric_limits<size_t>::max());
  for (size_t i = 0; i < sn; ++i) old_to_new[new_to_old[i]] = i;
  Graph s;
  s.nvtxs = sn;
  s.ncon = g.ncon;
  s.xadj.assign(sn + 1, 0);
  s.has_adjwgt = g.has_adjwgt;
  s.has_vwgt = g.has_vwgt;
  s.has_vsize = g.has_vsize;
  for (size_t i = 0; i < sn; ++i) {
    const size_t old = new_to_old[i];
    for (Idx j = g.xadj[old]; j < g.xadj[old + 1]; ++j) {
      const size_t u = (size_t)g.adjncy[j];
      if (part[u] == target) {
        s.adjncy.push_back((Idx)old_to_new[u]);
        if (g.has_adjwgt) s.adjwgt.push_back(g.edge_weight_at((size_t)j));
      }
    }
    s.xadj[i + 1] = (Idx)s.adjncy.size();
    if (g.has_vwgt)
      for (size_t c = 0; c < g.ncon; ++c) s.vwgt.push_back(g.vwgt[old * g.ncon + c]);
    if (g.has_vsize) s.vsize.push_back(g.vsize[old]);
  }
  return s;
}

// fm_refine / fm_pass (src/refine/fm.rs:12-127): every popped boundary
// vertex moves to the other side if that side stays feasible, whatever its
// gain; the pass then rolls back to the best cut seen. The queue's order among
// equal gains follows the k-way FM restatement (lowest vertex id first; the
// priority_queue crate's heap order is not restated). Note the reference's
// `improved` test compares with the cut before the rollback (fm.rs:118).
bool fm2_pass(const Graph& g, std::vector<Idx>& part, std::vector<Idx>& pw, const double* tpwgts,
              const double* ubvec) {
  const size_t n = g.nvtxs, ncon = g.ncon;
  std::vector<Idx> gains(n);
  for (size_t v = 0; v < n; ++v) gains[v] = compute_move_gain(g, v, part.data(), part[v], 1 - part[v]);
  auto cmp = [](const std::pair<Idx, size_t>& a, const std::pair<Idx, size_t>& b) {
    if (a.first != b.first) return a.first > b.first;
    return a.second < b.second;
  };
  std::set<std::pair<Idx, size_t>, decltype(cmp)> pq(cmp);
  std::vector<Idx> key(n);
  std::vector<char> queued(n, 0);
  auto on_boundary = [&](size_t v) {
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j)
      if (part[g.adjncy[j]] != part[v]) return true;
    return false;
  };
  auto push = [&](size_t v, Idx k) {
    if (queued[v]) pq.erase({key[v], v});
    key[v] = k;
    queued[v] = 1;
    pq.insert({k, v});
  };
  for (size_t v = 0; v < n; ++v)
    if (on_boundary(v)) push(v, gains[v]);
  std::vector<char> locked(n, 0);
  struct Move { size_t v; Idx from; };
  std::vector<Move> moves;
  Idx cut = g.edge_cut(part.data());
  Idx best_cut = cut;
  size_t best_len = 0;
  while (!pq.empty()) {
    auto top = *pq.begin();
    pq.erase(pq.begin());
    const size_t v = top.second;
    const Idx gain = top.first;
    queued[v] = 0;
    if (locked[v]) continue;
    const Idx from = part[v], to = 1 - from;
    bool feasible = true;
    for (size_t c = 0; c < ncon; ++c) {
      Idx new_w = (Idx)((uint32_t)pw[(size_t)to * ncon + c] + (uint32_t)g.vwgt_at(v, c));
      if (!((double)new_w <= tpwgts[(size_t)to * ncon + c] * ubvec[c])) { feasible = false; break; }
    }
    if (!feasible) continue;
    part[v] = to;
    for (size_t c = 0; c < ncon; ++c) {
      const uint32_t w = (uint32_t)g.vwgt_at(v, c);
      pw[(size_t)from * ncon + c] = (Idx)((uint32_t)pw[(size_t)from * ncon + c] - w);
      pw[(size_t)to * ncon + c] = (Idx)((uint32_t)pw[(size_t)to * ncon + c] + w);
    }
    locked[v] = 1;
    moves.push_back({v, from});
    cut = (Idx)((uint32_t)cut - (uint32_t)gain);
    if (cut < best_cut) { best_cut = cut; best_len = moves.size(); }
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j) {
      const size_t u = (size_t)g.adjncy[j];
      if (locked[u]) continue;
      gains[u] = compute_move_gain(g, u, part.data(), part[u], 1 - part[u]);
      if (queued[u]) push(u, gains[u]);
      else if (on_boundary(u)) push(u, gains[u]);
    }
  }
  const bool improved = best_len > 0 && best_cut < g.edge_cut(part.data());
  for (size_t i = moves.size(); i-- > best_len;) {
    const Move& m = moves[i];
    const Idx cur = part[m.v];
    for (size_t c = 0; c < ncon; ++c) {
      const uint32_t w = (uint32_t)g.vwgt_at(m.v, c);
      pw[(size_t)cur * ncon + c] = (Idx)((uint32_t)pw[(size_t)cur * ncon + c] - w);
      pw[(size_t)m.from * ncon + c] = (Idx)((uint32_t)pw[(size_t)m.from * ncon + c] + w);
    }
    part[m.v] = m.from;
  }
  return improved;
}

Idx fm2_refine(const Graph& g, std::vector<Idx>& part, const double* tpwgts, const double* ubvec, size_t niter) {
  std::vector<Idx> pw = g.partition_weights(part.data(), 2);
  for (size_t it = 0; it < niter; ++it)
    if (!fm2_pass(g, part, pw, tpwgts, ubvec)) break;
  return g.edge_cut(part.data());
}

// refine_2way (src/refine/mod.rs:12-23)
void refine_2way(const Graph& g, std::vector<Idx>& part, const double* t, const double* ub, const Options& opt) {
  if (opt.rtype == 1) greedy_refine(g, part, 2, t, ub, (size_t)opt.niter, nullptr);
  else fm2_refine(g, part, t, ub, (size_t)opt.niter);
}

// coarsen (src/coarsen/mod.rs:24-71) with one rank.
void coarsen_levels(const Graph& graph, size_t nparts, const Options& opt, SmallRng& rng, std::vector<Graph>& levels,
                    std::vector<std::vector<size_t>>& cmaps) {
  const size_t limit = std::max<size_t>(20 * nparts, 20);
  levels.reserve(128);
  const Graph* current = &graph;
  for (;;) {
    std::vector<size_t> matching = opt.ctype == 0 ? random_matching(*current, rng) : shem_matching(*current, rng);
    std::vector<size_t> cmap;
    Graph cg = current->build_coarse_graph(matching, cmap);
    const float ratio = (float)cg.nvtxs / (float)current->nvtxs;
    levels.push_back(std::move(cg));
    cmaps.push_back(std::move(cmap));
    const Graph& last = levels.back();
    if (last.nvtxs <= limit || ratio > 0.95f) break;
    current = &levels.back();
  }
}

// multilevel_bisect (src/partition/recursive.rs:133-187). Returns -4 when the
// grow step would need more distinct seeds than the coarsest graph has
// vertices (the reference's seed draw never ends there).
int multilevel_bisect(const Graph& graph, const float* tpwgts2, const double* ub, const Options& opt, SmallRng& rng,
                      std::vector<Idx>& part) {
  if (graph.nvtxs <= 2) {
    part.resize(graph.nvtxs);
    for (size_t v = 0; v < graph.nvtxs; ++v) part[v] = (Idx)v;
    return 1;
  }
  std::vector<Graph> levels;
  std::vector<std::vector<size_t>> cmaps;
  coarsen_levels(graph, 2, opt, rng, levels, cmaps);
  const Graph& coarsest = levels.empty() ? graph : levels.back();
  std::vector<double> ct = coarsest.compute_target_weights(2, tpwgts2);
  if (opt.iptype == 1) {
    part = random_partition(coarsest, 2, rng);
  } else {
    if (coarsest.nvtxs < 2) return -4;
    part = grow_partition(coarsest, 2, ct.data(), &rng, nullptr, nullptr);
  }
  refine_2way(coarsest, part, ct.data(), ub, opt);
  for (size_t i = levels.size(); i-- > 0;) {
    const Graph& fine = (i == 0) ? graph : levels[i - 1];
    std::vector<Idx> fine_part(fine.nvtxs);
    for (size_t v = 0; v < fine.nvtxs; ++v) fine_part[v] = part[cmaps[i][v]];
    std::vector<double> t = fine.compute_target_weights(2, tpwgts2);
    refine_2way(fine, fine_part, t.data(), ub, opt);
    part = std::move(fine_part);
  }
  return 1;
}

// rb_recurse (src/partition/recursive.rs:61-131). Real arithmetic is f32 as
// in the reference (sums in index order).
int rb_recurse(const Graph& graph, size_t nparts, size_t offset, const std::vector<float>& tpwgts, const double* ub,
               const Options& opt, SmallRng& rng, std::vector<Idx>& part) {
  if (nparts == 1) {
    for (size_t v = 0; v < graph.nvtxs; ++v) part[v] = (Idx)offset;
    return 1;
  }
  if (graph.nvtxs <= nparts) {
    for (size_t v = 0; v < graph.nvtxs; ++v) part[v] = (Idx)(offset + std::min(v, nparts - 1));
    return 1;
  }
  const size_t k1 = nparts / 2, k2 = nparts - k1, ncon = graph.ncon;
  std::vector<float> lw(ncon, 0.0f), rw(ncon, 0.0f);
  for (size_t c = 0; c < ncon; ++c) {
    for (size_t i = c; i < k1 * ncon; i += ncon) lw[c] += tpwgts[i];
    for (size_t i = k1 * ncon + c; i < nparts * ncon; i += ncon) rw[c] += tpwgts[i];
  }
  const float total = lw[0] + rw[0];
  std::vector<float> bis;
  for (size_t c = 0; c < ncon; ++c) bis.push_back(lw[c] / total);
  for (size_t c = 0; c < ncon; ++c) bis.push_back(rw[c] / total);
  std::vector<Idx> bp;
  int rc = multilevel_bisect(graph, bis.data(), ub, opt, rng, bp);
  if (rc != 1) return rc;
  std::vector<size_t> n2o0, n2o1;
  Graph g0 = extract_subgraph(graph, bp.data(), 0, n2o0);
  Graph g1 = extract_subgraph(graph, bp.data(), 1, n2o1);
  std::vector<float> ltp, rtp;
  for (size_t i = 0; i < k1 * ncon; ++i) ltp.push_back(tpwgts[i] / lw[0]);
  for (size_t i = k1 * ncon; i < nparts * ncon; ++i) rtp.push_back(tpwgts[i] / rw[0]);
  std::vector<Idx> sp0(g0.nvtxs, 0), sp1(g1.nvtxs, 0);
  rc = rb_recurse(g0, k1, 0, ltp, ub, opt, rng, sp0);
  if (rc != 1) return rc;
  rc = rb_recurse(g1, k2, 0, rtp, ub, opt, rng, sp1);
  if (rc != 1) return rc;
  for (size_t i = 0; i < n2o0.size(); ++i) part[n2o0[i]] = sp0[i] + (Idx)offset;
  for (size_t i = 0; i < n2o1.size(); ++i) part[n2o1[i]] = sp1[i] + (Idx)(offset + k1);
  return 1;
}

// partition_recursive (src/partition/recursive.rs:12-57): one RNG for the
// whole recursion, seeded with options.seed (entropy when 0).
int partition_recursive(const Graph& graph, size_t nparts, const float* tpwgts, const float* ubvec, const Options& opt,
                        std::vector<Idx>& part, Idx& obj) {
  if (nparts < 2) return -2;
  if (nparts > graph.nvtxs) return -2;
  uint64_t seed;
  if (opt.seed == 0) {
    std::random_device rd;
    seed = ((uint64_t)rd() << 32) ^ (uint64_t)rd();
  } else {
    seed = opt.seed;
  }
  SmallRng rng = SmallRng::seed_from_u64(seed);
  const size_t ncon = graph.ncon;
  std::vector<float> tp;
  if (tpwgts) tp.assign(tpwgts, tpwgts + nparts * ncon);
  else tp.assign(nparts * ncon, 1.0f / (float)nparts);
  std::vector<double> ub(ncon);
  for (size_t c = 0; c < ncon; ++c) ub[c] = ubvec ? (double)ubvec[c] : 1.0 + (double)opt.ufactor / 1000.0;
  part.assign(graph.nvtxs, 0);
  int rc = rb_recurse(graph, nparts, 0, tp, ub.data(), opt, rng, part);
  if (rc != 1) return rc;
  obj = graph.edge_cut(part.data());
  return 1;
}

// ---------------------------------------------------------------------------
// Nested dissection (src/partition/nd.rs:15-110, src/separator/mod.rs:9-61).
// ---------------------------------------------------------------------------

// find_node_separator (src/separator/mod.rs:9-61): a recursive bisection with
// targets (0.5, 0.5) and ub 1.05 (seeded from options.seed, not from the
// caller's generator), then every vertex of the lighter side (constraint 0)
// with a neighbour across becomes a separator vertex.
void find_node_separator(const Graph& g, const Options& opt, std::vector<size_t>& left, std::vector<size_t>& right,
                         std::vector<size_t>& sep) {
  const float tp[2] = {0.5f, 0.5f};
  const float ub[1] = {1.05f};
  std::vector<Idx> part;
  Idx obj = 0;
  if (partition_recursive(g, 2, tp, ub, opt, part, obj) != 1) {
    part.assign(g.nvtxs, 0);                                   // separator/mod.rs:22-27
    for (size_t v = 0; v < g.nvtxs; ++v) part[v] = v < g.nvtxs / 2 ? 0 : 1;
  }
  std::vector<Idx> pw = g.partition_weights(part.data(), 2);
  const Idx smaller = pw[0] <= pw[g.ncon] ? 0 : 1;
  std::vector<char> in_sep(g.nvtxs, 0);
  for (size_t v = 0; v < g.nvtxs; ++v) {
    if (part[v] != smaller) continue;
    for (Idx j = g.xadj[v]; j < g.xadj[v + 1]; ++j)
      if (part[g.adjncy[j]] != part[v]) { in_sep[v] = 1; break; }
  }
  left.clear(); right.clear(); sep.clear();
  for (size_t v = 0; v < g.nvtxs; ++v) {
    if (in_sep[v]) sep.push_back(v);
    else if (part[v] == smaller) left.push_back(v);
    else right.push_back(v);
  }
}

// nd_recurse (src/partition/nd.rs:51-110): small graphs (<= 100 vertices) and
// degenerate separators (>= n/2) are numbered in order; otherwise the left
// side, then the right side, then the separator.
void nd_recurse(const Graph& g, const std::vector<size_t>& orig, const Options& opt, std::vector<Idx>& perm,
                size_t& counter) {
  const size_t n = g.nvtxs;
  if (n <= 100) {
    for (size_t o : orig) perm[o] = (Idx)counter++;
    return;
  }
  std::vector<size_t> left, right, sep;
  find_node_separator(g, opt, left, right, sep);
  if (sep.size() >= n / 2) {
    for (size_t o : orig) perm[o] = (Idx)counter++;
    return;
  }
  std::vector<Idx> side(n, 2);
  for (size_t v : left) side[v] = 0;
  for (size_t v : right) side[v] = 1;
  for (Idx s = 0; s < 2; ++s) {
    if ((s == 0 ? left : right).empty()) continue;
    std::vector<size_t> n2o;
    Graph sub = extract_subgraph(g, side.data(), s, n2o);
    std::vector<size_t> sub_orig(n2o.size());
    for (size_t i = 0; i < n2o.size(); ++i) sub_orig[i] = orig[n2o[i]];
    nd_recurse(sub, sub_orig, opt, perm, counter);
  }
  for (size_t v : sep) perm[orig[v]] = (Idx)counter++;
}

// node_nd (src/partition/nd.rs:15-43): perm[v] = new position of v,
// iperm its inverse.
void node_nd(const Graph& g, const Options& opt, std::vector<Idx>& perm, std::vector<Idx>& iperm) {
  const size_t n = g.nvtxs;
  perm.assign(n, 0);
  iperm.assign(n, 0);
  std::vector<size_t> orig(n);
  for (size_t v = 0; v < n; ++v) orig[v] = v;
  size_t counter = 0;
  nd_recurse(g, orig, opt, perm, counter);
  for (size_t v = 0; v < n; ++v) iperm[(size_t)perm[v]] = (Idx)v;
}

Graph make_graph(int64_t n, int64_t ncon, const Idx* xadj, const Idx* adjncy, const Idx* vwgt,
                 const Idx* adjwgt, const Idx* vsize) {
  Graph g;
  g.nvtxs = (size_t)n;
  g.ncon = (size_t)ncon;
  g.xadj.assign(xadj, xadj + n + 1);
  size_t ne = (size_t)xadj[n];
  g.adjncy.assign(adjncy, adjncy + ne);
  if (vwgt) { g.has_vwgt = true; g.vwgt.assign(vwgt, vwgt + n * ncon); }
  if (adjwgt) { g.has_adjwgt = true; g.adjwgt.assign(adjwgt, adjwgt + ne); }
  if (vsize) { g.has_vsize = true; g.vsize.assign(vsize, vsize + n); }
  return g;
}

}  // namespace

// ---------------------------------------------------------------------------
// extern "C" surface used by the tests (ctypes) and by bench.py's CPU legs.
// ---------------------------------------------------------------------------
extern "C" {

// SmallRng helpers for known-answer checks of the RNG restatement.
void orc_rng_seed_from_u64(uint64_t seed, uint64_t* state) {
  SmallRng r = SmallRng::seed_from_u64(seed);
  std::memcpy(state, r.s, sizeof(r.s));
}
void orc_rng_from_state_next_u64(uint64_t* state, int64_t count, uint64_t* out) {
  SmallRng r;
  std::memcpy(r.s, state, sizeof(r.s));
  for (int64_t i = 0; i < count; ++i) out[i] = r.next_u64();
  std::memcpy(state, r.s, sizeof(r.s));
}
uint64_t orc_rng_gen_range(uint64_t* state, uint64_t low, uint64_t high) {
  SmallRng r;
  std::memcpy(r.s, state, sizeof(r.s));
  uint64_t v = r.gen_range(low, high);
  std::memcpy(state, r.s, sizeof(r.s));
  return v;
}

int orc_validate_csr(int64_t nvtxs, int64_t ncon, const Idx* xadj, int64_t xadj_len,
                     const Idx* adjncy, int64_t adjncy_len, const Idx* vwgt, int64_t vwgt_len,
                     const Idx* adjwgt, int64_t adjwgt_len) {
  return validate_csr((size_t)nvtxs, (size_t)ncon, xadj, (size_t)xadj_len, adjncy,
                      (size_t)adjncy_len, vwgt, (size_t)vwgt_len, adjwgt, (size_t)adjwgt_len);
}

Idx orc_edge_cut(int64_t n, const Idx* xadj, const Idx* adjncy, const Idx* adjwgt, const Idx* part) {
  Graph g = make_graph(n, 1, xadj, adjncy, nullptr, adjwgt, nullptr);
  return g.edge_cut(part);
}

void orc_partition_weights(int64_t n, int64_t ncon, const Idx* vwgt, const Idx* part, int64_t nparts,
                           Idx* out) {
  Graph g;
  g.nvtxs = (size_t)n;
  g.ncon = (size_t)ncon;
  if (vwgt) { g.has_vwgt = true; g.vwgt.assign(vwgt, vwgt + n * ncon); }
  std::vector<Idx> pw = g.partition_weights(part, (size_t)nparts);
  std::memcpy(out, pw.data(), pw.size() * sizeof(Idx));
}

void orc_total_weight(int64_t n, int64_t ncon, const Idx* vwgt, Idx* out) {
  Graph g;
  g.nvtxs = (size_t)n;
  g.ncon = (size_t)ncon;
  if (vwgt) { g.has_vwgt = true; g.vwgt.assign(vwgt, vwgt + n * ncon); }
  std::vector<Idx> tw = g.total_weight();
  std::memcpy(out, tw.data(), tw.size() * sizeof(Idx));
}

int64_t orc_boundary_vertices(int64_t n, const Idx* xadj, const Idx* adjncy, const Idx* part,
                              Idx* out) {
  Graph g = make_graph(n, 1, xadj, adjncy, nullptr, nullptr, nullptr);
  std::vector<size_t> b = g.boundary_vertices(part);
  for (size_t i = 0; i < b.size(); ++i) out[i] = (Idx)b[i];
  return (int64_t)b.size();
}

Idx orc_compute_move_gain(int64_t n, const Idx* xadj, const Idx* adjncy, const Idx* adjwgt,
                          int64_t v, const Idx* part, Idx from, Idx to) {
  Graph g = make_graph(n, 1, xadj, adjncy, nullptr, adjwgt, nullptr);
  return compute_move_gain(g, (size_t)v, part, from, to);
}

// build_coarse_graph. Outputs: cmap[n], cxadj[cn+1], cadjncy/cadjwgt[m upper
// bound], cvwgt[cn*ncon] (written only when vwgt given). flags: bit0 = coarse
// graph keeps adjwgt, bit1 = coarse graph has vwgt. Returns cn.
int64_t orc_build_coarse_graph(int64_t n, int64_t ncon, const Idx* xadj, const Idx* adjncy,
                               const Idx* vwgt, const Idx* adjwgt, const Idx* matching, Idx* cmap,
                               Idx* cxadj, Idx* cadjncy, Idx* cadjwgt, Idx* cvwgt, int32_t* flags) {
  Graph g = make_graph(n, ncon, xadj, adjncy, vwgt, adjwgt, nullptr);
  std::vector<size_t> m((size_t)n), cm;
  for (int64_t v = 0; v < n; ++v) m[v] = (size_t)matching[v];
  Graph cg = g.build_coarse_graph(m, cm);
  for (int64_t v = 0; v < n; ++v) cmap[v] = (Idx)cm[v];
  std::memcpy(cxadj, cg.xadj.data(), cg.xadj.size() * sizeof(Idx));
  std::memcpy(cadjncy, cg.adjncy.data(), cg.adjncy.size() * sizeof(Idx));
  for (size_t j = 0; j < cg.adjncy.size(); ++j) cadjwgt[j] = cg.edge_weight_at(j);
  if (cg.has_vwgt) std::memcpy(cvwgt, cg.vwgt.data(), cg.vwgt.size() * sizeof(Idx));
  *flags = (cg.has_adjwgt ? 1 : 0) | (cg.has_vwgt ? 2 : 0);
  return (int64_t)cg.nvtxs;
}

void orc_shem_matching(int64_t n, const Idx* xadj, const Idx* adjncy, const Idx* adjwgt,
                       uint64_t* rng_state, Idx* out) {
  Graph g = make_graph(n, 1, xadj, adjncy, nullptr, adjwgt, nullptr);
  SmallRng r;
  std::memcpy(r.s, rng_state, sizeof(r.s));
  std::vector<size_t> m = shem_matching(g, r);
  std::memcpy(rng_state, r.s, sizeof(r.s));
  for (int64_t v = 0; v < n; ++v) out[v] = (Idx)m[v];
}

void orc_random_matching(int64_t n, const Idx* xadj, const Idx* adjncy, uint64_t* rng_state,
                         Idx* out) {
  Graph g = make_graph(n, 1, xadj, adjncy, nullptr, nullptr, nullptr);
  SmallRng r;
  std::memcpy(r.s, rng_state, sizeof(r.s));
  std::vector<size_t> m = random_matching(g, r);
  std::memcpy(rng_state, r.s, sizeof(r.s));
  for (int64_t v = 0; v < n; ++v) out[v] = (Idx)m[v];
}

void orc_compute_target_weights(int64_t n, int64_t ncon, const Idx* vwgt, int64_t nparts,
                                 const float* tpwgts, double* out) {
  Graph g;
  g.nvtxs = (size_t)n;
  g.ncon = (size_t)ncon;
  if (vwgt) { g.has_vwgt = true; g.vwgt.assign(vwgt, vwgt + n * ncon); }
  std::vector<double> t = g.compute_target_weights((size_t)nparts, tpwgts);
  std::memcpy(out, t.data(), t.size() * sizeof(double));
}

// grow_partition; seeds == NULL draws them from rng_state (which is advanced),
// otherwise uses the given seeds. seeds_out (optional) receives the seeds.
void orc_grow_partition(int64_t n, int64_t ncon, const Idx* xadj, const Idx* adjncy,
                        const Idx* vwgt, int64_t nparts, const double* tpwgts, uint64_t* rng_state,
                        const Idx* seeds, Idx* seeds_out, Idx* part_out) {
  Graph g = make_graph(n, ncon, xadj, adjncy, vwgt, nullptr, nullptr);
  SmallRng r;
  if (rng_state) std::memcpy(r.s, rng_state, sizeof(r.s));
  std::vector<Idx> so;
  std::vector<Idx> part = grow_partition(g, (size_t)nparts, tpwgts, rng_state ? &r : nullptr, seeds, &so);
  if (rng_state) std::memcpy(rng_state, r.s, sizeof(r.s));
  if (seeds_out) std::memcpy(seeds_out, so.data(), so.size() * sizeof(Idx));
  std::memcpy(part_out, part.data(), part.size() * sizeof(Idx));
}

// greedy_refine on a graph; part is updated in place; returns the edge cut.
// moves_out (optional, length >= niter+1) receives the moves of each pass;
// *npasses receives the number of passes run.
Idx orc_greedy_refine(int64_t n, int64_t ncon, const Idx* xadj, const Idx* adjncy, const Idx* vwgt,
                      const Idx* adjwgt, Idx* part, int64_t nparts, const double* tpwgts,
                      const double* ubvec, int64_t niter, int64_t* moves_out, int64_t* npasses) {
  Graph g = make_graph(n, ncon, xadj, adjncy, vwgt, adjwgt, nullptr);
  std::vector<Idx> p(part, part + n);
  std::vector<int64_t> mv;
  Idx cut = greedy_refine(g, p, (size_t)nparts, tpwgts, ubvec, (size_t)niter, &mv);
  std::memcpy(part, p.data(), n * sizeof(Idx));
  if (moves_out) for (size_t i = 0; i < mv.size(); ++i) moves_out[i] = mv[i];
  if (npasses) *npasses = (int64_t)mv.size();
  return cut;
}

// fm_kway_refine on a graph; part is updated in place; returns the edge cut.
// stats (optional): [passes run, moves kept].
Idx orc_fm_kway_refine(int64_t n, int64_t ncon, const Idx* xadj, const Idx* adjncy, const Idx* vwgt,
                       const Idx* adjwgt, Idx* part, int64_t nparts, const double* tpwgts, const double* ubvec,
                       int64_t niter, int64_t* stats) {
  Graph g = make_graph(n, ncon, xadj, adjncy, vwgt, adjwgt, nullptr);
  std::vector<Idx> p(part, part + n);
  FmStats st;
  Idx cut = fm_kway_refine(g, p, (size_t)nparts, tpwgts, ubvec, (size_t)niter, &st);
  std::memcpy(part, p.data(), n * sizeof(Idx));
  if (stats) { stats[0] = st.passes; stats[1] = st.moves; }
  return cut;
}

// fm_refine (src/refine/fm.rs:12-28) on a 2-way partition; returns the cut.
Idx orc_fm2_refine(int64_t n, int64_t ncon, const Idx* xadj, const Idx* adjncy, const Idx* vwgt, const Idx* adjwgt,
                   Idx* part, const double* tpwgts, const double* ubvec, int64_t niter) {
  Graph g = make_graph(n, ncon, xadj, adjncy, vwgt, adjwgt, nullptr);
  std::vector<Idx> p(part, part + n);
  Idx cut = fm2_refine(g, p, tpwgts, ubvec, (size_t)niter);
  std::memcpy(part, p.data(), n * sizeof(Idx));
  return cut;
}

// Restated RMETIS_SetDefaultOptions (src/ffi/c_api.rs:15-23).
int orc_SetDefaultOptions(Idx* options) {
  if (!options) return -2;
  Options o;
  to_raw(o, options);
  return 1;
}

// Restated RMETIS_PartGraphKway (src/ffi/c_api.rs:56-81, 140-222) with an
// optional script (matchings per level + grow seeds) for replay.
int orc_PartGraphKway_script(const Idx* nvtxs, const Idx* ncon, const Idx* xadj, const Idx* adjncy,
                             const Idx* vwgt, const Idx* vsize, const Idx* adjwgt, const Idx* nparts,
                             const float* tpwgts, const float* ubvec, const Idx* options, Idx* objval,
                             Idx* part, const Idx* script_matchings, const int64_t* script_offsets,
                             int64_t script_nlevels, const Idx* script_seeds, int64_t* stats_out) {
  if (!nvtxs || !ncon || !xadj || !adjncy || !nparts || !part) return -2;
  int64_t n = *nvtxs, nc = *ncon, np = *nparts;
  if (n <= 0 || nc <= 0 || np < 2) return -2;
  int64_t ne = xadj[n];
  if (ne < 0) return -2;
  Options o;
  if (options && options[0] != -1) o = from_raw(options);    // c_api.rs:211-222
  if (validate_csr((size_t)n, (size_t)nc, xadj, (size_t)n + 1, adjncy, (size_t)ne, vwgt,
                   vwgt ? (size_t)(n * nc) : 0, adjwgt, adjwgt ? (size_t)ne : 0) != 0)
    return -2;
  Graph g = make_graph(n, nc, xadj, adjncy, vwgt, adjwgt, vsize);
  Script sc;
  Script* sp = nullptr;
  if (script_matchings || script_seeds) {
    sc.matchings = script_matchings;
    sc.level_offsets = script_offsets;
    sc.nlevels = script_nlevels;
    sc.grow_seeds = script_seeds;
    sp = &sc;
  }
  std::vector<Idx> best;
  Idx obj = 0;
  KwayStats st;
  int rc = partition_kway(g, (size_t)np, tpwgts, ubvec, o, best, obj, sp, &st);
  if (rc != 1) return rc;
  std::memcpy(part, best.data(), n * sizeof(Idx));
  if (objval) *objval = obj;
  if (stats_out) {
    stats_out[0] = st.nlevels;
    for (int64_t i = 0; i <= st.nlevels && i < 63; ++i) {
      stats_out[1 + 2 * i] = st.level_n[i];
      stats_out[2 + 2 * i] = st.level_m[i];
    }
  }
  return 1;
}

// Restated RMETIS_PartGraphRecursive (src/ffi/c_api.rs:27-53, c_partition_impl
// :140-209 with kway = false).
int orc_PartGraphRecursive(const Idx* nvtxs, const Idx* ncon, const Idx* xadj, const Idx* adjncy, const Idx* vwgt,
                           const Idx* vsize, const Idx* adjwgt, const Idx* nparts, const float* tpwgts,
                           const float* ubvec, const Idx* options, Idx* objval, Idx* part) {
  if (!nvtxs || !ncon || !xadj || !adjncy || !nparts || !part) return -2;
  int64_t n = *nvtxs, nc = *ncon, np = *nparts;
  if (n <= 0 || nc <= 0 || np < 2) return -2;
  int64_t ne = xadj[n];
  if (ne < 0) return -2;
  Options o;
  if (options && options[0] != -1) o = from_raw(options);
  if (validate_csr((size_t)n, (size_t)nc, xadj, (size_t)n + 1, adjncy, (size_t)ne, vwgt,
                   vwgt ? (size_t)(n * nc) : 0, adjwgt, adjwgt ? (size_t)ne : 0) != 0)
    return -2;
  Graph g = make_graph(n, nc, xadj, adjncy, vwgt, adjwgt, vsize);
  std::vector<Idx> best;
  Idx obj = 0;
  int rc = partition_recursive(g, (size_t)np, tpwgts, ubvec, o, best, obj);
  if (rc != 1) return rc;
  std::memcpy(part, best.data(), n * sizeof(Idx));
  if (objval) *objval = obj;
  return 1;
}

// Restated RMETIS_NodeND (src/ffi/c_api.rs:85-132): one constraint, vwgt
// optional, perm and iperm written.
int orc_NodeND(const Idx* nvtxs, const Idx* xadj, const Idx* adjncy, const Idx* vwgt, const Idx* options, Idx* perm,
               Idx* iperm) {
  if (!nvtxs || !xadj || !adjncy || !perm || !iperm) return -2;
  int64_t n = *nvtxs;
  if (n <= 0) return -2;
  int64_t ne = xadj[n];
  if (ne < 0) return -2;
  Options o;
  if (options && options[0] != -1) o = from_raw(options);
  if (validate_csr((size_t)n, 1, xadj, (size_t)n + 1, adjncy, (size_t)ne, vwgt, vwgt ? (size_t)n : 0, nullptr, 0) != 0)
    return -2;
  Graph g = make_graph(n, 1, xadj, adjncy, vwgt, nullptr, nullptr);
  std::vector<Idx> p, ip;
  node_nd(g, o, p, ip);
  std::memcpy(perm, p.data(), n * sizeof(Idx));
  std::memcpy(iperm, ip.data(), n * sizeof(Idx));
  return 1;
}

int orc_PartGraphKway(const Idx* nvtxs, const Idx* ncon, const Idx* xadj, const Idx* adjncy,
                      const Idx* vwgt, const Idx* vsize, const Idx* adjwgt, const Idx* nparts,
                      const float* tpwgts, const float* ubvec, const Idx* options, Idx* objval,
                      Idx* part) {
  return orc_PartGraphKway_script(nvtxs, ncon, xadj, adjncy, vwgt, vsize, adjwgt, nparts, tpwgts,
                                  ubvec, options, objval, part, nullptr, nullptr, 0, nullptr, nullptr);
}

}  // extern "C"
