// Invariant checks of the pipeline (debug mode, RMETIS_B200_CHECKS=1) and
// the per-level trace (RMETIS_B200_TRACE_JSON=<path>).
//
// The checks run after every contraction and every level's refinement and
// never trap: a violated invariant is counted in a device word, the host reads
// it back and throws METIS_ERROR with the invariant's name. They cover what a
// wrong kernel would break first: cmap maps onto [0, cn) and every coarse
// vertex has one or two members (a contraction of a matching that is not an
// involution breaks it), coarse vertex weights sum to the fine ones, part ids
// lie in [0, k) and the refined part weights sum to the level's total.
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "engine.h"

namespace rmb {

namespace {

// bad[0]: values outside [lo, hi); bad[1]: coarse ids hit by no fine vertex
// or by more than two.
__global__ void k_check_cmap(const idx_t* __restrict__ cmap, int32_t n, int32_t cn, int32_t* __restrict__ hits,
                             int32_t* __restrict__ bad) {
  RMB_GRID_STRIDE(v, n) {
    const int32_t c = cmap[v];
    if (c < 0 || c >= cn) atomicAdd(&bad[0], 1);
    else atomicAdd(&hits[c], 1);
  }
}

__global__ void k_check_hits(const int32_t* __restrict__ hits, int32_t cn, int32_t* __restrict__ bad) {
  RMB_GRID_STRIDE(c, cn) {
    if (hits[c] < 1 || hits[c] > 2) atomicAdd(&bad[1], 1);
  }
}

__global__ void k_check_range(const idx_t* __restrict__ a, int32_t n, int32_t lo, int32_t hi,
                              int32_t* __restrict__ bad) {
  RMB_GRID_STRIDE(v, n) {
    if (a[v] < lo || a[v] >= hi) atomicAdd(bad, 1);
  }
}

void fail(const char* what) {
  std::fprintf(stderr, "rmetis_b200: invariant violated: %s\n", what);
  throw Error(-4, std::string("invariant violated: ") + what);
}

}  // namespace

bool checks_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("RMETIS_B200_CHECKS");
    return e && *e && *e != '0';
  }();
  return on;
}

void check_contraction(const DGraph& fine, const DGraph& coarse, const idx_t* cmap, Arena& arena, cudaStream_t st,
                       int32_t* h_scratch) {
  Arena::Mark mk = arena.mark();
  int32_t* hits = arena.alloc<int32_t>((size_t)coarse.n + 1);
  int32_t* bad = arena.alloc<int32_t>(2);
  long long* tot = arena.alloc<long long>(2 * (size_t)fine.ncon);
  RMB_CUDA(cudaMemsetAsync(hits, 0, sizeof(int32_t) * ((size_t)coarse.n + 1), st));
  RMB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t) * 2, st));
  k_check_cmap<<<grid_for(fine.n, 256), 256, 0, st>>>(cmap, fine.n, coarse.n, hits, bad);
  RMB_LAUNCH_CHECK();
  k_check_hits<<<grid_for(coarse.n, 256), 256, 0, st>>>(hits, coarse.n, bad);
  RMB_LAUNCH_CHECK();
  const bool weights = fine.vwgt && coarse.vwgt;
  if (weights) {
    total_weight(fine, tot, st);
    total_weight(coarse, tot + fine.ncon, st);
  }
  RMB_CUDA(cudaMemcpyAsync(h_scratch, bad, sizeof(int32_t) * 2, cudaMemcpyDeviceToHost, st));
  long long ht[16] = {0};
  if (weights)
    RMB_CUDA(cudaMemcpyAsync(ht, tot, sizeof(long long) * 2 * (size_t)fine.ncon, cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  arena.reset_to(mk);
  if (h_scratch[0]) fail("cmap maps a fine vertex outside [0, cn)");
  if (h_scratch[1]) fail("a coarse vertex has no member or more than two");
  for (int c = 0; weights && c < fine.ncon; ++c)
    if (ht[c] != ht[fine.ncon + c]) fail("coarse vertex weights do not sum to the fine ones");
}

void check_refined(const DGraph& g, const idx_t* part, int k, Arena& arena, cudaStream_t st, int32_t* h_scratch) {
  Arena::Mark mk = arena.mark();
  int32_t* bad = arena.alloc<int32_t>(1);
  long long* pw = arena.alloc<long long>((size_t)k * g.ncon);
  long long* tot = arena.alloc<long long>((size_t)g.ncon);
  RMB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
  k_check_range<<<grid_for(g.n, 256), 256, 0, st>>>(part, g.n, 0, k, bad);
  RMB_LAUNCH_CHECK();
  RMB_CUDA(cudaMemcpyAsync(h_scratch, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  if (h_scratch[0]) {
    arena.reset_to(mk);
    fail("a part id lies outside [0, k)");
  }
  partition_weights_only(g, part, k, pw, st);
  if (g.vwgt) total_weight(g, tot, st);
  std::vector<long long> hpw((size_t)k * g.ncon), ht(g.ncon, g.n);
  RMB_CUDA(cudaMemcpyAsync(hpw.data(), pw, sizeof(long long) * hpw.size(), cudaMemcpyDeviceToHost, st));
  if (g.vwgt) RMB_CUDA(cudaMemcpyAsync(ht.data(), tot, sizeof(long long) * ht.size(), cudaMemcpyDeviceToHost, st));
  RMB_CUDA(cudaStreamSynchronize(st));
  arena.reset_to(mk);
  for (int c = 0; c < g.ncon; ++c) {
    long long s = 0;
    for (int p = 0; p < k; ++p) s += hpw[(size_t)p * g.ncon + c];
    if (s != ht[c]) fail("part weights do not sum to the level's total weight");
  }
}

// ---- per-level trace -------------------------------------------------------
const char* trace_json_path() {
  static const char* p = std::getenv("RMETIS_B200_TRACE_JSON");
  return p && *p ? p : nullptr;
}

void trace_json_write(const std::string& line) {
  static std::mutex mu;
  const char* path = trace_json_path();
  if (!path) return;
  std::lock_guard<std::mutex> lk(mu);
  if (FILE* f = std::fopen(path, "a")) {
    std::fputs(line.c_str(), f);
    std::fputc('\n', f);
    std::fclose(f);
  }
}

}  // namespace rmb
