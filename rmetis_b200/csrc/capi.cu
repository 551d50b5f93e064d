// extern "C" boundary: the reference's C ABI (src/ffi/c_api.rs) plus the GPU
// extensions declared in include/rmetis.h.
#include <future>
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <condition_variable>
#include <thread>
#include <memory>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/rmetis.h"
#include "engine.h"
#include "prof.h"
#include "scan.cuh"

using namespace rmb;

namespace {

// Options::from_raw (src/types.rs:190-224) as read by parse_options
// (src/ffi/c_api.rs:211-222): NULL or options[0] == -1 means all defaults.
KwayOptions parse_options(const idx_t* a) {
  KwayOptions o;
  if (!a || a[METIS_OPTION_PTYPE] == -1) return o;
  if (a[METIS_OPTION_CTYPE] == 0) o.ctype = 0;
  if (a[METIS_OPTION_IPTYPE] == 1) o.iptype = 1;
  else if (a[METIS_OPTION_IPTYPE] == 4) o.iptype = 4;
  if (a[METIS_OPTION_RTYPE] == 1) o.rtype = 1;
  if (a[METIS_OPTION_NCUTS] > 0) o.ncuts = a[METIS_OPTION_NCUTS];
  if (a[METIS_OPTION_NITER] > 0) o.niter = a[METIS_OPTION_NITER];
  o.seed = (uint64_t)(a[METIS_OPTION_SEED] > 0 ? a[METIS_OPTION_SEED] : 0);
  if (a[METIS_OPTION_UFACTOR] > 0) o.ufactor = (uint32_t)a[METIS_OPTION_UFACTOR];
  // objtype, no2hop, minconn, contig, numbering and dbglvl are decoded by the
  // reference but never read on its k-way path; they have no effect here either.
  return o;
}

struct Tuning {
  int grow_trials = 32;
  int match_rounds = 24;
  int summed_unit_weights = 0;
  int parallel_attempts = 1;
  int fused_max_n = 4096;
  int tail_max_n = 4096;
  int exact_max_n = 16384;
  int contract_thread_max = 32;
  int gain_block = 256;
  int fm_fused_max_n = 4096;
  int fused_edge_factor = 4;
};
// 1: batches run through the batched kernels (RMETIS_GPU_SetBatchMode).
int& batch_mode() {
  static int m = 1;
  return m;
}
// Graphs of a batch with more vertices than this run on the worker pool,
// alongside the batched launches of the others.
int& batch_max_n() {
  static int m = 262144;
  return m;
}
Tuning& tuning() {
  static Tuning t;
  return t;
}

void apply_tuning(KwayOptions& o) {
  o.grow_trials = tuning().grow_trials;
  o.match_rounds = tuning().match_rounds;
  o.summed_unit_weights = tuning().summed_unit_weights;
  o.parallel_attempts = tuning().parallel_attempts;
  o.fused_max_n = tuning().fused_max_n;
  o.tail_max_n = tuning().tail_max_n;
  o.exact_max_n = tuning().exact_max_n;
  o.contract_thread_max = tuning().contract_thread_max;
  o.gain_block = tuning().gain_block;
  o.fm_fused_max_n = tuning().fm_fused_max_n;
  o.fused_edge_factor = tuning().fused_edge_factor;
}

// Launch-shape knobs of jobs that share the device with other jobs (batch
// graphs and submitted requests); -1 = the single-call value. A single-block
// launch occupies one SM, which costs a lone call the idle rest of the device
// but not a job running beside others, so the best sizes differ.
struct PoolTuning {
  int fused_max_n = -1;
  int tail_max_n = -1;
};
PoolTuning& pool_tuning() {
  static PoolTuning t;
  return t;
}

void apply_pool_tuning(KwayOptions& o) {
  apply_tuning(o);
  if (pool_tuning().fused_max_n >= 0) o.fused_max_n = pool_tuning().fused_max_n;
  if (pool_tuning().tail_max_n >= 0) o.tail_max_n = pool_tuning().tail_max_n;
  o.parallel_attempts = 0;  // the jobs already run concurrently
}

template <typename F>
int guarded(F f) {
  try {
    return f();
  } catch (const rmb::Error& e) {
    if (std::getenv("RMETIS_B200_VERBOSE")) std::fprintf(stderr, "rmetis_b200: %s\n", e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    return METIS_ERROR_MEMORY;
  } catch (...) {
    return METIS_ERROR;
  }
}

// Upload a host array into arena memory (nullptr stays nullptr).
template <typename T>
T* upload(Engine& E, const T* h, size_t count) {
  if (!h) return nullptr;
  T* d = E.arena().alloc<T>(count ? count : 1);
  if (count) RMB_CUDA(cudaMemcpyAsync(d, h, sizeof(T) * count, cudaMemcpyHostToDevice, E.stream()));
  return d;
}

template <typename T>
void download(Engine& E, T* h, const T* d, size_t count) {
  if (count) RMB_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * count, cudaMemcpyDeviceToHost, E.stream()));
}

// The shared body of the host- and device-pointer entry points.
int kway_common(Engine& E, int32_t n, int32_t nc, int32_t np, const idx_t* d_xadj, const idx_t* d_adj, int64_t ne,
                const idx_t* d_vwgt, const idx_t* d_adjwgt, const real_t* tpwgts, const real_t* ubvec,
                const idx_t* options, idx_t* objval, idx_t* d_part, KwayTrace* trace,
                const KwayOptions* preset = nullptr) {
  KwayOptions o = preset ? *preset : parse_options(options);
  if (!preset) apply_tuning(o);
  DGraph g;
  g.n = n;
  g.m = ne;
  g.ncon = nc;
  g.xadj = d_xadj;
  g.adjncy = d_adj;
  g.adjwgt = d_adjwgt;
  g.vwgt = d_vwgt;
  // validate_csr (src/graph/validate.rs:16-142) on the device.
  if (validate_device(g, E.arena(), E.stream(), E.host_scratch()) != 0)
    throw Error(METIS_ERROR_INPUT, "graph failed validation");
  if (np > n) throw Error(METIS_ERROR_INPUT, "nparts > nvtxs");  // kway.rs:34-37
  int32_t obj = 0;
  E.partition_kway(g, np, tpwgts, ubvec, o, d_part, &obj, trace);
  if (objval) *objval = obj;
  return METIS_OK;
}

int kway_host(const idx_t* nvtxs, const idx_t* ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
              const idx_t* adjwgt, const idx_t* nparts, const real_t* tpwgts, const real_t* ubvec,
              const idx_t* options, idx_t* objval, idx_t* part, KwayTrace* trace) {
  // Mandatory pointers and scalar checks (src/ffi/c_api.rs:157-167).
  if (!nvtxs || !ncon || !xadj || !adjncy || !nparts || !part) return METIS_ERROR_INPUT;
  const int32_t n = *nvtxs, nc = *ncon, np = *nparts;
  if (n <= 0 || nc <= 0 || np < 2) return METIS_ERROR_INPUT;
  if (xadj[0] != 0 || xadj[n] < 0) return METIS_ERROR_INPUT;
  const int64_t ne = xadj[n];
  Engine& E = engine_for_current_device();
  std::lock_guard<std::mutex> lk(E.mu);
  Arena::Mark mk = E.arena().mark();
  struct Rewind {
    Engine& E;
    Arena::Mark m;
    ~Rewind() { E.arena().reset_to(m); }
  } rw{E, mk};
  idx_t* d_xadj = upload(E, xadj, (size_t)n + 1);
  idx_t* d_adj = upload(E, adjncy, (size_t)ne);
  idx_t* d_vwgt = upload(E, vwgt, (size_t)n * nc);
  idx_t* d_adjwgt = upload(E, adjwgt, (size_t)ne);
  idx_t* d_part = E.arena().alloc<idx_t>((size_t)n);
  int rc = kway_common(E, n, nc, np, d_xadj, d_adj, ne, d_vwgt, d_adjwgt, tpwgts, ubvec, options, objval, d_part,
                       trace);
  download(E, part, d_part, (size_t)n);
  RMB_CUDA(cudaStreamSynchronize(E.stream()));
  return rc;
}

// Host arrays for the single-function entry points.
struct HostCall {
  Engine& E;
  std::lock_guard<std::mutex> lk;
  Arena::Mark mk;
  HostCall() : E(engine_for_current_device()), lk(E.mu), mk(E.arena().mark()) {}
  ~HostCall() { E.arena().reset_to(mk); }
  cudaStream_t st() { return E.stream(); }
  void sync() { RMB_CUDA(cudaStreamSynchronize(E.stream())); }
};

// Host-side structural checks for the single-function entry points: every
// index a kernel will follow must be in range before anything is uploaded.
void check_csr(idx_t n, const idx_t* xadj, const idx_t* adjncy) {
  if (xadj[0] != 0) throw Error(METIS_ERROR_INPUT, "xadj[0] != 0");
  for (idx_t i = 0; i < n; ++i)
    if (xadj[i] > xadj[i + 1]) throw Error(METIS_ERROR_INPUT, "xadj not monotone");
  for (int64_t j = 0; j < xadj[n]; ++j)
    if (adjncy[j] < 0 || adjncy[j] >= n) throw Error(METIS_ERROR_INPUT, "adjncy out of range");
}

void check_range(const idx_t* a, int64_t len, idx_t hi, const char* what) {
  for (int64_t i = 0; i < len; ++i)
    if (a[i] < 0 || a[i] >= hi) throw Error(METIS_ERROR_INPUT, what);
}

DGraph dgraph(HostCall& h, idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
              const idx_t* adjwgt) {
  check_csr(n, xadj, adjncy);
  DGraph g;
  g.n = n;
  g.ncon = ncon;
  g.m = xadj ? xadj[n] : 0;
  g.xadj = upload(h.E, xadj, (size_t)n + 1);
  g.adjncy = upload(h.E, adjncy, (size_t)g.m);
  g.adjwgt = upload(h.E, adjwgt, (size_t)g.m);
  g.vwgt = upload(h.E, vwgt, (size_t)n * ncon);
  return g;
}

// ---- recursive bisection (src/partition/recursive.rs:12-187) --------------
// The recursion's bookkeeping and the target arithmetic (f32, as the
// reference's Real) run on the host; the subgraphs stay on the device, every
// bisection with more than two vertices and at least one edge is a 2-way
// multilevel partition on the GPU (coarsening, grow trials and refinement of
// the engine), and the sides are extracted by kernels (rb_levels_dev). Nested
// dissection keeps host subgraphs (HostGraph, extract_sub).
struct HostGraph {
  int32_t n = 0;
  int32_t ncon = 1;
  std::vector<idx_t> xadj{0}, adj, vwgt, adjw;
  bool has_vw = false, has_w = false;
  idx_t vw(int32_t v, int c) const { return has_vw ? vwgt[(size_t)v * ncon + c] : 1; }
};

// Graph::extract_subgraph (src/graph/mod.rs:209-273).
HostGraph extract_sub(const HostGraph& g, const std::vector<idx_t>& part, idx_t target, std::vector<int32_t>& n2o) {
  n2o.clear();
  for (int32_t v = 0; v < g.n; ++v)
    if (part[v] == target) n2o.push_back(v);
  std::vector<int32_t> o2n(g.n, -1);
  for (size_t i = 0; i < n2o.size(); ++i) o2n[n2o[i]] = (int32_t)i;
  HostGraph s;
  s.n = (int32_t)n2o.size();
  s.ncon = g.ncon;
  s.has_vw = g.has_vw;
  s.has_w = g.has_w;
  s.xadj.assign((size_t)s.n + 1, 0);
  for (int32_t i = 0; i < s.n; ++i) {
    const int32_t old = n2o[i];
    for (idx_t j = g.xadj[old]; j < g.xadj[old + 1]; ++j) {
      const idx_t u = g.adj[j];
      if (part[u] != target) continue;
      s.adj.push_back(o2n[u]);
      if (g.has_w) s.adjw.push_back(g.adjw[j]);
    }
    s.xadj[(size_t)i + 1] = (idx_t)s.adj.size();
    if (g.has_vw)
      for (int c = 0; c < g.ncon; ++c) s.vwgt.push_back(g.vwgt[(size_t)old * g.ncon + c]);
  }
  return s;
}

// multilevel_bisect (recursive.rs:133-187) on the GPU. A bisection without
// edges has cut 0 whatever it does; it is split on the host in vertex order,
// each vertex to the side it leaves least loaded relative to its targets on
// all constraints.
void bisect(Engine& E, const HostGraph& g, const std::vector<float>& tp2, const real_t* ubvec, const KwayOptions& o,
            uint64_t seed, std::vector<idx_t>& part) {
  part.assign((size_t)g.n, 0);
  if (g.n <= 2) {  // recursive.rs:141-144
    for (int32_t v = 0; v < g.n; ++v) part[v] = v;
    return;
  }
  if (g.xadj[g.n] == 0) {
    // Each vertex, in order, goes to the side whose largest relative load
    // (weight / target over the constraints) stays lower with it (side 0 on
    // ties), which keeps both sides near their targets on every constraint.
    const int nc = g.ncon;
    std::vector<double> tot(nc, 0.0), w[2] = {std::vector<double>(nc, 0.0), std::vector<double>(nc, 0.0)};
    for (int32_t v = 0; v < g.n; ++v)
      for (int c = 0; c < nc; ++c) tot[c] += g.vw(v, c);
    auto load = [&](int side, int32_t v) {
      double worst = 0.0;
      for (int c = 0; c < nc; ++c) {
        const double t = (double)tp2[(size_t)side * nc + c] * tot[c];
        const double x = w[side][c] + g.vw(v, c);
        worst = std::max(worst, t > 0 ? x / t : (x > 0 ? 1e300 : 0.0));
      }
      return worst;
    };
    for (int32_t v = 0; v < g.n; ++v) {
      const int side = load(0, v) <= load(1, v) ? 0 : 1;
      part[v] = side;
      for (int c = 0; c < nc; ++c) w[side][c] += g.vw(v, c);
    }
    return;
  }
  Arena::Mark mk = E.arena().mark();
  struct Rewind {
    Engine& E;
    Arena::Mark m;
    ~Rewind() { E.arena().reset_to(m); }
  } rw{E, mk};
  DGraph dg;
  dg.n = g.n;
  dg.m = g.xadj[g.n];
  dg.ncon = g.ncon;
  dg.xadj = upload(E, g.xadj.data(), (size_t)g.n + 1);
  dg.adjncy = upload(E, g.adj.data(), (size_t)dg.m);
  dg.adjwgt = g.has_w ? upload(E, g.adjw.data(), (size_t)dg.m) : nullptr;
  dg.vwgt = g.has_vw ? upload(E, g.vwgt.data(), (size_t)g.n * g.ncon) : nullptr;
  idx_t* d_part = E.arena().alloc<idx_t>((size_t)g.n);
  KwayOptions ob = o;
  ob.seed = seed;
  ob.ncuts = 1;
  ob.parallel_attempts = 0;
  ob.bisect_fm2 = 1;  // refine_2way (recursive.rs:184-186): the 2-way FM of fm.rs for rtype Fm
  int32_t obj = 0;
  E.partition_kway(dg, 2, tp2.data(), ubvec, ob, d_part, &obj, nullptr);
  download(E, part.data(), d_part, (size_t)g.n);
  RMB_CUDA(cudaStreamSynchronize(E.stream()));
}


// ---- independent bisections at once --------------------------------------
// The subgraphs of one level of a recursion do not depend on each other:
// their bisections run concurrently on the device's worker pool (each worker
// has its own stream and workspace), instead of one after another.
struct BisectJob {
  const HostGraph* g = nullptr;
  std::vector<float> tp2;
  uint64_t seed = 0;
  std::vector<idx_t> part;
};

void bisect_all(std::vector<BisectJob>& jobs, const real_t* ubvec, const KwayOptions& o) {
  if (jobs.empty()) return;
  int dev = 0;
  RMB_CUDA(cudaGetDevice(&dev));
  WorkerPool& pool = pool_for_device(dev);
  std::vector<std::future<int>> fut;
  fut.reserve(jobs.size());
  for (BisectJob& j : jobs) {
    BisectJob* jp = &j;
    fut.push_back(pool.submit(footprint_bytes(j.g->n, j.g->xadj[j.g->n], 2, j.g->ncon), [jp, ubvec, &o](Engine& W) {
      bisect(W, *jp->g, jp->tp2, ubvec, o, jp->seed, jp->part);
      return 1;
    }));
  }
  int rc = 1;
  for (auto& f : fut) {
    const int r = f.get();
    if (r != 1 && rc == 1) rc = r;
  }
  if (rc != 1) throw Error(rc, "a bisection failed");
}

// rb_recurse (recursive.rs:61-131), one recursion level at a time (the
// device form below, rb_levels_dev): a node with nparts parts is bisected with
// the summed f32 targets of its halves (k1 = nparts / 2), both sides are
// extracted as subgraphs and become the next level's nodes with their targets
// divided by constraint 0's sum; a node with one part, or no more vertices
// than parts, is assigned directly. The bisections of a level run
// concurrently on the worker pool. The reference draws every bisection from
// one generator; here the bisection at position h of the recursion tree (root
// 0, children 2h+1 and 2h+2) runs with seed + h (0 stays 0: an entropy seed
// per bisection).
// ---- the recursion on the device -------------------------------------------
// The subgraphs of every level stay on the device: a level's bisections run on
// the worker pool reading their subgraph in place, and both sides of each are
// extracted by kernels (Graph::extract_subgraph, src/graph/mod.rs:209-273:
// the side's vertices in ascending old id, each row keeping its same-side
// neighbours in CSR order, renumbered). Per level the host reads back only the
// children's sizes.
struct DevNode {
  DGraph g;
  idx_t* orig = nullptr;  // [n] original vertex ids
  int32_t nparts = 2, offset = 0;
  std::vector<float> tp;
  uint64_t heap = 0;
};

struct LoadSide0 {
  const idx_t* side;
  __device__ idx_t operator()(int64_t i) const { return side[i] == 0 ? 1 : 0; }
};

// kdeg of each vertex (its same-side neighbours) at its position in its side.
__global__ void k_rb_kdeg(int32_t n, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                          const idx_t* __restrict__ side, const idx_t* __restrict__ pos0, idx_t* __restrict__ kdeg0,
                          idx_t* __restrict__ kdeg1) {
  RMB_GRID_STRIDE(v, n) {
    const idx_t s = side[v];
    int32_t c = 0;
    for (int32_t j = xadj[v]; j < xadj[v + 1]; ++j) c += side[adj[j]] == s ? 1 : 0;
    if (s == 0) kdeg0[pos0[v]] = c;
    else kdeg1[v - pos0[v]] = c;
  }
}

struct RbSide {
  idx_t* xadj;
  idx_t* adj;
  idx_t* adjw;
  idx_t* vwgt;
  idx_t* orig;
};

__global__ void k_rb_fill(int32_t n, int32_t ncon, const idx_t* __restrict__ xadj, const idx_t* __restrict__ adj,
                          const idx_t* __restrict__ adjw, const idx_t* __restrict__ vwgt,
                          const idx_t* __restrict__ orig, const idx_t* __restrict__ side,
                          const idx_t* __restrict__ pos0, RbSide s0, RbSide s1) {
  RMB_GRID_STRIDE(v, n) {
    const idx_t s = side[v];
    const RbSide& o = s == 0 ? s0 : s1;
    const int32_t i = s == 0 ? pos0[v] : (int32_t)v - pos0[v];
    int32_t k = o.xadj[i];
    for (int32_t j = xadj[v]; j < xadj[v + 1]; ++j) {
      const int32_t u = adj[j];
      if (side[u] != s) continue;
      o.adj[k] = s == 0 ? pos0[u] : u - pos0[u];
      if (adjw) o.adjw[k] = adjw[j];
      ++k;
    }
    if (vwgt)
      for (int c = 0; c < ncon; ++c) o.vwgt[(int64_t)i * ncon + c] = vwgt[(int64_t)v * ncon + c];
    o.orig[i] = orig[v];
  }
}

// part[orig[v]] = offset (mode 0) or offset + min(v, nparts - 1) (mode 1).
__global__ void k_rb_assign(int32_t n, const idx_t* __restrict__ orig, int32_t offset, int32_t nparts, int mode,
                            idx_t* __restrict__ part) {
  RMB_GRID_STRIDE(v, n) part[orig[v]] = mode == 0 ? offset : offset + min((int32_t)v, nparts - 1);
}

__global__ void k_rb_iota(int32_t n, idx_t* __restrict__ a) {
  RMB_GRID_STRIDE(v, n) a[v] = (idx_t)v;
}

// multilevel_bisect (recursive.rs:133-187) of a device-resident subgraph into
// d_side: two vertices or fewer by position; a subgraph without edges on the
// host (as bisect does); otherwise a 2-way partition on the GPU.
void bisect_dev(Engine& E, const DGraph& g, const std::vector<float>& tp2, const real_t* ubvec, const KwayOptions& o,
                uint64_t seed, idx_t* d_side) {
  cudaStream_t st = E.stream();
  if (g.n <= 2) {  // recursive.rs:141-144
    k_rb_iota<<<1, 32, 0, st>>>(g.n, d_side);
    RMB_LAUNCH_CHECK();
    RMB_CUDA(cudaStreamSynchronize(st));
    return;
  }
  if (g.m == 0) {
    HostGraph h;
    h.n = g.n;
    h.ncon = g.ncon;
    h.xadj.assign((size_t)g.n + 1, 0);
    h.has_vw = g.vwgt != nullptr;
    if (h.has_vw) {
      h.vwgt.resize((size_t)g.n * g.ncon);
      download(E, h.vwgt.data(), g.vwgt, h.vwgt.size());
      RMB_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<idx_t> side;
    bisect(E, h, tp2, ubvec, o, seed, side);
    RMB_CUDA(cudaMemcpyAsync(d_side, side.data(), sizeof(idx_t) * side.size(), cudaMemcpyHostToDevice, st));
    RMB_CUDA(cudaStreamSynchronize(st));
    return;
  }
  KwayOptions ob = o;
  ob.seed = seed;
  ob.ncuts = 1;
  ob.parallel_attempts = 0;
  ob.bisect_fm2 = 1;  // refine_2way (recursive.rs:184-186): the 2-way FM of fm.rs for rtype Fm
  int32_t obj = 0;
  E.partition_kway(g, 2, tp2.data(), ubvec, ob, d_side, &obj, nullptr);
}

// rb_recurse (recursive.rs:61-131) level by level on the device (targets,
// seeds and direct assignments as described above). root.g and root.orig are
// device arrays; d_part gets the parts.
void rb_levels_dev(Engine& E, DevNode root, const real_t* ubvec, const KwayOptions& o, idx_t* d_part) {
  cudaStream_t st = E.stream();
  const int32_t n_in = root.g.n;
  const int64_t m_in = root.g.m;
  const int nc = root.g.ncon;
  const bool has_w = root.g.adjwgt != nullptr, has_vw = root.g.vwgt != nullptr;
  // Two regions, alternating by depth, hold the subgraphs of a level (the
  // children of one level sum to at most the input's vertices and entries).
  const size_t max_children = 2 * (size_t)std::max(root.nparts, 2) + 2;
  const size_t region_bytes = sizeof(idx_t) * (2 * ((size_t)n_in + max_children) + 2 * (size_t)m_in * (has_w ? 2 : 1) +
                                               2 * (size_t)n_in * (has_vw ? nc : 0) + 2 * (size_t)n_in) +
                              max_children * 5 * 256 + 256;
  char* region[2] = {E.arena().alloc<char>(region_bytes), E.arena().alloc<char>(region_bytes)};
  std::vector<DevNode> frontier;
  frontier.push_back(std::move(root));
  int depth = 0;
  int dev = 0;
  RMB_CUDA(cudaGetDevice(&dev));
  WorkerPool& pool = pool_for_device(dev);
  while (!frontier.empty()) {
    std::vector<DevNode*> split;
    for (DevNode& nd : frontier) {
      if (nd.nparts == 1 || nd.g.n <= nd.nparts) {
        k_rb_assign<<<grid_for(nd.g.n, 256), 256, 0, st>>>(nd.g.n, nd.orig, nd.offset, nd.nparts,
                                                           nd.nparts == 1 ? 0 : 1, d_part);
        RMB_LAUNCH_CHECK();
        continue;
      }
      split.push_back(&nd);
    }
    if (split.empty()) break;
    const size_t S = split.size();
    Arena::Mark mk = E.arena().mark();
    std::vector<std::vector<float>> tp2(S), lws(S), rws(S);
    std::vector<idx_t*> d_side(S);
    for (size_t i = 0; i < S; ++i) {
      const DevNode& nd = *split[i];
      const int32_t k1 = nd.nparts / 2;
      lws[i].assign(nc, 0.0f);
      rws[i].assign(nc, 0.0f);
      for (int c = 0; c < nc; ++c) {
        for (int32_t t = c; t < k1 * nc; t += nc) lws[i][c] += nd.tp[t];
        for (int32_t t = k1 * nc + c; t < nd.nparts * nc; t += nc) rws[i][c] += nd.tp[t];
      }
      const float total = lws[i][0] + rws[i][0];
      for (int c = 0; c < nc; ++c) tp2[i].push_back(lws[i][c] / total);
      for (int c = 0; c < nc; ++c) tp2[i].push_back(rws[i][c] / total);
      d_side[i] = E.arena().alloc<idx_t>((size_t)nd.g.n);
    }
    RMB_CUDA(cudaStreamSynchronize(st));  // the level's subgraphs are complete before the workers read them
    {
      std::vector<std::future<int>> fut;
      for (size_t i = 0; i < S; ++i) {
        const DevNode* nd = split[i];
        const std::vector<float>* t2 = &tp2[i];
        idx_t* ds = d_side[i];
        const uint64_t seed = o.seed == 0 ? 0 : o.seed + nd->heap;
        fut.push_back(pool.submit(footprint_bytes(nd->g.n, nd->g.m, 2, nc), [nd, t2, ds, seed, ubvec, &o](Engine& W) {
          bisect_dev(W, nd->g, *t2, ubvec, o, seed, ds);
          return 1;
        }));
      }
      int rc = 1;
      for (auto& f : fut) {
        const int r = f.get();
        if (r != 1 && rc == 1) rc = r;
      }
      if (rc != 1) throw Error(rc, "a bisection failed");
    }
    // Side sizes: n0 per node (one read-back for the level).
    idx_t* d_cnt = E.arena().alloc<idx_t>(S);
    std::vector<idx_t*> pos0(S);
    for (size_t i = 0; i < S; ++i) {
      pos0[i] = E.arena().alloc<idx_t>((size_t)split[i]->g.n);
      exclusive_scan<idx_t>(LoadSide0{d_side[i]}, StoreArr<idx_t>{pos0[i]}, split[i]->g.n, d_cnt + i, E.arena(), st);
    }
    std::vector<idx_t> n0(S);
    download(E, n0.data(), d_cnt, S);
    RMB_CUDA(cudaStreamSynchronize(st));
    // Children's row offsets (in this depth's region) and entry counts.
    char* reg = region[depth & 1];
    size_t off = 0;
    auto take = [&](size_t count) {
      idx_t* p = reinterpret_cast<idx_t*>(reg + off);
      off += (count * sizeof(idx_t) + 255) & ~(size_t)255;
      if (off > region_bytes) throw Error(-4, "recursion region overflow");
      return p;
    };
    std::vector<std::array<DevNode, 2>> kids(S);
    for (size_t i = 0; i < S; ++i) {
      const DevNode& nd = *split[i];
      const int32_t ns[2] = {n0[i], nd.g.n - n0[i]};
      idx_t* kdeg[2] = {E.arena().alloc<idx_t>((size_t)ns[0] + 1), E.arena().alloc<idx_t>((size_t)ns[1] + 1)};
      k_rb_kdeg<<<grid_for(nd.g.n, 256), 256, 0, st>>>(nd.g.n, nd.g.xadj, nd.g.adjncy, d_side[i], pos0[i], kdeg[0],
                                                       kdeg[1]);
      RMB_LAUNCH_CHECK();
      for (int sd = 0; sd < 2; ++sd) {
        DevNode& ch = kids[i][sd];
        ch.g.n = ns[sd];
        ch.g.ncon = nc;
        idx_t* cx = take((size_t)ns[sd] + 1);
        exclusive_scan_arr<idx_t>(kdeg[sd], cx, ns[sd], cx + ns[sd], E.arena(), st);
        ch.g.xadj = cx;
      }
    }
    std::vector<idx_t> ms(2 * S);
    for (size_t i = 0; i < S; ++i)
      for (int sd = 0; sd < 2; ++sd)
        download(E, &ms[2 * i + sd], kids[i][sd].g.xadj + kids[i][sd].g.n, 1);
    RMB_CUDA(cudaStreamSynchronize(st));
    std::vector<DevNode> next;
    for (size_t i = 0; i < S; ++i) {
      const DevNode& nd = *split[i];
      const int32_t k1 = nd.nparts / 2, k2 = nd.nparts - k1;
      RbSide so[2];
      for (int sd = 0; sd < 2; ++sd) {
        DevNode& ch = kids[i][sd];
        ch.g.m = ms[2 * i + sd];
        idx_t* ca = take((size_t)ch.g.m);
        idx_t* cw = has_w ? take((size_t)ch.g.m) : nullptr;
        idx_t* cv = has_vw ? take((size_t)ch.g.n * nc) : nullptr;
        ch.orig = take((size_t)ch.g.n);
        ch.g.adjncy = ca;
        ch.g.adjwgt = cw;
        ch.g.vwgt = cv;
        so[sd] = RbSide{const_cast<idx_t*>(ch.g.xadj), ca, cw, cv, ch.orig};
        ch.nparts = sd == 0 ? k1 : k2;
        ch.offset = sd == 0 ? nd.offset : nd.offset + k1;
        const float div = sd == 0 ? lws[i][0] : rws[i][0];
        for (int32_t t = sd == 0 ? 0 : k1 * nc; t < (sd == 0 ? k1 * nc : nd.nparts * nc); ++t)
          ch.tp.push_back(nd.tp[t] / div);
        ch.heap = 2 * nd.heap + 1 + (uint64_t)sd;
      }
      k_rb_fill<<<grid_for(nd.g.n, 256), 256, 0, st>>>(nd.g.n, nc, nd.g.xadj, nd.g.adjncy, nd.g.adjwgt, nd.g.vwgt,
                                                       nd.orig, d_side[i], pos0[i], so[0], so[1]);
      RMB_LAUNCH_CHECK();
      next.push_back(std::move(kids[i][0]));
      next.push_back(std::move(kids[i][1]));
    }
    RMB_CUDA(cudaStreamSynchronize(st));  // the children are written before the level's scratch is dropped
    E.arena().reset_to(mk);
    frontier = std::move(next);
    ++depth;
  }
  RMB_CUDA(cudaStreamSynchronize(st));
}

int recursive_host(const idx_t* nvtxs, const idx_t* ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                   const idx_t* adjwgt, const idx_t* nparts, const real_t* tpwgts, const real_t* ubvec,
                   const idx_t* options, idx_t* objval, idx_t* part) {
  // Mandatory pointers and scalar checks (src/ffi/c_api.rs:157-167).
  if (!nvtxs || !ncon || !xadj || !adjncy || !nparts || !part) return METIS_ERROR_INPUT;
  const int32_t n = *nvtxs, nc = *ncon, np = *nparts;
  if (n <= 0 || nc <= 0 || np < 2) return METIS_ERROR_INPUT;
  if (xadj[0] != 0 || xadj[n] < 0) return METIS_ERROR_INPUT;
  if (nc > 8) return METIS_ERROR_INPUT;
  const int64_t ne = xadj[n];
  KwayOptions o = parse_options(options);
  apply_tuning(o);
  Engine& E = engine_for_current_device();
  std::lock_guard<std::mutex> lk(E.mu);
  Arena::Mark mk = E.arena().mark();
  struct Rewind {
    Engine& E;
    Arena::Mark m;
    ~Rewind() { E.arena().reset_to(m); }
  } rw{E, mk};
  // The input on the device: validate_csr (src/graph/validate.rs:16-142) as
  // Graph::new does, then the root of the recursion, read in place.
  DGraph g;
  g.n = n;
  g.m = ne;
  g.ncon = nc;
  g.xadj = upload(E, xadj, (size_t)n + 1);
  g.adjncy = upload(E, adjncy, (size_t)ne);
  g.vwgt = upload(E, vwgt, (size_t)n * nc);
  g.adjwgt = upload(E, adjwgt, (size_t)ne);
  if (validate_device(g, E.arena(), E.stream(), E.host_scratch()) != 0)
    throw Error(METIS_ERROR_INPUT, "graph failed validation");
  if (np > n) return METIS_ERROR_INPUT;  // recursive.rs:22-26
  std::vector<float> tp;
  if (tpwgts) tp.assign(tpwgts, tpwgts + (size_t)np * nc);
  else tp.assign((size_t)np * nc, 1.0f / (float)np);  // recursive.rs:38-43
  DevNode root;
  root.g = g;
  root.orig = E.arena().alloc<idx_t>((size_t)n);
  k_rb_iota<<<grid_for(n, 256), 256, 0, E.stream()>>>(n, root.orig);
  RMB_LAUNCH_CHECK();
  root.nparts = np;
  root.tp = std::move(tp);
  idx_t* d_part = E.arena().alloc<idx_t>((size_t)n);
  rb_levels_dev(E, std::move(root), ubvec, o, d_part);
  std::vector<idx_t> out((size_t)n, 0);
  download(E, out.data(), d_part, (size_t)n);
  RMB_CUDA(cudaStreamSynchronize(E.stream()));
  // edge_cut (src/graph/mod.rs:123-137): i32 sum over both directions, / 2.
  uint32_t cut = 0;
  for (int32_t v = 0; v < n; ++v)
    for (idx_t j = xadj[v]; j < xadj[v + 1]; ++j)
      if (out[adjncy[j]] != out[v]) cut += (uint32_t)(adjwgt ? adjwgt[j] : 1);
  std::memcpy(part, out.data(), sizeof(idx_t) * (size_t)n);
  if (objval) *objval = (idx_t)cut / 2;
  return METIS_OK;
}

// ---- nested dissection (src/partition/nd.rs:16-111, src/separator/mod.rs:10-61)
// The reference recurses depth first: a graph of more than 100 vertices is
// bisected by partition_recursive (targets 0.5/0.5, ubvec 1.05, the caller's
// options, so every bisection starts from options.seed), the boundary of the
// lighter side (constraint 0, ties to side 0) becomes the separator, and the
// two sides without it are ordered first (lighter side first), the separator
// last; a separator of n/2 vertices or more, or a graph of at most 100
// vertices, is ordered as it stands. Here the recursion tree is built level by
// level, every bisection of a level at once on the worker pool; the numbering
// is then assigned in the reference's depth-first order.
struct NdNode {
  HostGraph g;
  std::vector<int32_t> orig;  // original id of each local vertex
  int left = -1, right = -1;  // children (node indices), -1 if none
  std::vector<int32_t> sep;   // local ids of the separator, ascending
  bool leaf = true;
};

constexpr int32_t kNdThreshold = 100;  // nd.rs:13

void nd_order(std::vector<NdNode>& nodes, const KwayOptions& o) {
  const real_t ub[1] = {1.05f};  // separator/mod.rs:21
  std::vector<int> frontier{0};
  while (!frontier.empty()) {
    std::vector<int> split;
    for (int id : frontier)
      if (nodes[id].g.n > kNdThreshold) split.push_back(id);
    std::vector<BisectJob> jobs(split.size());
    for (size_t i = 0; i < split.size(); ++i) {
      jobs[i].g = &nodes[split[i]].g;
      jobs[i].tp2 = {0.5f, 0.5f};
      jobs[i].seed = o.seed;
    }
    bisect_all(jobs, ub, o);
    std::vector<int> next;
    for (size_t i = 0; i < split.size(); ++i) {
      const int id = split[i];
      const HostGraph& g = nodes[id].g;
      const std::vector<idx_t>& part = jobs[i].part;
      int32_t pw[2] = {0, 0};  // partition_weights, i32 as the reference sums them
      for (int32_t v = 0; v < g.n; ++v) pw[part[v]] = (int32_t)((uint32_t)pw[part[v]] + (uint32_t)g.vw(v, 0));
      const idx_t smaller = pw[0] <= pw[1] ? 0 : 1;
      std::vector<idx_t> code((size_t)g.n);
      std::vector<int32_t> sep;
      for (int32_t v = 0; v < g.n; ++v) {
        bool cut = false;
        if (part[v] == smaller)
          for (idx_t j = g.xadj[v]; j < g.xadj[v + 1] && !cut; ++j) cut = part[g.adj[j]] != part[v];
        if (cut) sep.push_back(v);
        code[v] = cut ? 2 : (part[v] == smaller ? 0 : 1);
      }
      if ((int64_t)sep.size() >= g.n / 2) continue;  // degenerate separator: ordered as it stands (nd.rs:78-84)
      nodes[id].leaf = false;
      nodes[id].sep = std::move(sep);
      for (idx_t side = 0; side < 2; ++side) {
        std::vector<int32_t> n2o;
        HostGraph sub = extract_sub(nodes[id].g, code, side, n2o);
        if (sub.n == 0) continue;
        NdNode child;
        child.g = std::move(sub);
        child.orig.resize(n2o.size());
        for (size_t t = 0; t < n2o.size(); ++t) child.orig[t] = nodes[id].orig[n2o[t]];
        nodes.push_back(std::move(child));  // may move nodes: index, not reference
        const int cid = (int)nodes.size() - 1;
        (side == 0 ? nodes[id].left : nodes[id].right) = cid;
        next.push_back(cid);
      }
    }
    frontier = std::move(next);
  }
}

int nodend_host(const idx_t* nvtxs, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                const idx_t* options, idx_t* perm, idx_t* iperm) {
  // Pointer and size checks (src/ffi/c_api.rs:95-99).
  if (!nvtxs || !xadj || !adjncy || !perm || !iperm) return METIS_ERROR_INPUT;
  const int32_t n = *nvtxs;
  if (n <= 0) return METIS_ERROR_INPUT;
  if (xadj[0] != 0 || xadj[n] < 0) return METIS_ERROR_INPUT;
  const int64_t ne = xadj[n];
  KwayOptions o = parse_options(options);
  apply_tuning(o);
  Engine& E = engine_for_current_device();
  {
    // Graph::new (validate_csr) on the device: ncon 1, vwgt, no edge weights.
    std::lock_guard<std::mutex> lk(E.mu);
    Arena::Mark mk = E.arena().mark();
    struct Rewind {
      Engine& E;
      Arena::Mark m;
      ~Rewind() { E.arena().reset_to(m); }
    } rw{E, mk};
    DGraph g;
    g.n = n;
    g.m = ne;
    g.ncon = 1;
    g.xadj = upload(E, xadj, (size_t)n + 1);
    g.adjncy = upload(E, adjncy, (size_t)ne);
    g.vwgt = upload(E, vwgt, (size_t)n);
    if (validate_device(g, E.arena(), E.stream(), E.host_scratch()) != 0)
      throw Error(METIS_ERROR_INPUT, "graph failed validation");
  }
  std::vector<NdNode> nodes(1);
  HostGraph& g = nodes[0].g;
  g.n = n;
  g.ncon = 1;
  g.xadj.assign(xadj, xadj + n + 1);
  g.adj.assign(adjncy, adjncy + ne);
  g.has_vw = vwgt != nullptr;
  if (vwgt) g.vwgt.assign(vwgt, vwgt + n);
  nodes[0].orig.resize(n);
  for (int32_t v = 0; v < n; ++v) nodes[0].orig[v] = v;
  nd_order(nodes, o);
  // Depth-first numbering: left subtree, right subtree, then the separator
  // (nd.rs:88-110); a leaf in its own vertex order (nd.rs:57-63).
  int32_t counter = 0;
  std::vector<std::pair<int, int>> stack{{0, 0}};  // (node, stage)
  while (!stack.empty()) {
    auto& top = stack.back();
    const NdNode& nd = nodes[top.first];
    if (nd.leaf) {
      for (int32_t v : nd.orig) perm[v] = counter++;
      stack.pop_back();
    } else if (top.second == 0) {
      top.second = 1;
      if (nd.left >= 0) stack.push_back({nd.left, 0});
    } else if (top.second == 1) {
      top.second = 2;
      if (nd.right >= 0) stack.push_back({nd.right, 0});
    } else {
      for (int32_t v : nd.sep) perm[nd.orig[v]] = counter++;
      stack.pop_back();
    }
  }
  for (int32_t v = 0; v < n; ++v) iperm[perm[v]] = v;
  return METIS_OK;
}

}  // namespace

extern "C" {

int RMETIS_SetDefaultOptions(idx_t* options) {
  if (!options) return METIS_ERROR_INPUT;
  // Options::default().to_raw() (src/types.rs:77-95, :227-245)
  for (int i = 0; i < METIS_NOPTIONS; ++i) options[i] = -1;
  options[METIS_OPTION_CTYPE] = 1;      // Shem
  options[METIS_OPTION_IPTYPE] = 0;     // Grow
  options[METIS_OPTION_RTYPE] = 0;      // Fm
  options[METIS_OPTION_OBJTYPE] = 0;    // Cut
  options[METIS_OPTION_NO2HOP] = 0;
  options[METIS_OPTION_NCUTS] = 1;
  options[METIS_OPTION_NITER] = 10;
  options[METIS_OPTION_SEED] = 0;
  options[METIS_OPTION_MINCONN] = 0;
  options[METIS_OPTION_CONTIG] = 0;
  options[METIS_OPTION_UFACTOR] = 30;
  options[METIS_OPTION_NUMBERING] = 0;
  options[METIS_OPTION_DBGLVL] = 0;
  return METIS_OK;
}

int RMETIS_PartGraphKway(const idx_t* nvtxs, const idx_t* ncon, const idx_t* xadj, const idx_t* adjncy,
                         const idx_t* vwgt, const idx_t* vsize, const idx_t* adjwgt, const idx_t* nparts,
                         const real_t* tpwgts, const real_t* ubvec, const idx_t* options, idx_t* objval,
                         idx_t* part) {
  (void)vsize;  // aggregated by the reference's contraction but never read on the k-way path
  return guarded([&] {
    return kway_host(nvtxs, ncon, xadj, adjncy, vwgt, adjwgt, nparts, tpwgts, ubvec, options, objval, part,
                     nullptr);
  });
}

int RMETIS_PartGraphRecursive(const idx_t* nvtxs, const idx_t* ncon, const idx_t* xadj, const idx_t* adjncy,
                              const idx_t* vwgt, const idx_t* vsize, const idx_t* adjwgt, const idx_t* nparts,
                              const real_t* tpwgts, const real_t* ubvec, const idx_t* options, idx_t* objval,
                              idx_t* part) {
  (void)vsize;  // carried by the reference's subgraphs but never read
  return guarded([&] {
    return recursive_host(nvtxs, ncon, xadj, adjncy, vwgt, adjwgt, nparts, tpwgts, ubvec, options, objval, part);
  });
}

int RMETIS_NodeND(const idx_t* nvtxs, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt, const idx_t* options,
                  idx_t* perm, idx_t* iperm) {
  return guarded([&] { return nodend_host(nvtxs, xadj, adjncy, vwgt, options, perm, iperm); });
}

int RMETIS_GPU_PartGraphKwayDevice(const idx_t* nvtxs, const idx_t* ncon, const idx_t* d_xadj,
                                   const idx_t* d_adjncy, const idx_t* d_vwgt, const idx_t* d_adjwgt,
                                   const idx_t* nparts, const real_t* tpwgts, const real_t* ubvec,
                                   const idx_t* options, idx_t* objval, idx_t* d_part) {
  return guarded([&] {
    if (!nvtxs || !ncon || !d_xadj || !d_adjncy || !nparts || !d_part) return METIS_ERROR_INPUT;
    const int32_t n = *nvtxs, nc = *ncon, np = *nparts;
    if (n <= 0 || nc <= 0 || np < 2) return METIS_ERROR_INPUT;
    Engine& E = engine_for_current_device();
    std::lock_guard<std::mutex> lk(E.mu);
    int32_t* hs = E.host_scratch();
    RMB_CUDA(cudaMemcpyAsync(hs, d_xadj, sizeof(idx_t), cudaMemcpyDeviceToHost, E.stream()));
    RMB_CUDA(cudaMemcpyAsync(hs + 1, d_xadj + n, sizeof(idx_t), cudaMemcpyDeviceToHost, E.stream()));
    RMB_CUDA(cudaStreamSynchronize(E.stream()));
    if (hs[0] != 0 || hs[1] < 0) return METIS_ERROR_INPUT;
    const int64_t ne = hs[1];
    Arena::Mark mk = E.arena().mark();
    int rc;
    try {
      rc = kway_common(E, n, nc, np, d_xadj, d_adjncy, ne, d_vwgt, d_adjwgt, tpwgts, ubvec, options, objval, d_part,
                       nullptr);
      RMB_CUDA(cudaStreamSynchronize(E.stream()));
    } catch (...) {
      E.arena().reset_to(mk);
      throw;
    }
    E.arena().reset_to(mk);
    return rc;
  });
}

int RMETIS_GPU_SetStream(void* stream) {
  return guarded([&] {
    Engine& E = engine_for_current_device();
    std::lock_guard<std::mutex> lk(E.mu);
    E.set_stream(reinterpret_cast<cudaStream_t>(stream));
    return METIS_OK;
  });
}

int RMETIS_GPU_SetTuning(int grow_trials, int match_rounds, int summed_unit_weights, int parallel_attempts,
                         int fused_max_n, int tail_max_n) {
  if (grow_trials >= 0) tuning().grow_trials = grow_trials > 0 ? grow_trials : 1;
  if (match_rounds >= 0) tuning().match_rounds = match_rounds > 0 ? match_rounds : 1;
  if (summed_unit_weights >= 0) tuning().summed_unit_weights = summed_unit_weights ? 1 : 0;
  if (parallel_attempts >= 0) tuning().parallel_attempts = parallel_attempts ? 1 : 0;
  if (fused_max_n >= 0) tuning().fused_max_n = fused_max_n;
  if (tail_max_n >= 0) tuning().tail_max_n = tail_max_n;
  return METIS_OK;
}

int RMETIS_GPU_SetRefineMode(int exact_max_n) {
  if (exact_max_n < -1) return METIS_ERROR_INPUT;
  tuning().exact_max_n = exact_max_n == -1 ? INT32_MAX : exact_max_n;
  return METIS_OK;
}

int RMETIS_GPU_SetKernelShapes(int contract_thread_max, int gain_block) {
  if (contract_thread_max != -1 && contract_thread_max != 16 && contract_thread_max != 32) return METIS_ERROR_INPUT;
  if (gain_block != -1 && gain_block != 128 && gain_block != 256 && gain_block != 512) return METIS_ERROR_INPUT;
  if (contract_thread_max != -1) tuning().contract_thread_max = contract_thread_max;
  if (gain_block != -1) tuning().gain_block = gain_block;
  return METIS_OK;
}

int RMETIS_GPU_SetCoopMatching(int on) {
  if (on < 0 || on > 1) return METIS_ERROR_INPUT;
  coop_matching() = on;
  return METIS_OK;
}

int RMETIS_GPU_SetFusedEdgeFactor(int factor) {
  if (factor < -1 || factor == 0) return METIS_ERROR_INPUT;
  if (factor > 0) tuning().fused_edge_factor = factor;
  return METIS_OK;
}

int RMETIS_GPU_SetFmFusedMax(int max_n) {
  if (max_n < -1) return METIS_ERROR_INPUT;
  if (max_n >= 0) tuning().fm_fused_max_n = max_n;
  return METIS_OK;
}

int RMETIS_GPU_SetBatchMode(int mode, int max_n) {
  if (mode < -1 || mode > 1 || max_n < -1) return METIS_ERROR_INPUT;
  if (mode >= 0) batch_mode() = mode;
  if (max_n >= 0) batch_max_n() = max_n;
  return METIS_OK;
}

int RMETIS_GPU_SetPoolTuning(int fused_max_n, int tail_max_n) {
  if (fused_max_n >= -1) pool_tuning().fused_max_n = fused_max_n;
  if (tail_max_n >= -1) pool_tuning().tail_max_n = tail_max_n;
  return METIS_OK;
}

int RMETIS_GPU_SetProfiling(int on) {
  return guarded([&] {
    profiler().on = on != 0;
    profiler().reset();
    return METIS_OK;
  });
}

int RMETIS_GPU_GetProfile(int64_t* launches, double* ms, double* bytes, int max_ids) {
  return guarded([&] {
    profiler().collect();
    const int n = max_ids < (int)kProfCount ? max_ids : (int)kProfCount;
    for (int i = 0; i < n; ++i) {
      if (launches) launches[i] = profiler().totals.launches[i];
      if (ms) ms[i] = profiler().totals.ms[i];
      if (bytes) bytes[i] = profiler().totals.bytes[i];
    }
    // One slot past the kernel ids: all kernel launches of this library so far.
    if (max_ids > (int)kProfCount && launches) launches[kProfCount] = launch_counter();
    return (int)kProfCount;
  });
}

int RMETIS_GPU_PartGraphKwayBatch(idx_t ngraphs, idx_t ncon, const int64_t* vtx_off, const int64_t* edge_off,
                                  const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt, const idx_t* adjwgt,
                                  const idx_t* nparts, const real_t* ubvec, const idx_t* options, idx_t* objval,
                                  idx_t* part, idx_t* status) {
  return guarded([&] {
    if (ngraphs <= 0 || ncon <= 0 || !vtx_off || !edge_off || !xadj || !adjncy || !nparts || !part || !objval ||
        !status)
      return METIS_ERROR_INPUT;
    if (vtx_off[0] != 0 || edge_off[0] != 0) return METIS_ERROR_INPUT;
    for (idx_t g = 0; g < ngraphs; ++g) {
      const int64_t n = vtx_off[g + 1] - vtx_off[g], m = edge_off[g + 1] - edge_off[g];
      if (n <= 0 || n > INT32_MAX || m < 0 || m > INT32_MAX) return METIS_ERROR_INPUT;
      const idx_t* x = xadj + vtx_off[g] + g;
      if (x[0] != 0 || x[n] != m) return METIS_ERROR_INPUT;
    }
    KwayOptions o = parse_options(options);
    apply_pool_tuning(o);
    const int64_t ntot = vtx_off[ngraphs], mtot = edge_off[ngraphs];
    Engine& E = engine_for_current_device();
    std::lock_guard<std::mutex> lk(E.mu);
    Arena::Mark mk = E.arena().mark();
    struct Rewind {
      Engine& E;
      Arena::Mark m;
      ~Rewind() { E.arena().reset_to(m); }
    } rw{E, mk};
    // One upload of the concatenated batch; the workers read it in place.
    idx_t* d_xadj = upload(E, xadj, (size_t)(ntot + ngraphs));
    idx_t* d_adj = upload(E, adjncy, (size_t)mtot);
    idx_t* d_vwgt = upload(E, vwgt, (size_t)ntot * ncon);
    idx_t* d_adjwgt = upload(E, adjwgt, (size_t)mtot);
    idx_t* d_part = E.arena().alloc<idx_t>((size_t)ntot);
    std::vector<int> done(ngraphs, 0);
    std::vector<int32_t> objs(ngraphs, 0);
    // Graphs for the batched kernels: eligible and at most batch_max_n
    // vertices (a large graph's levels take one block each there, so it runs
    // faster on the pool's grid-wide kernels).
    std::vector<char> batched(ngraphs, 0);
    if (batch_mode() == 1)
      for (idx_t g = 0; g < ngraphs; ++g) {
        const int32_t n = (int32_t)(vtx_off[g + 1] - vtx_off[g]);
        batched[g] = batch_eligible(o, n, nparts[g], ncon) && n <= batch_max_n();
      }
    RMB_CUDA(cudaStreamSynchronize(E.stream()));  // the upload is complete before other streams read it
    int dev = 0;
    RMB_CUDA(cudaGetDevice(&dev));
    WorkerPool& pool = pool_for_device(dev);
    std::vector<std::future<int>> fut(ngraphs);
    std::vector<char> submitted(ngraphs, 0);
    auto submit = [&](idx_t g) {
      const int64_t v0 = vtx_off[g], e0 = edge_off[g];
      const int32_t n = (int32_t)(vtx_off[g + 1] - v0);
      const int64_t m = edge_off[g + 1] - e0;
      const int32_t k = nparts[g];
      int32_t* obj_g = &objs[g];
      submitted[g] = 1;
      fut[g] = pool.submit(footprint_bytes(n, m, std::max(k, 2), ncon), [=](Engine& W) {
        DGraph gr;
        gr.n = n;
        gr.m = m;
        gr.ncon = ncon;
        gr.xadj = d_xadj + v0 + g;
        gr.adjncy = d_adj + e0;
        gr.adjwgt = d_adjwgt ? d_adjwgt + e0 : nullptr;
        gr.vwgt = d_vwgt ? d_vwgt + v0 * ncon : nullptr;
        if (k < 2 || k > n) return (int)METIS_ERROR_INPUT;
        if (validate_device(gr, W.arena(), W.stream(), W.host_scratch()) != 0) return (int)METIS_ERROR_INPUT;
        return W.partition_kway(gr, k, nullptr, ubvec, o, d_part + v0, obj_g, nullptr);
      });
    };
    // The pool's graphs first, largest first: they run on the workers'
    // streams while the batched launches run on this engine's stream.
    {
      std::vector<idx_t> rest;
      for (idx_t g = 0; g < ngraphs; ++g)
        if (!batched[g]) rest.push_back(g);
      std::stable_sort(rest.begin(), rest.end(), [&](idx_t x, idx_t y) {
        return edge_off[x + 1] - edge_off[x] > edge_off[y + 1] - edge_off[y];
      });
      for (idx_t g : rest) submit(g);
    }
    std::vector<BatchItem> items;
    std::vector<idx_t> which;
    for (idx_t g = 0; g < ngraphs; ++g) {
      if (!batched[g]) continue;
      const int64_t v0 = vtx_off[g], e0 = edge_off[g];
      BatchItem it;
      it.g.n = (int32_t)(vtx_off[g + 1] - v0);
      it.g.m = edge_off[g + 1] - e0;
      it.g.ncon = ncon;
      it.g.xadj = d_xadj + v0 + g;
      it.g.adjncy = d_adj + e0;
      it.g.adjwgt = d_adjwgt ? d_adjwgt + e0 : nullptr;
      it.g.vwgt = d_vwgt ? d_vwgt + v0 * ncon : nullptr;
      it.k = nparts[g];
      it.part_out = d_part + v0;
      items.push_back(it);
      which.push_back(g);
    }
    if (!items.empty()) {
      std::exception_ptr err;
      try {
        E.partition_kway_batch(items, ubvec, o);
      } catch (const Error& e) {
        if (e.code == METIS_ERROR_MEMORY) {
          for (BatchItem& it : items) it.status = 0;  // out of device memory: every graph alone
        } else {
          err = std::current_exception();
        }
      } catch (...) {
        err = std::current_exception();
      }
      if (err) {  // the pool's jobs read this call's buffers: let them finish first
        for (idx_t g = 0; g < ngraphs; ++g)
          if (submitted[g]) fut[g].wait();
        std::rethrow_exception(err);
      }
      for (size_t i = 0; i < items.size(); ++i) {
        const idx_t g = which[i];
        if (items[i].status == 0) {
          submit(g);  // the batched kernels could not finish it: alone
          continue;
        }
        done[g] = 1;
        status[g] = items[i].status;
        objval[g] = items[i].objval;
      }
    }
    int rc = METIS_OK;
    for (idx_t g = 0; g < ngraphs; ++g) {
      if (!done[g]) {
        status[g] = fut[g].get();
        objval[g] = objs[g];
      }
      if (status[g] != METIS_OK && rc == METIS_OK) rc = status[g];
    }
    download(E, part, d_part, (size_t)ntot);
    RMB_CUDA(cudaStreamSynchronize(E.stream()));
    return rc;
  });
}

namespace {

// ---- continuous batching of small requests --------------------------------
// A request of RMETIS_GPU_SubmitKway that the batched kernels can take goes to
// the device's dispatcher instead of the worker pool: a thread that, whenever
// it is idle, takes every request queued meanwhile and runs them as one batch
// (Engine::partition_kway_batch on its own engine and stream), grouped by
// options (all but the seed), ncon and ubvec. Requests that arrive while a
// batch runs form the next one, so batches grow with the load. Large requests
// keep running on the pool at the same time.
struct BatchReq {
  int32_t n = 0, nc = 1, np = 2;
  int64_t ne = 0;
  const idx_t* xadj = nullptr;
  const idx_t* adjncy = nullptr;
  const idx_t* vwgt = nullptr;
  const idx_t* adjwgt = nullptr;
  idx_t* objval = nullptr;
  idx_t* part = nullptr;
  KwayOptions o;
  std::vector<real_t> ub;
  std::promise<int> prom;
  bool done = false;
  void finish(int rc) {
    if (!done) {
      done = true;
      prom.set_value(rc);
    }
  }
};

std::vector<long long> group_key(const BatchReq& r) {
  const KwayOptions& o = r.o;
  std::vector<long long> k = {r.nc, o.ctype, o.iptype, o.rtype, o.niter, o.ncuts, (long long)o.ufactor,
                              o.grow_trials, o.match_rounds, o.summed_unit_weights, o.fused_max_n, o.tail_max_n,
                              o.exact_max_n, o.contract_thread_max, o.gain_block, o.fused_edge_factor,
                              o.fm_fused_max_n, (long long)r.ub.size()};
  for (real_t u : r.ub) {
    uint32_t bits;
    std::memcpy(&bits, &u, sizeof(bits));
    k.push_back(bits);
  }
  return k;
}

class Dispatcher {
 public:
  explicit Dispatcher(int dev) : dev_(dev) { th_ = std::thread([this] { run(); }); }
  std::future<int> submit(std::unique_ptr<BatchReq> r) {
    std::future<int> f = r->prom.get_future();
    {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(std::move(r));
    }
    cv_.notify_one();
    return f;
  }

 private:
  void run() {
    cudaSetDevice(dev_);
    Engine E(true);
    for (;;) {
      std::vector<std::unique_ptr<BatchReq>> take;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !q_.empty(); });
        take.swap(q_);
      }
      std::map<std::vector<long long>, std::vector<BatchReq*>> groups;
      for (auto& r : take) groups[group_key(*r)].push_back(r.get());
      for (auto& kv : groups) run_group(E, kv.second);
      for (auto& r : take) r->finish(METIS_ERROR);  // (every request is finished above)
    }
  }

  static void run_group(Engine& E, std::vector<BatchReq*>& grp) {
    Arena::Mark mk = E.arena().mark();
    try {
      std::vector<BatchItem> items(grp.size());
      for (size_t i = 0; i < grp.size(); ++i) {
        BatchReq& r = *grp[i];
        BatchItem& it = items[i];
        it.g.n = r.n;
        it.g.m = r.ne;
        it.g.ncon = r.nc;
        it.g.xadj = upload(E, r.xadj, (size_t)r.n + 1);
        it.g.adjncy = upload(E, r.adjncy, (size_t)r.ne);
        it.g.vwgt = upload(E, r.vwgt, (size_t)r.n * r.nc);
        it.g.adjwgt = upload(E, r.adjwgt, (size_t)r.ne);
        it.k = r.np;
        it.part_out = E.arena().alloc<idx_t>((size_t)r.n);
        it.seed = (int64_t)r.o.seed;
      }
      const BatchReq& r0 = *grp[0];
      bool batched = true;
      try {
        E.partition_kway_batch(items, r0.ub.empty() ? nullptr : r0.ub.data(), r0.o);
      } catch (const Error& e) {
        if (e.code != METIS_ERROR_MEMORY) throw;
        batched = false;  // out of device memory: one request at a time
      }
      for (size_t i = 0; i < grp.size(); ++i) {
        BatchReq& r = *grp[i];
        BatchItem& it = items[i];
        if (!batched || it.status == 0) {
          try {
            // (validated by the batch unless it never ran)
            if (!batched && validate_device(it.g, E.arena(), E.stream(), E.host_scratch()) != 0)
              throw Error(METIS_ERROR_INPUT, "graph failed validation");
            int32_t obj = 0;
            E.partition_kway(it.g, r.np, nullptr, r.ub.empty() ? nullptr : r.ub.data(), r.o, it.part_out, &obj,
                             nullptr);
            it.status = METIS_OK;
            it.objval = obj;
          } catch (const Error& e) {
            it.status = e.code;
          }
        }
        if (it.status == METIS_OK) download(E, r.part, it.part_out, (size_t)r.n);
      }
      RMB_CUDA(cudaStreamSynchronize(E.stream()));
      for (size_t i = 0; i < grp.size(); ++i) {
        if (items[i].status == METIS_OK && grp[i]->objval) *grp[i]->objval = items[i].objval;
        grp[i]->finish(items[i].status);
      }
    } catch (const Error& e) {
      cudaStreamSynchronize(E.stream());
      for (BatchReq* r : grp) r->finish(e.code);
    } catch (...) {
      cudaStreamSynchronize(E.stream());
      for (BatchReq* r : grp) r->finish(METIS_ERROR);
    }
    E.arena().reset_to(mk);
  }

  int dev_;
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<std::unique_ptr<BatchReq>> q_;
};

Dispatcher& dispatcher_for_device(int dev) {
  static std::mutex m;
  static std::vector<Dispatcher*> ds;
  std::lock_guard<std::mutex> lk(m);
  if ((int)ds.size() <= dev) ds.resize(dev + 1, nullptr);
  if (!ds[dev]) ds[dev] = new Dispatcher(dev);  // lives until process exit
  return *ds[dev];
}

}  // namespace

namespace {
struct Tickets {
  std::mutex mu;
  int64_t next = 1;
  std::map<int64_t, std::shared_future<int>> pending;
};
Tickets& tickets() {
  static Tickets t;
  return t;
}
}  // namespace

int64_t RMETIS_GPU_SubmitKway(const idx_t* nvtxs, const idx_t* ncon, const idx_t* xadj, const idx_t* adjncy,
                              const idx_t* vwgt, const idx_t* adjwgt, const idx_t* nparts, const real_t* tpwgts,
                              const real_t* ubvec, const idx_t* options, idx_t* objval, idx_t* part) {
  try {
    if (!nvtxs || !ncon || !xadj || !adjncy || !nparts || !part) return METIS_ERROR_INPUT;
    const int32_t n = *nvtxs, nc = *ncon, np = *nparts;
    if (n <= 0 || nc <= 0 || np < 2) return METIS_ERROR_INPUT;
    if (xadj[0] != 0 || xadj[n] < 0) return METIS_ERROR_INPUT;
    const int64_t ne = xadj[n];
    KwayOptions o = parse_options(options);
    apply_pool_tuning(o);
    // tpwgts and ubvec are copied now; the CSR arrays, part and objval are
    // read and written by the worker until the request completes.
    std::vector<real_t> tp, ub;
    if (tpwgts) tp.assign(tpwgts, tpwgts + (size_t)np * nc);
    if (ubvec) ub.assign(ubvec, ubvec + nc);
    int dev = 0;
    RMB_CUDA(cudaGetDevice(&dev));
    if (batch_mode() == 1 && !tpwgts && n <= batch_max_n() && batch_eligible(o, n, np, nc)) {
      auto r = std::make_unique<BatchReq>();
      r->n = n;
      r->nc = nc;
      r->np = np;
      r->ne = ne;
      r->xadj = xadj;
      r->adjncy = adjncy;
      r->vwgt = vwgt;
      r->adjwgt = adjwgt;
      r->objval = objval;
      r->part = part;
      r->o = o;
      r->ub = ub;
      std::shared_future<int> f = dispatcher_for_device(dev).submit(std::move(r)).share();
      std::lock_guard<std::mutex> lk(tickets().mu);
      const int64_t id = tickets().next++;
      tickets().pending.emplace(id, f);
      return id;
    }
    WorkerPool& pool = pool_for_device(dev);
    std::shared_future<int> f =
        pool.submit(footprint_bytes(n, ne, np, nc), [=](Engine& W) {
              Arena::Mark mk = W.arena().mark();
              idx_t* d_xadj = upload(W, xadj, (size_t)n + 1);
              idx_t* d_adj = upload(W, adjncy, (size_t)ne);
              idx_t* d_vwgt = upload(W, vwgt, (size_t)n * nc);
              idx_t* d_adjwgt = upload(W, adjwgt, (size_t)ne);
              idx_t* d_part = W.arena().alloc<idx_t>((size_t)n);
              const int rc = kway_common(W, n, nc, np, d_xadj, d_adj, ne, d_vwgt, d_adjwgt,
                                         tp.empty() ? nullptr : tp.data(), ub.empty() ? nullptr : ub.data(), nullptr,
                                         objval, d_part, nullptr, &o);
              download(W, part, d_part, (size_t)n);
              RMB_CUDA(cudaStreamSynchronize(W.stream()));
              W.arena().reset_to(mk);
              return rc;
            }).share();
    std::lock_guard<std::mutex> lk(tickets().mu);
    const int64_t id = tickets().next++;
    tickets().pending.emplace(id, f);
    return id;
  } catch (const rmb::Error& e) {
    return e.code;
  } catch (...) {
    return METIS_ERROR;
  }
}

int RMETIS_GPU_PollKway(int64_t ticket) {
  std::lock_guard<std::mutex> lk(tickets().mu);
  auto it = tickets().pending.find(ticket);
  if (it == tickets().pending.end()) return METIS_ERROR_INPUT;
  return it->second.wait_for(std::chrono::seconds(0)) == std::future_status::ready ? 1 : 0;
}

int RMETIS_GPU_WaitKway(int64_t ticket) {
  std::shared_future<int> f;
  {
    std::lock_guard<std::mutex> lk(tickets().mu);
    auto it = tickets().pending.find(ticket);
    if (it == tickets().pending.end()) return METIS_ERROR_INPUT;
    f = it->second;
    tickets().pending.erase(it);
  }
  return f.get();
}

int RMETIS_GPU_PartGraphKwayTrace(const idx_t* nvtxs, const idx_t* ncon, const idx_t* xadj, const idx_t* adjncy,
                                  const idx_t* vwgt, const idx_t* adjwgt, const idx_t* nparts,
                                  const real_t* tpwgts, const real_t* ubvec, const idx_t* options, idx_t* objval,
                                  idx_t* part, idx_t* matchings, int64_t matchings_cap, int64_t* level_off,
                                  int64_t level_off_cap, int64_t* nlevels, idx_t* grow_seeds, int64_t* stats) {
  return guarded([&] {
    KwayTrace tr;
    int rc = kway_host(nvtxs, ncon, xadj, adjncy, vwgt, adjwgt, nparts, tpwgts, ubvec, options, objval, part, &tr);
    if (rc != METIS_OK) return rc;
    const int64_t L = (int64_t)tr.matchings.size();
    if (level_off_cap < L + 1) return METIS_ERROR_MEMORY;
    int64_t off = 0;
    for (int64_t i = 0; i < L; ++i) {
      level_off[i] = off;
      const int64_t len = (int64_t)tr.matchings[i].size();
      if (off + len > matchings_cap) return METIS_ERROR_MEMORY;
      std::memcpy(matchings + off, tr.matchings[i].data(), sizeof(idx_t) * len);
      off += len;
    }
    level_off[L] = off;
    if (nlevels) *nlevels = L;
    if (grow_seeds && !tr.grow_seeds.empty())
      std::memcpy(grow_seeds, tr.grow_seeds.data(), sizeof(idx_t) * tr.grow_seeds.size());
    if (stats) {
      stats[0] = tr.refine_passes;
      stats[1] = tr.refine_moves;
      stats[2] = tr.decide_rounds;
    }
    return METIS_OK;
  });
}

int RMETIS_GPU_EdgeCut(idx_t n, const idx_t* xadj, const idx_t* adjncy, const idx_t* adjwgt, const idx_t* part,
                       idx_t* cut) {
  return guarded([&] {
    if (n <= 0 || !xadj || !adjncy || !part || !cut) return METIS_ERROR_INPUT;
    HostCall h;
    DGraph g = dgraph(h, n, 1, xadj, adjncy, nullptr, adjwgt);
    idx_t* d_part = upload(h.E, part, (size_t)n);
    unsigned long long* acc = h.E.arena().alloc<unsigned long long>(1);
    cut_and_weights(g, d_part, 1, acc, nullptr, h.st());
    unsigned long long v = 0;
    RMB_CUDA(cudaMemcpyAsync(h.E.host_scratch(), acc, sizeof(v), cudaMemcpyDeviceToHost, h.st()));
    h.sync();
    std::memcpy(&v, h.E.host_scratch(), sizeof(v));
    *cut = (idx_t)(uint32_t)v / 2;
    return METIS_OK;
  });
}

int RMETIS_GPU_PartitionWeights(idx_t n, idx_t ncon, const idx_t* vwgt, const idx_t* part, idx_t nparts,
                                idx_t* pw) {
  return guarded([&] {
    if (n <= 0 || ncon <= 0 || nparts <= 0 || !part || !pw) return METIS_ERROR_INPUT;
    HostCall h;
    DGraph g;
    g.n = n;
    g.ncon = ncon;
    g.vwgt = upload(h.E, vwgt, (size_t)n * ncon);
    idx_t* d_part = upload(h.E, part, (size_t)n);
    const size_t K = (size_t)nparts * ncon;
    long long* d_pw = h.E.arena().alloc<long long>(K);
    partition_weights_only(g, d_part, nparts, d_pw, h.st());
    std::vector<long long> tmp(K);
    download(h.E, tmp.data(), d_pw, K);
    h.sync();
    for (size_t i = 0; i < K; ++i) pw[i] = (idx_t)(uint32_t)(unsigned long long)tmp[i];
    return METIS_OK;
  });
}

int RMETIS_GPU_BuildCoarseGraph(idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                                const idx_t* adjwgt, const idx_t* match, idx_t* cn, idx_t* cmap, idx_t* cxadj,
                                idx_t* cadjncy, idx_t* cadjwgt, idx_t* cvwgt) {
  return guarded([&] {
    if (n <= 0 || ncon <= 0 || !xadj || !adjncy || !match || !cn || !cmap || !cxadj || !cadjncy || !cadjwgt)
      return METIS_ERROR_INPUT;
    check_range(match, n, n, "match out of range");
    for (idx_t v = 0; v < n; ++v)
      if (match[match[v]] != v) return METIS_ERROR_INPUT;  // must be an involution
    HostCall h;
    DGraph g = dgraph(h, n, ncon, xadj, adjncy, vwgt, adjwgt);
    idx_t* d_match = upload(h.E, match, (size_t)n);
    CoarseResult r = contract(g, d_match, vwgt ? 1 : 0, h.E.arena(), h.st(), h.E.host_scratch(),
                              tuning().contract_thread_max);
    *cn = r.g.n;
    download(h.E, cmap, r.cmap, (size_t)n);
    download(h.E, cxadj, r.xadj, (size_t)r.g.n + 1);
    download(h.E, cadjncy, r.adjncy, (size_t)r.g.m);
    download(h.E, cadjwgt, r.adjwgt, (size_t)r.g.m);
    if (vwgt && cvwgt) download(h.E, cvwgt, r.vwgt, (size_t)r.g.n * ncon);
    h.sync();
    return METIS_OK;
  });
}

int RMETIS_GPU_Project(idx_t n_fine, const idx_t* cmap, idx_t n_coarse, const idx_t* coarse_part,
                       idx_t* fine_part) {
  return guarded([&] {
    if (n_fine <= 0 || n_coarse <= 0 || !cmap || !coarse_part || !fine_part) return METIS_ERROR_INPUT;
    check_range(cmap, n_fine, n_coarse, "cmap out of range");
    HostCall h;
    idx_t* d_cmap = upload(h.E, cmap, (size_t)n_fine);
    idx_t* d_cp = upload(h.E, coarse_part, (size_t)n_coarse);
    idx_t* d_fp = h.E.arena().alloc<idx_t>((size_t)n_fine);
    project(n_fine, d_cmap, d_cp, d_fp, h.st());
    download(h.E, fine_part, d_fp, (size_t)n_fine);
    h.sync();
    return METIS_OK;
  });
}

int RMETIS_GPU_GainTable(idx_t n, const idx_t* xadj, const idx_t* adjncy, const idx_t* adjwgt, const idx_t* part,
                         idx_t nparts, idx_t* boundary, idx_t* ncand, idx_t* wfrom, idx_t* cand_part,
                         idx_t* cand_gain) {
  return guarded([&] {
    if (n <= 0 || nparts <= 0 || !xadj || !adjncy || !part || !boundary || !ncand || !wfrom || !cand_part ||
        !cand_gain)
      return METIS_ERROR_INPUT;
    check_range(part, n, nparts, "part out of range");
    HostCall h;
    DGraph g = dgraph(h, n, 1, xadj, adjncy, nullptr, adjwgt);
    idx_t* d_part = upload(h.E, part, (size_t)n);
    idx_t* d_b = h.E.arena().alloc<idx_t>((size_t)n);
    idx_t* d_nc = h.E.arena().alloc<idx_t>((size_t)n);
    idx_t* d_wf = h.E.arena().alloc<idx_t>((size_t)n);
    idx_t* d_cp = h.E.arena().alloc<idx_t>((size_t)g.m + 1);
    idx_t* d_cg = h.E.arena().alloc<idx_t>((size_t)g.m + 1);
    idx_t* d_heavy = h.E.arena().alloc<idx_t>((size_t)n);
    const int32_t nh = heavy_list(g, d_heavy, h.E.arena(), h.st(), h.E.host_scratch());
    RMB_CUDA(cudaMemsetAsync(d_nc, 0, sizeof(idx_t) * n, h.st()));
    RMB_CUDA(cudaMemsetAsync(d_wf, 0, sizeof(idx_t) * n, h.st()));
    gain_table(g, d_part, nparts, d_b, d_nc, d_wf, d_cp, d_cg, d_heavy, nh, h.st());
    download(h.E, boundary, d_b, (size_t)n);
    download(h.E, ncand, d_nc, (size_t)n);
    download(h.E, wfrom, d_wf, (size_t)n);
    download(h.E, cand_part, d_cp, (size_t)g.m);
    download(h.E, cand_gain, d_cg, (size_t)g.m);
    h.sync();
    return METIS_OK;
  });
}

int RMETIS_GPU_Match(idx_t n, const idx_t* xadj, const idx_t* adjncy, const idx_t* adjwgt, int mode, uint64_t seed,
                     int rounds, idx_t* match) {
  return guarded([&] {
    if (n <= 0 || !xadj || !adjncy || !match || rounds <= 0) return METIS_ERROR_INPUT;
    HostCall h;
    DGraph g = dgraph(h, n, 1, xadj, adjncy, nullptr, adjwgt);
    idx_t* d_heavy = h.E.arena().alloc<idx_t>((size_t)n);
    const int32_t nh = heavy_list(g, d_heavy, h.E.arena(), h.st(), h.E.host_scratch());
    idx_t* d_match = h.E.arena().alloc<idx_t>((size_t)n);
    match_parallel(g, mode ? 1 : 0, seed, rounds, d_match, d_heavy, nh, h.E.arena(), h.st(), h.E.host_scratch());
    download(h.E, match, d_match, (size_t)n);
    h.sync();
    return METIS_OK;
  });
}

int RMETIS_GPU_GrowPartition(idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                             const idx_t* adjwgt, idx_t nparts, const double* targets, idx_t ntrials,
                             const idx_t* seeds, idx_t* parts, int64_t* cuts) {
  return guarded([&] {
    if (n <= 0 || ncon <= 0 || nparts <= 0 || ntrials <= 0 || !xadj || !adjncy || !targets || !seeds || !parts)
      return METIS_ERROR_INPUT;
    check_range(seeds, (int64_t)ntrials * nparts, n, "seed out of range");
    for (idx_t t = 0; t < ntrials; ++t) {  // seeds of one trial are distinct (grow.rs:26-32)
      std::vector<char> used(n, 0);
      for (idx_t p = 0; p < nparts; ++p) {
        const idx_t sv = seeds[(int64_t)t * nparts + p];
        if (used[sv]) return METIS_ERROR_INPUT;
        used[sv] = 1;
      }
    }
    HostCall h;
    DGraph g = dgraph(h, n, ncon, xadj, adjncy, vwgt, adjwgt);
    const size_t K = (size_t)nparts * ncon;
    std::vector<long long> grow(K);
    for (size_t i = 0; i < K; ++i) {
      long long f, o;
      threshold_values(targets[i], 1.0, &f, &o, &grow[i]);
    }
    long long* d_grow = upload(h.E, grow.data(), K);
    idx_t* d_seeds = upload(h.E, seeds, (size_t)ntrials * nparts);
    idx_t* d_parts = h.E.arena().alloc<idx_t>((size_t)ntrials * n);
    long long* d_cuts = h.E.arena().alloc<long long>((size_t)ntrials);
    grow_trials(g, nparts, ntrials, d_seeds, d_grow, d_parts, d_cuts, h.E.arena(), h.st());
    download(h.E, parts, d_parts, (size_t)ntrials * n);
    std::vector<long long> c(ntrials);
    download(h.E, c.data(), d_cuts, (size_t)ntrials);
    h.sync();
    if (cuts)
      for (int i = 0; i < ntrials; ++i) cuts[i] = c[i];
    return METIS_OK;
  });
}

// The refinement of a host graph and partition by greedy_refine (fm 0),
// fm_refine (fm 1) or the 2-way fm2_refine (fm 2).
static int refine_entry(int fm, idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                        const idx_t* adjwgt, idx_t* part, idx_t nparts, const double* targets, const double* ubvec,
                        idx_t niter, idx_t* cut, int64_t* stats) {
  return guarded([&] {
    if (n <= 0 || ncon <= 0 || nparts <= 0 || niter < 0 || !xadj || !adjncy || !part || !targets || !ubvec)
      return METIS_ERROR_INPUT;
    check_range(part, n, nparts, "part out of range");
    HostCall h;
    DGraph g = dgraph(h, n, ncon, xadj, adjncy, vwgt, adjwgt);
    const size_t K = (size_t)nparts * ncon;
    std::vector<long long> feas(K), over(K), grow(K);
    for (int p = 0; p < nparts; ++p)
      for (int c = 0; c < ncon; ++c) {
        const size_t i = (size_t)p * ncon + c;
        threshold_values(targets[i], ubvec[c], &feas[i], &over[i], &grow[i]);
      }
    long long* d_feas = upload(h.E, feas.data(), K);
    long long* d_over = upload(h.E, over.data(), K);
    idx_t* d_part = upload(h.E, part, (size_t)n);
    idx_t* d_heavy = h.E.arena().alloc<idx_t>((size_t)n);
    const int32_t nh = heavy_list(g, d_heavy, h.E.arena(), h.st(), h.E.host_scratch());
    RefineParams rp;
    rp.k = nparts;
    rp.niter = niter;
    rp.feas_max = d_feas;
    rp.over_thr = d_over;
    rp.collect_stats = stats != nullptr;
    rp.fused_max_n = tuning().fused_max_n;
    rp.fm_fused_max_n = tuning().fm_fused_max_n;
    rp.fused_edge_factor = tuning().fused_edge_factor;
    rp.exact_max_n = tuning().exact_max_n;
    rp.gain_block = tuning().gain_block;
    {
      std::vector<long long> tot(ncon, 0);
      for (int64_t v = 0; v < n; ++v)
        for (int c = 0; c < ncon; ++c) tot[c] += vwgt ? vwgt[v * ncon + c] : 1;
      rp.small_weights = weights_fit_int32(tot.data(), ncon, feas.data(), over.data(), K);
    }
    RefineStats rs = fm == 2   ? fm2_refine(g, d_part, rp, h.E.arena(), h.st(), h.E.host_scratch())
                     : fm == 1 ? fm_refine(g, d_part, rp, d_heavy, nh, h.E.arena(), h.st(), h.E.host_scratch())
                               : greedy_refine(g, d_part, rp, d_heavy, nh, h.E.arena(), h.st(), h.E.host_scratch());
    unsigned long long* acc = h.E.arena().alloc<unsigned long long>(1);
    cut_and_weights(g, d_part, nparts, acc, nullptr, h.st());
    download(h.E, part, d_part, (size_t)n);
    unsigned long long v = 0;
    RMB_CUDA(cudaMemcpyAsync(h.E.host_scratch(), acc, sizeof(v), cudaMemcpyDeviceToHost, h.st()));
    h.sync();
    std::memcpy(&v, h.E.host_scratch(), sizeof(v));
    if (cut) *cut = (idx_t)(uint32_t)v / 2;
    if (stats) {
      stats[0] = rs.passes;
      stats[1] = rs.moves;
      stats[2] = rs.decide_iters;
      stats[3] = rs.movers;
    }
    return METIS_OK;
  });
}

int RMETIS_GPU_GreedyRefine(idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                            const idx_t* adjwgt, idx_t* part, idx_t nparts, const double* targets,
                            const double* ubvec, idx_t niter, idx_t* cut, int64_t* stats) {
  return refine_entry(0, n, ncon, xadj, adjncy, vwgt, adjwgt, part, nparts, targets, ubvec, niter, cut, stats);
}

int RMETIS_GPU_FmRefine(idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                        const idx_t* adjwgt, idx_t* part, idx_t nparts, const double* targets, const double* ubvec,
                        idx_t niter, idx_t* cut, int64_t* stats) {
  return refine_entry(1, n, ncon, xadj, adjncy, vwgt, adjwgt, part, nparts, targets, ubvec, niter, cut, stats);
}

int RMETIS_GPU_Fm2Refine(idx_t n, idx_t ncon, const idx_t* xadj, const idx_t* adjncy, const idx_t* vwgt,
                         const idx_t* adjwgt, idx_t* part, const double* targets, const double* ubvec, idx_t niter,
                         idx_t* cut, int64_t* stats) {
  return refine_entry(2, n, ncon, xadj, adjncy, vwgt, adjwgt, part, 2, targets, ubvec, niter, cut, stats);
}

}  // extern "C"
