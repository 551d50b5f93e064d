// Host orchestration of the multilevel k-way pipeline on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <functional>
#include <future>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "arena.h"
#include "kernels.h"

namespace rmb {

// Decoded options of the reference (src/types.rs:52-95, from_raw :190-224)
// plus engine knobs that have no slot in the METIS option array.
struct KwayOptions {
  int ctype = 1;    // 0 = Rm, 1 = Shem
  int iptype = 0;   // 0 = Grow, 1 = Random, 4 = MetisRb (grown like Grow)
  int rtype = 0;    // 0 = Fm, 1 = Greedy
  int niter = 10;
  int ncuts = 1;
  uint64_t seed = 0;
  uint32_t ufactor = 30;
  // engine knobs
  int grow_trials = 32;       // grown partitions per attempt; the lowest cut is kept
  int match_rounds = 24;     // proposal rounds per coarsening level (upper bound)
  int summed_unit_weights = 0;  // 1: a graph without vwgt gets summed coarse weights
  int parallel_attempts = 1;    // 1: ncuts > 1 attempts run concurrently on the worker pool
  int fused_max_n = 4096;       // levels up to this size (and 4x its edges) refine in one launch
  int tail_max_n = 4096;        // from a level of at most this size, coarsening runs in one launch
  int exact_max_n = 16384;      // larger levels decide cut passes by parallel admission
  int contract_thread_max = 32; // coarse rows with a longer bound are merged by a warp (16 or 32)
  int gain_block = 256;         // threads per block of the gain-table kernel
  int fused_edge_factor = 4;    // ... with at most this many entries per vertex of fused_max_n
  int fm_fused_max_n = 4096;    // FM levels up to this size refine in one launch
  int bisect_fm2 = 0;           // 1: a 2-way partition with rtype Fm refines with the 2-way FM of fm.rs
};

// Per-kernel-family device time, measured with CUDA events on the engine's
// stream when profiling is on.
struct KernelStat {
  int64_t launches = 0;
  double ms = 0.0;
  double bytes = 0.0;  // algorithmic bytes (counted per launch from sizes)
};
enum StatId { kStatMatch = 0, kStatContract, kStatGrow, kStatRefine, kStatProject, kStatCut, kStatCount };

// Optional record of the random choices of the kept attempt, so that a
// checker can replay them.
struct KwayTrace {
  std::vector<std::vector<int32_t>> matchings;
  std::vector<int32_t> grow_seeds;
  std::vector<int64_t> level_n, level_m;
  int64_t refine_passes = 0, refine_moves = 0, decide_rounds = 0;
};

// One graph of a batched call: a device-resident graph, its part count and
// its output (part_out on the device); objval and status are filled in.
struct BatchItem {
  DGraph g;
  int k = 2;
  idx_t* part_out = nullptr;
  int64_t seed = -1;  // >= 0: this item's options seed instead of the shared one
  int32_t objval = 0;
  int status = 0;
};

// Whether the batched kernels can run a graph with these options: Greedy
// refinement, one attempt, grown initial partitions, ncon <= 2,
// 2 <= k <= min(n, 256).
bool batch_eligible(const KwayOptions& o, int32_t n, int k, int ncon);

class Engine {
 public:
  // A worker engine (one per pool thread) never hands work to the pool.
  explicit Engine(bool is_worker = false);
  ~Engine();

  // The whole k-way partition of a device-resident graph. part_out is a
  // device array of g.n entries. tpwgts/ubvec are host arrays (or null).
  // Returns 1 (METIS_OK) or throws rmb::Error.
  int partition_kway(const DGraph& g, int nparts, const float* tpwgts, const float* ubvec, const KwayOptions& o,
                     idx_t* part_out, int32_t* objval, KwayTrace* trace);

  // One attempt (kway.rs:62-98) with seed seed64: coarsen, grow, refine and
  // project; writes the partition to part_out (device, g.n) and its cut to
  // *objval. g must be complete before this engine's stream reads it.
  void run_attempt(const DGraph& g, int k, const float* tpwgts, const std::vector<double>& ub,
                   const std::vector<int32_t>& total0, const KwayOptions& o, uint64_t seed64, idx_t* part_out,
                   int32_t* objval, KwayTrace* trace);

  // Every graph of a batch through the pipeline in a handful of launches,
  // one block per graph and step (batch.cu). Each item's result equals the
  // single call partition_kway(item.g, item.k, nullptr, ubvec, o, ...).
  // Items must be eligible (batch_eligible); an item the batched kernels could
  // not finish (a coarsening deeper than the level table) is left with
  // status 0 for the caller to run alone. status: 1 done, -2 invalid graph.
  void partition_kway_batch(std::vector<BatchItem>& items, const float* ubvec, const KwayOptions& o);

  void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
  cudaStream_t stream() const { return stream_; }
  Arena& arena() { return arena_; }
  int32_t* host_scratch() { return h_scratch_; }

  void set_profiling(bool on) { profiling_ = on; }
  void reset_stats();
  const KernelStat* stats() const { return stats_; }

  std::mutex mu;

 private:
  // Thresholds of every level at once: totals[l] per level, written to
  // d_thr[l][3][k*ncon] (feas, over, grow) with a single upload.
  void thresholds(const std::vector<std::vector<int32_t>>& totals, int k, int ncon, const float* tpwgts,
                  const std::vector<double>& ub, long long* d_thr);

  struct Timer;
  Arena arena_;
  bool is_worker_ = false;
  int device_ = 0;
  cudaStream_t own_stream_ = nullptr;
  cudaStream_t stream_ = nullptr;
  int32_t* h_scratch_ = nullptr;   // pinned
  TailOut* h_tail_ = nullptr;      // pinned level table of the coarse-tail kernel
  long long* h_thr_ = nullptr;     // pinned staging for thresholds
  size_t h_thr_cap_ = 0;
  bool profiling_ = false;
  KernelStat stats_[kStatCount];
};

// One engine per device, created on first use.
Engine& engine_for_current_device();

// Device memory one partition of a graph of n vertices, m CSR entries, k
// parts and ncon constraints may hold at once (input, hierarchy, refinement
// and grow scratch), rounded up: the admission estimate of the pool.
size_t footprint_bytes(int64_t n, int64_t m, int k, int ncon);

// Worker threads on one device, each with its own Engine (stream, workspace,
// pinned staging), running submitted jobs concurrently. Jobs start in
// submission order when their footprint fits in the budget next to the jobs
// running (a job larger than the whole budget runs alone). A job's return
// value (or the code of the rmb::Error it throws) completes its future; the
// worker's workspace is rewound after every job. The footprint is an
// estimate: a job that runs out of device memory next to others is retried
// once alone, after every worker has freed the workspace it keeps between
// jobs (so jobs must be safe to run again).
class WorkerPool {
 public:
  WorkerPool(int device, int nworkers, size_t budget_bytes);
  ~WorkerPool();
  std::future<int> submit(size_t footprint, std::function<int(Engine&)> fn);
  int workers() const { return (int)threads_.size(); }
  size_t budget() const { return budget_; }
  void set_budget(size_t b);

 private:
  struct Job {
    size_t footprint;
    std::function<int(Engine&)> fn;
    std::promise<int> prom;
    bool alone = false;  // retry after running out of memory: nothing else runs
  };
  void worker_main(int idx);
  int device_;
  std::vector<std::thread> threads_;
  std::deque<std::unique_ptr<Job>> queue_;
  std::mutex mu_;
  std::condition_variable cv_;
  size_t budget_;
  size_t in_use_ = 0;
  int running_ = 0;
  bool stop_ = false;
  unsigned trim_epoch_ = 0;  // bumped when a job ran out of memory: workers free their workspace
  std::vector<unsigned> worker_epoch_;  // the last epoch each worker has freed its workspace for
};

// The pool of a device, created on first use: RMETIS_B200_WORKERS threads
// (default 8) and a budget of RMETIS_B200_POOL_BYTES (default 150 GB).
WorkerPool& pool_for_device(int device);

// Debug invariant checks (checks.cu; on when RMETIS_B200_CHECKS is set): a
// violation throws Error(-4) naming the invariant.
bool checks_enabled();
void check_contraction(const DGraph& fine, const DGraph& coarse, const idx_t* cmap, Arena& arena, cudaStream_t st,
                       int32_t* h_scratch);
void check_refined(const DGraph& g, const idx_t* part, int k, Arena& arena, cudaStream_t st, int32_t* h_scratch);
// Per-level trace: one JSON line per attempt appended to the file named by
// RMETIS_B200_TRACE_JSON (null: tracing off).
const char* trace_json_path();
void trace_json_write(const std::string& line);

// Host-side threshold form of the reference's f64 tests:
//   feasible   (pw + vw) as f64 <= t * ub   <=>  pw + vw <= feas
//   overweight  pw as f64 > t * ub          <=>  pw > over
//   at target   pw as f64 >= t              <=>  pw >= grow
void threshold_values(double t, double ub, long long* feas, long long* over, long long* grow);

}  // namespace rmb
