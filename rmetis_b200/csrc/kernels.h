// Launchers for the sm_100a kernels of the k-way hot path. Each launcher
// names the reference function it replaces.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>

#include "arena.h"
#include "common.cuh"

namespace rmb {

// Device view of one CSR level. adjwgt == nullptr means unit edge weights,
// vwgt == nullptr means unit vertex weights (the reference's `None`).
struct DGraph {
  int32_t n = 0;
  int64_t m = 0;
  int32_t ncon = 1;
  const idx_t* xadj = nullptr;
  const idx_t* adjncy = nullptr;
  const idx_t* adjwgt = nullptr;
  const idx_t* vwgt = nullptr;
};

// Vertices whose degree exceeds this go to the warp-per-vertex paths.
constexpr int kHeavyDegree = 64;
// Coarse vertices whose merged row bound exceeds this use the warp merge.
constexpr int kContractThreadMax = 16;
// The same bound in the grid-wide contraction kernel, whose threads have more
// registers to spare than those of the 1024-thread coarse-tail block.
constexpr int kContractThreadMaxGrid = 32;
// Movers per block in the refinement decision kernel.
constexpr int kDecideBlock = 256;

// ---- graph_kernels.cu ----------------------------------------------------
// Validation of a device CSR (src/graph/validate.rs:16-142). Returns a bit
// mask of failed checks (0 = valid). Requires xadj[0]==0 and xadj[n]==m,
// checked by the caller on the host.
int validate_device(const DGraph& g, Arena& arena, cudaStream_t st, int32_t* h_scratch);

// edge_cut (src/graph/mod.rs:123-137) and partition_weights (:140-149) in one
// pass. Results stay on the device: cut_acc (u64, sum of cross weights taken
// mod 2^32 later), pw (i64 [k][ncon]). Both are zeroed here.
void cut_and_weights(const DGraph& g, const idx_t* part, int k, unsigned long long* cut_acc,
                     long long* pw, cudaStream_t st);
void partition_weights_only(const DGraph& g, const idx_t* part, int k, long long* pw, cudaStream_t st);
// Edge cuts (both directions) of ntrials partitions parts[trial][g.n].
void trial_cuts(const DGraph& g, const idx_t* parts, int ntrials, long long* cuts, cudaStream_t st);

// total_weight (src/graph/mod.rs:152-160): i64 sums per constraint (zeroed here).
void total_weight(const DGraph& g, long long* tot, cudaStream_t st);

// Projection fine[v] = coarse[cmap[v]] (src/partition/kway.rs:81-84).
void project(int32_t n_fine, const idx_t* cmap, const idx_t* coarse_part, idx_t* fine_part,
             cudaStream_t st);

// boundary flags (src/graph/mod.rs:164-171): flag[v] = 1 if v has a
// neighbour in another part.
void boundary_flags(const DGraph& g, const idx_t* part, idx_t* flag, cudaStream_t st);

// Compact the ids v with flag[v] != 0 into out (ascending). count_dev gets
// the number written.
void compact_flags(const idx_t* flag, int32_t n, idx_t* out, idx_t* count_dev, Arena& arena,
                   cudaStream_t st);

// ---- coarsen.cu ----------------------------------------------------------
// Parallel matching (replaces shem_matching src/coarsen/shem.rs:13-56 and
// random_matching src/coarsen/rm.rs:13-43). mode 1 = heavy edge first
// (SHEM), 0 = random (RM). match[v] is an involution, self = unmatched.
// heavy/nheavy: precomputed list of vertices with degree > kHeavyDegree.
// coop: the rounds may run in one cooperative launch (coop_matching()).
void match_parallel(const DGraph& g, int mode, uint64_t seed, int rounds, idx_t* match,
                    const idx_t* heavy, int32_t nheavy, Arena& arena, cudaStream_t st,
                    int32_t* h_scratch, bool coop = true);

struct CoarseResult {
  DGraph g;
  idx_t* cmap = nullptr;
  idx_t* xadj = nullptr;
  idx_t* adjncy = nullptr;
  idx_t* adjwgt = nullptr;
  idx_t* vwgt = nullptr;
};

// build_coarse_graph (src/graph/mod.rs:284-384): cmap numbering by ascending
// leader, merged rows in first-appearance order with summed weights.
// coarse_vwgt: 0 = coarse graph has no vwgt (reference rule when the fine
// graph has none), 1 = sum (materialising 1 for a unit fine graph).
CoarseResult contract(const DGraph& g, const idx_t* match, int coarse_vwgt, Arena& arena,
                      cudaStream_t st, int32_t* h_scratch, int thread_max = kContractThreadMaxGrid);

// Degree > kHeavyDegree vertex list of a level (ascending ids).
int32_t heavy_list(const DGraph& g, idx_t* out, Arena& arena, cudaStream_t st, int32_t* h_scratch);

// The level table written by the coarse-tail kernel: heavy lists (and the
// matching, null for a level that was not matched) of the levels it started
// from, in order, and the coarse levels it kept. finished = 1 when the stop
// rule ended coarsening; 0 when the workspace or the table ran out and the
// host loop goes on from the last kept level.
constexpr int kTailMaxLevels = 32;
struct TailOut {
  int32_t levels, ncoarse, finished, pad;
  long long heavy[kTailMaxLevels];
  int32_t nheavy[kTailMaxLevels];
  long long match[kTailMaxLevels];
  long long cmap[kTailMaxLevels], xadj[kTailMaxLevels], adj[kTailMaxLevels], adjw[kTailMaxLevels],
      vwgt[kTailMaxLevels];
  int32_t cn[kTailMaxLevels];
  long long cm[kTailMaxLevels];
  int32_t coarse_vw[kTailMaxLevels];
};

// 1 (default): the matching rounds of a level run in one cooperative launch
// (grid-wide barriers between phases); 0: one launch per phase. The same
// matching either way.
int& coop_matching();

// Arguments of one graph's coarsening in a single block (coarsen_tail and
// the batched form).
struct TailArgs {
  DGraph g;
  int has_vw, summed_unit, mode, lvl0, k, rounds;
  uint64_t seed64;
  long long limit;
  char* ws;           // workspace of tail_workspace_bytes(g, rounds), 256-byte aligned; TailOut at its start
  long long ws_bytes;
};

// Workspace bytes of one graph's single-block coarsening.
int64_t tail_workspace_bytes(const DGraph& g, int rounds);

// Every graph of a batch coarsened in one launch, one block per graph
// (d_args[order[b]] for block b); graphs with d_bad set are skipped. Each
// graph's level table is the TailOut at the start of its workspace.
void coarsen_tail_batch(const TailArgs* d_args, const int32_t* d_order, const int32_t* d_bad, int ngraphs,
                        cudaStream_t st);

// The coarsening loop of coarsen/mod.rs:36-71 from level lvl0 (graph g) on,
// in one single-block launch: per level the heavy list, match_parallel (same
// seeds, rounds and progress checks) and contract, then the stop rule (cn < k
// keeps the finer level; cn <= limit or cn/n > 0.95 stops). The levels are
// the ones the host loop would produce. has_vw: g carries vertex weights;
// summed_unit: coarse levels of a unit-weight graph get summed weights. The
// level data lives in a workspace taken from the arena; the table is copied
// to h_out (pinned) before return.
void coarsen_tail(const DGraph& g, int has_vw, int summed_unit, int mode, uint64_t seed64, int lvl0, int k,
                  int64_t limit, int rounds, Arena& arena, cudaStream_t st, TailOut* h_out);

// ---- initial.cu ----------------------------------------------------------
// grow_partition (src/initial/grow.rs:12-103), exact given the seed vertices:
// one warp per trial. seeds: [ntrials][k]; grow_tgt: [k][ncon] integer form of
// the `pw as f64 >= t` test (pw >= grow_tgt). parts: [ntrials][n]. cuts:
// [ntrials] edge cut of each grown partition.
void grow_trials(const DGraph& g, int k, int ntrials, const idx_t* seeds, const long long* grow_tgt,
                 idx_t* parts, long long* cuts, Arena& arena, cudaStream_t st);

// One coarsest graph's grow trials in the batched launch.
struct GrowJob {
  const idx_t* xadj;
  const idx_t* adjncy;
  const idx_t* adjwgt;
  const idx_t* vwgt;
  int32_t n, ncon, k, trials;
  const idx_t* seeds;         // [trials][k]
  const long long* grow_tgt;  // [k][ncon]
  idx_t* parts;               // [trials][n]
  long long* cuts;            // [trials] directed edge cut of each trial
  unsigned char* scratch;     // [trials][scratch_bytes] when use_smem is 0
  long long scratch_bytes;
  int32_t use_smem;
  int32_t first_block;        // the job's trials are blocks first_block ..
};

// Bytes of one grow trial's state (shared memory or global scratch).
size_t grow_scratch_bytes(int32_t n, int k, int ncon);

// Every grow trial of a batch in one launch (block b: job d_block_job[b]);
// dyn_smem covers the jobs with use_smem set.
void grow_trials_batch(const GrowJob* d_jobs, const int32_t* d_block_job, int nblocks, size_t dyn_smem,
                       cudaStream_t st);

// ---- batch.cu ------------------------------------------------------------
// One graph's validation in the batched launch (the checks of validate_device)
// and the total weight per constraint (64-bit sums).
struct ValJob {
  const idx_t* xadj;
  const idx_t* adjncy;
  const idx_t* vwgt;
  int32_t n, ncon;
  int32_t* degcheck;  // [n], zero on entry
  int32_t* flag;      // validate_device's bits, zero on entry
  long long* total;   // [ncon]
};

// ---- refine.cu -----------------------------------------------------------
struct RefineParams {
  int k = 2;
  int niter = 10;
  const long long* feas_max = nullptr;  // [k][ncon]: feasible iff pw + vw <= feas_max
  const long long* over_thr = nullptr;  // [k][ncon]: overweight iff pw > over_thr
  bool collect_stats = false;           // read the per-pass counts back (one sync)
  // Set when every part weight (|pw| <= total < 2^28) and every threshold
  // (|feas|, |over| < 2^29) is small: the walk may then keep 32-bit slacks.
  bool small_weights = false;
  // Levels with at most this many vertices and fused_edge_factor times as
  // many adjacency entries (and k <= 256, ncon <= 2) run all their passes in one
  // single-block launch (k_refine_level); 0 = never.
  int32_t fused_max_n = 0;
  // ... and at most this many adjacency entries per vertex of fused_max_n
  // (the edge bound is fused_edge_factor * fused_max_n).
  int32_t fused_edge_factor = 4;
  // FM levels with at most this many vertices (k <= 256, ncon <= 2, exact
  // walk) run all their passes and rounds in one single-block launch
  // (k_fm_level); 0 = never.
  int32_t fm_fused_max_n = 0;
  // Cut passes of levels with more vertices than this decide by parallel
  // admission (admit.cu) instead of the exact sequential walk.
  int32_t exact_max_n = INT32_MAX;
  // Threads per block of the gain-table kernel (128, 256 or 512; the same
  // table whatever the size).
  int gain_block = 256;
};

// True when the totals and thresholds allow 32-bit slacks in the walk.
inline bool weights_fit_int32(const long long* total, int ncon, const long long* feas, const long long* over,
                              size_t K) {
  for (int c = 0; c < ncon; ++c)
    if (total[c] < 0 || total[c] >= (1LL << 28)) return false;
  for (size_t i = 0; i < K; ++i) {
    const long long lim = 1LL << 29;
    if (feas[i] <= -lim || feas[i] >= lim || over[i] <= -lim || over[i] >= lim) return false;
  }
  return true;
}

struct RefineStats {
  int passes = 0;
  int64_t moves = 0;
  int decide_iters = 0;
  int64_t movers = 0;
};

// greedy_refine_with_comm with one rank (src/refine/greedy.rs:36-193):
// balance-repair pass, then up to niter positive-gain passes, every pass
// bit-identical to the sequential reference pass. part is updated in place.
RefineStats greedy_refine(const DGraph& g, idx_t* part, const RefineParams& rp, const idx_t* heavy,
                          int32_t nheavy, Arena& arena, cudaStream_t st, int32_t* h_scratch);

// fm_kway_refine (src/refine/fm_kway.rs:12-158): up to niter passes of
// positive-gain moves of local-maximum vertices in rounds, each move's target
// feasible, moved vertices locked for the pass; stops after a pass without a
// move. part is updated in place. Stats: passes, moves, rounds with movers,
// selected movers.
RefineStats fm_refine(const DGraph& g, idx_t* part, const RefineParams& rp, const idx_t* heavy, int32_t nheavy,
                      Arena& arena, cudaStream_t st, int32_t* h_scratch);

// fm_refine (src/refine/fm.rs:12-127) of a bisection (k = 2): passes of
// moves of free boundary vertices, negative gains included, then a rollback
// to the lowest cut of the pass; in rounds of non-adjacent local-maximum
// moves admitted by the parallel admission. Stats: passes, moves kept,
// rounds, selected movers.
RefineStats fm2_refine(const DGraph& g, idx_t* part, const RefineParams& rp, Arena& arena, cudaStream_t st,
                       int32_t* h_scratch);

// Gain table of one pass (boundary_vertices + compute_move_gain,
// src/graph/mod.rs:164-171, src/refine/greedy.rs:197-218): per vertex the
// boundary flag, w_from and the explicit candidate list sorted by
// (gain desc, part asc), stored at cand[xadj[v] ..].
void gain_table(const DGraph& g, const idx_t* part, int k, idx_t* boundary, idx_t* ncand,
                idx_t* wfrom, idx_t* cand_p, idx_t* cand_g, const idx_t* heavy, int32_t nheavy,
                cudaStream_t st);

// One graph's level in a step of the batched refinement (k_batch_level and,
// for an admission level, k_batch_admit). Scratch arrays are the graph's own,
// sized for its finest level.
struct LevelJob {
  const idx_t* xadj;
  const idx_t* adjncy;
  const idx_t* adjwgt;
  const idx_t* vwgt;
  int32_t n, ncon, k, niter;
  // start partition: the best grow trial (trial_parts set) or the projection
  // part[v] = cpart[cmap[v]] of the coarser level's
  const idx_t* trial_parts;
  const long long* trial_cuts;
  int32_t trials;
  int32_t admit;  // 1: cut passes by parallel admission (k_batch_admit), 0: exact walk
  const idx_t* cmap;
  const idx_t* cpart;
  idx_t* part;
  const long long* feas;
  const long long* over;
  const idx_t* heavy;
  int32_t nheavy;
  int32_t pad;
  long long* pw;
  long long* in_max;
  long long* out_max;
  idx_t* mover;
  idx_t* ncand;
  idx_t* wfrom;
  idx_t* cand_p;
  idx_t* cand_g;
  idx_t* movers;
  int32_t* rec_pv;
  int32_t* rec_ne;
  int32_t* rec_wf;
  int32_t* rec_coff;
  int32_t* rec_known;
  int32_t* rec_cp;
  int32_t* rec_cg;
  int32_t* rec_vw;
  int32_t* rec_np;
  int32_t* ghist;     // [32][k]
  int32_t* counters;  // [2 * (niter + 1)]
  int32_t* long_flag;
  int32_t* a_tgt;
  int32_t* a_src;
  int32_t* a_w;
  int32_t* a_rank;
  int32_t* a_gsrc;
  int32_t* a_cut;
  long long* a_pref;
  long long* a_out;   // [k][ncon], zero on entry
  idx_t* touched[2];
};

// Inline candidate slots of a mover record (the walk's record layout).
constexpr int kRecInline = 4;

// A step of the batched refinement over njobs levels of one kind (edge
// weights, 32-bit slacks, the k bucket of k, ncon 1 or 2): projection or
// best trial, part weights, repair pass and, unless the job's admit is set,
// the cut passes with the exact walk; one block (512 threads) per job.
void batch_level_launch(const LevelJob* d_jobs, int njobs, bool has_w, bool small_weights, int k, int ncon,
                        cudaStream_t st);

// The cut passes of admission levels, one block (1024 threads) per job:
// gain table (after the first pass only where the last pass moved), picks,
// admission fixed point and moves, as admit_cut_pass does with grid kernels.
void batch_admit_launch(const LevelJob* d_jobs, int njobs, bool has_w, cudaStream_t st);

// ---- admit.cu -----------------------------------------------------------
// Parallel admission of one greedy cut pass (src/refine/greedy.rs:126-190 in
// a parallel form): picks, stable grouping by target part and a monotone
// admission fixed point, all in one single-block launch. Scratch holds nm
// entries each (pref: nm * ncon).
constexpr size_t kAdmitMaxSmem = 200 * 1024;
struct AdmitScratch {
  int32_t* tgt = nullptr;      // [n] target of each mover (-1: none)
  int32_t* src = nullptr;      // [n] its part
  int32_t* w = nullptr;        // [n * ncon] its weights
  int32_t* rank = nullptr;     // [n] its place in its target's in-list
  long long* pref = nullptr;   // [n * ncon] running sums (when shared memory is short)
  int32_t* gsrc = nullptr;     // [n] sources in grouped order (same)
  long long* out = nullptr;    // [k * ncon] out-weights of a pass's picks: zero before the level's first pass
  int32_t* cut = nullptr;      // [k] admitted prefix per part
};
size_t admit_smem_bytes(int k, int ncon);
bool admit_supported(int k, int ncon);
// Returns the profiler handle of the pass. nmax bounds the movers (grid
// size); nmoves gets the moves admitted, rounds_out (optional) the admission
// rounds (negative: the bound was hit). With apply = false the part vector is
// left to the caller: mover j moves to s.tgt[j] when s.tgt[j] >= 0 and
// s.rank[j] < s.cut[s.tgt[j]]. With `touched` (n flags), the moved vertices
// and their neighbours are flagged there.
int admit_cut_pass(const DGraph& g, int k, int32_t nmax, const int32_t* nm_dev, const idx_t* movers,
                   const idx_t* ncand, const idx_t* wfrom, const idx_t* cand_p, const idx_t* cand_g, idx_t* part,
                   long long* pw, const long long* feas, int32_t* nmoves, int32_t* rounds_out,
                   const AdmitScratch& s, cudaStream_t st, bool apply = true, idx_t* touched = nullptr,
                   bool any_gain = false);

// Opts a kernel in to `bytes` of dynamic shared memory on the current device
// (once per kernel and device; safe from several host threads).
void allow_dyn_smem(const void* kernel, size_t bytes);

}  // namespace rmb
