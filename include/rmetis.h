/*
 * rmetis-b200: B200-native multilevel k-way partitioning behind the C ABI of
 * javagg/rmetis.
 *
 * Drop-in entry points (same names, argument meaning, ownership and return
 * codes as the reference's C ABI, src/ffi/c_api.rs):
 *   RMETIS_SetDefaultOptions   replaces src/ffi/c_api.rs:15-23
 *   RMETIS_PartGraphKway       replaces src/ffi/c_api.rs:56-81 (+ c_partition_impl :140-209,
 *                              parse_options :211-222)
 *   RMETIS_PartGraphRecursive  replaces src/ffi/c_api.rs:27-53 (same helpers)
 *   RMETIS_NodeND              replaces src/ffi/c_api.rs:84-132
 *
 * The k-way path computes on the GPU (CType Shem/Rm, IpType Grow/Random/MetisRb,
 * RType Greedy and Fm). Greedy is refined pass for pass as the reference does;
 * Fm (the reference's default, src/refine/fm_kway.rs) runs the same move rule
 * in parallel rounds, so its partitions match the reference's in quality
 * rather than bit for bit (RMETIS_GPU_FmRefine). Callers select Greedy with
 * options[METIS_OPTION_PTYPE] != -1 and options[METIS_OPTION_RTYPE] = 1,
 * exactly as the reference's from_raw (src/types.rs:190-224) decodes them.
 *
 * Everything after the drop-in section is additive: a device-pointer variant,
 * stream/tuning/profiling controls, and one entry point per reference function
 * of the hot path (used by the parity tests and available to users).
 *
 * Types follow the reference: idx_t = int32_t (src/types.rs:4), real_t = float
 * (src/types.rs:6). Return codes (src/types.rs:164-167): METIS_OK 1,
 * METIS_ERROR_INPUT -2, METIS_ERROR_MEMORY -3, METIS_ERROR -4.
 */
#ifndef RMETIS_B200_H
#define RMETIS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t idx_t;
typedef float real_t;

#if defined(__GNUC__)
#define RMETIS_API __attribute__((visibility("default")))
#else
#define RMETIS_API
#endif

#define METIS_OK 1
#define METIS_ERROR_INPUT (-2)
#define METIS_ERROR_MEMORY (-3)
#define METIS_ERROR (-4)

#define METIS_NOPTIONS 40
#define METIS_OPTION_PTYPE 0
#define METIS_OPTION_OBJTYPE 1
#define METIS_OPTION_CTYPE 2
#define METIS_OPTION_IPTYPE 3
#define METIS_OPTION_RTYPE 4
#define METIS_OPTION_DBGLVL 5
#define METIS_OPTION_NITER 6
#define METIS_OPTION_NCUTS 7
#define METIS_OPTION_SEED 8
#define METIS_OPTION_NO2HOP 9
#define METIS_OPTION_MINCONN 10
#define METIS_OPTION_CONTIG 11
#define METIS_OPTION_UFACTOR 16
#define METIS_OPTION_NUMBERING 17

/* ---- drop-in ---------------------------------------------------------- */

/* Fills options[0..40) with the reference's Options::default().to_raw()
 * (src/types.rs:77-95, :227-245). options[0] stays -1, which the partitioner
 * reads as "all defaults". NULL -> METIS_ERROR_INPUT. */
RMETIS_API int RMETIS_SetDefaultOptions(idx_t *options);

/* Multilevel k-way partition (src/ffi/c_api.rs:56-81). Host pointers.
 * Required: nvtxs, ncon, xadj[n+1], adjncy[xadj[n]], nparts, part[n].
 * Optional (NULL = default): vwgt[n*ncon] (unit), vsize (ignored, as in the
 * reference), adjwgt[xadj[n]] (unit), tpwgts[nparts*ncon] (1/nparts),
 * ubvec[ncon] (1 + ufactor/1000), options (defaults), objval (not written).
 * The caller owns all buffers; the library copies the inputs and writes only
 * part[0..n) and *objval. One difference from the reference, which has no
 * such limit: ncon above 8 returns METIS_ERROR_INPUT (the refinement kernels
 * hold at most 8 constraints per part). */
RMETIS_API int RMETIS_PartGraphKway(const idx_t *nvtxs, const idx_t *ncon, const idx_t *xadj, const idx_t *adjncy,
                         const idx_t *vwgt, const idx_t *vsize, const idx_t *adjwgt, const idx_t *nparts,
                         const real_t *tpwgts, const real_t *ubvec, const idx_t *options, idx_t *objval,
                         idx_t *part);

/* Multilevel recursive bisection (src/ffi/c_api.rs:27-53 with
 * src/partition/recursive.rs:12-187). Same arguments, ownership and return
 * codes as RMETIS_PartGraphKway; the options are decoded the same way, and the
 * reference's Options::for_recursive() (iptype MetisRb, rtype Fm, ufactor 1)
 * is what its callers pass. The recursion and the f32 target arithmetic
 * follow the reference on the host; the subgraphs stay on the device (the
 * input is uploaded once, both sides of every bisection are extracted there as
 * extract_subgraph does), each bisection is a 2-way multilevel partition on
 * the GPU (coarsening to 40 vertices, grow trials, refinement), and the
 * bisections of one recursion level run concurrently on the device's worker
 * pool. With rtype Fm every bisection is
 * refined by the reference's 2-way FM rule (src/refine/fm.rs: negative moves
 * and a rollback to the lowest cut) in parallel rounds (RMETIS_GPU_Fm2Refine).
 * Differences: the order of those moves, and the bisection at position h of the recursion tree (root 0,
 * children 2h+1, 2h+2) runs with seed + h where the reference draws all
 * bisections from one generator; partitions match the reference's in quality,
 * not bit for bit. Graphs with more than 8 constraints return
 * METIS_ERROR_INPUT (as RMETIS_PartGraphKway). */
RMETIS_API int RMETIS_PartGraphRecursive(const idx_t *nvtxs, const idx_t *ncon, const idx_t *xadj,
                                         const idx_t *adjncy, const idx_t *vwgt, const idx_t *vsize,
                                         const idx_t *adjwgt, const idx_t *nparts, const real_t *tpwgts,
                                         const real_t *ubvec, const idx_t *options, idx_t *objval, idx_t *part);

/* Nested dissection ordering (replaces src/ffi/c_api.rs:84-132, node_nd
 * src/partition/nd.rs:16-111, find_node_separator src/separator/mod.rs:10-61).
 * nvtxs, xadj, adjncy, perm and iperm are required (NULL or nvtxs <= 0 ->
 * METIS_ERROR_INPUT); vwgt[nvtxs] and options are optional; a graph failing
 * validation returns METIS_ERROR_INPUT. Writes perm[v] = new position of
 * vertex v and iperm = its inverse. A graph of more than 100 vertices is
 * bisected (targets 0.5/0.5, ubvec 1.05, the caller's options and seed), the
 * boundary of the lighter side becomes the separator, and the two sides are
 * ordered recursively (lighter side first) before the separator, as the
 * reference does. Each bisection is a 2-way multilevel partition on the GPU;
 * the bisections of one recursion level run concurrently on the device's
 * worker pool. The bisections differ from the reference's (parallel matching,
 * the 2-way FM moves in parallel rounds for rtype Fm), so orderings match it in quality
 * (separator sizes, fill), not bit for bit. */
RMETIS_API int RMETIS_NodeND(const idx_t *nvtxs, const idx_t *xadj, const idx_t *adjncy, const idx_t *vwgt,
                             const idx_t *options, idx_t *perm, idx_t *iperm);

/* ---- GPU extensions ---------------------------------------------------- */

/* Same contract as RMETIS_PartGraphKway, but xadj, adjncy, vwgt, adjwgt and part
 * are device pointers (current device). Scalars, tpwgts, ubvec, options and
 * objval stay on the host. No reference counterpart (additive). */
RMETIS_API int RMETIS_GPU_PartGraphKwayDevice(const idx_t *nvtxs, const idx_t *ncon, const idx_t *d_xadj,
                                   const idx_t *d_adjncy, const idx_t *d_vwgt, const idx_t *d_adjwgt,
                                   const idx_t *nparts, const real_t *tpwgts, const real_t *ubvec,
                                   const idx_t *options, idx_t *objval, idx_t *d_part);

/* Runs the engine of the current device on `stream` (a cudaStream_t; NULL =
 * the engine's own stream). */
RMETIS_API int RMETIS_GPU_SetStream(void *stream);

/* Engine knobs without a METIS option slot: grown partitions per attempt
 * (lowest cut kept), matching rounds per level, whether a graph without
 * vertex weights gets summed coarse weights (1) or the reference's unit coarse
 * weights (0, default), whether ncuts > 1 attempts run concurrently on the
 * device's worker pool (1, default) or one after another (0), the largest
 * level (vertices; its adjacency entries at most 4 times that) whose
 * refinement runs in one single-block launch (default 4096, 0 = never), and
 * the largest level (vertices; its adjacency entries at most 64 times that)
 * from which all remaining coarsening levels run in one single-block launch
 * (default 4096, 0 = never); the last three never change a result. Values
 * < 0 leave a knob unchanged. */
RMETIS_API int RMETIS_GPU_SetTuning(int grow_trials, int match_rounds, int summed_unit_weights,
                                    int parallel_attempts, int fused_max_n, int tail_max_n);

/* How greedy cut passes decide (no counterpart in the reference, whose pass
 * is sequential, src/refine/greedy.rs:126-190). Levels with at most
 * exact_max_n vertices (default 16384) decide every pass exactly as the
 * reference's sequential pass does; larger levels decide each cut pass by
 * parallel admission in one launch: every mover takes its best positive-gain
 * part that its move alone keeps feasible, and each part admits the longest
 * prefix (by vertex id) of its incoming moves that fits its limit given the
 * admitted moves out of it. Balance holds as in the reference (every part
 * that receives a move ends within floor(t*ub)); the decisions differ, so
 * results are compared by quality. -1 = exact everywhere. Returns
 * METIS_ERROR_INPUT for values below -1. */
RMETIS_API int RMETIS_GPU_SetRefineMode(int exact_max_n);

/* Kernel shapes that never change a result (no counterpart in the
 * reference): contract_thread_max (16 or 32) is the longest merged-row bound
 * a single thread merges in registers during contraction (longer rows go to
 * a warp each); gain_block (128, 256 or 512) is the block size of the
 * gain-table kernel. -1 leaves a knob unchanged; other values return
 * METIS_ERROR_INPUT. rmetis_b200/autotune.py measures them. */
RMETIS_API int RMETIS_GPU_SetKernelShapes(int contract_thread_max, int gain_block);

/* The last two knobs of RMETIS_GPU_SetTuning for jobs that share the device
 * with other jobs: the graphs of RMETIS_GPU_PartGraphKwayBatch and requests of
 * RMETIS_GPU_SubmitKway (no counterpart in the reference). A single-block
 * launch leaves most SMs idle in a lone call but not beside other jobs, so
 * the best sizes differ; rmetis_b200/autotune.py measures both. -1 = use the
 * RMETIS_GPU_SetTuning value (default); values < -1 leave a knob unchanged.
 * Neither knob changes a result. */
RMETIS_API int RMETIS_GPU_SetPoolTuning(int fused_max_n, int tail_max_n);

/* Many graphs in one call (no counterpart in the reference, which partitions
 * one graph per call). Host arrays of the concatenated batch: graph g has
 * n_g = vtx_off[g+1]-vtx_off[g] vertices and m_g = edge_off[g+1]-edge_off[g]
 * CSR entries; its xadj (n_g+1 local offsets) starts at xadj[vtx_off[g]+g],
 * its adjncy/adjwgt (local vertex ids) at edge_off[g], its vwgt at
 * vtx_off[g]*ncon, its part at part[vtx_off[g]]. nparts[g] per graph; ncon,
 * ubvec and options are shared. The batch is uploaded once. With Greedy
 * refinement (options[METIS_OPTION_RTYPE] = 1), ncuts 1, a grown initial
 * partition, ncon <= 2 and nparts[g] <= 256, graphs of up to 262144
 * vertices (RMETIS_GPU_SetBatchMode) go through the pipeline together: each
 * step (validation, coarsening, grow trials, the refinement of one level per
 * graph, the cut) is one launch over them, one thread block per graph; the
 * other graphs are partitioned concurrently on the device's worker pool. Either way each result equals the one of a
 * separate RMETIS_PartGraphKway call. status[g] gets each graph's return code;
 * the call returns METIS_OK or the first failing code. */
RMETIS_API int RMETIS_GPU_PartGraphKwayBatch(idx_t ngraphs, idx_t ncon, const int64_t *vtx_off,
                                             const int64_t *edge_off, const idx_t *xadj, const idx_t *adjncy,
                                             const idx_t *vwgt, const idx_t *adjwgt, const idx_t *nparts,
                                             const real_t *ubvec, const idx_t *options, idx_t *objval,
                                             idx_t *part, idx_t *status);

/* 1 (default): the matching rounds of a coarsening level run in one
 * cooperative launch, with grid-wide barriers between their phases and the
 * progress checks on the device; 0: one launch per phase and a host check
 * every other round (no counterpart in the reference). The same matching
 * either way; other values return METIS_ERROR_INPUT. */
RMETIS_API int RMETIS_GPU_SetCoopMatching(int on);

/* The edge bound of the single-block levels of RMETIS_GPU_SetTuning's
 * fused_max_n: a level runs all its passes in one launch when it has at most
 * fused_max_n vertices and factor * fused_max_n adjacency entries (default
 * factor 4; no counterpart in the reference). Never changes a result; -1
 * leaves it unchanged, 0 or other negative values return METIS_ERROR_INPUT. */
RMETIS_API int RMETIS_GPU_SetFusedEdgeFactor(int factor);

/* FM levels (rtype Fm) of at most max_n vertices (default 4096) run all their
 * passes and rounds in one single-block launch instead of about ten launches
 * per round (no counterpart in the reference); 0 = never, -1 leaves it
 * unchanged, other negative values return METIS_ERROR_INPUT. Never changes a
 * result. */
RMETIS_API int RMETIS_GPU_SetFmFusedMax(int max_n);

/* How RMETIS_GPU_PartGraphKwayBatch runs its graphs (no counterpart in the
 * reference; results are the same either way). mode 1 (default): eligible
 * graphs with at most max_n vertices (default 262144) go through the batched
 * launches, while the others run on the worker pool at the same time (a
 * large graph's levels take one thread block each in the batched launches,
 * so it finishes sooner on the pool's grid-wide kernels); mode 0: every graph
 * on the worker pool. -1 leaves a value unchanged; other negative values, or
 * a mode above 1, return METIS_ERROR_INPUT. */
RMETIS_API int RMETIS_GPU_SetBatchMode(int mode, int max_n);

/* Asynchronous requests for a serving loop (no counterpart in the reference).
 * Same arguments as RMETIS_PartGraphKway without vsize; returns a ticket > 0,
 * or a negative METIS error code. The request starts on the device's worker
 * pool once its estimated device-memory footprint fits in the pool's budget
 * next to the requests running; xadj, adjncy, vwgt, adjwgt, part and objval
 * must stay valid until RMETIS_GPU_WaitKway returns. Poll: 0 pending, 1 done
 * (the ticket stays valid). Wait: blocks, returns the request's code and
 * releases the ticket. */
RMETIS_API int64_t RMETIS_GPU_SubmitKway(const idx_t *nvtxs, const idx_t *ncon, const idx_t *xadj,
                                         const idx_t *adjncy, const idx_t *vwgt, const idx_t *adjwgt,
                                         const idx_t *nparts, const real_t *tpwgts, const real_t *ubvec,
                                         const idx_t *options, idx_t *objval, idx_t *part);
RMETIS_API int RMETIS_GPU_PollKway(int64_t ticket);
RMETIS_API int RMETIS_GPU_WaitKway(int64_t ticket);

/* Per-launch CUDA-event timing of the hot kernels (off by default).
 * RMETIS_GPU_GetProfile fills, per kernel id (0 gain, 1 decide, 2 propose,
 * 3 contract, 4 cut, 5 grow, 6 single-block level refinement, 7 single-block
 * coarse tail), launches[i], ms[i] (summed device time) and
 * bytes[i] (summed algorithmic bytes); returns the number of ids. With
 * max_ids above that number, launches[ids] receives the count of all kernel
 * launches made by this library in the process so far. */
RMETIS_API int RMETIS_GPU_SetProfiling(int on);
RMETIS_API int RMETIS_GPU_GetProfile(int64_t *launches, double *ms, double *bytes, int max_ids);

/* Like RMETIS_PartGraphKway, and also returns the random choices of the kept
 * attempt: the matching of every coarsening level (concatenated into
 * matchings, level offsets in level_off[0..nlevels]) and the nparts grow seeds.
 * matchings_cap / level_off_cap are the capacities of those arrays; a trace
 * that does not fit returns METIS_ERROR_MEMORY. stats (optional, 3 entries):
 * refinement passes, moves, decision rounds of the kept attempt. */
RMETIS_API int RMETIS_GPU_PartGraphKwayTrace(const idx_t *nvtxs, const idx_t *ncon, const idx_t *xadj, const idx_t *adjncy,
                                  const idx_t *vwgt, const idx_t *adjwgt, const idx_t *nparts,
                                  const real_t *tpwgts, const real_t *ubvec, const idx_t *options, idx_t *objval,
                                  idx_t *part, idx_t *matchings, int64_t matchings_cap, int64_t *level_off,
                                  int64_t level_off_cap, int64_t *nlevels, idx_t *grow_seeds, int64_t *stats);

/* ---- hot-path functions (host pointers; one call = upload, kernels, download) */

/* Graph::edge_cut (src/graph/mod.rs:123-137). adjwgt may be NULL. */
RMETIS_API int RMETIS_GPU_EdgeCut(idx_t n, const idx_t *xadj, const idx_t *adjncy, const idx_t *adjwgt, const idx_t *part,
                       idx_t *cut);

/* Graph::partition_weights (src/graph/mod.rs:140-149): pw[nparts*ncon]. */
RMETIS_API int RMETIS_GPU_PartitionWeights(idx_t n, idx_t ncon, const idx_t *vwgt, const idx_t *part, idx_t nparts,
                                idx_t *pw);

/* Graph::build_coarse_graph (src/graph/mod.rs:284-384) for a given matching
 * (an involution; match[v] == v means unmatched). Outputs cmap[n],
 * cxadj[n+1], cadjncy/cadjwgt[xadj[n]] capacity, cvwgt[n*ncon] (written when
 * vwgt != NULL), *cn. Coarse edge weights are always returned (1 where the
 * reference keeps no coarse adjwgt). */
RMETIS_API int RMETIS_GPU_BuildCoarseGraph(idx_t n, idx_t ncon, const idx_t *xadj, const idx_t *adjncy, const idx_t *vwgt,
                                const idx_t *adjwgt, const idx_t *match, idx_t *cn, idx_t *cmap, idx_t *cxadj,
                                idx_t *cadjncy, idx_t *cadjwgt, idx_t *cvwgt);

/* Projection fine[v] = coarse[cmap[v]] (src/partition/kway.rs:81-84). */
RMETIS_API int RMETIS_GPU_Project(idx_t n_fine, const idx_t *cmap, idx_t n_coarse, const idx_t *coarse_part,
                       idx_t *fine_part);

/* Gain table of a partition (boundary_vertices src/graph/mod.rs:164-171 and
 * compute_move_gain src/refine/greedy.rs:197-218): boundary[n] flags,
 * wfrom[n], ncand[n] and, at cand_part/cand_gain[xadj[v]..], the parts with
 * nonzero connection weight sorted by (gain desc, part asc). For any other
 * part p != part[v], gain(v, p) = -wfrom[v]. */
RMETIS_API int RMETIS_GPU_GainTable(idx_t n, const idx_t *xadj, const idx_t *adjncy, const idx_t *adjwgt, const idx_t *part,
                         idx_t nparts, idx_t *boundary, idx_t *ncand, idx_t *wfrom, idx_t *cand_part,
                         idx_t *cand_gain);

/* Parallel matching replacing shem_matching / random_matching
 * (src/coarsen/shem.rs:13-56, src/coarsen/rm.rs:13-43): mode 1 = heavy
 * edge, 0 = random. match[n] is an involution. */
RMETIS_API int RMETIS_GPU_Match(idx_t n, const idx_t *xadj, const idx_t *adjncy, const idx_t *adjwgt, int mode, uint64_t seed,
                     int rounds, idx_t *match);

/* grow_partition (src/initial/grow.rs:12-103) for ntrials seed sets
 * seeds[ntrials*nparts]; targets[nparts*ncon] are the f64 targets the
 * reference passes in (compute_target_weights). parts[ntrials*n], cuts[ntrials]
 * (sum over both directions). */
RMETIS_API int RMETIS_GPU_GrowPartition(idx_t n, idx_t ncon, const idx_t *xadj, const idx_t *adjncy, const idx_t *vwgt,
                             const idx_t *adjwgt, idx_t nparts, const double *targets, idx_t ntrials,
                             const idx_t *seeds, idx_t *parts, int64_t *cuts);

/* greedy_refine (src/refine/greedy.rs:12-22, :36-193): part updated in place;
 * targets[nparts*ncon] and ubvec[ncon] in f64 as the reference passes them.
 * *cut receives the edge cut afterwards; stats (optional, 4 entries): passes,
 * moves, decision rounds, movers. Every pass is the reference's sequential
 * pass bit for bit, except the cut passes of a graph with more vertices than
 * the RMETIS_GPU_SetRefineMode threshold (default 16384), which decide by
 * parallel admission. */
RMETIS_API int RMETIS_GPU_GreedyRefine(idx_t n, idx_t ncon, const idx_t *xadj, const idx_t *adjncy, const idx_t *vwgt,
                            const idx_t *adjwgt, idx_t *part, idx_t nparts, const double *targets,
                            const double *ubvec, idx_t niter, idx_t *cut, int64_t *stats);

/* fm_kway_refine (src/refine/fm_kway.rs:12-158, selected through
 * refine_kway src/refine/mod.rs:26-38): up to niter passes of positive-gain
 * moves to each vertex's best adjacent part, every target feasible
 * ((pw+vw) as f64 <= target*ub), moved vertices locked for the pass; stops
 * after a pass without a move. Same arguments as RMETIS_GPU_GreedyRefine;
 * stats (optional, 4 entries): passes, moves, rounds with movers, movers.
 * The cut never rises and ends at a fixed point of the reference's move rule;
 * the order of the moves differs from the reference's queue, so partitions
 * match it in quality, not bit for bit. */
RMETIS_API int RMETIS_GPU_FmRefine(idx_t n, idx_t ncon, const idx_t *xadj, const idx_t *adjncy, const idx_t *vwgt,
                                   const idx_t *adjwgt, idx_t *part, idx_t nparts, const double *targets,
                                   const double *ubvec, idx_t niter, idx_t *cut, int64_t *stats);

/* fm_refine (src/refine/fm.rs:12-127) of a bisection: the refinement that
 * RMETIS_PartGraphRecursive applies to every bisection with rtype Fm
 * (refine_2way, src/partition/recursive.rs:184-186). A pass moves free
 * boundary vertices to the other side, negative gains included, each move
 * feasible ((pw+vw) as f64 <= target*ub), moved vertices locked for the pass,
 * then undoes the moves after the lowest cut of the pass; passes repeat while
 * one improves (at most niter). Here a pass moves rounds of non-adjacent
 * local-maximum vertices and rolls back to the best round, so results match
 * the reference in quality, not bit for bit. targets: [2][ncon]; stats
 * (optional, 4 entries): passes, moves kept, rounds, selected movers. The cut
 * never rises; each side ends at most at max(its start weight,
 * floor(target*ub)). */
RMETIS_API int RMETIS_GPU_Fm2Refine(idx_t n, idx_t ncon, const idx_t *xadj, const idx_t *adjncy, const idx_t *vwgt,
                                    const idx_t *adjwgt, idx_t *part, const double *targets, const double *ubvec,
                                    idx_t niter, idx_t *cut, int64_t *stats);

/* Edge cut and partition weights of a device-resident graph without any
 * allocation, for callers that cannot allocate device memory at the point of
 * the call (a host that gives the library a fixed memory budget or its own
 * pool and forbids it to grow, or a loop where cudaMalloc/cudaFree would
 * synchronise the device). No counterpart in the reference: it is an additive
 * variant of RMETIS_GPU_EdgeCut plus RMETIS_GPU_PartitionWeights.
 * Inputs and outputs are device pointers on the current device: d_xadj[n+1],
 * d_adjncy/d_adjwgt[nnz] (d_adjwgt and d_vwgt may be NULL for unit weights),
 * d_part[n]; outputs *d_cut and d_pw[nparts*ncon]. The work is queued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and the call returns
 * without waiting; outputs are ready once that stream has reached them.
 * Scratch is a fixed array in device memory of the library (about 128 KiB per
 * GPU, kept until exit): nparts*ncon above 16384 returns METIS_ERROR_INPUT with
 * a message on stderr. The first call on a device looks up that array's device
 * address, so make that first call before any stream capture. All calls share
 * the array and each clears it first: calls that overlap on the GPU race and
 * must be serialised by the caller. Out-of-range indices (in d_part, d_xadj or
 * d_adjncy) are skipped and make *d_cut = -1; d_pw is then meaningless. A
 * valid graph whose cut sum wraps to -1 in 32 bits (as the reference's i32 sum
 * can) gives the same -1, so a caller that can meet such sums should check its
 * inputs itself. */
RMETIS_API int RMETIS_GPU_EdgeCutWeightsNoAlloc(idx_t n, idx_t ncon, int64_t nnz, const idx_t *d_xadj,
                                                const idx_t *d_adjncy, const idx_t *d_adjwgt, const idx_t *d_vwgt,
                                                const idx_t *d_part, idx_t nparts, idx_t *d_cut, idx_t *d_pw,
                                                void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RMETIS_B200_H */
