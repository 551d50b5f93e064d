"""One GPU call per reference function of the k-way hot path.

Each wraps an entry point of include/rmetis.h and mirrors the reference
function's arguments: shem_matching/random_matching (src/coarsen/shem.rs:13,
rm.rs:13), grow_partition (src/initial/grow.rs:12), greedy_refine
(src/refine/greedy.rs:12-22), the projection of src/partition/kway.rs:81-84.
Graph-level ones (edge_cut, partition_weights, build_coarse_graph,
boundary_vertices) are methods of rmetis_b200.Graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import Graph, _i32, _p, _raise_for
from ._lib import F64P, I64P

SHEM = 1
RM = 0


def match(graph: Graph, mode: int = SHEM, seed: int = 1, rounds: int = 16) -> np.ndarray:
    """Parallel matching (an involution; match[v] == v means unmatched)."""
    out = np.zeros(graph.nvtxs, np.int32)
    rc = _lib.load().RMETIS_GPU_Match(graph.nvtxs, _p(graph.xadj), _p(graph.adjncy), _p(graph.adjwgt), int(mode),
                                      ctypes.c_uint64(seed), int(rounds), _p(out))
    _raise_for(rc, "match")
    return out


def project(cmap, coarse_part) -> np.ndarray:
    cmap = _i32(cmap)
    cp = _i32(coarse_part)
    out = np.zeros(len(cmap), np.int32)
    rc = _lib.load().RMETIS_GPU_Project(len(cmap), _p(cmap), len(cp), _p(cp), _p(out))
    _raise_for(rc, "project")
    return out


def grow_partition(graph: Graph, nparts: int, targets, seeds):
    """grow_partition for one or more seed sets (seeds: [ntrials, nparts]).
    Returns (parts [ntrials, n], cuts [ntrials])."""
    seeds = np.atleast_2d(_i32(seeds))
    ntr = seeds.shape[0]
    t = np.ascontiguousarray(targets, dtype=np.float64)
    parts = np.zeros((ntr, graph.nvtxs), np.int32)
    cuts = np.zeros(ntr, np.int64)
    rc = _lib.load().RMETIS_GPU_GrowPartition(graph.nvtxs, graph.ncon, _p(graph.xadj), _p(graph.adjncy),
                                              _p(graph.vwgt), _p(graph.adjwgt), nparts, _p(t, F64P), ntr,
                                              _p(np.ascontiguousarray(seeds)), _p(parts), _p(cuts, I64P))
    _raise_for(rc, "grow_partition")
    return parts, cuts


def greedy_refine(graph: Graph, part, nparts: int, targets, ubvec, niter: int = 10):
    """Returns (refined part, edge cut, stats[passes, moves, decision rounds, movers])."""
    part = np.array(part, dtype=np.int32)
    t = np.ascontiguousarray(targets, dtype=np.float64)
    ub = np.ascontiguousarray(ubvec, dtype=np.float64)
    cut = ctypes.c_int32(0)
    stats = np.zeros(4, np.int64)
    rc = _lib.load().RMETIS_GPU_GreedyRefine(graph.nvtxs, graph.ncon, _p(graph.xadj), _p(graph.adjncy),
                                             _p(graph.vwgt), _p(graph.adjwgt), _p(part), nparts, _p(t, F64P),
                                             _p(ub, F64P), niter, ctypes.byref(cut), _p(stats, I64P))
    _raise_for(rc, "greedy_refine")
    return part, int(cut.value), stats


def fm2_refine(graph: Graph, part, targets, ubvec, niter: int = 10):
    """2-way fm_refine (src/refine/fm.rs:12-28) of a bisection on the GPU.
    Returns (refined part, edge cut, stats[passes, moves kept, rounds, movers])."""
    part = np.array(part, dtype=np.int32)
    t = np.ascontiguousarray(targets, dtype=np.float64)
    ub = np.ascontiguousarray(ubvec, dtype=np.float64)
    cut = ctypes.c_int32(0)
    stats = np.zeros(4, np.int64)
    rc = _lib.load().RMETIS_GPU_Fm2Refine(graph.nvtxs, graph.ncon, _p(graph.xadj), _p(graph.adjncy),
                                          _p(graph.vwgt), _p(graph.adjwgt), _p(part), _p(t, F64P), _p(ub, F64P),
                                          niter, ctypes.byref(cut), _p(stats, I64P))
    _raise_for(rc, "fm2_refine")
    return part, int(cut.value), stats


def fm_refine(graph: Graph, part, nparts: int, targets, ubvec, niter: int = 10):
    """fm_kway_refine (src/refine/fm_kway.rs:12-31) on the GPU. Returns
    (refined part, edge cut, stats[passes, moves, rounds with movers, movers])."""
    part = np.array(part, dtype=np.int32)
    t = np.ascontiguousarray(targets, dtype=np.float64)
    ub = np.ascontiguousarray(ubvec, dtype=np.float64)
    cut = ctypes.c_int32(0)
    stats = np.zeros(4, np.int64)
    rc = _lib.load().RMETIS_GPU_FmRefine(graph.nvtxs, graph.ncon, _p(graph.xadj), _p(graph.adjncy),
                                         _p(graph.vwgt), _p(graph.adjwgt), _p(part), nparts, _p(t, F64P),
                                         _p(ub, F64P), niter, ctypes.byref(cut), _p(stats, I64P))
    _raise_for(rc, "fm_refine")
    return part, int(cut.value), stats
