"""rmetis_b200 — B200-native multilevel k-way graph partitioning.

A Python mirror of the reference's public k-way API (javagg/rmetis:
`Graph` src/graph/mod.rs:13-50, `Options` src/types.rs:52-117,
`part_graph_kway` src/lib.rs:48-56, `PartitionResult` src/types.rs:125-130,
`MetisError` src/types.rs:146-161) over the C ABI in include/rmetis.h. All
compute runs in librmetis_gpu.so on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import F32P, F64P, I32P, I64P

__all__ = [
    "CType", "IpType", "RType", "ObjType", "Options", "Graph", "PartitionResult", "MetisError", "InputError",
    "OutOfMemoryError", "InternalError", "part_graph_kway", "part_graph_recursive", "set_default_options",
    "node_nd", "NDResult",
    "METIS_OK",
    "METIS_ERROR_INPUT", "METIS_ERROR_MEMORY", "METIS_ERROR", "METIS_NOPTIONS",
]

METIS_OK = 1
METIS_ERROR_INPUT = -2
METIS_ERROR_MEMORY = -3
METIS_ERROR = -4
METIS_NOPTIONS = 40

(OPT_PTYPE, OPT_OBJTYPE, OPT_CTYPE, OPT_IPTYPE, OPT_RTYPE, OPT_DBGLVL, OPT_NITER, OPT_NCUTS, OPT_SEED,
 OPT_NO2HOP, OPT_MINCONN, OPT_CONTIG) = range(12)
OPT_UFACTOR = 16
OPT_NUMBERING = 17


class CType(enum.IntEnum):
    Rm = 0
    Shem = 1


class IpType(enum.IntEnum):
    Grow = 0
    Random = 1
    MetisRb = 4


class RType(enum.IntEnum):
    Fm = 0
    Greedy = 1


class ObjType(enum.IntEnum):
    Cut = 0
    Vol = 1


class MetisError(Exception):
    """Base error (src/types.rs:146-161)."""
    code = METIS_ERROR


class InputError(MetisError):
    code = METIS_ERROR_INPUT


class OutOfMemoryError(MetisError):
    code = METIS_ERROR_MEMORY


class InternalError(MetisError):
    code = METIS_ERROR


def _raise_for(rc: int, what: str):
    if rc == METIS_OK:
        return
    if rc == METIS_ERROR_INPUT:
        raise InputError(f"{what}: input error")
    if rc == METIS_ERROR_MEMORY:
        raise OutOfMemoryError(f"{what}: out of memory")
    raise InternalError(f"{what}: error {rc}")


@dataclass
class Options:
    """All tuning parameters (src/types.rs:52-95); defaults mirror
    Options::default(), including rtype Fm."""
    ctype: CType = CType.Shem
    iptype: IpType = IpType.Grow
    rtype: RType = RType.Fm
    objtype: ObjType = ObjType.Cut
    no2hop: bool = False
    ncuts: int = 1
    niter: int = 10
    seed: int = 0
    minconn: bool = False
    contig: bool = False
    ufactor: int = 30
    numbering: int = 0
    dbglvl: int = 0

    @classmethod
    def for_kway(cls) -> "Options":  # src/types.rs:109-116
        return cls(iptype=IpType.Grow, rtype=RType.Fm, ufactor=30)

    @classmethod
    def for_recursive(cls) -> "Options":  # src/types.rs:99-106
        return cls(iptype=IpType.MetisRb, rtype=RType.Fm, ufactor=1)

    def to_raw(self) -> np.ndarray:  # src/types.rs:227-245
        a = np.full(METIS_NOPTIONS, -1, dtype=np.int32)
        a[OPT_CTYPE] = int(self.ctype)
        a[OPT_IPTYPE] = int(self.iptype)
        a[OPT_RTYPE] = int(self.rtype)
        a[OPT_OBJTYPE] = int(self.objtype)
        a[OPT_NO2HOP] = int(self.no2hop)
        a[OPT_NCUTS] = self.ncuts
        a[OPT_NITER] = self.niter
        a[OPT_SEED] = np.int64(self.seed).astype(np.int32)
        a[OPT_MINCONN] = int(self.minconn)
        a[OPT_CONTIG] = int(self.contig)
        a[OPT_UFACTOR] = self.ufactor
        a[OPT_NUMBERING] = self.numbering
        a[OPT_DBGLVL] = self.dbglvl
        return a

    @classmethod
    def from_raw(cls, a) -> "Options":  # src/types.rs:190-224
        a = np.asarray(a, dtype=np.int32)
        o = cls()
        if a[OPT_CTYPE] == 0:
            o.ctype = CType.Rm
        if a[OPT_IPTYPE] == 1:
            o.iptype = IpType.Random
        elif a[OPT_IPTYPE] == 4:
            o.iptype = IpType.MetisRb
        if a[OPT_RTYPE] == 1:
            o.rtype = RType.Greedy
        if a[OPT_OBJTYPE] == 1:
            o.objtype = ObjType.Vol
        if a[OPT_NO2HOP] != 0:
            o.no2hop = True
        if a[OPT_NCUTS] > 0:
            o.ncuts = int(a[OPT_NCUTS])
        if a[OPT_NITER] > 0:
            o.niter = int(a[OPT_NITER])
        o.seed = max(int(a[OPT_SEED]), 0)
        o.minconn = bool(a[OPT_MINCONN] != 0)
        o.contig = bool(a[OPT_CONTIG] != 0)
        if a[OPT_UFACTOR] > 0:
            o.ufactor = int(a[OPT_UFACTOR])
        o.numbering = int(a[OPT_NUMBERING]) & 0xFF
        o.dbglvl = int(a[OPT_DBGLVL])
        return o

    def c_array(self) -> np.ndarray:
        """The option array the C ABI reads: to_raw() with PTYPE set so that the
        partitioner does not fall back to all defaults (src/ffi/c_api.rs:217)."""
        a = self.to_raw()
        a[OPT_PTYPE] = 0
        return a


@dataclass
class PartitionResult:
    part: np.ndarray
    objval: int


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _p(a, t=I32P):
    return None if a is None else a.ctypes.data_as(t)


def _validate(nvtxs, ncon, xadj, adjncy, vwgt, adjwgt):
    """validate_csr (src/graph/validate.rs:16-142) on host arrays."""
    if nvtxs <= 0:
        raise InputError("nvtxs must be > 0")
    if ncon <= 0:
        raise InputError("ncon must be > 0")
    if len(xadj) != nvtxs + 1:
        raise InputError(f"xadj.len()={len(xadj)} but expected nvtxs+1={nvtxs + 1}")
    if xadj[0] != 0:
        raise InputError(f"xadj[0]={xadj[0]} but must be 0")
    if np.any(np.diff(xadj.astype(np.int64)) < 0):
        raise InputError("xadj is not monotone")
    ne = int(xadj[nvtxs])
    if len(adjncy) != ne:
        raise InputError(f"adjncy.len()={len(adjncy)} but xadj[nvtxs]={ne}")
    if ne:
        if adjncy.min() < 0 or adjncy.max() >= nvtxs:
            raise InputError("adjncy out of range")
        src = np.repeat(np.arange(nvtxs, dtype=np.int64), np.diff(xadj.astype(np.int64)))
        if np.any(src == adjncy):
            raise InputError("self-loop detected")
    deg_check = np.bincount(adjncy, minlength=nvtxs) if ne else np.zeros(nvtxs, np.int64)
    if np.any(deg_check != np.diff(xadj.astype(np.int64))):
        raise InputError("graph is not symmetric")
    if adjwgt is not None and len(adjwgt) != ne:
        raise InputError("adjwgt length mismatch")
    if vwgt is not None:
        if len(vwgt) != nvtxs * ncon:
            raise InputError("vwgt length mismatch")
        if np.any(vwgt <= 0):
            raise InputError("vwgt must be > 0")


class Graph:
    """CSR graph (src/graph/mod.rs:13-50). Edge-level queries run on the GPU."""

    def __init__(self, nvtxs, ncon, xadj, adjncy, vwgt=None, adjwgt=None, vsize=None, validate=True):
        self.nvtxs = int(nvtxs)
        self.ncon = int(ncon)
        self.xadj = _i32(xadj)
        self.adjncy = _i32(adjncy)
        self.vwgt = _i32(vwgt)
        self.adjwgt = _i32(adjwgt)
        self.vsize = _i32(vsize)
        if validate:
            _validate(self.nvtxs, self.ncon, self.xadj, self.adjncy, self.vwgt, self.adjwgt)
        self.nedges = len(self.adjncy) // 2

    @classmethod
    def new(cls, nvtxs, ncon, xadj, adjncy, vwgt=None, adjwgt=None, vsize=None) -> "Graph":
        return cls(nvtxs, ncon, xadj, adjncy, vwgt, adjwgt, vsize)

    @classmethod
    def new_unweighted(cls, nvtxs, xadj, adjncy) -> "Graph":
        return cls(nvtxs, 1, xadj, adjncy)

    def neighbors(self, v):
        return self.adjncy[self.xadj[v]:self.xadj[v + 1]]

    def degree(self, v):
        return int(self.xadj[v + 1] - self.xadj[v])

    def edge_cut(self, part) -> int:
        part = _i32(part)
        cut = ctypes.c_int32(0)
        rc = _lib.load().RMETIS_GPU_EdgeCut(self.nvtxs, _p(self.xadj), _p(self.adjncy), _p(self.adjwgt), _p(part),
                                            ctypes.byref(cut))
        _raise_for(rc, "edge_cut")
        return int(cut.value)

    def partition_weights(self, part, nparts) -> np.ndarray:
        part = _i32(part)
        out = np.zeros(nparts * self.ncon, dtype=np.int32)
        rc = _lib.load().RMETIS_GPU_PartitionWeights(self.nvtxs, self.ncon, _p(self.vwgt), _p(part), nparts,
                                                     _p(out))
        _raise_for(rc, "partition_weights")
        return out.reshape(nparts, self.ncon)

    def total_weight(self) -> np.ndarray:
        if self.vwgt is None:
            return np.full(self.ncon, self.nvtxs, dtype=np.int32)
        return self.vwgt.reshape(self.nvtxs, self.ncon).astype(np.int64).sum(axis=0).astype(np.int32)

    def gain_table(self, part, nparts):
        """Boundary flags, w_from and sorted explicit candidates (see
        RMETIS_GPU_GainTable)."""
        part = _i32(part)
        n = self.nvtxs
        m = len(self.adjncy)
        b = np.zeros(n, np.int32); nc = np.zeros(n, np.int32); wf = np.zeros(n, np.int32)
        cp = np.zeros(max(m, 1), np.int32); cg = np.zeros(max(m, 1), np.int32)
        rc = _lib.load().RMETIS_GPU_GainTable(n, _p(self.xadj), _p(self.adjncy), _p(self.adjwgt), _p(part), nparts,
                                              _p(b), _p(nc), _p(wf), _p(cp), _p(cg))
        _raise_for(rc, "gain_table")
        return b, nc, wf, cp, cg

    def boundary_vertices(self, part) -> np.ndarray:
        part = _i32(part)
        b, *_ = self.gain_table(part, int(part.max()) + 1 if len(part) else 1)
        return np.nonzero(b)[0].astype(np.int64)

    def build_coarse_graph(self, matching):
        """Returns (coarse Graph, cmap) (src/graph/mod.rs:284-384)."""
        matching = _i32(matching)
        n = self.nvtxs
        m = len(self.adjncy)
        cn = ctypes.c_int32(0)
        cmap = np.zeros(n, np.int32); cx = np.zeros(n + 1, np.int32)
        ca = np.zeros(max(m, 1), np.int32); cw = np.zeros(max(m, 1), np.int32)
        cv = np.zeros(max(n * self.ncon, 1), np.int32)
        rc = _lib.load().RMETIS_GPU_BuildCoarseGraph(n, self.ncon, _p(self.xadj), _p(self.adjncy), _p(self.vwgt),
                                                     _p(self.adjwgt), _p(matching), ctypes.byref(cn), _p(cmap),
                                                     _p(cx), _p(ca), _p(cw), _p(cv))
        _raise_for(rc, "build_coarse_graph")
        c = cn.value
        cx = cx[:c + 1]
        ce = int(cx[c])
        cw = cw[:ce]
        keep = self.adjwgt is not None or bool(np.any(cw != 1))
        g = Graph(c, self.ncon, cx, ca[:ce], vwgt=None if self.vwgt is None else cv[:c * self.ncon],
                  adjwgt=cw if keep else None, validate=False)
        return g, cmap

    def __repr__(self):
        return f"Graph(nvtxs={self.nvtxs}, nedges={self.nedges}, ncon={self.ncon})"


def set_default_options() -> np.ndarray:
    a = np.zeros(METIS_NOPTIONS, dtype=np.int32)
    _raise_for(_lib.load().RMETIS_SetDefaultOptions(_p(a)), "set_default_options")
    return a


def part_graph_kway(graph: Graph, nparts: int, tpwgts=None, ubvec=None, options: Options | None = None
                    ) -> PartitionResult:
    """Multilevel k-way partition (src/lib.rs:48-56) on the GPU.

    RType::Greedy refines pass for pass as the reference does; RType::Fm (the
    default) runs the reference's FM move rule in parallel rounds, equal to
    the reference's in quality rather than bit for bit."""
    options = options or Options()
    if nparts < 2:
        raise InputError(f"nparts must be >= 2, got {nparts}")
    if nparts > graph.nvtxs:
        raise InputError(f"nparts={nparts} > nvtxs={graph.nvtxs}")
    opts = options.c_array()
    part = np.zeros(graph.nvtxs, dtype=np.int32)
    obj = ctypes.c_int32(0)
    nv = ctypes.c_int32(graph.nvtxs); nc = ctypes.c_int32(graph.ncon); npr = ctypes.c_int32(nparts)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    rc = _lib.load().RMETIS_PartGraphKway(ctypes.byref(nv), ctypes.byref(nc), _p(graph.xadj), _p(graph.adjncy),
                                          _p(graph.vwgt), _p(graph.vsize), _p(graph.adjwgt), ctypes.byref(npr),
                                          _p(tp, F32P), _p(ub, F32P), _p(opts), ctypes.byref(obj), _p(part))
    _raise_for(rc, "part_graph_kway")
    return PartitionResult(part=part, objval=int(obj.value))


def part_graph_recursive(graph: Graph, nparts: int, tpwgts=None, ubvec=None, options: Options | None = None
                         ) -> PartitionResult:
    """Multilevel recursive bisection (src/lib.rs part_graph_recursive,
    src/partition/recursive.rs:12-187): the reference's recursion and target
    arithmetic, each bisection a 2-way multilevel partition on the GPU. Pass
    Options.for_recursive() for the reference's defaults of this call."""
    options = options or Options()
    if nparts < 2:
        raise InputError(f"nparts must be >= 2, got {nparts}")
    if nparts > graph.nvtxs:
        raise InputError(f"nparts={nparts} > nvtxs={graph.nvtxs}")
    opts = options.c_array()
    part = np.zeros(graph.nvtxs, dtype=np.int32)
    obj = ctypes.c_int32(0)
    nv = ctypes.c_int32(graph.nvtxs); nc = ctypes.c_int32(graph.ncon); npr = ctypes.c_int32(nparts)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    rc = _lib.load().RMETIS_PartGraphRecursive(ctypes.byref(nv), ctypes.byref(nc), _p(graph.xadj),
                                               _p(graph.adjncy), _p(graph.vwgt), _p(graph.vsize), _p(graph.adjwgt),
                                               ctypes.byref(npr), _p(tp, F32P), _p(ub, F32P), _p(opts),
                                               ctypes.byref(obj), _p(part))
    _raise_for(rc, "part_graph_recursive")
    return PartitionResult(part=part, objval=int(obj.value))


def part_graph_kway_trace(graph: Graph, nparts: int, tpwgts=None, ubvec=None, options: Options | None = None):
    """part_graph_kway plus the random choices of the kept attempt:
    returns (PartitionResult, matchings per level, grow seeds, stats)."""
    options = options or Options()
    opts = options.c_array()
    n = graph.nvtxs
    part = np.zeros(n, dtype=np.int32)
    obj = ctypes.c_int32(0)
    nv = ctypes.c_int32(n); nc = ctypes.c_int32(graph.ncon); npr = ctypes.c_int32(nparts)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    cap = 24 * n + 64
    mats = np.zeros(cap, np.int32)
    off = np.zeros(130, np.int64)
    nl = ctypes.c_int64(0)
    seeds = np.zeros(nparts, np.int32)
    stats = np.zeros(4, np.int64)
    rc = _lib.load().RMETIS_GPU_PartGraphKwayTrace(
        ctypes.byref(nv), ctypes.byref(nc), _p(graph.xadj), _p(graph.adjncy), _p(graph.vwgt), _p(graph.adjwgt),
        ctypes.byref(npr), _p(tp, F32P), _p(ub, F32P), _p(opts), ctypes.byref(obj), _p(part), _p(mats), cap,
        _p(off, I64P), len(off), ctypes.byref(nl), _p(seeds), _p(stats, I64P))
    _raise_for(rc, "part_graph_kway_trace")
    L = nl.value
    matchings = [mats[off[i]:off[i + 1]].copy() for i in range(L)]
    return PartitionResult(part=part, objval=int(obj.value)), matchings, seeds, stats


def set_tuning(grow_trials: int = -1, match_rounds: int = -1, summed_unit_weights: int = -1,
               parallel_attempts: int = -1, fused_max_n: int = -1, tail_max_n: int = -1):
    """Engine knobs without an options slot (-1 leaves a knob unchanged)."""
    _raise_for(_lib.load().RMETIS_GPU_SetTuning(grow_trials, match_rounds, summed_unit_weights, parallel_attempts,
                                                fused_max_n, tail_max_n), "set_tuning")


def set_refine_mode(exact_max_n: int = 16384):
    """Levels with at most exact_max_n vertices decide greedy cut passes
    exactly as the reference's sequential pass; larger levels by parallel
    admission (-1: exact everywhere)."""
    _raise_for(_lib.load().RMETIS_GPU_SetRefineMode(exact_max_n), "set_refine_mode")


def set_kernel_shapes(contract_thread_max: int = -1, gain_block: int = -1):
    """Result-neutral kernel shapes: the longest merged-row bound one thread
    merges in contraction (16 or 32) and the gain-table block size (128, 256
    or 512); -1 leaves a knob unchanged."""
    _raise_for(_lib.load().RMETIS_GPU_SetKernelShapes(contract_thread_max, gain_block), "set_kernel_shapes")


def set_pool_tuning(fused_max_n: int = -2, tail_max_n: int = -2):
    """Launch-shape knobs for batch graphs and submitted requests, which share
    the device with other jobs (-1 = the set_tuning value, -2 leaves a knob
    unchanged). Neither changes a result; rmetis_b200.autotune measures them."""
    _raise_for(_lib.load().RMETIS_GPU_SetPoolTuning(fused_max_n, tail_max_n), "set_pool_tuning")


def set_coop_matching(on: int = 1):
    """1 (default): a level's matching rounds run in one cooperative launch;
    0: one launch per phase. The same matching either way."""
    _raise_for(_lib.load().RMETIS_GPU_SetCoopMatching(on), "set_coop_matching")


def set_fused_edge_factor(factor: int = -1):
    """Edge bound of the single-block levels: at most factor * fused_max_n
    adjacency entries (default 4). Never changes a result."""
    _raise_for(_lib.load().RMETIS_GPU_SetFusedEdgeFactor(factor), "set_fused_edge_factor")


def set_fm_fused_max(max_n: int = -1):
    """FM levels of at most max_n vertices (default 4096) run all their passes
    and rounds in one single-block launch; 0 = never. Never changes a result."""
    _raise_for(_lib.load().RMETIS_GPU_SetFmFusedMax(max_n), "set_fm_fused_max")


def set_batch_mode(mode: int = -1, max_n: int = -1):
    """How part_graph_kway_batch runs its graphs. mode 1 (default): eligible
    graphs (Greedy, ncuts 1, grown initial partitions, ncon <= 2,
    nparts <= 256) of at most max_n vertices (default 262144) go through the
    batched launches, one step of the pipeline for all of them at a time,
    while the others run on the worker pool at the same time; mode 0: every
    graph on the worker pool. -1 leaves a value unchanged. Results are the
    same either way."""
    _raise_for(_lib.load().RMETIS_GPU_SetBatchMode(mode, max_n), "set_batch_mode")


def part_graph_kway_batch(graphs, nparts, ubvec=None, options: Options | None = None):
    """Partition many graphs in one call: the batch is uploaded once; eligible
    graphs go through the pipeline together (one launch per step, one block
    per graph, see set_batch_mode), the others run concurrently on the
    device's worker pool. Returns one
    PartitionResult per graph, each equal to part_graph_kway's for that graph.
    `nparts` is an int or one value per graph; all graphs share ncon and
    either all have vertex (edge) weights or none has."""
    options = options or Options()
    graphs = list(graphs)
    G = len(graphs)
    if G == 0:
        return []
    ncon = graphs[0].ncon
    if any(g.ncon != ncon for g in graphs):
        raise InputError("all graphs of a batch need the same ncon")
    nps = np.full(G, nparts, np.int32) if np.isscalar(nparts) else np.ascontiguousarray(nparts, dtype=np.int32)
    if len(nps) != G:
        raise InputError("nparts needs one value per graph")
    for g, k in zip(graphs, nps):
        if k < 2 or k > g.nvtxs:
            raise InputError(f"nparts={k} is outside [2, nvtxs={g.nvtxs}]")
    have_vw = {g.vwgt is not None for g in graphs}
    have_ew = {g.adjwgt is not None for g in graphs}
    if len(have_vw) > 1 or len(have_ew) > 1:
        raise InputError("either every graph of a batch has vertex (edge) weights or none has")
    vtx_off = np.zeros(G + 1, np.int64)
    edge_off = np.zeros(G + 1, np.int64)
    vtx_off[1:] = np.cumsum([g.nvtxs for g in graphs])
    edge_off[1:] = np.cumsum([len(g.adjncy) for g in graphs])
    xadj = np.concatenate([g.xadj for g in graphs]).astype(np.int32)
    adjncy = np.concatenate([g.adjncy for g in graphs]).astype(np.int32)
    vwgt = np.concatenate([g.vwgt for g in graphs]).astype(np.int32) if have_vw.pop() else None
    adjwgt = np.concatenate([g.adjwgt for g in graphs]).astype(np.int32) if have_ew.pop() else None
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    part = np.zeros(int(vtx_off[-1]), np.int32)
    obj = np.zeros(G, np.int32)
    status = np.zeros(G, np.int32)
    opts = options.c_array()
    rc = _lib.load().RMETIS_GPU_PartGraphKwayBatch(G, ncon, _p(vtx_off, I64P), _p(edge_off, I64P), _p(xadj),
                                                   _p(adjncy), _p(vwgt), _p(adjwgt), _p(nps), _p(ub, F32P),
                                                   _p(opts), _p(obj), _p(part), _p(status))
    _raise_for(rc, "part_graph_kway_batch")
    return [PartitionResult(part=part[vtx_off[i]:vtx_off[i + 1]].copy(), objval=int(obj[i])) for i in range(G)]


class KwayRequest:
    """An asynchronous k-way request on the device's worker pool (see
    submit_kway). It holds the host arrays the worker reads and writes until
    wait() returns."""

    def __init__(self, ticket, keep, part, obj):
        self._ticket = ticket
        self._keep = keep
        self._part = part
        self._obj = obj
        self._result = None

    def done(self) -> bool:
        if self._result is not None:
            return True
        rc = _lib.load().RMETIS_GPU_PollKway(self._ticket)
        if rc < 0:
            _raise_for(rc, "poll")
        return rc == 1

    def wait(self) -> PartitionResult:
        if self._result is None:
            rc = _lib.load().RMETIS_GPU_WaitKway(self._ticket)
            self._keep = None
            _raise_for(rc, "submit_kway")
            self._result = PartitionResult(part=self._part, objval=int(self._obj.value))
        return self._result


def submit_kway(graph: Graph, nparts: int, tpwgts=None, ubvec=None, options: Options | None = None) -> KwayRequest:
    """Queue a k-way partition on the device's worker pool and return at once.
    Requests start in submission order as their estimated memory footprint
    fits the pool's budget; the result equals part_graph_kway's."""
    options = options or Options()
    if nparts < 2:
        raise InputError(f"nparts must be >= 2, got {nparts}")
    if nparts > graph.nvtxs:
        raise InputError(f"nparts={nparts} > nvtxs={graph.nvtxs}")
    opts = options.c_array()
    part = np.zeros(graph.nvtxs, dtype=np.int32)
    obj = ctypes.c_int32(0)
    nv = ctypes.c_int32(graph.nvtxs); nc = ctypes.c_int32(graph.ncon); npr = ctypes.c_int32(nparts)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    t = _lib.load().RMETIS_GPU_SubmitKway(ctypes.byref(nv), ctypes.byref(nc), _p(graph.xadj), _p(graph.adjncy),
                                          _p(graph.vwgt), _p(graph.adjwgt), ctypes.byref(npr), _p(tp, F32P),
                                          _p(ub, F32P), _p(opts), ctypes.byref(obj), _p(part))
    if t <= 0:
        _raise_for(int(t), "submit_kway")
    return KwayRequest(t, (graph, opts, nv, nc, npr, tp, ub), part, obj)


@dataclass
class NDResult:
    """Nested dissection ordering (src/types.rs:133-137): perm[v] is the new
    position of vertex v, iperm its inverse."""
    perm: np.ndarray
    iperm: np.ndarray


def node_nd(graph: Graph, options: Options | None = None) -> NDResult:
    """Nested dissection ordering (src/partition/nd.rs:16-44) through
    RMETIS_NodeND: separators from GPU bisections of each subgraph, lighter
    side first, separator last. The graph's vertex weights (constraint 0) are
    used; edge weights are not (the reference's C entry has none)."""
    options = options or Options()
    n = graph.nvtxs
    perm = np.zeros(n, np.int32)
    iperm = np.zeros(n, np.int32)
    vw = None if graph.vwgt is None else np.ascontiguousarray(graph.vwgt.reshape(n, graph.ncon)[:, 0])
    rc = _lib.load().RMETIS_NodeND(ctypes.byref(ctypes.c_int32(n)), _p(graph.xadj), _p(graph.adjncy), _p(vw),
                                   _p(options.c_array()), _p(perm), _p(iperm))
    _raise_for(rc, "node_nd")
    return NDResult(perm=perm, iperm=iperm)


from .graphio import format_metis_graph, parse_metis_graph, read_metis_graph, write_metis_graph  # noqa: E402
