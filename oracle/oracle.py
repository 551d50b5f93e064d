"""ctypes wrapper over the oracle (the CPU restatement in ref_kway.cpp).

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU
legs use it to check the CUDA path. The product (rmetis_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_kway.so")
_lib = None

I32P = ctypes.POINTER(ctypes.c_int32)
I64P = ctypes.POINTER(ctypes.c_int64)
U64P = ctypes.POINTER(ctypes.c_uint64)
F32P = ctypes.POINTER(ctypes.c_float)
F64P = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the restatement with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_edge_cut.restype = ctypes.c_int32
        _lib.orc_compute_move_gain.restype = ctypes.c_int32
        _lib.orc_boundary_vertices.restype = ctypes.c_int64
        _lib.orc_build_coarse_graph.restype = ctypes.c_int64
        _lib.orc_greedy_refine.restype = ctypes.c_int32
        _lib.orc_fm_kway_refine.restype = ctypes.c_int32
        _lib.orc_rng_gen_range.restype = ctypes.c_uint64
        _lib.orc_fm2_refine.restype = ctypes.c_int32
        for name in ("orc_validate_csr", "orc_SetDefaultOptions", "orc_PartGraphKway",
                     "orc_PartGraphKway_script", "orc_PartGraphRecursive", "orc_NodeND"):
            getattr(_lib, name).restype = ctypes.c_int
    return _lib


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


class SmallRng:
    """The reference's SmallRng (rand 0.8.5), state held in numpy."""

    def __init__(self, seed: int):
        self.state = np.zeros(4, dtype=np.uint64)
        lib().orc_rng_seed_from_u64(ctypes.c_uint64(seed), _p(self.state, U64P))

    @classmethod
    def from_state(cls, s):
        r = cls.__new__(cls)
        r.state = np.asarray(s, dtype=np.uint64).copy()
        return r

    def next_u64(self, count=1):
        out = np.zeros(count, dtype=np.uint64)
        lib().orc_rng_from_state_next_u64(_p(self.state, U64P), ctypes.c_int64(count), _p(out, U64P))
        return out

    def gen_range(self, low, high):
        return int(lib().orc_rng_gen_range(_p(self.state, U64P), ctypes.c_uint64(low), ctypes.c_uint64(high)))


def validate_csr(nvtxs, ncon, xadj, adjncy, vwgt=None, adjwgt=None) -> int:
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    return lib().orc_validate_csr(
        ctypes.c_int64(nvtxs), ctypes.c_int64(ncon), _p(xadj, I32P), ctypes.c_int64(len(xadj)),
        _p(adjncy, I32P), ctypes.c_int64(len(adjncy)), _p(vwgt, I32P),
        ctypes.c_int64(0 if vwgt is None else len(vwgt)), _p(adjwgt, I32P),
        ctypes.c_int64(0 if adjwgt is None else len(adjwgt)))


def edge_cut(xadj, adjncy, adjwgt, part) -> int:
    xadj = _i32(xadj); adjncy = _i32(adjncy); adjwgt = _i32(adjwgt); part = _i32(part)
    return int(lib().orc_edge_cut(ctypes.c_int64(len(xadj) - 1), _p(xadj, I32P), _p(adjncy, I32P),
                                  _p(adjwgt, I32P), _p(part, I32P)))


def partition_weights(n, ncon, vwgt, part, nparts):
    vwgt = _i32(vwgt); part = _i32(part)
    out = np.zeros(nparts * ncon, dtype=np.int32)
    lib().orc_partition_weights(ctypes.c_int64(n), ctypes.c_int64(ncon), _p(vwgt, I32P), _p(part, I32P),
                                ctypes.c_int64(nparts), _p(out, I32P))
    return out.reshape(nparts, ncon)


def total_weight(n, ncon, vwgt):
    vwgt = _i32(vwgt)
    out = np.zeros(ncon, dtype=np.int32)
    lib().orc_total_weight(ctypes.c_int64(n), ctypes.c_int64(ncon), _p(vwgt, I32P), _p(out, I32P))
    return out


def boundary_vertices(xadj, adjncy, part):
    xadj = _i32(xadj); adjncy = _i32(adjncy); part = _i32(part)
    n = len(xadj) - 1
    out = np.zeros(n, dtype=np.int32)
    cnt = lib().orc_boundary_vertices(ctypes.c_int64(n), _p(xadj, I32P), _p(adjncy, I32P), _p(part, I32P),
                                      _p(out, I32P))
    return out[:cnt]


def compute_move_gain(xadj, adjncy, adjwgt, v, part, frm, to) -> int:
    xadj = _i32(xadj); adjncy = _i32(adjncy); adjwgt = _i32(adjwgt); part = _i32(part)
    return int(lib().orc_compute_move_gain(ctypes.c_int64(len(xadj) - 1), _p(xadj, I32P), _p(adjncy, I32P),
                                           _p(adjwgt, I32P), ctypes.c_int64(v), _p(part, I32P),
                                           ctypes.c_int32(frm), ctypes.c_int32(to)))


def build_coarse_graph(xadj, adjncy, matching, vwgt=None, adjwgt=None, ncon=1):
    """Returns dict(cn, cmap, cxadj, cadjncy, cadjwgt, cvwgt|None, keeps_adjwgt)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    matching = _i32(matching)
    n = len(xadj) - 1
    m = len(adjncy)
    cmap = np.zeros(n, dtype=np.int32)
    cxadj = np.zeros(n + 1, dtype=np.int32)
    cadj = np.zeros(max(m, 1), dtype=np.int32)
    cw = np.zeros(max(m, 1), dtype=np.int32)
    cv = np.zeros(max(n * ncon, 1), dtype=np.int32)
    flags = ctypes.c_int32(0)
    cn = lib().orc_build_coarse_graph(ctypes.c_int64(n), ctypes.c_int64(ncon), _p(xadj, I32P), _p(adjncy, I32P),
                                      _p(vwgt, I32P), _p(adjwgt, I32P), _p(matching, I32P), _p(cmap, I32P),
                                      _p(cxadj, I32P), _p(cadj, I32P), _p(cw, I32P), _p(cv, I32P),
                                      ctypes.byref(flags))
    cxadj = cxadj[:cn + 1].copy()
    cm = int(cxadj[cn])
    return dict(cn=int(cn), cmap=cmap, cxadj=cxadj, cadjncy=cadj[:cm].copy(), cadjwgt=cw[:cm].copy(),
                cvwgt=(cv[:cn * ncon].copy() if (flags.value & 2) else None),
                keeps_adjwgt=bool(flags.value & 1))


def shem_matching(xadj, adjncy, adjwgt, rng: SmallRng):
    xadj = _i32(xadj); adjncy = _i32(adjncy); adjwgt = _i32(adjwgt)
    n = len(xadj) - 1
    out = np.zeros(n, dtype=np.int32)
    lib().orc_shem_matching(ctypes.c_int64(n), _p(xadj, I32P), _p(adjncy, I32P), _p(adjwgt, I32P),
                            _p(rng.state, U64P), _p(out, I32P))
    return out


def random_matching(xadj, adjncy, rng: SmallRng):
    xadj = _i32(xadj); adjncy = _i32(adjncy)
    n = len(xadj) - 1
    out = np.zeros(n, dtype=np.int32)
    lib().orc_random_matching(ctypes.c_int64(n), _p(xadj, I32P), _p(adjncy, I32P), _p(rng.state, U64P),
                              _p(out, I32P))
    return out


def compute_target_weights(n, ncon, vwgt, nparts, tpwgts=None):
    vwgt = _i32(vwgt)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    out = np.zeros(nparts * ncon, dtype=np.float64)
    lib().orc_compute_target_weights(ctypes.c_int64(n), ctypes.c_int64(ncon), _p(vwgt, I32P),
                                     ctypes.c_int64(nparts), _p(tp, F32P), _p(out, F64P))
    return out


def grow_partition(xadj, adjncy, nparts, tpwgts, vwgt=None, ncon=1, rng: SmallRng | None = None, seeds=None):
    """Returns (part, seeds)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); seeds = _i32(seeds)
    n = len(xadj) - 1
    tp = np.ascontiguousarray(tpwgts, dtype=np.float64)
    part = np.zeros(n, dtype=np.int32)
    so = np.zeros(nparts, dtype=np.int32)
    lib().orc_grow_partition(ctypes.c_int64(n), ctypes.c_int64(ncon), _p(xadj, I32P), _p(adjncy, I32P),
                             _p(vwgt, I32P), ctypes.c_int64(nparts), _p(tp, F64P),
                             None if rng is None else _p(rng.state, U64P), _p(seeds, I32P), _p(so, I32P),
                             _p(part, I32P))
    return part, so


def greedy_refine(xadj, adjncy, part, nparts, tpwgts, ubvec, niter, vwgt=None, adjwgt=None, ncon=1):
    """Returns (part, cut, moves_per_pass)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    part = np.array(part, dtype=np.int32)
    tp = np.ascontiguousarray(tpwgts, dtype=np.float64)
    ub = np.ascontiguousarray(ubvec, dtype=np.float64)
    moves = np.zeros(niter + 1, dtype=np.int64)
    npasses = ctypes.c_int64(0)
    cut = lib().orc_greedy_refine(ctypes.c_int64(len(xadj) - 1), ctypes.c_int64(ncon), _p(xadj, I32P),
                                  _p(adjncy, I32P), _p(vwgt, I32P), _p(adjwgt, I32P), _p(part, I32P),
                                  ctypes.c_int64(nparts), _p(tp, F64P), _p(ub, F64P), ctypes.c_int64(niter),
                                  _p(moves, I64P), ctypes.byref(npasses))
    return part, int(cut), moves[:npasses.value].copy()


def fm_kway_refine(xadj, adjncy, part, nparts, tpwgts, ubvec, niter, vwgt=None, adjwgt=None, ncon=1):
    """Restated fm_kway_refine (src/refine/fm_kway.rs:12-31). Returns
    (part, cut, passes, moves)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    part = np.array(part, dtype=np.int32)
    tp = np.ascontiguousarray(tpwgts, dtype=np.float64)
    ub = np.ascontiguousarray(ubvec, dtype=np.float64)
    st = np.zeros(2, dtype=np.int64)
    cut = lib().orc_fm_kway_refine(ctypes.c_int64(len(xadj) - 1), ctypes.c_int64(ncon), _p(xadj, I32P),
                                   _p(adjncy, I32P), _p(vwgt, I32P), _p(adjwgt, I32P), _p(part, I32P),
                                   ctypes.c_int64(nparts), _p(tp, F64P), _p(ub, F64P), ctypes.c_int64(niter),
                                   _p(st, I64P))
    return part, int(cut), int(st[0]), int(st[1])


def set_default_options():
    opts = np.zeros(40, dtype=np.int32)
    rc = lib().orc_SetDefaultOptions(_p(opts, I32P))
    return rc, opts


def fm2_refine(xadj, adjncy, part, tpwgts, ubvec, niter, vwgt=None, adjwgt=None, ncon=1):
    """Restated 2-way fm_refine (src/refine/fm.rs:12-28). Returns (part, cut)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    part = np.array(part, dtype=np.int32)
    tp = np.ascontiguousarray(tpwgts, dtype=np.float64)
    ub = np.ascontiguousarray(ubvec, dtype=np.float64)
    cut = lib().orc_fm2_refine(ctypes.c_int64(len(xadj) - 1), ctypes.c_int64(ncon), _p(xadj, I32P),
                               _p(adjncy, I32P), _p(vwgt, I32P), _p(adjwgt, I32P), _p(part, I32P), _p(tp, F64P),
                               _p(ub, F64P), ctypes.c_int64(niter))
    return part, int(cut)


def part_graph_recursive(xadj, adjncy, nparts, vwgt=None, adjwgt=None, ncon=1, tpwgts=None, ubvec=None,
                         options=None):
    """Restated RMETIS_PartGraphRecursive (src/ffi/c_api.rs:27-53,
    src/partition/recursive.rs:12-187). Returns (rc, part, objval)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    n = len(xadj) - 1
    part = np.zeros(n, dtype=np.int32)
    obj = ctypes.c_int32(0)
    nv = ctypes.c_int32(n); nc = ctypes.c_int32(ncon); npr = ctypes.c_int32(nparts)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    op = None if options is None else _i32(options)
    rc = lib().orc_PartGraphRecursive(ctypes.byref(nv), ctypes.byref(nc), _p(xadj, I32P), _p(adjncy, I32P),
                                      _p(vwgt, I32P), None, _p(adjwgt, I32P), ctypes.byref(npr), _p(tp, F32P),
                                      _p(ub, F32P), _p(op, I32P), ctypes.byref(obj), _p(part, I32P))
    return rc, part, int(obj.value)


def node_nd(xadj, adjncy, vwgt=None, options=None):
    """Restated RMETIS_NodeND (src/ffi/c_api.rs:85-132, src/partition/nd.rs).
    Returns (rc, perm, iperm)."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt)
    n = len(xadj) - 1
    perm = np.zeros(n, dtype=np.int32)
    iperm = np.zeros(n, dtype=np.int32)
    nv = ctypes.c_int32(n)
    op = None if options is None else _i32(options)
    rc = lib().orc_NodeND(ctypes.byref(nv), _p(xadj, I32P), _p(adjncy, I32P), _p(vwgt, I32P), _p(op, I32P),
                          _p(perm, I32P), _p(iperm, I32P))
    return rc, perm, iperm


def part_graph_kway(xadj, adjncy, nparts, vwgt=None, adjwgt=None, ncon=1, tpwgts=None, ubvec=None,
                    options=None, script=None, with_stats=False):
    """Restated RMETIS_PartGraphKway. script = (matchings list, seeds) replays
    given random choices. Returns (rc, part, objval[, stats])."""
    xadj = _i32(xadj); adjncy = _i32(adjncy); vwgt = _i32(vwgt); adjwgt = _i32(adjwgt)
    n = len(xadj) - 1
    part = np.zeros(n, dtype=np.int32)
    obj = ctypes.c_int32(0)
    nv = ctypes.c_int32(n); nc = ctypes.c_int32(ncon); npr = ctypes.c_int32(nparts)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, dtype=np.float32)
    op = None if options is None else _i32(options)
    sm = so = ss = None
    nl = 0
    if script is not None:
        mats, seeds = script
        if mats is not None:
            sm = np.concatenate([np.asarray(m, dtype=np.int32) for m in mats]) if mats else np.zeros(1, np.int32)
            so = np.zeros(len(mats) + 1, dtype=np.int64)
            so[1:] = np.cumsum([len(m) for m in mats])
            nl = len(mats)
        ss = None if seeds is None else _i32(seeds)
    stats = np.zeros(130, dtype=np.int64)
    rc = lib().orc_PartGraphKway_script(
        ctypes.byref(nv), ctypes.byref(nc), _p(xadj, I32P), _p(adjncy, I32P), _p(vwgt, I32P), None,
        _p(adjwgt, I32P), ctypes.byref(npr), _p(tp, F32P), _p(ub, F32P), _p(op, I32P), ctypes.byref(obj),
        _p(part, I32P), _p(sm, I32P), _p(so, I64P), ctypes.c_int64(nl), _p(ss, I32P), _p(stats, I64P))
    if with_stats:
        nlev = int(stats[0])
        st = dict(nlevels=nlev, level_n=[int(stats[1 + 2 * i]) for i in range(nlev + 1)],
                  level_m=[int(stats[2 + 2 * i]) for i in range(nlev + 1)])
        return rc, part, int(obj.value), st
    return rc, part, int(obj.value)
