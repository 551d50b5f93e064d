"""RMETIS_NodeND (nested dissection ordering) through the C ABI, against the
oracle's restatement of src/partition/nd.rs and src/separator/mod.rs.

The orderings come from different bisections (the GPU's parallel matching and
refinement), so they are compared by what an ordering is for: the fill of
the Cholesky factor it produces, summed over seeds, within 5% of the
oracle's. The reference's own test (nd.rs:115-150) and its C-ABI checks are
checked exactly.
"""
import ctypes

import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests.conftest import greedy_options

pytestmark = pytest.mark.gpu

I32P = ctypes.POINTER(ctypes.c_int32)


def nodend(rmb, x, a, vwgt=None, options=None):
    lib = rmb._lib.load()
    n = len(x) - 1
    keep = [np.ascontiguousarray(z, np.int32) if z is not None else None for z in (x, a, vwgt, options)]
    p = lambda z: None if z is None else z.ctypes.data_as(I32P)
    perm = np.full(n, -1, np.int32)
    iperm = np.full(n, -1, np.int32)
    rc = lib.RMETIS_NodeND(ctypes.byref(ctypes.c_int32(n)), p(keep[0]), p(keep[1]), p(keep[2]), p(keep[3]),
                           p(perm), p(iperm))
    return rc, perm, iperm


def factor_nnz(x, a, perm):
    """Entries of the Cholesky factor L (below the diagonal) of a matrix with
    this graph, eliminated in the order perm (perm[v] = position of v)."""
    n = len(x) - 1
    iperm = np.empty(n, np.int64)
    iperm[perm] = np.arange(n)
    children = [[] for _ in range(n)]
    struct = [None] * n
    total = 0
    for k in range(n):
        v = iperm[k]
        s = {int(perm[u]) for u in a[x[v]:x[v + 1]] if perm[u] > k}
        for c in children[k]:
            s |= struct[c]
            struct[c] = None
        s.discard(k)
        struct[k] = s
        total += len(s)
        if s:
            children[min(s)].append(k)
    return total


def check_perm(perm, iperm):
    n = len(perm)
    assert sorted(perm.tolist()) == list(range(n))
    assert (perm[iperm] == np.arange(n)).all()


def _options(seed):
    o = greedy_options(seed=seed)
    o[4] = 0  # rtype Fm: the reference's default, which node_nd passes on
    return o


def test_path10_reference_case(rmb):
    """nd.rs:115-150: a 10-vertex path with seed 42 gives a permutation and
    its inverse (at most 100 vertices: the identity order)."""
    x, a = G.path(10)
    rc, perm, iperm = nodend(rmb, x, a, options=_options(42))
    assert rc == 1
    check_perm(perm, iperm)
    assert (perm == np.arange(10)).all()


def test_nodend_errors(rmb):
    lib = rmb._lib.load()
    x, a = G.grid2d(4, 4)
    perm = np.zeros(16, np.int32)
    p = lambda z: z.ctypes.data_as(I32P)
    assert lib.RMETIS_NodeND(None, p(x), p(a), None, None, p(perm), p(perm)) == -2
    assert lib.RMETIS_NodeND(ctypes.byref(ctypes.c_int32(0)), p(x), p(a), None, None, p(perm), p(perm)) == -2
    bad = a.copy()
    bad[0] = 0  # a self-loop fails validation
    assert nodend(rmb, x, bad)[0] == -2


@pytest.mark.parametrize("name", ["grid2d_60", "grid3d_16", "rgg_6k", "grid2d_90_weighted"])
def test_nodend_fill_close_to_oracle(rmb, oracle, name):
    vw = None
    if name == "grid2d_60":
        x, a = G.grid2d(60, 60)
    elif name == "grid3d_16":
        x, a, _, _ = G.grid3d(16)
    elif name == "rgg_6k":
        x, a, _, _ = G.rgg2d(6000, 7)
    else:
        x, a = G.grid2d(90, 90)
        vw = np.random.default_rng(3).integers(1, 5, len(x) - 1).astype(np.int32)
    gpu = ref = 0
    for seed in (1, 2, 3):
        rc, perm, iperm = nodend(rmb, x, a, vwgt=vw, options=_options(seed))
        assert rc == 1
        check_perm(perm, iperm)
        rc2, perm2, _ = nodend(rmb, x, a, vwgt=vw, options=_options(seed))
        assert rc2 == 1 and (perm2 == perm).all(), "same seed, same ordering"
        orc, operm, oiperm = oracle.node_nd(x, a, vwgt=vw, options=_options(seed))
        assert orc == 1
        gpu += factor_nnz(x, a, perm)
        ref += factor_nnz(x, a, operm)
    assert gpu <= 1.05 * ref, (gpu, ref)


def test_python_node_nd(rmb):
    x, a = G.grid2d(40, 40)
    g = rmb.Graph.new_unweighted(len(x) - 1, x, a)
    res = rmb.node_nd(g, rmb.Options(seed=5))
    check_perm(res.perm, res.iperm)
    rc, perm, _ = nodend(rmb, x, a, options=rmb.Options(seed=5).c_array())
    assert rc == 1 and (perm == res.perm).all()
