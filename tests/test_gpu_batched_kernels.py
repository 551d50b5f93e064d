"""The batched launches of RMETIS_GPU_PartGraphKwayBatch (batch.cu): every
graph of a batch goes through validation, coarsening, grow trials, the
refinement of its levels and the cut in one launch per step, one block per
graph. Each result must equal the single call's for that graph, bit for bit
(src/partition/kway.rs:20-99 per graph), whichever path a graph takes:
the batched kernels, or the worker pool for graphs they do not take
(k > 256, ncon > 2, other options) or cannot finish.

The batch mixes what changes the kernel variant or the path of a level:
vertex and edge weights present or not, one or two constraints, k in every
walk bucket (<= 32, <= 64, <= 128, <= 256) and above, levels large enough for
the parallel admission (more than 16,384 vertices), isolated vertices (grow
leftovers), a graph barely larger than k, and an invalid graph.
"""
import ctypes

import numpy as np
import pytest

from rmetis_b200 import generators as G

pytestmark = pytest.mark.gpu


def greedy(rmb, seed, ufactor=30, **kw):
    return rmb.Options(rtype=rmb.RType.Greedy, seed=seed, ufactor=ufactor, **kw)


def graph_of(rmb, x, a, v=None, w=None, ncon=1):
    return rmb.Graph.new(len(x) - 1, ncon, x, a, vwgt=v, adjwgt=w)


@pytest.fixture
def batch_mode(rmb):
    yield
    rmb.set_batch_mode(1, 262144)


def _check(rmb, graphs, ks, opts):
    """Batched launches for every eligible graph; every graph on the pool;
    and graphs above 5,000 vertices on the pool while the batched launches
    run the others."""
    rmb.set_batch_mode(1, 1 << 30)
    batch = rmb.part_graph_kway_batch(graphs, ks, options=opts)
    rmb.set_batch_mode(0)
    pool = rmb.part_graph_kway_batch(graphs, ks, options=opts)
    rmb.set_batch_mode(1, 5000)
    mixed = rmb.part_graph_kway_batch(graphs, ks, options=opts)
    rmb.set_batch_mode(1, 262144)
    for i, (g, k, r, q, x) in enumerate(zip(graphs, ks, batch, pool, mixed)):
        solo = rmb.part_graph_kway(g, k, options=opts)
        for res in (r, q, x):
            assert res.objval == solo.objval, (i, k, res.objval, solo.objval)
            np.testing.assert_array_equal(res.part, solo.part)
    return batch


def test_batched_weighted_sizes_and_buckets(rmb, batch_mode):
    """Vertex and edge weights; k in every walk bucket and above 256;
    levels above 16,384 vertices (parallel admission)."""
    rng = np.random.default_rng(3)
    graphs, ks = [], []
    for i, n in enumerate([40000, 25000, 9000, 3000, 1200, 700]):
        x, a, w, _ = G.rgg2d(n, 100 + i, mean_degree=8.0)
        v = rng.integers(1, 6, size=n).astype(np.int32)
        graphs.append(graph_of(rmb, x, a, v, w))
        ks.append([8, 64, 100, 200, 16, 300][i])           # 300 > 256: the worker pool
    x, a, v, w = G.grid3d(30, 28, 26, weights_seed=2)        # weighted 3D grid, 21,840 vertices
    graphs.append(graph_of(rmb, x, a, v, w))
    ks.append(48)
    res = _check(rmb, graphs, ks, greedy(rmb, 5))
    for k, r in zip(ks, res):
        assert r.part.min() >= 0 and r.part.max() < k


def test_batched_unweighted(rmb, batch_mode):
    """No weights at all (the input level has no edge weights); a graph barely
    larger than k; isolated vertices (the grow's leftovers)."""
    graphs, ks = [], []
    x, a = G.grid2d(150, 150)                                 # 22,500 vertices
    graphs.append(graph_of(rmb, x, a))
    ks.append(32)
    x, a = G.grid2d(4, 5)
    graphs.append(graph_of(rmb, x, a))
    ks.append(16)
    x, a, _, _ = G.rgg2d(5000, 7, mean_degree=1.5)
    graphs.append(graph_of(rmb, x, a))
    ks.append(12)
    x, a, _, _ = G.rgg2d(12000, 8, mean_degree=7.0)
    graphs.append(graph_of(rmb, x, a))
    ks.append(130)
    _check(rmb, graphs, ks, greedy(rmb, 6))


def test_batched_two_constraints_many_graphs(rmb, batch_mode):
    rng = np.random.default_rng(11)
    graphs, ks = [], []
    for i in range(40):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(30000))))
        x, a, w, _ = G.rgg2d(n, 1000 + i, mean_degree=10.0)
        v = rng.integers(1, 9, size=2 * n).astype(np.int32)
        graphs.append(graph_of(rmb, x, a, v, w, ncon=2))
        ks.append(int(rng.choice([2, 4, 8, 16, 32, 64])))
    _check(rmb, graphs, ks, greedy(rmb, 1, ufactor=50))


def test_batched_summed_unit_weights_and_rm(rmb, batch_mode):
    graphs, ks = [], []
    for i, n in enumerate([20000, 6000, 2500]):
        x, a, w, _ = G.rgg2d(n, 300 + i, mean_degree=9.0)
        graphs.append(graph_of(rmb, x, a, None, w))
        ks.append([24, 8, 40][i])
    rmb.set_tuning(summed_unit_weights=1)
    try:
        _check(rmb, graphs, ks, greedy(rmb, 2))
    finally:
        rmb.set_tuning(summed_unit_weights=0)
    _check(rmb, graphs, ks, greedy(rmb, 4, ctype=rmb.CType.Rm))


def test_batched_invalid_graph_keeps_others(rmb, batch_mode):
    """An asymmetric graph is found by the batched validation: its status is
    METIS_ERROR_INPUT and the other graphs are partitioned as alone."""
    x1, a1 = G.grid2d(40, 40)
    xb = np.array([0, 2, 4, 6, 8], np.int32)
    ab = np.array([1, 3, 0, 2, 1, 3, 0, 0], np.int32)      # vertex 3 lists 0 twice: asymmetric
    x3, a3, w3, _ = G.rgg2d(3000, 9, mean_degree=8.0)
    I32P, I64P = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)
    ns = [1600, 4, 3000]
    ms = [len(a1), len(ab), len(a3)]
    vtx_off = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    edge_off = np.concatenate([[0], np.cumsum(ms)]).astype(np.int64)
    xadj = np.concatenate([x1, xb, x3]).astype(np.int32)
    adj = np.concatenate([a1, ab, a3]).astype(np.int32)
    w = np.concatenate([np.ones(len(a1), np.int32), np.ones(len(ab), np.int32), w3]).astype(np.int32)
    nps = np.array([8, 2, 16], np.int32)
    part = np.full(sum(ns), -1, np.int32)
    obj = np.zeros(3, np.int32)
    status = np.zeros(3, np.int32)
    opts = greedy(rmb, 3).c_array()
    p = lambda arr, t=I32P: arr.ctypes.data_as(t)
    rmb.set_batch_mode(1)
    rc = rmb._lib.load().RMETIS_GPU_PartGraphKwayBatch(3, 1, p(vtx_off, I64P), p(edge_off, I64P), p(xadj), p(adj),
                                                       None, p(w), p(nps), None, p(opts), p(obj), p(part),
                                                       p(status))
    assert rc == -2
    assert list(status) == [1, -2, 1]
    for gi, (x, a, ww, k) in enumerate([(x1, a1, np.ones(len(a1), np.int32), 8), (x3, a3, w3, 16)]):
        solo = rmb.part_graph_kway(graph_of(rmb, x, a, None, ww), k, options=greedy(rmb, 3))
        lo = 0 if gi == 0 else 1604
        assert obj[0 if gi == 0 else 2] == solo.objval
        np.testing.assert_array_equal(part[lo:lo + len(x) - 1], solo.part)


def test_submitted_requests_batched_equal_sync_calls(rmb, batch_mode):
    """Continuous batching: submitted requests that the batched kernels can take
    are collected by the device's dispatcher while earlier batches run, grouped
    by options, and partitioned together; each result equals the synchronous
    call's. The requests mix seeds, ufactors (two groups), k buckets, a graph
    above the batch size limit (the pool) and an invalid graph."""
    rng = np.random.default_rng(21)
    reqs = []
    for i in range(30):
        n = int(rng.integers(500, 12000))
        x, a, w, _ = G.rgg2d(n, 700 + i, mean_degree=8.0)
        v = rng.integers(1, 5, size=n).astype(np.int32) if i % 3 else None
        g = graph_of(rmb, x, a, v, w)
        reqs.append((g, int(rng.choice([4, 16, 40, 100])), greedy(rmb, 100 + i, ufactor=30 if i % 2 else 50)))
    rmb.set_batch_mode(1, 8000)   # graphs above 8,000 vertices on the pool
    try:
        tickets = [rmb.submit_kway(g, k, options=o) for g, k, o in reqs]
        bad = rmb.Graph(4, 1, np.array([0, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 0]), validate=False)
        bad_t = rmb.submit_kway(bad, 2, options=greedy(rmb, 1))
        results = [t.wait() for t in tickets]
        with pytest.raises(rmb.InputError):
            bad_t.wait()
    finally:
        rmb.set_batch_mode(1, 262144)
    for (g, k, o), r in zip(reqs, results):
        solo = rmb.part_graph_kway(g, k, options=o)
        assert r.objval == solo.objval
        np.testing.assert_array_equal(r.part, solo.part)
