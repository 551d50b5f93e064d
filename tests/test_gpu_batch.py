"""Concurrent work on one device: ncuts attempts on the worker pool, many graphs
in one batched call, and asynchronous requests. Each must give exactly the
partition that the plain one-graph, one-attempt-after-another call gives (the
reference partitions one graph per call and runs its attempts in a loop,
src/partition/kway.rs:54-99)."""
import ctypes

import numpy as np
import pytest

from rmetis_b200 import generators as G

pytestmark = pytest.mark.gpu


def greedy(seed, ncuts=1, ufactor=30):
    import rmetis_b200 as rmb
    return rmb.Options(rtype=rmb.RType.Greedy, seed=seed, ncuts=ncuts, ufactor=ufactor)


def graph_of(rmb, x, a, v=None, w=None, ncon=1):
    return rmb.Graph.new(len(x) - 1, ncon, x, a, vwgt=v, adjwgt=w)


@pytest.fixture
def restore_parallel(rmb):
    yield
    rmb.set_tuning(parallel_attempts=1)


@pytest.mark.parametrize("ncuts", [2, 5])
def test_parallel_attempts_equal_sequential(rmb, restore_parallel, ncuts):
    x, a, v, w = G.grid3d(20, weights_seed=3)
    g = graph_of(rmb, x, a, v, w)
    rmb.set_tuning(parallel_attempts=0)
    seq = rmb.part_graph_kway(g, 16, options=greedy(11, ncuts))
    rmb.set_tuning(parallel_attempts=1)
    par = rmb.part_graph_kway(g, 16, options=greedy(11, ncuts))
    assert par.objval == seq.objval
    np.testing.assert_array_equal(par.part, seq.part)
    one = rmb.part_graph_kway(g, 16, options=greedy(11, 1))
    assert par.objval <= one.objval


def test_parallel_attempts_keep_first_minimum(rmb):
    """Attempt a uses seed + a (src/partition/kway.rs:55-61): the best of
    ncuts attempts is the first single-attempt run with the lowest cut."""
    x, a = G.grid2d(40, 40)
    g = graph_of(rmb, x, a)
    runs = [rmb.part_graph_kway(g, 8, options=greedy(100 + s, 1)) for s in range(4)]
    best = min(range(4), key=lambda i: (runs[i].objval, i))
    par = rmb.part_graph_kway(g, 8, options=greedy(100, 4))
    assert par.objval == runs[best].objval
    np.testing.assert_array_equal(par.part, runs[best].part)


def _uneven_batch(ncon=1, count=12, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(300, 6000))
        x, a, w, _pts = G.rgg2d(n, int(rng.integers(1 << 30)), mean_degree=6.0)
        v = rng.integers(1, 5, size=n * ncon).astype(np.int32)
        out.append((x, a, v, w))
    return out


@pytest.mark.parametrize("ncon", [1, 2])
def test_batch_equals_individual_calls(rmb, ncon):
    graphs = [graph_of(rmb, x, a, v, w, ncon) for x, a, v, w in _uneven_batch(ncon)]
    ks = [4 + 3 * (i % 5) for i in range(len(graphs))]
    batch = rmb.part_graph_kway_batch(graphs, ks, options=greedy(9, ufactor=50))
    for g, k, r in zip(graphs, ks, batch):
        solo = rmb.part_graph_kway(g, k, options=greedy(9, ufactor=50))
        assert r.objval == solo.objval
        np.testing.assert_array_equal(r.part, solo.part)


def test_batch_reports_bad_graph_without_losing_others(rmb):
    """Through the C ABI: a graph with nparts > nvtxs gets METIS_ERROR_INPUT
    in its status slot and the call returns it, while the other graphs of the
    batch are still partitioned."""
    x1, a1 = G.grid2d(30, 30)
    x2, a2 = G.path(3)
    good = graph_of(rmb, x1, a1)
    I32P, I64P = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)
    vtx_off = np.array([0, 900, 903], np.int64)
    edge_off = np.array([0, len(a1), len(a1) + len(a2)], np.int64)
    xadj = np.concatenate([x1, x2]).astype(np.int32)
    adj = np.concatenate([a1, a2]).astype(np.int32)
    nps = np.array([4, 8], np.int32)
    part = np.full(903, -1, np.int32)
    obj = np.zeros(2, np.int32)
    status = np.zeros(2, np.int32)
    opts = greedy(1).c_array()
    p = lambda arr, t=I32P: arr.ctypes.data_as(t)
    rc = rmb._lib.load().RMETIS_GPU_PartGraphKwayBatch(2, 1, p(vtx_off, I64P), p(edge_off, I64P), p(xadj), p(adj),
                                                       None, None, p(nps), None, p(opts), p(obj), p(part),
                                                       p(status))
    assert rc == -2
    assert list(status) == [1, -2]
    solo = rmb.part_graph_kway(good, 4, options=greedy(1))
    assert obj[0] == solo.objval
    np.testing.assert_array_equal(part[:900], solo.part)


def test_async_requests_equal_sync_calls(rmb):
    """Requests that overlap on the device give the results they give alone."""
    graphs = [graph_of(rmb, x, a, v, w) for x, a, v, w in _uneven_batch(count=10, seed=8)]
    reqs = [rmb.submit_kway(g, 6 + i % 4, options=greedy(3 + i)) for i, g in enumerate(graphs)]
    results = [r.wait() for r in reqs]
    for i, (g, r) in enumerate(zip(graphs, results)):
        solo = rmb.part_graph_kway(g, 6 + i % 4, options=greedy(3 + i))
        assert r.objval == solo.objval
        np.testing.assert_array_equal(r.part, solo.part)
        assert reqs[i].done()


def test_async_error_codes(rmb):
    import rmetis_b200 as rmb_mod
    x, a = G.grid2d(10, 10)
    g = graph_of(rmb, x, a)
    bad = rmb_mod.Graph(4, 1, np.array([0, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 0]), validate=False)
    with pytest.raises(rmb_mod.InputError):                    # asymmetric: found by the device validation
        rmb.submit_kway(bad, 2, options=rmb_mod.Options(rtype=rmb_mod.RType.Greedy, seed=1)).wait()
    lib = rmb._lib.load()
    assert lib.RMETIS_GPU_WaitKway(123456789) == -2
    assert lib.RMETIS_GPU_PollKway(123456789) == -2


def test_ranks_path_single_rank_equals_plain(rmb):
    """The rank-striped best-of-ncuts with one rank runs every attempt there
    and equals the plain call's best of ncuts."""
    import socket
    import torch.distributed as dist
    from rmetis_b200 import distributed as D
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        x, a, v, w = G.grid3d(18, weights_seed=6)
        g = graph_of(rmb, x, a, v, w)
        res = D.part_graph_kway_ranks(g, 12, options=greedy(21, 4))
        plain = rmb.part_graph_kway(g, 12, options=greedy(21, 4))
        assert res.objval == plain.objval
        np.testing.assert_array_equal(res.part, plain.part)
    finally:
        dist.destroy_process_group()
