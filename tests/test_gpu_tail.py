"""The single-block coarse tail (every coarsening level from a small level on,
in one launch) produces exactly the levels of the host loop
(src/coarsen/mod.rs:36-71): the same matching at every level, the same grow
seeds and the same partition, whether the tail starts at the input graph,
part-way down, or not at all."""
import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests.test_gpu_parity import GRAPHS, load

pytestmark = pytest.mark.gpu

DEFAULT_TAIL = 4096


def _traced(rmb, g, k, o, tail, ubvec=None):
    rmb.set_tuning(tail_max_n=tail)
    try:
        return rmb.part_graph_kway_trace(g, k, ubvec=ubvec, options=o)
    finally:
        rmb.set_tuning(tail_max_n=DEFAULT_TAIL)


def _assert_same(a, b):
    ra, ma, sa, _ = a
    rb, mb, sb, _ = b
    assert len(ma) == len(mb)
    for lvl, (x, y) in enumerate(zip(ma, mb)):
        np.testing.assert_array_equal(x, y, err_msg=f"matching of level {lvl}")
    np.testing.assert_array_equal(sa, sb)
    assert ra.objval == rb.objval
    np.testing.assert_array_equal(ra.part, rb.part)


def _opts(rmb, seed, ctype):
    return rmb.Options(rtype=rmb.RType.Greedy, seed=seed, ctype=ctype)


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [4, 64])
@pytest.mark.parametrize("ctype", ["Shem", "Rm"])
def test_tail_from_the_input_equals_host_loop(rmb, name, k, ctype):
    x, a, v, w = load(name)
    g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
    o = _opts(rmb, 5 + k, getattr(rmb.CType, ctype))
    _assert_same(_traced(rmb, g, k, o, 1 << 30), _traced(rmb, g, k, o, 0))


@pytest.mark.parametrize("case", ["grid3d_24_w", "rmat_13", "rgg_20k"])
def test_tail_part_way_down_equals_host_loop(rmb, case):
    if case == "grid3d_24_w":
        x, a, v, w = G.grid3d(24, weights_seed=9)
    elif case == "rmat_13":
        (x, a), v, w = G.rmat(13, seed=4), None, None
    else:
        x, a, w, _ = G.rgg2d(20000, 17, mean_degree=8.0)
        v = None
    g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
    o = _opts(rmb, 2, rmb.CType.Shem)
    for k in (8, 48):
        on = _traced(rmb, g, k, o, DEFAULT_TAIL)
        assert len(on[1]) >= 2
        _assert_same(on, _traced(rmb, g, k, o, 0))


def test_tail_three_constraints(rmb):
    x, a, _, w = G.random_graph(6000, 8.0, seed=41)
    n = len(x) - 1
    v = np.random.default_rng(3).integers(1, 20, 3 * n).astype(np.int32)
    g = rmb.Graph(n, 3, x, a, vwgt=v, adjwgt=w)
    o = _opts(rmb, 7, rmb.CType.Shem)
    ub = np.array([1.05, 1.1, 1.2], np.float32)
    _assert_same(_traced(rmb, g, 16, o, 1 << 30, ub), _traced(rmb, g, 16, o, 0, ub))


def test_tail_summed_unit_weights(rmb):
    """A graph without vertex weights whose coarse levels get summed weights."""
    x, a = G.grid2d(70, 60)
    g = rmb.Graph(len(x) - 1, 1, x, a)
    o = _opts(rmb, 4, rmb.CType.Shem)
    rmb.set_tuning(summed_unit_weights=1)
    try:
        _assert_same(_traced(rmb, g, 10, o, 1 << 30), _traced(rmb, g, 10, o, 0))
    finally:
        rmb.set_tuning(summed_unit_weights=0)


def test_tail_stops_before_fewer_vertices_than_parts(rmb):
    """A contraction to fewer than k vertices is dropped and the finer level
    kept, inside the tail as in the host loop."""
    x, a = G.path(40)
    g = rmb.Graph(40, 1, x, a)
    o = _opts(rmb, 1, rmb.CType.Shem)
    on = _traced(rmb, g, 30, o, 1 << 30)
    assert len(on[1]) == 1  # one matching computed, its contraction dropped
    _assert_same(on, _traced(rmb, g, 30, o, 0))


def test_tail_batch_and_attempts(rmb):
    """Batched graphs and concurrent ncuts attempts on worker engines use the
    tail too and still equal the host loop."""
    specs = [G.rgg2d(int(n), s, mean_degree=7.0) for n, s in ((1500, 1), (5000, 2), (12000, 3))]
    graphs = [rmb.Graph(len(x) - 1, 1, x, a, adjwgt=w) for x, a, w, _ in specs]
    o = rmb.Options(rtype=rmb.RType.Greedy, seed=8, ncuts=3)
    rmb.set_tuning(tail_max_n=0)
    try:
        off = rmb.part_graph_kway_batch(graphs, [6, 12, 24], options=o)
    finally:
        rmb.set_tuning(tail_max_n=DEFAULT_TAIL)
    on = rmb.part_graph_kway_batch(graphs, [6, 12, 24], options=o)
    for r0, r1 in zip(off, on):
        assert r0.objval == r1.objval
        np.testing.assert_array_equal(r0.part, r1.part)
