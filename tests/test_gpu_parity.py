"""Bit-exact parity of the CUDA path against the oracle, through the C ABI.

Covers every RNG-free function of the hot path (edge cut, partition weights,
contraction given a matching, projection, gain table, grow given seeds,
greedy refinement given a partition) and the whole pipeline replayed with the
GPU's own random choices (matchings, grow seeds).
"""
import numpy as np
import pytest

from rmetis_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def exact_refinement(rmb):
    """Every pass of RMETIS_GPU_GreedyRefine the reference's sequential pass:
    levels above the refine-mode threshold (default 16384 vertices) would
    otherwise decide their cut passes by parallel admission."""
    rmb.set_refine_mode(-1)
    yield
    rmb.set_refine_mode(16384)


def star_graph(n_leaves, hub_extra=0, seed=0):
    """A hub joined to every leaf, leaves chained in a path (heavy rows)."""
    n = n_leaves + 1
    edges = [(0, i) for i in range(1, n)] + [(i, i + 1) for i in range(1, n - 1)]
    src = np.array([a for a, b in edges] + [b for a, b in edges])
    dst = np.array([b for a, b in edges] + [a for a, b in edges])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    xadj = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=xadj[1:])
    rng = np.random.default_rng(seed)
    w = G.symmetric_edge_weights(xadj.astype(np.int32), dst.astype(np.int32), rng, 1, 5)
    return xadj.astype(np.int32), dst.astype(np.int32), w


GRAPHS = {
    "grid2d_30x17": lambda: (*G.grid2d(30, 17), None, None),
    "grid3d_9x8x7_w": lambda: G.grid3d(9, 8, 7, weights_seed=3),
    "random_2k": lambda: G.random_graph(2000, 9.0, seed=5),
    "random_3k_deg40": lambda: G.random_graph(3000, 40.0, seed=6),
    "star_300": lambda: (*star_graph(300)[:2], None, star_graph(300)[2]),
    "star_1500": lambda: (*star_graph(1500)[:2], None, star_graph(1500)[2]),
}


def load(name):
    x, a, v, w = GRAPHS[name]()
    return np.asarray(x, np.int32), np.asarray(a, np.int32), v, w


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [2, 7, 64])
def test_edge_cut_and_weights(rmb, oracle, name, k):
    x, a, v, w = load(name)
    n = len(x) - 1
    part = np.random.default_rng(k).integers(0, k, n).astype(np.int32)
    g = rmb.Graph(n, 1, x, a, vwgt=v, adjwgt=w)
    assert g.edge_cut(part) == oracle.edge_cut(x, a, w, part)
    assert (g.partition_weights(part, k) == oracle.partition_weights(n, 1, v, part, k)).all()


def _check_contraction(rmb, oracle, x, a, v, w, m, ncon=1):
    n = len(x) - 1
    g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
    cg, cmap = g.build_coarse_graph(m)
    ref = oracle.build_coarse_graph(x, a, m, vwgt=v, adjwgt=w, ncon=ncon)
    assert cg.nvtxs == ref["cn"]
    assert (cmap == ref["cmap"]).all()
    assert (cg.xadj == ref["cxadj"]).all()
    assert (cg.adjncy == ref["cadjncy"]).all()
    gw = cg.adjwgt if cg.adjwgt is not None else np.ones(len(cg.adjncy), np.int32)
    assert (gw == ref["cadjwgt"]).all()
    assert (cg.adjwgt is not None) == ref["keeps_adjwgt"]
    if v is not None:
        assert (cg.vwgt == ref["cvwgt"]).all()


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("source", ["shem", "rm", "gpu"])
@pytest.mark.parametrize("thread_max", [16, 32])
def test_contraction_bit_exact(rmb, oracle, name, source, thread_max):
    """Rows merged by one thread (bound up to thread_max) and by a warp give
    the same coarse graph."""
    from rmetis_b200 import functions as F
    rmb.set_kernel_shapes(contract_thread_max=thread_max)
    x, a, v, w = load(name)
    n = len(x) - 1
    if source == "shem":
        m = oracle.shem_matching(x, a, w, oracle.SmallRng(11))
    elif source == "rm":
        m = oracle.random_matching(x, a, oracle.SmallRng(12))
    else:
        m = F.match(rmb.Graph(n, 1, x, a, adjwgt=w), mode=1, seed=13)
    try:
        _check_contraction(rmb, oracle, x, a, v, w, m)
    finally:
        rmb.set_kernel_shapes(contract_thread_max=32)


@pytest.mark.parametrize("source", ["shem", "gpu"])
@pytest.mark.parametrize("thread_max", [16, 32])
def test_contraction_isolated_vertices(rmb, oracle, source, thread_max):
    """R-MAT keeps thousands of isolated vertices: runs of coarse vertices
    whose merged rows are all empty (empty ranges in the compaction), short
    rows beside hub rows, and ranges that start and end off a multiple of
    four entries."""
    from rmetis_b200 import functions as F
    rmb.set_kernel_shapes(contract_thread_max=thread_max)
    x, a = G.rmat(13, seed=21)
    n = len(x) - 1
    assert int((np.diff(x) == 0).sum()) > 1000
    if source == "shem":
        m = oracle.shem_matching(x, a, None, oracle.SmallRng(14))
    else:
        m = F.match(rmb.Graph(n, 1, x, a), mode=1, seed=15)
    try:
        _check_contraction(rmb, oracle, x, a, None, None, m)
    finally:
        rmb.set_kernel_shapes(contract_thread_max=32)


def test_contraction_multiconstraint(rmb, oracle):
    x, a, _, w = G.random_graph(1500, 8.0, seed=9)
    n = len(x) - 1
    v = np.random.default_rng(1).integers(1, 9, 2 * n).astype(np.int32)
    m = oracle.shem_matching(x, a, w, oracle.SmallRng(3))
    _check_contraction(rmb, oracle, x, a, v, w, m, ncon=2)


def test_contraction_reference_path4(rmb):
    # src/graph/mod.rs:498-514
    g = rmb.Graph.new_unweighted(4, [0, 1, 3, 5, 6], [1, 0, 2, 1, 3, 2])
    cg, cmap = g.build_coarse_graph([1, 0, 3, 2])
    assert cg.nvtxs == 2 and cg.nedges == 1
    assert cmap[0] == cmap[1] and cmap[2] == cmap[3] and cmap[0] != cmap[2]


def test_projection(rmb):
    from rmetis_b200 import functions as F
    rng = np.random.default_rng(0)
    cmap = rng.integers(0, 500, 3000).astype(np.int32)
    cp = rng.integers(0, 16, 500).astype(np.int32)
    assert (F.project(cmap, cp) == cp[cmap]).all()


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [2, 5, 40])
def test_gain_table_matches_compute_move_gain(rmb, oracle, name, k):
    x, a, v, w = load(name)
    n = len(x) - 1
    # a partition with structure (blocks of ids) plus noise
    rng = np.random.default_rng(k)
    part = ((np.arange(n) * k) // n).astype(np.int32)
    flip = rng.random(n) < 0.1
    part[flip] = rng.integers(0, k, flip.sum())
    g = rmb.Graph(n, 1, x, a, adjwgt=w)
    b, nc, wf, cp, cg = g.gain_table(part, k)
    bref = oracle.boundary_vertices(x, a, part)
    assert (np.nonzero(b)[0] == bref).all()
    lib = oracle.lib()
    for vv in bref[:: max(1, len(bref) // 150)]:
        s = x[vv]
        exp = {int(cp[s + i]): int(cg[s + i]) for i in range(nc[vv])}
        gains = [(exp.get(p, int(np.int32(-wf[vv]))), p) for p in range(k) if p != part[vv]]
        for gval, p in gains:
            assert gval == oracle.compute_move_gain(x, a, w, int(vv), part, int(part[vv]), p), (vv, p)
        # explicit list is sorted by (gain desc, part asc)
        keys = [(-int(cg[s + i]), int(cp[s + i])) for i in range(nc[vv])]
        assert keys == sorted(keys)


@pytest.mark.parametrize("name", ["grid2d_30x17", "grid3d_9x8x7_w", "random_2k", "star_300"])
@pytest.mark.parametrize("k", [2, 6, 24])
def test_grow_exact_given_seeds(rmb, oracle, name, k):
    from rmetis_b200 import functions as F
    x, a, v, w = load(name)
    n = len(x) - 1
    t = oracle.compute_target_weights(n, 1, v, k)
    rng = np.random.default_rng(k + n)
    seeds = np.stack([rng.choice(n, k, replace=False) for _ in range(5)]).astype(np.int32)
    g = rmb.Graph(n, 1, x, a, vwgt=v, adjwgt=w)
    parts, cuts = F.grow_partition(g, k, t, seeds)
    for tr in range(len(seeds)):
        ref, _ = oracle.grow_partition(x, a, k, t, vwgt=v, seeds=seeds[tr])
        assert (parts[tr] == ref).all(), tr
        assert cuts[tr] == 2 * oracle.edge_cut(x, a, w, ref) or cuts[tr] == 2 * oracle.edge_cut(x, a, w, ref) + 1


def test_grow_disconnected_leftovers(rmb, oracle):
    from rmetis_b200 import functions as F
    # two grids side by side without edges between them plus isolated vertices
    x1, a1 = G.grid2d(6, 6)
    n1 = 36
    x = np.concatenate([x1, x1[1:] + x1[-1], np.full(5, 2 * x1[-1])]).astype(np.int32)
    a = np.concatenate([a1, a1 + n1]).astype(np.int32)
    n = len(x) - 1
    k = 3
    t = oracle.compute_target_weights(n, 1, None, k)
    seeds = np.array([[0, 5, 7]], np.int32)
    parts, _ = F.grow_partition(rmb.Graph(n, 1, x, a), k, t, seeds)
    ref, _ = oracle.grow_partition(x, a, k, t, seeds=seeds[0])
    assert (parts[0] == ref).all()


def test_grow_multiconstraint(rmb, oracle):
    from rmetis_b200 import functions as F
    x, a, _, w = G.random_graph(1200, 6.0, seed=21)
    n = len(x) - 1
    v = np.random.default_rng(2).integers(1, 9, 2 * n).astype(np.int32)
    k = 8
    t = oracle.compute_target_weights(n, 2, v, k)
    seeds = np.random.default_rng(4).choice(n, k, replace=False).astype(np.int32)[None]
    parts, _ = F.grow_partition(rmb.Graph(n, 2, x, a, vwgt=v, adjwgt=w), k, t, seeds)
    ref, _ = oracle.grow_partition(x, a, k, t, vwgt=v, ncon=2, seeds=seeds[0])
    assert (parts[0] == ref).all()


def _refine_case(rmb, oracle, x, a, v, w, part, k, ub, ncon=1, niter=10, tp=None):
    from rmetis_b200 import functions as F
    n = len(x) - 1
    t = oracle.compute_target_weights(n, ncon, v, k, tp)
    g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
    gp, gcut, stats = F.greedy_refine(g, part, k, t, ub, niter)
    rp, rcut, moves = oracle.greedy_refine(x, a, part, k, t, ub, niter, vwgt=v, adjwgt=w, ncon=ncon)
    assert gcut == rcut
    assert (gp == rp).all()
    assert stats[0] == len(moves)
    assert stats[1] == moves.sum()
    return stats


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [2, 8, 48])
def test_greedy_refine_bit_exact(rmb, oracle, name, k):
    x, a, v, w = load(name)
    n = len(x) - 1
    rng = np.random.default_rng(100 + k)
    part = ((np.arange(n) * k) // n).astype(np.int32)
    flip = rng.random(n) < 0.2
    part[flip] = rng.integers(0, k, flip.sum())
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.03])


@pytest.mark.parametrize("ub", [1.001, 1.03, 1.2])
def test_greedy_refine_repair_pass(rmb, oracle, ub):
    """Heavily imbalanced start: the repair pass moves many vertices, also to
    non-adjacent parts."""
    x, a, v, w = G.grid3d(16, 12, 10, weights_seed=5)
    n = len(x) - 1
    k = 12
    part = np.minimum((np.arange(n) * k * 2) // (3 * n), k - 1).astype(np.int32)  # last parts empty-ish
    _refine_case(rmb, oracle, x, a, v, w, part, k, [ub])


def test_greedy_refine_large_parallel_rounds(rmb, oracle):
    """Enough movers for the multi-block decision rounds."""
    x, a, v, w = G.grid3d(40, 40, 30, weights_seed=8)
    n = len(x) - 1
    k = 16
    rng = np.random.default_rng(3)
    part = rng.integers(0, k, n).astype(np.int32)
    stats = _refine_case(rmb, oracle, x, a, v, w, part, k, [1.03], niter=4)
    assert stats[3] > 4 * 256


def test_greedy_refine_multiconstraint_tpwgts(rmb, oracle):
    x, a, _, w = G.random_graph(4000, 7.0, seed=33)
    n = len(x) - 1
    v = np.random.default_rng(7).integers(1, 9, 2 * n).astype(np.int32)
    k = 6
    tp = np.random.default_rng(8).random((k, 2)).astype(np.float32)
    tp /= tp.sum(axis=0, keepdims=True)
    part = np.random.default_rng(9).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.05, 1.1], ncon=2, tp=tp.ravel())


def test_reference_greedy_cycle4_cases(rmb, oracle):
    # src/refine/greedy.rs:229-251, tests/parallel.rs:91-116
    x = np.array([0, 2, 4, 6, 8], np.int32); a = np.array([1, 3, 0, 2, 1, 3, 0, 2], np.int32)
    for init in ([0, 0, 1, 1], [0, 1, 0, 1], [0, 1, 1, 0]):
        _refine_case(rmb, oracle, x, a, None, None, np.array(init, np.int32), 2, [1.03])


@pytest.mark.parametrize("mode", [0, 1])
def test_matching_properties(rmb, mode):
    from rmetis_b200 import functions as F
    for name in ["grid2d_30x17", "random_3k_deg40", "star_1500"]:
        x, a, v, w = load(name)
        n = len(x) - 1
        g = rmb.Graph(n, 1, x, a, adjwgt=w)
        m = F.match(g, mode=mode, seed=5)
        assert (m[m] == np.arange(n)).all()                      # involution
        src = np.repeat(np.arange(n), np.diff(x))
        pairs = set(zip(src.tolist(), a.tolist()))
        for vv in np.nonzero(m != np.arange(n))[0]:
            assert (int(vv), int(m[vv])) in pairs                # matched pairs are edges
        assert (F.match(g, mode=mode, seed=5) == m).all()          # deterministic
        # (almost) maximal: few edges join two unmatched vertices
        un = m == np.arange(n)
        assert np.count_nonzero(un[src] & un[a]) <= 0.005 * n + 2


def test_pipeline_replay_bit_exact(rmb, oracle):
    """The whole k-way pipeline equals the oracle's when the oracle replays
    the GPU's random choices (matchings and grow seeds)."""
    from tests.conftest import greedy_options
    cases = [
        (G.grid2d(64, 64) + (None, None), 8, 1),
        (G.grid3d(20, 18, 16, weights_seed=7), 16, 7),
        (G.random_graph(6000, 8.0, seed=2), 10, 3),
    ]
    for (x, a, v, w), k, seed in cases:
        n = len(x) - 1
        g = rmb.Graph(n, 1, x, a, vwgt=v, adjwgt=w)
        opts = rmb.Options(rtype=rmb.RType.Greedy, seed=seed)
        res, mats, seeds, _ = rmb.part_graph_kway_trace(g, k, options=opts)
        rc, part, obj = oracle.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, options=greedy_options(seed=seed),
                                               script=(mats, seeds))
        assert rc == 1
        assert obj == res.objval
        assert (part == res.part).all()


def test_greedy_refine_large_weights(rmb, oracle):
    """Totals above 2^28 take the 64-bit slack path of the walk."""
    x, a, _, w = G.grid3d(14, 12, 10, weights_seed=4)
    n = len(x) - 1
    v = np.random.default_rng(5).integers(200_000, 400_000, n).astype(np.int32)
    assert v.astype(np.int64).sum() > (1 << 28)
    k = 9
    part = np.random.default_rng(6).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.03])


@pytest.mark.parametrize("k,ub,start", [(128, 1.03, "random"), (256, 1.03, "random"), (256, 1.01, "skewed"),
                                        (200, 1.05, "skewed")])
def test_greedy_refine_many_candidates(rmb, oracle, k, ub, start):
    """R-MAT hubs touch many parts: candidate lists far longer than the
    walk's inline slots, and (skewed start) repair moves to parts the vertex
    has no edge to."""
    x, a = G.rmat(12, seed=5)
    n = len(x) - 1
    rng = np.random.default_rng(k)
    if start == "random":
        part = rng.integers(0, k, n).astype(np.int32)
    else:
        part = np.minimum((np.arange(n) * k * 3) // (4 * n), k - 1).astype(np.int32)
        flip = rng.random(n) < 0.3
        part[flip] = rng.integers(0, k, flip.sum())
    stats = _refine_case(rmb, oracle, x, a, None, None, part, k, [ub])
    assert stats[1] > 0


def test_greedy_refine_many_candidates_two_constraints(rmb, oracle):
    x, a = G.rmat(11, seed=9)
    n = len(x) - 1
    v = np.random.default_rng(1).integers(1, 9, 2 * n).astype(np.int32)
    w = G.symmetric_edge_weights(x, a, np.random.default_rng(2), 1, 10)
    k = 160
    part = np.random.default_rng(3).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.05, 1.1], ncon=2)


def test_greedy_refine_many_candidates_large_weights(rmb, oracle):
    x, a = G.rmat(11, seed=10)
    n = len(x) - 1
    v = np.random.default_rng(4).integers(200_000, 400_000, n).astype(np.int32)
    k = 96
    part = np.random.default_rng(5).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, None, part, k, [1.03])


def test_pipeline_replay_rmat_k256(rmb, oracle):
    """Skewed graph, k=256: coarsening stops early (isolated vertices never
    match), grow leaves many vertices to the lightest-part rule."""
    from tests.conftest import greedy_options
    x, a = G.rmat(13, seed=3)
    n = len(x) - 1
    g = rmb.Graph(n, 1, x, a)
    res, mats, seeds, _ = rmb.part_graph_kway_trace(g, 256, options=rmb.Options(rtype=rmb.RType.Greedy, seed=4))
    rc, part, obj = oracle.part_graph_kway(x, a, 256, options=greedy_options(seed=4), script=(mats, seeds))
    assert rc == 1
    assert obj == res.objval
    assert (part == res.part).all()


@pytest.mark.parametrize("k", [7, 64, 200, 1024, 1100])
def test_grow_leftovers_unweighted(rmb, oracle, k):
    """Thousands of isolated vertices (R-MAT) go to the lightest part one by
    one (src/initial/grow.rs:88-100); unweighted graphs take the level-by-level
    form of that rule up to k = 1024 and the plain argmin above it."""
    from rmetis_b200 import functions as F
    x, a = G.rmat(12, seed=7)
    n = len(x) - 1
    assert (np.diff(x) == 0).sum() > 500
    t = oracle.compute_target_weights(n, 1, None, k)
    seeds = np.stack([np.random.default_rng(40 + i).choice(n, k, replace=False) for i in range(3)]).astype(np.int32)
    parts, _ = F.grow_partition(rmb.Graph(n, 1, x, a), k, t, seeds)
    for i in range(3):
        ref, _ = oracle.grow_partition(x, a, k, t, seeds=seeds[i])
        assert (parts[i] == ref).all()


def test_grow_leftovers_skewed_levels(rmb, oracle):
    """Parts of very different weights before the leftovers: the levels pass
    many part weights before every part takes part."""
    from rmetis_b200 import functions as F
    # a long path, a few short paths and many isolated vertices
    xs, as_ = [], []
    off = 0
    sizes = [3000, 40, 25, 5] + [1] * 4000
    for sz in sizes:
        if sz == 1:
            xs.append(np.array([0], np.int64)); as_.append(np.zeros(0, np.int64))
        else:
            px, pa = G.path(sz)
            xs.append(px[:-1].astype(np.int64)); as_.append(pa.astype(np.int64) + off)
        off += sz
    nnz = np.cumsum([0] + [len(q) for q in as_])
    x = np.concatenate([xs[i] + nnz[i] for i in range(len(xs))] + [np.array([nnz[-1]])]).astype(np.int32)
    a = np.concatenate(as_).astype(np.int32)
    n = len(x) - 1
    k = 24
    t = oracle.compute_target_weights(n, 1, None, k)
    seeds = np.array([[0, 1500, 2999, 3000, 3040, 3065] + list(range(3070, 3088))], np.int32)
    parts, _ = F.grow_partition(rmb.Graph(n, 1, x, a), k, t, seeds)
    ref, _ = oracle.grow_partition(x, a, k, t, seeds=seeds[0])
    assert (parts[0] == ref).all()


@pytest.mark.parametrize("L,shift", [(100, 100), (60, 33), (300, 150)])
def test_grow_duplicate_neighbours(rmb, oracle, L, shift):
    """A hub's row lists every leaf twice (the reference does not reject
    duplicate entries, src/graph/validate.rs:88-108): the second occurrence,
    in a later chunk or group of the row scan, must not be claimed again
    (src/initial/grow.rs:60-80)."""
    from rmetis_b200 import functions as F
    n = L + 1 + 40
    rows = [[] for _ in range(n)]
    leaves = list(range(1, L + 1))
    order = leaves[shift % L:] + leaves[:shift % L]
    rows[0] = leaves + order                  # each leaf twice, far apart
    for u in leaves:
        rows[u] = [0, 0]
    for i in range(L + 1, n - 1):             # a path elsewhere
        rows[i].append(i + 1)
        rows[i + 1].append(i)
    x = np.zeros(n + 1, np.int32)
    x[1:] = np.cumsum([len(r) for r in rows])
    a = np.array([u for r in rows for u in r], np.int32)
    assert oracle.validate_csr(n, 1, x, a) == 0
    k = 3
    t = oracle.compute_target_weights(n, 1, None, k)
    seeds = np.array([[0, L + 1, n - 1], [3, L + 5, 0]], np.int32)
    parts, _ = F.grow_partition(rmb.Graph(n, 1, x, a), k, t, seeds)
    for i in range(2):
        ref, _ = oracle.grow_partition(x, a, k, t, seeds=seeds[i])
        assert (parts[i] == ref).all()


@pytest.mark.parametrize("k", [300, 700])
def test_greedy_refine_general_walk(rmb, oracle, k):
    """More than 256 parts: the windowed walk against shared-memory weights
    (k * ncon <= 4096), on long candidate lists."""
    x, a = G.rmat(12, seed=17)
    n = len(x) - 1
    part = np.random.default_rng(k).integers(0, k, n).astype(np.int32)
    stats = _refine_case(rmb, oracle, x, a, None, None, part, k, [1.03])
    assert stats[1] > 0


def test_greedy_refine_general_walk_global_weights(rmb, oracle):
    """k * ncon above 4096: part weights and thresholds stay in global memory;
    heavy rows with k above the shared histogram of the warp gain path."""
    x, a, v, w = load("star_1500")
    n = len(x) - 1
    k = 2100
    v2 = np.random.default_rng(3).integers(1, 5, 2 * n).astype(np.int32)
    part = np.random.default_rng(4).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v2, w, part, k, [1.2, 1.3], ncon=2)


@pytest.mark.parametrize("ncon", [3, 5])
def test_greedy_refine_many_constraints(rmb, oracle, ncon):
    x, a, _, w = G.random_graph(3000, 8.0, seed=41 + ncon)
    n = len(x) - 1
    v = np.random.default_rng(ncon).integers(1, 9, ncon * n).astype(np.int32)
    k = 20
    part = np.random.default_rng(5).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.05 + 0.02 * c for c in range(ncon)], ncon=ncon)


@pytest.mark.parametrize("k,ncon", [(300, 1), (24, 3)])
def test_pipeline_replay_general_walk(rmb, oracle, k, ncon):
    from tests.conftest import greedy_options
    x, a, _, w = G.random_graph(9000, 10.0, seed=61)
    n = len(x) - 1
    v = np.random.default_rng(62).integers(1, 6, ncon * n).astype(np.int32)
    g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
    res, mats, seeds, _ = rmb.part_graph_kway_trace(g, k, options=rmb.Options(rtype=rmb.RType.Greedy, seed=8))
    rc, part, obj = oracle.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, ncon=ncon, options=greedy_options(seed=8),
                                           script=(mats, seeds))
    assert rc == 1
    assert obj == res.objval
    assert (part == res.part).all()
