"""Pins the oracle (CPU restatement) to the reference's own known answers.

Every case below restates a unit or integration test of the reference
(file:line given per test) against the oracle, plus the published
xoshiro256++ reference outputs for the RNG core. No GPU needed.
"""
import numpy as np
import pytest

from tests.conftest import greedy_options

CYCLE4 = (np.array([0, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 2]))
PATH4 = (np.array([0, 1, 3, 5, 6]), np.array([1, 0, 2, 1, 3, 2]))
GRID4 = (np.array([0, 2, 4, 6, 8]), np.array([1, 2, 0, 3, 0, 3, 1, 2]))  # grow.rs:121-128


def grid_graph(rows, cols):
    """tests/parallel.rs:15-33 builder (neighbour order: up, down, left, right)."""
    xadj = [0]
    adj = []
    for r in range(rows):
        for c in range(cols):
            nb = []
            if r > 0: nb.append((r - 1) * cols + c)
            if r + 1 < rows: nb.append((r + 1) * cols + c)
            if c > 0: nb.append(r * cols + c - 1)
            if c + 1 < cols: nb.append(r * cols + c + 1)
            adj += nb
            xadj.append(len(adj))
    return np.array(xadj), np.array(adj)


def build_undirected(n, edges):
    """tests/correctness.rs:36-50 builder (sorted neighbours)."""
    adj = [[] for _ in range(n)]
    for u, v in edges:
        adj[u].append(v)
        adj[v].append(u)
    xadj = [0]
    out = []
    for v in range(n):
        out += sorted(adj[v])
        xadj.append(len(out))
    return np.array(xadj), np.array(out)


def grid4x4():
    edges = []
    for r in range(4):
        for c in range(4):
            v = r * 4 + c
            if c + 1 < 4: edges.append((v, v + 1))
            if r + 1 < 4: edges.append((v, v + 4))
    return build_undirected(16, edges)


# ---- RNG core --------------------------------------------------------------

def test_xoshiro256pp_reference_vectors(oracle):
    # Outputs of the published xoshiro256++ reference for state (1, 2, 3, 4).
    r = oracle.SmallRng.from_state([1, 2, 3, 4])
    got = [int(x) for x in r.next_u64(10)]
    assert got == [41943041, 58720359, 3588806011781223, 3591011842654386, 9228616714210784205,
                   9973669472204895162, 14011001112246962877, 12406186145184390807, 15849039046786891736,
                   10450023813501588000]


def test_gen_range_bounds_and_determinism(oracle):
    a = oracle.SmallRng(42)
    b = oracle.SmallRng(42)
    xs = [a.gen_range(0, 7) for _ in range(200)]
    ys = [b.gen_range(0, 7) for _ in range(200)]
    assert xs == ys
    assert min(xs) >= 0 and max(xs) < 7 and len(set(xs)) == 7


# ---- src/graph/mod.rs tests -------------------------------------------------

def test_edge_cut_partition(oracle):          # mod.rs:454-461
    assert oracle.edge_cut(*CYCLE4, None, [0, 0, 1, 1]) == 2


def test_partition_weights_uniform(oracle):   # mod.rs:463-470
    pw = oracle.partition_weights(4, 1, None, [0, 0, 1, 1], 2)
    assert pw.tolist() == [[2], [2]]


def test_total_weight_uniform(oracle):        # mod.rs:472-476
    assert oracle.total_weight(4, 1, None).tolist() == [4]


def test_boundary_vertices(oracle):           # mod.rs:478-485
    assert sorted(oracle.boundary_vertices(*CYCLE4, [0, 0, 1, 1]).tolist()) == [0, 1, 2, 3]


def test_build_coarse_graph_path(oracle):     # mod.rs:498-514
    r = oracle.build_coarse_graph(*PATH4, [1, 0, 3, 2])
    assert r["cn"] == 2
    assert len(r["cadjncy"]) // 2 == 1
    cmap = r["cmap"]
    assert cmap[0] == cmap[1] and cmap[2] == cmap[3] and cmap[0] != cmap[2]


# ---- src/graph/validate.rs tests --------------------------------------------

def test_validate_cases(oracle):              # validate.rs:151-188
    assert oracle.validate_csr(4, 1, *CYCLE4) == 0
    assert oracle.validate_csr(4, 1, np.array([0, 2, 4]), CYCLE4[1]) != 0
    assert oracle.validate_csr(4, 1, np.array([0, 3, 5, 7, 9]), np.array([0, 1, 3, 0, 2, 1, 3, 0, 2])) != 0
    assert oracle.validate_csr(4, 1, np.array([0, 1, 1, 0, 0]), np.array([1])) != 0
    assert oracle.validate_csr(4, 1, *CYCLE4, vwgt=np.array([1, 1, 1])) != 0


# ---- matching tests ---------------------------------------------------------

def test_shem_prefers_heavy_edge(oracle):     # shem.rs:80-106
    xadj = np.array([0, 3, 4, 5, 6]); adj = np.array([1, 2, 3, 0, 0, 0])
    w = np.array([1, 3, 1, 1, 3, 1])
    m = oracle.shem_matching(xadj, adj, w, oracle.SmallRng(1))
    assert all(m[m[v]] == v for v in range(4))
    assert sum(1 for v in range(4) if m[v] != v) >= 2


@pytest.mark.parametrize("seed", [42, 0])
def test_random_matching(oracle, seed):       # rm.rs:56-74
    m = oracle.random_matching(*PATH4, oracle.SmallRng(seed))
    assert all(m[m[v]] == v for v in range(4))
    assert sum(1 for v in range(4) if m[v] != v) >= 2


# ---- grow.rs tests ----------------------------------------------------------

@pytest.mark.parametrize("seed", [42, 7])
def test_grow_all_assigned(oracle, seed):     # grow.rs:121-139
    part, seeds = oracle.grow_partition(*GRID4, 2, [2.0, 2.0], rng=oracle.SmallRng(seed))
    assert all(0 <= p < 2 for p in part)
    assert (part == 0).sum() + (part == 1).sum() == 4
    assert len(set(seeds.tolist())) == 2


def test_grow_seeded_replay_equals_drawn(oracle):
    xadj, adj = grid_graph(6, 5)
    t = [10.0, 10.0, 10.0]
    p1, s1 = oracle.grow_partition(xadj, adj, 3, t, rng=oracle.SmallRng(3))
    p2, s2 = oracle.grow_partition(xadj, adj, 3, t, seeds=s1)
    assert (p1 == p2).all()


# ---- greedy.rs / tests/parallel.rs ------------------------------------------

def test_refine_does_not_increase_cut(oracle):     # greedy.rs:229-239
    before = oracle.edge_cut(*CYCLE4, None, [0, 1, 0, 1])
    part, cut, _ = oracle.greedy_refine(*CYCLE4, [0, 1, 0, 1], 2, [2.0, 2.0], [1.03], 10)
    assert cut <= before


@pytest.mark.parametrize("init", [[0, 0, 1, 1], [0, 1, 0, 1], [0, 1, 1, 0]])
def test_greedy_deterministic(oracle, init):        # tests/parallel.rs:91-116
    a = oracle.greedy_refine(*CYCLE4, init, 2, [2.0, 2.0], [1.03], 10)
    b = oracle.greedy_refine(*CYCLE4, init, 2, [2.0, 2.0], [1.03], 10)
    assert a[1] == b[1] and (a[0] == b[0]).all()


def test_greedy_rows_no_cut_increase(oracle):       # tests/parallel.rs:118-132
    xadj, adj = grid_graph(4, 4)
    part = np.arange(16) // 4
    before = oracle.edge_cut(xadj, adj, None, part)
    _, after, _ = oracle.greedy_refine(xadj, adj, part, 4, [4.0] * 4, [1.05], 10)
    assert after <= before


def test_compute_move_gain_known(oracle):
    # cycle4 with part [0,0,1,1]: moving 1 to part 1 gains +1 - 1 = 0
    assert oracle.compute_move_gain(*CYCLE4, None, 1, [0, 0, 1, 1], 0, 1) == 0
    # path4 weighted 1,3,1: vertex 1 in part 0 with 0|1|1|1 -> to part 1: +3 - 1
    xadj, adj = PATH4
    w = np.array([1, 1, 3, 3, 1, 1])
    assert oracle.compute_move_gain(xadj, adj, w, 1, [0, 0, 1, 1], 0, 1) == 2


# ---- kway integration (tests/correctness.rs, tests/parallel.rs) --------------

def _balanced(oracle, xadj, adj, part, k, ufactor, vwgt=None):
    # correctness.rs:68-79 balance check (with its +1 slack)
    n = len(xadj) - 1
    pw = oracle.partition_weights(n, 1, vwgt, part, k)
    total = oracle.total_weight(n, 1, vwgt)[0]
    max_allowed = total * (1.0 + ufactor / 1000.0) / k
    return all(w[0] <= max_allowed + 1.0 for w in pw)


def test_kway_grid4x4_k4_greedy_ncuts5(oracle):   # correctness.rs:120-128
    xadj, adj = grid4x4()
    rc, part, obj = oracle.part_graph_kway(xadj, adj, 4, options=greedy_options(seed=1, ncuts=5))
    assert rc == 1
    assert ((part >= 0) & (part < 4)).all()
    assert _balanced(oracle, xadj, adj, part, 4, 30)
    assert obj == oracle.edge_cut(xadj, adj, None, part)


def test_kway_cycle4_k2(oracle):                  # correctness.rs:100-108 (Greedy path)
    rc, part, obj = oracle.part_graph_kway(*CYCLE4, 2, options=greedy_options(seed=1))
    assert rc == 1 and obj <= 4


def test_kway_deterministic(oracle):              # correctness.rs:179-187
    xadj, adj = grid4x4()
    o = greedy_options(seed=123)
    r1 = oracle.part_graph_kway(xadj, adj, 4, options=o)
    r2 = oracle.part_graph_kway(xadj, adj, 4, options=o)
    assert r1[2] == r2[2] and (r1[1] == r2[1]).all()


def test_kway_errors(oracle):                     # correctness.rs:203-215
    assert oracle.part_graph_kway(*CYCLE4, 10, options=greedy_options())[0] == -2
    assert oracle.part_graph_kway(*CYCLE4, 1, options=greedy_options())[0] == -2


def test_kway_weighted(oracle):                   # correctness.rs:221-235
    rc, part, obj = oracle.part_graph_kway(*CYCLE4, 2, vwgt=[2, 1, 2, 1], adjwgt=[3, 1, 3, 1, 3, 1, 3, 1],
                                           options=greedy_options(seed=5))
    assert rc == 1 and ((part >= 0) & (part < 2)).all()


def test_kway_explicit_valid_nonempty(oracle):    # tests/parallel.rs:163-187 (Greedy path)
    xadj, adj = grid_graph(4, 4)
    rc, part, obj = oracle.part_graph_kway(xadj, adj, 4, options=greedy_options(seed=1, ncuts=3))
    assert rc == 1
    assert obj == oracle.edge_cut(xadj, adj, None, part)
    assert all((part == p).sum() > 0 for p in range(4))


def test_kway_more_cuts_not_worse(oracle):        # tests/parallel.rs:202-215
    xadj, adj = grid_graph(6, 6)
    r1 = oracle.part_graph_kway(xadj, adj, 4, options=greedy_options(seed=42, ncuts=1))
    r4 = oracle.part_graph_kway(xadj, adj, 4, options=greedy_options(seed=42, ncuts=4))
    assert r4[2] <= r1[2]


def test_hierarchy_valid(oracle):                 # tests/parallel.rs:136-159
    xadj, adj = grid_graph(4, 4)
    rc, part, obj, st = oracle.part_graph_kway(xadj, adj, 2, options=greedy_options(seed=42), with_stats=True)
    assert rc == 1 and st["nlevels"] >= 1
    assert st["level_n"][0] == 16
    assert all(st["level_n"][i + 1] <= st["level_n"][i] for i in range(st["nlevels"]))


def test_set_default_options(oracle):             # c_api.rs:15-23, types.rs:227-245
    rc, a = oracle.set_default_options()
    assert rc == 1
    assert a[0] == -1 and a[2] == 1 and a[3] == 0 and a[4] == 0 and a[6] == 10 and a[7] == 1 and a[16] == 30


def test_script_replay_reproduces_run(oracle):
    """A script holding the oracle's own SHEM matchings replays its run."""
    from rmetis_b200 import generators as G
    xadj, adj = G.grid2d(20, 20)
    o = greedy_options(seed=9)
    rc, part, obj = oracle.part_graph_kway(xadj, adj, 4, options=o)
    # replay with the same RNG: recompute matchings through the restated SHEM
    rng = oracle.SmallRng(9)
    mats = []
    cur_x, cur_a, cur_w = xadj, adj, None
    while True:
        m = oracle.shem_matching(cur_x, cur_a, cur_w, rng)
        mats.append(m)
        r = oracle.build_coarse_graph(cur_x, cur_a, m, adjwgt=cur_w)
        ratio = np.float32(r["cn"]) / np.float32(len(cur_x) - 1)
        cur_x, cur_a = r["cxadj"], r["cadjncy"]
        cur_w = r["cadjwgt"] if r["keeps_adjwgt"] else None
        if r["cn"] <= 80 or ratio > np.float32(0.95):
            break
    t = oracle.compute_target_weights(len(cur_x) - 1, 1, None, 4)
    _, seeds = oracle.grow_partition(cur_x, cur_a, 4, t, rng=rng)
    rc2, part2, obj2 = oracle.part_graph_kway(xadj, adj, 4, options=o, script=(mats, seeds))
    assert rc2 == 1 and obj2 == obj and (part2 == part).all()


# ---- fm_kway.rs (k-way FM, the reference's default rtype) -------------------

from tests.conftest import fm_options  # noqa: E402
from tests import fm_check  # noqa: E402


def grid3x3():
    return grid_graph(3, 3)


def test_fm_kway_does_not_increase_cut(oracle):    # fm_kway.rs:207-219
    xadj, adj = grid3x3()
    part0 = [v // 3 for v in range(9)]
    before = oracle.edge_cut(xadj, adj, None, part0)
    part, cut, passes, moves = oracle.fm_kway_refine(xadj, adj, part0, 3, [3.0, 3.0, 3.0], [1.1], 5)
    assert cut <= before
    assert cut == oracle.edge_cut(xadj, adj, None, part)


def _fm_case(seed):
    from rmetis_b200 import generators as G
    rng = np.random.default_rng(seed)
    x, a, _, w = G.random_graph(int(rng.integers(60, 400)), 6.0, seed)
    k = int(rng.choice([2, 3, 5, 8]))
    n = len(x) - 1
    ncon = int(rng.choice([1, 2]))
    vw = rng.integers(1, 5, size=n * ncon).astype(np.int32)
    part0 = rng.integers(0, k, size=n).astype(np.int32)
    tot = vw.reshape(n, ncon).sum(axis=0)
    t = np.repeat(tot[None, :] / k, k, axis=0).reshape(-1)
    ub = np.full(ncon, 1.05)
    return x, a, w, vw, ncon, k, part0, t, ub


@pytest.mark.parametrize("seed", range(8))
def test_fm_kway_properties(oracle, seed):
    """Cut never rises and equals edge_cut; parts only receive while feasible;
    after a pass without a move no vertex has a feasible positive-gain best
    move; the same input gives the same output."""
    x, a, w, vw, ncon, k, part0, t, ub = _fm_case(seed)
    before = oracle.edge_cut(x, a, w, part0)
    part, cut, passes, moves = oracle.fm_kway_refine(x, a, part0, k, t, ub, 50, vwgt=vw, adjwgt=w, ncon=ncon)
    assert cut <= before and cut == oracle.edge_cut(x, a, w, part)
    assert fm_check.balance_bound_holds(part0, part, k, vw, ncon, t, ub)
    assert passes < 50
    assert fm_check.fixed_point_violations(x, a, w, vw, part, k, ncon, t, ub) == []
    again = oracle.fm_kway_refine(x, a, part0, k, t, ub, 50, vwgt=vw, adjwgt=w, ncon=ncon)
    assert again[1] == cut and (again[0] == part).all()


def test_kway_cycle4_k2_fm(oracle):               # correctness.rs:100-108
    rc, part, obj = oracle.part_graph_kway(*CYCLE4, 2, options=fm_options(seed=1))
    assert rc == 1 and ((part >= 0) & (part < 2)).all()
    assert _balanced(oracle, *CYCLE4, part, 2, 30)
    assert obj <= 4


def test_kway_grid2x3_k2_fm(oracle):              # correctness.rs:110-117
    xadj, adj = grid_graph(2, 3)
    rc, part, obj = oracle.part_graph_kway(xadj, adj, 2, options=fm_options(seed=42))
    assert rc == 1 and ((part >= 0) & (part < 2)).all()
    assert _balanced(oracle, xadj, adj, part, 2, 30)


def test_kway_deterministic_fm(oracle):           # correctness.rs:179-187
    xadj, adj = grid4x4()
    r1 = oracle.part_graph_kway(xadj, adj, 4, options=fm_options(seed=123))
    r2 = oracle.part_graph_kway(xadj, adj, 4, options=fm_options(seed=123))
    assert r1[0] == 1 and r1[2] == r2[2] and (r1[1] == r2[1]).all()


def test_kway_weighted_fm(oracle):                # correctness.rs:221-235
    rc, part, obj = oracle.part_graph_kway(*CYCLE4, 2, vwgt=[2, 1, 2, 1], adjwgt=[3, 1, 3, 1, 3, 1, 3, 1],
                                           options=fm_options(seed=5))
    assert rc == 1 and ((part >= 0) & (part < 2)).all()


def test_kway_default_options_run_fm(oracle):     # c_api.rs:217-219: NULL options = defaults (rtype Fm)
    xadj, adj = grid_graph(8, 8)
    rc, part, obj = oracle.part_graph_kway(xadj, adj, 4, options=None)
    assert rc == 1 and obj == oracle.edge_cut(xadj, adj, None, part)


# ---- recursive.rs / fm.rs (recursive bisection, 2-way FM) -------------------

def _recursive_options(seed, rtype=0):
    import rmetis_b200 as rmb
    o = rmb.Options.for_recursive()               # types.rs:99-106: MetisRb, Fm, ufactor 1
    o.seed = seed
    o.rtype = rmb.RType(rtype)
    return o.c_array()


def test_fm2_does_not_increase_cut(oracle):        # fm.rs:145-159
    x = np.array([0, 2, 4, 6, 8, 10, 12]); a = np.array([1, 5, 0, 2, 1, 3, 2, 4, 3, 5, 4, 0])
    part0 = [0, 0, 0, 1, 1, 1]
    before = oracle.edge_cut(x, a, None, part0)
    part, cut = oracle.fm2_refine(x, a, part0, [3.0, 3.0], [1.05], 10)
    assert cut <= before and cut == oracle.edge_cut(x, a, None, part)


def test_recursive_cycle4_k2(oracle):             # correctness.rs:130-137
    rc, part, obj = oracle.part_graph_recursive(*CYCLE4, 2, options=_recursive_options(7))
    assert rc == 1 and ((part >= 0) & (part < 2)).all()
    assert _balanced(oracle, *CYCLE4, part, 2, 5)


@pytest.mark.parametrize("k", [4, 8])
def test_recursive_grid4x4(oracle, k):            # correctness.rs:139-153
    xadj, adj = grid4x4()
    rc, part, obj = oracle.part_graph_recursive(xadj, adj, k, options=_recursive_options(42))
    assert rc == 1 and ((part >= 0) & (part < k)).all()
    assert obj == oracle.edge_cut(xadj, adj, None, part)


def test_recursive_deterministic(oracle):         # correctness.rs:189-197
    xadj, adj = grid4x4()
    r1 = oracle.part_graph_recursive(xadj, adj, 4, options=_recursive_options(99))
    r2 = oracle.part_graph_recursive(xadj, adj, 4, options=_recursive_options(99))
    assert r1[0] == 1 and r1[2] == r2[2] and (r1[1] == r2[1]).all()


@pytest.mark.parametrize("rtype", [0, 1])
def test_recursive_properties(oracle, rtype):
    """Every part used, objval equals the edge cut, the error rules of
    partition_recursive (recursive.rs:19-26), with either 2-way refinement."""
    from rmetis_b200 import generators as G
    x, a, v, w = G.grid3d(12, 10, 8, weights_seed=2)
    for k in (2, 3, 7, 16):
        rc, part, obj = oracle.part_graph_recursive(x, a, k, vwgt=v, adjwgt=w, options=_recursive_options(5, rtype))
        assert rc == 1 and obj == oracle.edge_cut(x, a, w, part)
        assert sorted(set(part.tolist())) == list(range(k))
    assert oracle.part_graph_recursive(*CYCLE4, 10, options=_recursive_options(1))[0] == -2
    assert oracle.part_graph_recursive(*CYCLE4, 1, options=_recursive_options(1))[0] == -2


# ---- nd.rs / separator (nested dissection) ----------------------------------

def _nd_valid(n, perm, iperm):                    # correctness.rs:81-94
    assert len(perm) == n and len(iperm) == n
    assert sorted(perm.tolist()) == list(range(n))
    assert all(perm[iperm[v]] == v for v in range(n))


def _default_options(seed):
    import rmetis_b200 as rmb
    o = rmb.Options()
    o.seed = seed
    return o.c_array()


def test_nd_path10(oracle):                       # nd.rs:115-150
    n = 10
    x = [0]; a = []
    for v in range(n):
        if v > 0:
            a.append(v - 1)
        if v < n - 1:
            a.append(v + 1)
        x.append(len(a))
    rc, perm, iperm = oracle.node_nd(np.array(x), np.array(a), options=_default_options(42))
    assert rc == 1
    _nd_valid(n, perm, iperm)


def test_nd_cycle4_and_grid4x4(oracle):           # correctness.rs:159-176
    rc, perm, iperm = oracle.node_nd(*CYCLE4, options=_default_options(1))
    assert rc == 1
    _nd_valid(4, perm, iperm)
    xadj, adj = grid4x4()
    rc, perm, iperm = oracle.node_nd(xadj, adj, options=_default_options(42))
    assert rc == 1
    _nd_valid(16, perm, iperm)


def test_nd_separators_on_a_larger_grid(oracle):
    """A 30x30 grid (900 > 100 vertices) goes through separators: still a
    permutation, the same for the same seed, and the last positions hold the
    top-level separator, which splits the grid."""
    xadj, adj = grid_graph(30, 30)
    rc, perm, iperm = oracle.node_nd(xadj, adj, options=_default_options(3))
    assert rc == 1
    _nd_valid(900, perm, iperm)
    rc2, perm2, _ = oracle.node_nd(xadj, adj, options=_default_options(3))
    assert (perm2 == perm).all()
    assert (perm != np.arange(900)).any()    # separators moved to the end, not the plain order
    assert oracle.node_nd(np.array([0, 1, 1, 0, 0]), np.array([1]))[0] == -2   # asymmetric: validation
