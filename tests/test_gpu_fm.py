"""k-way FM refinement on the GPU (src/refine/fm_kway.rs:12-158), the
reference's default rtype, through the C ABI.

RMETIS_GPU_FmRefine is checked against the reference's move rule directly:
the cut never rises and equals the edge cut of the result, a part only
receives vertices while it stays feasible ((pw+vw) as f64 <= target*ub), and
a refinement that stopped at a pass without a move leaves no vertex whose
best move (largest positive gain to an adjacent part, lowest id on ties) is
feasible. Its moves run in parallel rounds, so the partition is compared with
the oracle's restatement by quality (summed cut within 5%), not bit for bit.
Full partitions with rtype Fm are checked for validity, objval, determinism
and quality against the oracle's FM pipeline over the same seeds."""
import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests import fm_check
from tests.conftest import fm_options
from tests.test_gpu_kway import CASES, call_c_abi
from tests.test_gpu_parity import GRAPHS, load

pytestmark = pytest.mark.gpu


def _fm_case(rmb, oracle, x, a, v, w, part, k, ub, ncon=1, niter=50, tp=None, fixed_point=True):
    from rmetis_b200 import functions as F
    n = len(x) - 1
    t = oracle.compute_target_weights(n, ncon, v, k, tp)
    g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
    before = oracle.edge_cut(x, a, w, part)
    gp, gcut, stats = F.fm_refine(g, part, k, t, ub, niter)
    assert ((gp >= 0) & (gp < k)).all()
    assert gcut == oracle.edge_cut(x, a, w, gp)
    assert gcut <= before
    assert (gcut < before) == (stats[1] > 0)
    assert fm_check.balance_bound_holds(part, gp, k, v, ncon, t, ub)
    if fixed_point and stats[0] < niter:
        assert fm_check.fixed_point_violations(x, a, w, v, gp, k, ncon, t, ub) == []
    again = F.fm_refine(g, part, k, t, ub, niter)
    assert again[1] == gcut and (again[0] == gp).all()
    rp, rcut, passes, moves = oracle.fm_kway_refine(x, a, part, k, t, ub, niter, vwgt=v, adjwgt=w, ncon=ncon)
    return gcut, rcut, before, stats


def _start(n, k, seed, flip=0.2):
    rng = np.random.default_rng(seed)
    part = ((np.arange(n) * k) // n).astype(np.int32)
    f = rng.random(n) < flip
    part[f] = rng.integers(0, k, f.sum())
    return part


def test_fm_reference_grid3x3():                        # fm_kway.rs:207-219
    import rmetis_b200 as rmb
    from rmetis_b200 import functions as F
    x, a = G.grid2d(3, 3)
    g = rmb.Graph(9, 1, x, a)
    part0 = np.array([v // 3 for v in range(9)], np.int32)
    before = g.edge_cut(part0)
    part, cut, stats = F.fm_refine(g, part0, 3, [3.0, 3.0, 3.0], [1.1], 5)
    assert cut <= before and cut == g.edge_cut(part)


def test_fm_refine_rule_and_quality(rmb, oracle):
    """Every graph of the parity set, k = 2, 8, 48, from a blocked start with
    20% of the vertices moved at random: the rule checks per case, and the
    summed cut within 5% of the oracle's FM."""
    g_sum = r_sum = 0
    for name in GRAPHS:
        x, a, v, w = load(name)
        n = len(x) - 1
        for k in (2, 8, 48):
            gcut, rcut, before, stats = _fm_case(rmb, oracle, x, a, v, w, _start(n, k, 100 + k), k, [1.03])
            g_sum += gcut
            r_sum += rcut
    assert g_sum <= 1.05 * r_sum, (g_sum, r_sum)


def test_fm_refine_random_start_many_rounds(rmb, oracle):
    """A random start on a 3D grid: many movers per round and many rounds."""
    x, a, v, w = G.grid3d(40, 40, 30, weights_seed=8)
    n = len(x) - 1
    k = 16
    part = np.random.default_rng(3).integers(0, k, n).astype(np.int32)
    gcut, rcut, before, stats = _fm_case(rmb, oracle, x, a, v, w, part, k, [1.03], niter=10, fixed_point=False)
    assert stats[2] > 10 and stats[3] > 10_000
    assert gcut <= 1.05 * rcut, (gcut, rcut)


def test_fm_refine_multiconstraint_tpwgts(rmb, oracle):
    x, a, _, w = G.random_graph(4000, 7.0, seed=33)
    n = len(x) - 1
    v = np.random.default_rng(7).integers(1, 9, 2 * n).astype(np.int32)
    k = 6
    tp = np.random.default_rng(8).random((k, 2)).astype(np.float32)
    tp /= tp.sum(axis=0, keepdims=True)
    part = np.random.default_rng(9).integers(0, k, n).astype(np.int32)
    gcut, rcut, _, _ = _fm_case(rmb, oracle, x, a, v, w, part, k, [1.05, 1.1], ncon=2, tp=tp.ravel())
    assert gcut <= 1.05 * rcut, (gcut, rcut)


def test_fm_refine_hubs_many_parts(rmb, oracle):
    """R-MAT hubs (warp-per-vertex gain rows, long neighbour lists in the
    selection) and k = 128."""
    x, a = G.rmat(12, seed=5)
    n = len(x) - 1
    part = np.random.default_rng(128).integers(0, 128, n).astype(np.int32)
    gcut, rcut, before, stats = _fm_case(rmb, oracle, x, a, None, None, part, 128, [1.03], niter=10,
                                         fixed_point=False)
    assert stats[1] > 0


def test_fm_refine_large_weights(rmb, oracle):
    """Totals above 2^28 take the 64-bit slack path of the walk."""
    x, a, _, w = G.grid3d(14, 12, 10, weights_seed=4)
    n = len(x) - 1
    v = np.random.default_rng(5).integers(200_000, 400_000, n).astype(np.int32)
    part = np.random.default_rng(6).integers(0, 9, n).astype(np.int32)
    _fm_case(rmb, oracle, x, a, v, w, part, 9, [1.03])


@pytest.mark.parametrize("name,make,k", CASES)
def test_kway_fm_valid_deterministic_and_close_to_reference(rmb, oracle, name, make, k):
    x, a, v, w = make()
    seeds = range(1, 5)
    cuts, ref = [], []
    for seed in seeds:
        rc, part, obj = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, options=fm_options(seed=seed))
        assert rc == 1 and ((part >= 0) & (part < k)).all()
        assert obj == oracle.edge_cut(x, a, w, part)
        rc2, part2, obj2 = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, options=fm_options(seed=seed))
        assert rc2 == 1 and obj2 == obj and (part2 == part).all()
        cuts.append(obj)
        rc, _, robj = oracle.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, options=fm_options(seed=seed))
        assert rc == 1
        ref.append(robj)
    assert np.mean(cuts) <= 1.05 * np.mean(ref), (cuts, ref)


def test_kway_default_options_run(rmb, oracle):
    """NULL options select the reference's defaults (rtype Fm) and partition."""
    x, a = G.grid2d(32, 32)
    rc, part, obj = call_c_abi(rmb, x, a, 4, options=None)
    assert rc == 1 and ((part >= 0) & (part < 4)).all()
    assert obj == oracle.edge_cut(x, a, None, part)


def test_fm_batch_and_async_equal_single_calls(rmb):
    import rmetis_b200 as rmb_mod
    graphs, ks = [], []
    for i, (n, k) in enumerate(((3000, 4), (9000, 16), (1500, 2))):
        x, a, w, _ = G.rgg2d(n, 40 + i)
        v = np.random.default_rng(i).integers(1, 9, 2 * (len(x) - 1)).astype(np.int32)
        graphs.append(rmb_mod.Graph(len(x) - 1, 2, x, a, vwgt=v, adjwgt=w))
        ks.append(k)
    o = rmb_mod.Options(rtype=rmb_mod.RType.Fm, seed=3)
    solo = [rmb_mod.part_graph_kway(g, k, options=o) for g, k in zip(graphs, ks)]
    batch = rmb_mod.part_graph_kway_batch(graphs, ks, options=o)
    reqs = [rmb_mod.submit_kway(g, k, options=o) for g, k in zip(graphs, ks)]
    for s, b, r in zip(solo, batch, reqs):
        res = r.wait()
        assert s.objval == b.objval == res.objval
        np.testing.assert_array_equal(s.part, b.part)
        np.testing.assert_array_equal(s.part, res.part)
