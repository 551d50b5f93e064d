"""The single-block refinement of a level (all passes in one launch) and the
multi-kernel path decide every pass identically: both are checked against the
oracle's greedy refinement (src/refine/greedy.rs:36-193) on the same cases,
and full partitions are identical either way."""
import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests.test_gpu_parity import GRAPHS, _refine_case, load

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["fused", "multi"])
def refine_path(rmb, request):
    rmb.set_tuning(fused_max_n=(1 << 30) if request.param == "fused" else 0)
    yield request.param
    rmb.set_tuning(fused_max_n=4096)


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [2, 8, 48])
def test_refine_paths_bit_exact(rmb, oracle, refine_path, name, k):
    x, a, v, w = load(name)
    n = len(x) - 1
    rng = np.random.default_rng(300 + k)
    part = ((np.arange(n) * k) // n).astype(np.int32)
    flip = rng.random(n) < 0.2
    part[flip] = rng.integers(0, k, flip.sum())
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.03])


@pytest.mark.parametrize("ub", [1.001, 1.2])
def test_refine_paths_repair(rmb, oracle, refine_path, ub):
    x, a, v, w = G.grid3d(16, 12, 10, weights_seed=5)
    n = len(x) - 1
    k = 12
    part = np.minimum((np.arange(n) * k * 2) // (3 * n), k - 1).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [ub])


@pytest.mark.parametrize("k", [128, 256])
def test_refine_paths_long_lists(rmb, oracle, refine_path, k):
    x, a = G.rmat(12, seed=5)
    n = len(x) - 1
    part = np.random.default_rng(k).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, None, None, part, k, [1.03])


def test_refine_paths_two_constraints_large_weights(rmb, oracle, refine_path):
    x, a, _, w = G.random_graph(3000, 7.0, seed=35)
    n = len(x) - 1
    v = np.random.default_rng(11).integers(200_000, 400_000, 2 * n).astype(np.int32)
    k = 40
    part = np.random.default_rng(12).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.05, 1.1], ncon=2)


def test_refine_paths_heavy_rows(rmb, oracle, refine_path):
    """Rows above the heavy degree take the warp gain path inside the fused
    kernel too."""
    x, a, v, w = load("star_1500")
    n = len(x) - 1
    k = 9
    part = np.random.default_rng(13).integers(0, k, n).astype(np.int32)
    _refine_case(rmb, oracle, x, a, v, w, part, k, [1.03])


def test_full_partitions_identical_across_paths(rmb):
    cases = [(G.grid3d(24, weights_seed=7), 32), (G.grid2d(90, 90) + (None, None), 16)]
    for (x, a, v, w), k in cases:
        g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
        o = rmb.Options(rtype=rmb.RType.Greedy, seed=3)
        try:
            rmb.set_tuning(fused_max_n=0)
            multi = rmb.part_graph_kway(g, k, options=o)
            rmb.set_tuning(fused_max_n=1 << 30)
            fused = rmb.part_graph_kway(g, k, options=o)
        finally:
            rmb.set_tuning(fused_max_n=4096)
        assert multi.objval == fused.objval
        np.testing.assert_array_equal(multi.part, fused.part)


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [2, 9, 48])
def test_fm_level_paths_identical(rmb, name, k):
    """The single-block FM level (k_fm_level: every pass and round of
    fm_kway_refine in one launch) and the multi-kernel rounds decide every
    round identically: same partition, cut and statistics."""
    from rmetis_b200 import functions as F
    x, a, v, w = load(name)
    n = len(x) - 1
    rng = np.random.default_rng(500 + k)
    part = ((np.arange(n) * k) // n).astype(np.int32)
    flip = rng.random(n) < 0.15
    part[flip] = rng.integers(0, k, flip.sum())
    g = rmb.Graph(n, 1, x, a, vwgt=v, adjwgt=w)
    tot = n if v is None else int(np.asarray(v).sum())
    t = np.full(k, tot / k, np.float64)
    out = {}
    try:
        for path, fm in (("multi", 0), ("fused", 1 << 30)):
            rmb.set_fm_fused_max(fm)
            out[path] = F.fm_refine(g, part, k, t, [1.03], 10)
    finally:
        rmb.set_fm_fused_max(4096)
    assert out["multi"][1] == out["fused"][1]
    np.testing.assert_array_equal(out["multi"][0], out["fused"][0])
    np.testing.assert_array_equal(out["multi"][2], out["fused"][2])


def test_fm_full_partitions_identical_across_paths(rmb):
    cases = [(G.grid3d(24, weights_seed=7), 32), (G.grid2d(90, 90) + (None, None), 16),
             (G.random_graph(6000, 8.0, seed=9), 24)]
    for (x, a, v, w), k in cases:
        g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
        o = rmb.Options(rtype=rmb.RType.Fm, seed=4)
        try:
            rmb.set_fm_fused_max(0)
            multi = rmb.part_graph_kway(g, k, options=o)
            rmb.set_fm_fused_max(1 << 30)
            fused = rmb.part_graph_kway(g, k, options=o)
        finally:
            rmb.set_fm_fused_max(4096)
        assert multi.objval == fused.objval
        np.testing.assert_array_equal(multi.part, fused.part)


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("mode", [0, 1])
def test_coop_matching_identical(rmb, name, mode):
    """The matching rounds in one cooperative launch (grid-wide barriers,
    progress checks on the device) and one launch per phase with host checks
    give the same matching."""
    from rmetis_b200 import functions as F
    x, a, v, w = load(name)
    g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
    out = {}
    try:
        for on in (0, 1):
            rmb.set_coop_matching(on)
            out[on] = F.match(g, mode=mode, seed=77, rounds=24)
    finally:
        rmb.set_coop_matching(1)
    np.testing.assert_array_equal(out[0], out[1])
    m = out[1]
    assert (m[m] == np.arange(len(m))).all()


def test_coop_matching_full_partitions(rmb):
    cases = [(G.grid3d(40, weights_seed=2), 64), (G.random_graph(30000, 9.0, seed=4), 16)]
    for (x, a, v, w), k in cases:
        g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
        o = rmb.Options(rtype=rmb.RType.Greedy, seed=8)
        try:
            rmb.set_coop_matching(0)
            plain = rmb.part_graph_kway(g, k, options=o)
            rmb.set_coop_matching(1)
            coop = rmb.part_graph_kway(g, k, options=o)
        finally:
            rmb.set_coop_matching(1)
        assert plain.objval == coop.objval
        np.testing.assert_array_equal(plain.part, coop.part)
