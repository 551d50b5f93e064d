"""The parallel admission of greedy cut passes (rmetis_b200/csrc/admit.cu)
against its numpy model (tests/admit_model.py), bit for bit, and full
partitions decided that way against the oracle.

RMETIS_GPU_GreedyRefine decides the cut passes of graphs above the
RMETIS_GPU_SetRefineMode threshold by admission; the tests set the threshold
to 0 (every level) and restore the default afterwards. The repair pass stays
the reference's sequential pass, so the model starts from the oracle's
repaired partition (oracle.greedy_refine with niter=0).
"""
import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests import admit_model as M
from tests.conftest import greedy_options
from tests.test_gpu_kway import call_c_abi
from tests.test_gpu_quality import overshoot

pytestmark = pytest.mark.gpu

DEFAULT_EXACT_MAX_N = 16384


@pytest.fixture
def admit_everywhere(rmb):
    rmb.set_refine_mode(0)
    yield
    rmb.set_refine_mode(DEFAULT_EXACT_MAX_N)


def _start(n, k, seed, frac=1.0):
    rng = np.random.default_rng(seed)
    part = ((np.arange(n) * k) // n).astype(np.int32)
    flip = rng.random(n) < frac
    part[flip] = rng.integers(0, k, flip.sum())
    return part


def _check_passes(rmb, oracle, x, a, v, w, part, k, ub, ncon=1, niter=4, tp=None):
    from rmetis_b200 import functions as F
    n = len(x) - 1
    t = oracle.compute_target_weights(n, ncon, v, k, tp)
    g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
    gp, gcut, stats = F.greedy_refine(g, part, k, t, ub, niter)
    # the model: the reference's repair pass, then admission cut passes
    rp, _, rmoves = oracle.greedy_refine(x, a, part, k, t, ub, 0, vwgt=v, adjwgt=w, ncon=ncon)
    feas = M.feasible_limits(t, ub, k, ncon)
    pw = M.part_weights(v, rp, k, ncon)
    cur = rp
    total_moves = int(rmoves.sum())
    passes = 1
    moved_any = False
    for _ in range(niter):
        cur, pw, moves, rounds, conv = M.admit_pass(x, a, v, w, cur, k, ncon, feas, pw)
        total_moves += moves
        passes += 1
        moved_any |= moves > 0
        if moves == 0:
            break
    assert (gp == cur).all(), f"{int((gp != cur).sum())} vertices differ from the model"
    assert gcut == oracle.edge_cut(x, a, w, gp)
    assert stats[0] == passes and stats[1] == total_moves
    # every part that received a vertex ends within its limit
    start_pw = M.part_weights(v, rp, k, ncon)
    recv = np.zeros(k, bool)
    recv[np.unique(gp[gp != rp])] = True
    assert (pw[recv] <= feas[recv]).all()
    assert (pw[~recv] <= np.maximum(start_pw[~recv], feas[~recv])).all()
    return total_moves, moved_any


@pytest.mark.parametrize("k", [4, 16, 64])
def test_admission_matches_model_grid3d(rmb, oracle, admit_everywhere, k):
    x, a, v, w = G.grid3d(40, 40, 30, weights_seed=8)
    part = _start(len(x) - 1, k, 3, frac=0.3)
    moves, moved = _check_passes(rmb, oracle, x, a, v, w, part, k, [1.03])
    assert moved


def test_admission_matches_model_unweighted_grid(rmb, oracle, admit_everywhere):
    x, a = G.grid2d(300, 300)
    part = _start(len(x) - 1, 8, 5, frac=0.1)
    _check_passes(rmb, oracle, x, a, None, None, part, 8, [1.05], niter=6)


def test_admission_matches_model_two_constraints_tpwgts(rmb, oracle, admit_everywhere):
    x, a, _, w = G.random_graph(60000, 8.0, seed=12)
    n = len(x) - 1
    v = np.random.default_rng(4).integers(1, 9, 2 * n).astype(np.int32)
    k = 32
    tp = np.random.default_rng(5).random(k * 2).astype(np.float32)
    tp = (tp.reshape(k, 2) / tp.reshape(k, 2).sum(axis=0)).reshape(-1)
    part = _start(n, k, 6, frac=0.5)
    _check_passes(rmb, oracle, x, a, v, w, part, k, [1.05, 1.05], ncon=2, tp=tp)


def test_admission_matches_model_rmat_hubs(rmb, oracle, admit_everywhere):
    x, a = G.rmat(15, seed=8)
    part = _start(len(x) - 1, 64, 7, frac=1.0)
    _check_passes(rmb, oracle, x, a, None, None, part, 64, [1.03])


def test_admission_tight_limits(rmb, oracle, admit_everywhere):
    """ub barely above 1: most picks are dropped and the rounds cascade."""
    x, a, v, w = G.grid3d(48, 40, 30, weights_seed=2)
    part = _start(len(x) - 1, 24, 9, frac=0.05)
    _check_passes(rmb, oracle, x, a, v, w, part, 24, [1.0005])


@pytest.mark.parametrize("name", ["grid3d_40_w", "rgg_30k"])
def test_full_partition_with_admission(rmb, oracle, admit_everywhere, name):
    """Whole partitions with every large level decided by admission: valid,
    reproducible, within the reference's limit where the oracle is, and a
    summed cut within 5% of the oracle's over 8 seeds."""
    if name == "grid3d_40_w":
        x, a, v, w = G.grid3d(40, 40, 30, weights_seed=8)
        k = 32
    else:
        x, a, w, _ = G.rgg2d(30000, 4)
        v, k = None, 16
    gpu, ref = [], []
    for s in range(1, 9):
        rc, part, obj = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, options=greedy_options(seed=s))
        assert rc == 1 and obj == oracle.edge_cut(x, a, w, part)
        rc2, part2, obj2 = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, options=greedy_options(seed=s))
        assert obj2 == obj and (part2 == part).all()
        gpu.append((obj, overshoot(oracle, x, v, part, k, 1)))
        rc, p_, o_ = oracle.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, options=greedy_options(seed=s))
        ref.append((o_, overshoot(oracle, x, v, p_, k, 1)))
    assert sum(c for c, _ in gpu) <= 1.05 * sum(c for c, _ in ref), (gpu, ref)
    assert max(o for _, o in gpu) <= max(0.0, max(o for _, o in ref))
