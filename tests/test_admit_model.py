"""CPU checks of the parallel-admission rule (tests/admit_model.py, the model
the GPU kernel is compared with): every move is a positive-gain move its
mover could make alone, each part admits a prefix of its picks in vertex-id
order, and every part that receives a move ends within floor(t * ub) on
every constraint, whatever the cascade of dropped moves."""
import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests import admit_model as M


def _case(seed, n=3000, k=12, ncon=1, ub=1.03):
    x, a, _, w = G.random_graph(n, 7.0, seed=seed)
    rng = np.random.default_rng(seed)
    v = rng.integers(1, 6, n * ncon).astype(np.int32)
    part = rng.integers(0, k, n).astype(np.int32)
    t = np.tile(v.reshape(n, ncon).sum(axis=0) / k, k)
    feas = M.feasible_limits(t, [ub] * ncon, k, ncon)
    return x, a, v, w, part, k, ncon, feas


@pytest.mark.parametrize("seed,ncon,ub", [(1, 1, 1.03), (2, 1, 1.001), (3, 2, 1.05), (4, 3, 1.2)])
def test_admission_rule_properties(seed, ncon, ub):
    x, a, v, w, part, k, ncon, feas = _case(seed, ncon=ncon, ub=ub)
    pw = M.part_weights(v, part, k, ncon)
    tgt = M.picks(x, a, v, w, part, k, ncon, feas, pw)
    new, pw2, moves, rounds, conv = M.admit_pass(x, a, v, w, part, k, ncon, feas, pw)
    moved = np.nonzero(new != part)[0]
    assert moves == len(moved)
    # every move is its mover's pick
    assert (new[moved] == tgt[moved]).all()
    conn = M.connection(x, a, w, part, k)
    gains = conn[moved, new[moved]] - conn[moved, part[moved]]
    assert (gains > 0).all()
    vw = M.vertex_weights(v, len(part), ncon)
    assert (pw[new[moved]] + vw[moved] <= feas[new[moved]]).all()
    # admitted moves into a part are a prefix (by id) of its picks
    for p in range(k):
        picks_p = np.nonzero(tgt == p)[0]
        took = np.isin(picks_p, moved)
        if took.any():
            assert took[:took.sum()].all()
    # weights: recomputed from scratch, receiving parts within the limit
    assert (pw2 == M.part_weights(v, new, k, ncon)).all()
    recv = np.zeros(k, bool)
    recv[np.unique(new[moved])] = True
    assert (pw2[recv] <= feas[recv]).all()
    assert (pw2[~recv] <= pw[~recv]).all()
    assert rounds >= 1


def test_admission_counts_moves_out_of_a_part():
    """Part 1 has room for one vertex alone, but two of its vertices leave in
    the same pass, so it admits all three vertices that pick it."""
    # edges (weight): 0-1 (1), 0-3 (5), 1-3 (5), 2-3 (1), 2-4 (5)
    edges = [(0, 1, 1), (0, 3, 5), (1, 3, 5), (2, 3, 1), (2, 4, 5)]
    n = 5
    src = np.array([u for u, v, _ in edges] + [v for u, v, _ in edges])
    dst = np.array([v for u, v, _ in edges] + [u for u, v, _ in edges])
    wt = np.array([c for _, _, c in edges] * 2)
    order = np.lexsort((dst, src))
    x = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(src, minlength=n), out=x[1:])
    a, w = dst[order].astype(np.int32), wt[order].astype(np.int32)
    part = np.array([0, 0, 1, 1, 2], np.int32)
    feas = np.full((3, 1), 3, np.int64)
    pw = M.part_weights(None, part, 3, 1)
    tgt = M.picks(x, a, None, w, part, 3, 1, feas, pw)
    assert list(tgt) == [1, 1, 2, 0, 1]
    new, pw2, moves, rounds, conv = M.admit_pass(x, a, None, w, part, 3, 1, feas, pw)
    assert conv and moves == 5 and list(new) == [1, 1, 2, 0, 1] and list(pw2[:, 0]) == [1, 3, 1]
