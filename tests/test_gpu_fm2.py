"""2-way FM refinement of bisections on the GPU (RMETIS_GPU_Fm2Refine,
src/refine/fm.rs:12-127) against the oracle's restatement (fm2_refine).

The reference moves one queued vertex at a time, negative gains included,
and undoes the moves after the lowest cut; the GPU moves rounds of
non-adjacent free boundary vertices of the largest gain and undoes the rounds
after the lowest cut. Checked: the cut never rises and equals the edge cut of the result;
every side ends at most at max(its start weight, floor(t * ub)); the same
input gives the same output; and the summed cut over the cases is within 5%
of the oracle's. The reference's own case (fm.rs:145-159) is checked too.
"""
import numpy as np
import pytest

from rmetis_b200 import generators as G

pytestmark = pytest.mark.gpu


def _case(rmb, oracle, x, a, v, w, part, ub, ncon=1, niter=10, tp=(0.5, 0.5)):
    from rmetis_b200 import functions as F
    n = len(x) - 1
    t = oracle.compute_target_weights(n, ncon, v, 2, np.repeat(np.asarray(tp, np.float32), ncon))
    g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
    before = oracle.edge_cut(x, a, w, part)
    gp, gcut, stats = F.fm2_refine(g, part, t, ub, niter)
    assert set(np.unique(gp).tolist()) <= {0, 1}
    assert gcut == oracle.edge_cut(x, a, w, gp) and gcut <= before
    vw = np.ones((n, ncon), np.int64) if v is None else np.asarray(v, np.int64).reshape(n, ncon)
    lim = np.floor(np.asarray(t, np.float64).reshape(2, ncon) * np.asarray(ub, np.float64)[None, :])
    p0 = np.zeros((2, ncon), np.int64)
    p1 = np.zeros((2, ncon), np.int64)
    np.add.at(p0, part, vw)
    np.add.at(p1, gp, vw)
    assert (p1 <= np.maximum(p0, lim)).all()
    again = F.fm2_refine(g, part, t, ub, niter)
    assert again[1] == gcut and (again[0] == gp).all()
    op, ocut = oracle.fm2_refine(x, a, part, t, ub, niter, vwgt=v, adjwgt=w, ncon=ncon)
    return gcut, ocut, before


def test_fm2_reference_case(rmb, oracle):
    """fm.rs:145-159: a 2x4 grid split badly improves."""
    x, a = G.grid2d(2, 4)
    part = np.array([0, 1, 0, 1, 1, 0, 1, 0], np.int32)
    gcut, ocut, before = _case(rmb, oracle, x, a, None, None, part, [1.5])
    assert gcut < before


def _starts(n, seed, noise):
    rng = np.random.default_rng(seed)
    part = (np.arange(n) >= n // 2).astype(np.int32)
    flip = rng.random(n) < noise
    part[flip] = 1 - part[flip]
    return part


@pytest.mark.parametrize("ub", [1.001, 1.05])
def test_fm2_quality_against_the_oracle(rmb, oracle, ub):
    cases = []
    x, a = G.grid2d(60, 60)
    cases.append((x, a, None, None))
    x, a, v, w = G.grid3d(20, 18, 16, weights_seed=4)
    cases.append((x, a, v, w))
    x, a, _, w = G.random_graph(5000, 7.0, seed=3)
    cases.append((x, a, None, w))
    x, a, w, pts = G.rgg2d(8000, 9)
    cases.append((x, a, None, w))
    tot_g = tot_o = 0
    for i, (x, a, v, w) in enumerate(cases):
        n = len(x) - 1
        for seed, noise in ((1, 0.02), (2, 0.1)):
            part = _starts(n, 10 * i + seed, noise)
            if i == 3:  # the RGG's ids are random in space: split it by x instead
                half = (pts[:, 0] >= np.median(pts[:, 0])).astype(np.int32)
                flip = np.random.default_rng(10 * i + seed).random(n) < noise
                part = np.where(flip, 1 - half, half).astype(np.int32)
            gcut, ocut, before = _case(rmb, oracle, x, a, v, w, part, [ub])
            tot_g += gcut
            tot_o += ocut
    print(f"\n2-way FM ub={ub}: GPU summed cut {tot_g}, oracle {tot_o}, ratio {tot_g / tot_o:.3f}")
    assert tot_g <= 1.05 * tot_o, (tot_g, tot_o)


def test_fm2_two_constraints(rmb, oracle):
    x, a, _, w = G.random_graph(4000, 8.0, seed=21)
    n = len(x) - 1
    v = np.random.default_rng(2).integers(1, 9, 2 * n).astype(np.int32)
    part = _starts(n, 5, 0.05)
    _case(rmb, oracle, x, a, v, w, part, [1.05, 1.05], ncon=2)
