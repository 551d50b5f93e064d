"""A numpy model of the parallel admission of a greedy cut pass
(rmetis_b200/csrc/admit.cu), used to check the kernel bit for bit.

The reference's cut pass (src/refine/greedy.rs:126-190) decides movers one
after another in ascending id; the parallel form decides them together:

1. pick: every boundary vertex takes the part with the best positive gain
   (lowest part id on ties) among the parts its move alone keeps feasible
   under the start-of-pass weights: pw[p][c] + vw[c] <= feas[p][c] for all c;
2. each part's in-list is its picks in ascending vertex id; a part admits
   the longest prefix of its in-list whose summed weight fits
   feas - pw + (weight of the admitted moves out of it), on every
   constraint; dropping moves lowers other parts' out-credit, so this is
   repeated until nothing changes (at most 64 rounds, after which each part
   keeps only the prefix that fits with no out-credit);
3. the admitted moves apply together.

Gains use the start-of-pass part vector, as in the reference.
"""
from __future__ import annotations

import numpy as np

MAX_ROUNDS = 64


def connection(x, a, w, part, k):
    """conn[v][p] = summed weight of v's edges into part p."""
    n = len(x) - 1
    src = np.repeat(np.arange(n), np.diff(np.asarray(x, np.int64)))
    wt = np.ones(len(a), np.int64) if w is None else np.asarray(w, np.int64)
    conn = np.zeros((n, k), np.int64)
    np.add.at(conn, (src, np.asarray(part)[np.asarray(a)]), wt)
    return conn


def vertex_weights(v, n, ncon):
    return np.ones((n, ncon), np.int64) if v is None else np.asarray(v, np.int64).reshape(n, ncon)


def picks(x, a, v, w, part, k, ncon, feas, pw):
    """Target part of every vertex (-1: no move)."""
    n = len(x) - 1
    part = np.asarray(part)
    conn = connection(x, a, w, part, k)
    ids = np.arange(n)
    wfrom = conn[ids, part]
    gain = conn - wfrom[:, None]
    others = np.arange(k)[None, :] != part[:, None]
    boundary = ((conn > 0) & others).any(axis=1)
    vw = vertex_weights(v, n, ncon)
    alone = (pw[None, :, :] + vw[:, None, :] <= feas[None, :, :]).all(axis=2)
    ok = (gain > 0) & alone & others & boundary[:, None]
    best = np.where(ok, gain, np.iinfo(np.int64).min).argmax(axis=1)  # first max: lowest part
    return np.where(ok.any(axis=1), best, -1)


def admit_pass(x, a, v, w, part, k, ncon, feas, pw):
    """One cut pass. Returns (new part, new pw, moves, rounds, converged)."""
    n = len(x) - 1
    part = np.array(part, np.int32)
    vw = vertex_weights(v, n, ncon)
    tgt = picks(x, a, v, w, part, k, ncon, feas, pw)
    inlist = [np.nonzero(tgt == p)[0] for p in range(k)]
    cums = [np.cumsum(vw[l], axis=0) for l in inlist]
    cut = [len(l) for l in inlist]

    def fit(p, imax, budget):
        if imax == 0 or (budget < 0).any():
            return 0
        ok = (cums[p][:imax] <= budget[None, :]).all(axis=1)
        bad = np.nonzero(~ok)[0]
        return int(bad[0]) if len(bad) else imax

    rounds, converged = 0, False
    while rounds < MAX_ROUNDS:
        rounds += 1
        out = np.zeros((k, ncon), np.int64)
        for p in range(k):
            acc = inlist[p][:cut[p]]
            np.add.at(out, part[acc], vw[acc])
        changed = False
        new = []
        for p in range(k):
            c = fit(p, cut[p], feas[p] - pw[p] + out[p])
            changed |= c < cut[p]
            new.append(c)
        cut = new
        if not changed:
            converged = True
            break
    if not converged:
        cut = [fit(p, cut[p], feas[p] - pw[p]) for p in range(k)]
    pw = pw.copy()
    moves = 0
    for p in range(k):
        acc = inlist[p][:cut[p]]
        np.add.at(pw, part[acc], -vw[acc])
        pw[p] += vw[acc].sum(axis=0)
        moves += len(acc)
    for p in range(k):
        part[inlist[p][:cut[p]]] = p
    return part, pw, moves, rounds, converged


def feasible_limits(targets, ubvec, k, ncon):
    """floor(t * ub) per part and constraint (the integer form of the
    reference's f64 test)."""
    t = np.asarray(targets, np.float64).reshape(k, ncon)
    return np.floor(t * np.asarray(ubvec, np.float64)[None, :]).astype(np.int64)


def part_weights(v, part, k, ncon):
    n = len(part)
    pw = np.zeros((k, ncon), np.int64)
    np.add.at(pw, np.asarray(part), vertex_weights(v, n, ncon))
    return pw
