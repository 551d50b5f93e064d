"""Checks shared by the FM tests (src/refine/fm_kway.rs): the best move of a
vertex as the reference's compute_move_gain closure defines it, and the
balance and fixed-point properties of a refined partition."""
import numpy as np


def best_moves(xadj, adjncy, adjwgt, part, k):
    """Per vertex (best part or -1, its gain): the adjacent part p != part[v]
    with the largest edge_to[p] - edge_to[part[v]] > 0, lowest p on ties
    (fm_kway.rs:47-71)."""
    n = len(xadj) - 1
    bp = np.full(n, -1, np.int64)
    bg = np.zeros(n, np.int64)
    for v in range(n):
        s, e = int(xadj[v]), int(xadj[v + 1])
        to = {}
        for j in range(s, e):
            q = int(part[adjncy[j]])
            to[q] = to.get(q, 0) + (1 if adjwgt is None else int(adjwgt[j]))
        pv = int(part[v])
        wf = to.get(pv, 0)
        best, bgain = -1, 0
        for q in sorted(to):
            if q == pv or to[q] == 0:
                continue
            g = to[q] - wf
            if g > bgain:
                best, bgain = q, g
        bp[v], bg[v] = best, bgain
    return bp, bg


def part_weights(part, k, vwgt, ncon):
    n = len(part)
    w = np.ones((n, ncon), np.int64) if vwgt is None else np.asarray(vwgt, np.int64).reshape(n, ncon)
    pw = np.zeros((k, ncon), np.int64)
    np.add.at(pw, np.asarray(part, np.int64), w)
    return pw


def feasible(pw_row, vw, targets_row, ubvec):
    """The reference's test (fm_kway.rs:103-106): (pw + vw) as f64 <= t * ub on
    every constraint."""
    return all(float(pw_row[c] + vw[c]) <= float(targets_row[c]) * float(ubvec[c]) for c in range(len(vw)))


def balance_bound_holds(part0, part1, k, vwgt, ncon, targets, ubvec):
    """A part only receives a vertex while it stays feasible, so every final
    part weight is at most max(its start weight, the largest feasible one)."""
    p0 = part_weights(part0, k, vwgt, ncon)
    p1 = part_weights(part1, k, vwgt, ncon)
    t = np.asarray(targets, np.float64).reshape(k, ncon)
    for p in range(k):
        for c in range(ncon):
            if p1[p, c] > p0[p, c] and not float(p1[p, c]) <= t[p, c] * float(ubvec[c]):
                return False
    return True


def fixed_point_violations(xadj, adjncy, adjwgt, vwgt, part, k, ncon, targets, ubvec):
    """Vertices whose best move has a positive gain and is feasible: after a
    pass without a move there are none."""
    bp, bg = best_moves(xadj, adjncy, adjwgt, part, k)
    pw = part_weights(part, k, vwgt, ncon)
    n = len(part)
    w = np.ones((n, ncon), np.int64) if vwgt is None else np.asarray(vwgt, np.int64).reshape(n, ncon)
    t = np.asarray(targets, np.float64).reshape(k, ncon)
    bad = []
    for v in range(n):
        if bp[v] >= 0 and feasible(pw[bp[v]], w[v], t[bp[v]], ubvec):
            bad.append(v)
    return bad
