"""Seeded synthetic graph generators (int32 CSR, symmetric, no self-loops).

These produce the benchmark workloads: 2D 5-point and 3D 7-point grids with
row-major vertex ids and ascending neighbour lists (the layout of the
reference's own grid builder, benches/partition.rs:4-23), R-MAT graphs and 2D
random geometric graphs. All are plain numpy.
"""
from __future__ import annotations

import numpy as np


def _csr_from_pairs(n: int, src: np.ndarray, dst: np.ndarray, w: np.ndarray | None = None):
    """Symmetric CSR from directed pairs that already contain both directions.

    Rows are sorted by neighbour id; `w` (optional) follows the pairs.
    """
    order = np.lexsort((dst, src))
    src = src[order]
    dst = dst[order]
    counts = np.bincount(src, minlength=n)
    xadj = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=xadj[1:])
    out_w = None if w is None else np.ascontiguousarray(w[order], dtype=np.int32)
    return xadj.astype(np.int32), dst.astype(np.int32), out_w


def _stencil_csr(shape):
    """CSR of an axis-aligned grid stencil (2*len(shape) neighbours), row-major
    ids with the last axis fastest. Returns (xadj, adjncy, slots, mask) where
    slots[v, s] is the neighbour in slot s (slots ordered by ascending
    neighbour id: -stride_0 ... -stride_last, +stride_last ... +stride_0)."""
    dims = list(shape)
    n = int(np.prod(dims))
    strides = [int(np.prod(dims[i + 1:])) for i in range(len(dims))]
    coords = np.indices(dims).reshape(len(dims), -1)
    v = np.arange(n, dtype=np.int64)
    nd = len(dims)
    slots = np.full((n, 2 * nd), -1, dtype=np.int64)
    # backward slots: largest stride first (smallest neighbour id first)
    for i in range(nd):
        ok = coords[i] > 0
        slots[ok, i] = v[ok] - strides[i]
    # forward slots: smallest stride first
    for j, i in enumerate(reversed(range(nd))):
        ok = coords[i] < dims[i] - 1
        slots[ok, nd + j] = v[ok] + strides[i]
    mask = slots >= 0
    deg = mask.sum(axis=1)
    xadj = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=xadj[1:])
    adjncy = slots[mask]
    return xadj.astype(np.int32), adjncy.astype(np.int32), slots, mask, strides


def _stencil_weights(slots, mask, strides, rng, lo, hi):
    """Edge weights drawn once per undirected edge (u < v, in CSR order) and
    mirrored: forward slots in vertex-major order are exactly the CSR order of
    the u < v entries."""
    n, s2 = slots.shape
    nd = s2 // 2
    W = np.zeros((n, s2), dtype=np.int32)
    fwd = mask[:, nd:]
    W[:, nd:][fwd] = rng.integers(lo, hi + 1, size=int(fwd.sum()), dtype=np.int32)
    for j, i in enumerate(reversed(range(nd))):
        # backward slot i of v mirrors forward slot nd+j of v - strides[i]
        ok = mask[:, i]
        src = np.nonzero(ok)[0] - strides[i]
        W[ok, i] = W[src, nd + j]
    return W[mask]


def grid2d(rows: int, cols: int):
    """2D 5-point grid, row-major ids, neighbours ascending."""
    xadj, adjncy, _, _, _ = _stencil_csr((rows, cols))
    return xadj, adjncy


def grid3d(nx: int, ny: int | None = None, nz: int | None = None, weights_seed: int | None = None):
    """3D 7-point grid, row-major ids (x fastest), neighbours ascending.

    With `weights_seed`, draws vwgt ~ U{1..4} per vertex and adjwgt ~ U{1..10}
    once per undirected edge (u < v, in CSR order) and mirrors it, from
    numpy default_rng(weights_seed). Returns (xadj, adjncy, vwgt, adjwgt).
    """
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    xadj, adjncy, slots, mask, strides = _stencil_csr((nz, ny, nx))
    if weights_seed is None:
        return xadj, adjncy, None, None
    rng = np.random.default_rng(weights_seed)
    n = nx * ny * nz
    vwgt = rng.integers(1, 5, size=n, dtype=np.int32)
    adjwgt = _stencil_weights(slots, mask, strides, rng, 1, 10)
    return xadj, adjncy, vwgt, adjwgt


def grid_weighted(shape, seed: int, wmax: int = 10):
    """Grid of any dimension with edge weights U{1..wmax} (symmetric)."""
    xadj, adjncy, slots, mask, strides = _stencil_csr(tuple(shape))
    rng = np.random.default_rng(seed)
    return xadj, adjncy, _stencil_weights(slots, mask, strides, rng, 1, wmax)


def symmetric_edge_weights(xadj, adjncy, rng, lo: int, hi: int):
    """Edge weights U{lo..hi} drawn once per undirected edge (u < v, CSR
    order) and mirrored onto (v, u)."""
    n = len(xadj) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(xadj).astype(np.int64))
    dst = adjncy.astype(np.int64)
    fwd = src < dst
    w = np.zeros(len(adjncy), dtype=np.int32)
    w[fwd] = rng.integers(lo, hi + 1, size=int(fwd.sum()), dtype=np.int32)
    # mirror: position of (v,u) for each (u,v) with u<v via key lookup
    key_fwd = src[fwd] * n + dst[fwd]
    key_all = src * n + dst
    rev = ~fwd
    key_rev = dst[rev] * n + src[rev]
    order = np.argsort(key_fwd)
    pos = np.searchsorted(key_fwd[order], key_rev)
    w[rev] = w[fwd][order[pos]]
    del key_all
    return w


def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 22):
    """R-MAT graph with 2**scale vertices and edge_factor * 2**scale generated
    pairs; symmetrised, self-loops and duplicates removed, isolated vertices
    kept, neighbours ascending."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    ne = edge_factor * n
    src = np.zeros(ne, dtype=np.int64)
    dst = np.zeros(ne, dtype=np.int64)
    ab = a + b
    c_norm = c / (1.0 - ab)
    a_norm = a / ab
    for bit in range(scale):
        ii = rng.random(ne) > ab
        jj = rng.random(ne) > np.where(ii, c_norm, a_norm)
        src |= ii.astype(np.int64) << bit
        dst |= jj.astype(np.int64) << bit
    keep = src != dst
    src, dst = src[keep], dst[keep]
    s2 = np.concatenate([src, dst])
    d2 = np.concatenate([dst, src])
    key = np.unique(s2 * n + d2)
    s2 = key // n
    d2 = key % n
    xadj, adjncy, _ = _csr_from_pairs(n, s2, d2)
    return xadj, adjncy


def rmat_device(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 22, device="cuda"):
    """R-MAT built on a CUDA device with torch (a seeded torch.Generator on that
    device), for scales whose host-side sort and dedup take minutes. Same
    construction as rmat(): symmetrised, self-loops and duplicates removed,
    isolated vertices kept, neighbours ascending. The random stream differs
    from rmat()'s numpy one, so the two give different graphs for one seed.
    Returns host numpy (xadj, adjncy)."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    n = 1 << scale
    ne = edge_factor * n
    src = torch.zeros(ne, dtype=torch.int64, device=device)
    dst = torch.zeros(ne, dtype=torch.int64, device=device)
    ab = a + b
    c_norm = c / (1.0 - ab)
    a_norm = a / ab
    for bit in range(scale):
        ii = torch.rand(ne, generator=gen, device=device) > ab
        thr = torch.where(ii, torch.tensor(c_norm, device=device), torch.tensor(a_norm, device=device))
        jj = torch.rand(ne, generator=gen, device=device) > thr
        src |= ii.to(torch.int64) << bit
        dst |= jj.to(torch.int64) << bit
        del ii, jj, thr
    keep = src != dst
    src, dst = src[keep], dst[keep]
    key = torch.unique(torch.cat([src * n + dst, dst * n + src]), sorted=True)
    del src, dst, keep
    s2 = key // n
    adjncy = (key % n).to(torch.int32)
    xadj = torch.zeros(n + 1, dtype=torch.int64, device=device)
    xadj[1:] = torch.cumsum(torch.bincount(s2, minlength=n), 0)
    out = xadj.to(torch.int32).cpu().numpy(), adjncy.cpu().numpy()
    del key, s2, adjncy, xadj
    torch.cuda.empty_cache()
    return out


def rgg2d(n: int, seed, mean_degree: float = 10.0):
    """2D random geometric graph: points U[0,1]^2, radius r = sqrt(mean_degree
    / (pi n)); edge weight 1 + floor(10 * (1 - d / r)). Returns (xadj, adjncy,
    adjwgt, points)."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    r = float(np.sqrt(mean_degree / (np.pi * n)))
    cells = max(1, int(1.0 / r))
    cx = np.minimum((pts[:, 0] * cells).astype(np.int64), cells - 1)
    cy = np.minimum((pts[:, 1] * cells).astype(np.int64), cells - 1)
    cell = cy * cells + cx
    order = np.argsort(cell, kind="stable")
    cell_sorted = cell[order]
    starts = np.searchsorted(cell_sorted, np.arange(cells * cells))
    ends = np.searchsorted(cell_sorted, np.arange(cells * cells), side="right")
    srcs, dsts, ws = [], [], []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            ncx = cx + dx
            ncy = cy + dy
            ok = (ncx >= 0) & (ncx < cells) & (ncy >= 0) & (ncy < cells)
            idx = np.nonzero(ok)[0]
            nc = ncy[idx] * cells + ncx[idx]
            s = starts[nc]
            e = ends[nc]
            cnt = e - s
            rep = np.repeat(idx, cnt)
            offs = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
            cand = order[np.repeat(s, cnt) + offs]
            d = np.sqrt(((pts[rep] - pts[cand]) ** 2).sum(axis=1))
            m = (d < r) & (rep != cand)
            srcs.append(rep[m]); dsts.append(cand[m])
            ws.append(1 + np.floor(10.0 * (1.0 - d[m] / r)).astype(np.int64))
    src = np.concatenate(srcs)
    dst = np.concatenate(dsts)
    w = np.concatenate(ws).astype(np.int32)
    xadj, adjncy, adjwgt = _csr_from_pairs(n, src, dst, w)
    return xadj, adjncy, adjwgt, pts


def rgg2d_device(n: int, seed: int, mean_degree: float = 10.0, device="cuda"):
    """rgg2d() built on a CUDA device with torch (seeded torch.Generator), for
    batches of many graphs: points U[0,1]^2, radius r = sqrt(mean_degree /
    (pi n)), edge weight 1 + floor(10 * (1 - d / r)), neighbours ascending.
    Returns host numpy (xadj, adjncy, adjwgt)."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    pts = torch.rand((n, 2), generator=gen, device=device, dtype=torch.float64)
    r = float(np.sqrt(mean_degree / (np.pi * n)))
    cells = max(1, int(1.0 / r))
    cxy = torch.clamp((pts * cells).to(torch.int64), max=cells - 1)
    cell = cxy[:, 1] * cells + cxy[:, 0]
    order = torch.argsort(cell, stable=True)
    cell_sorted = cell[order]
    ar = torch.arange(cells * cells, device=device)
    starts = torch.searchsorted(cell_sorted, ar)
    ends = torch.searchsorted(cell_sorted, ar, right=True)
    srcs, dsts, ws = [], [], []
    idx_all = torch.arange(n, device=device)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            ncx = cxy[:, 0] + dx
            ncy = cxy[:, 1] + dy
            ok = (ncx >= 0) & (ncx < cells) & (ncy >= 0) & (ncy < cells)
            idx = idx_all[ok]
            nc = ncy[ok] * cells + ncx[ok]
            st = starts[nc]
            cnt = ends[nc] - st
            rep = torch.repeat_interleave(idx, cnt)
            base = torch.repeat_interleave(st - (torch.cumsum(cnt, 0) - cnt), cnt)
            cand = order[base + torch.arange(int(cnt.sum()), device=device)]
            d = torch.sqrt(((pts[rep] - pts[cand]) ** 2).sum(dim=1))
            m = (d < r) & (rep != cand)
            srcs.append(rep[m]); dsts.append(cand[m])
            ws.append(1 + torch.floor(10.0 * (1.0 - d[m] / r)).to(torch.int64))
    src = torch.cat(srcs); dst = torch.cat(dsts); w = torch.cat(ws)
    key = src * n + dst
    o = torch.argsort(key)
    src, dst, w = src[o], dst[o], w[o]
    xadj = torch.zeros(n + 1, dtype=torch.int64, device=device)
    xadj[1:] = torch.cumsum(torch.bincount(src, minlength=n), 0)
    return (xadj.to(torch.int32).cpu().numpy(), dst.to(torch.int32).cpu().numpy(),
            w.to(torch.int32).cpu().numpy())


def path(n: int):
    src = np.concatenate([np.arange(n - 1), np.arange(1, n)])
    dst = np.concatenate([np.arange(1, n), np.arange(n - 1)])
    xadj, adjncy, _ = _csr_from_pairs(n, src, dst)
    return xadj, adjncy


def random_graph(n: int, avg_deg: float, seed: int, max_w: int = 10):
    """Erdos-Renyi-like symmetric graph with random weights; used by tests."""
    rng = np.random.default_rng(seed)
    ne = int(n * avg_deg / 2)
    a = rng.integers(0, n, ne)
    b = rng.integers(0, n, ne)
    keep = a != b
    a, b = a[keep], b[keep]
    lo = np.minimum(a, b); hi = np.maximum(a, b)
    key = np.unique(lo * n + hi)
    lo = key // n; hi = key % n
    src = np.concatenate([lo, hi]); dst = np.concatenate([hi, lo])
    xadj, adjncy, _ = _csr_from_pairs(n, src, dst)
    adjwgt = symmetric_edge_weights(xadj, adjncy, rng, 1, max_w)
    vwgt = rng.integers(1, 5, size=n, dtype=np.int32)
    return xadj, adjncy, vwgt, adjwgt
