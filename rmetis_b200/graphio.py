"""METIS `.graph` files (the format the reference documents for its test
inputs, DEVELOPMENT_GUIDE.md:844-866, which also describes a
`load_metis_graph` test helper that the reference does not ship):

    % comment lines start with '%'
    nvtxs nedges [fmt [ncon]]
    one line per vertex: [vsize] [w_1 .. w_ncon] u [ew] u [ew] ...

`nedges` counts undirected edges; neighbours are 1-based in the file and
0-based in memory. `fmt` has up to three digits "abc": a = vertex sizes
present, b = vertex weights present (`ncon` of them, default 1), c = edge
weights present (0, 1, 10, 11, 100, ... as in METIS). Reading checks the
counts and the neighbour range and then runs the same validation as
`Graph.new` (src/graph/validate.rs:16-142).
"""
from __future__ import annotations

import io
import os

import numpy as np


def _lines(text: str):
    for raw in text.splitlines():
        line = raw.strip()
        if line.startswith("%"):
            continue
        yield line


def parse_metis_graph(text: str):
    """Parse the text of a `.graph` file into a Graph."""
    from . import Graph, InputError
    it = _lines(text)
    header = None
    for line in it:
        if line:
            header = line.split()
            break
    if header is None:
        raise InputError("empty graph file")
    if len(header) < 2 or len(header) > 4:
        raise InputError(f"bad header: {' '.join(header)}")
    n, m = int(header[0]), int(header[1])
    fmt = header[2] if len(header) >= 3 else "0"
    if not fmt.isdigit() or len(fmt) > 3 or any(c not in "01" for c in fmt):
        raise InputError(f"bad fmt field: {fmt} (up to three digits, each 0 or 1)")
    fmt = fmt.zfill(3)
    has_vsize, has_vwgt, has_ewgt = fmt[0] == "1", fmt[1] == "1", fmt[2] == "1"
    ncon = int(header[3]) if len(header) == 4 else 1
    if len(header) == 4 and not has_vwgt:
        raise InputError("ncon given without vertex weights in fmt")
    if n <= 0 or m < 0 or ncon <= 0:
        raise InputError(f"bad sizes: nvtxs={n} nedges={m} ncon={ncon}")
    xadj = np.zeros(n + 1, dtype=np.int64)
    adj, ew = [], []
    vwgt = np.zeros(n * ncon, dtype=np.int64) if has_vwgt else None
    vsize = np.zeros(n, dtype=np.int64) if has_vsize else None
    v = 0
    for line in it:
        if v == n:
            if line:
                raise InputError(f"more than {n} vertex lines")
            continue
        tok = [int(t) for t in line.split()] if line else []
        pos = 0
        if has_vsize:
            if pos >= len(tok):
                raise InputError(f"vertex {v + 1}: missing size")
            vsize[v] = tok[pos]
            pos += 1
        if has_vwgt:
            if pos + ncon > len(tok):
                raise InputError(f"vertex {v + 1}: missing weights")
            vwgt[v * ncon:(v + 1) * ncon] = tok[pos:pos + ncon]
            pos += ncon
        step = 2 if has_ewgt else 1
        rest = tok[pos:]
        if len(rest) % step:
            raise InputError(f"vertex {v + 1}: neighbour without edge weight")
        for j in range(0, len(rest), step):
            u = rest[j]
            if u < 1 or u > n:
                raise InputError(f"vertex {v + 1}: neighbour {u} outside 1..{n}")
            adj.append(u - 1)
            if has_ewgt:
                ew.append(rest[j + 1])
        v += 1
        xadj[v] = len(adj)
    if v != n:
        raise InputError(f"{v} vertex lines for {n} vertices")
    if len(adj) != 2 * m:
        raise InputError(f"{len(adj)} neighbour entries for {m} edges (expected {2 * m})")
    i32 = lambda a: None if a is None else np.asarray(a, dtype=np.int64).astype(np.int32)
    return Graph.new(n, ncon, i32(xadj), i32(adj), vwgt=i32(vwgt), adjwgt=i32(ew) if has_ewgt else None,
                     vsize=i32(vsize))


def read_metis_graph(path: str | os.PathLike):
    """Read a `.graph` file into a Graph (1-based ids become 0-based)."""
    with open(path) as f:
        return parse_metis_graph(f.read())


def format_metis_graph(graph) -> str:
    """The text of a `.graph` file for `graph` (0-based ids become 1-based)."""
    n = graph.nvtxs
    xadj = np.asarray(graph.xadj, dtype=np.int64)
    adj = np.asarray(graph.adjncy, dtype=np.int64)
    if len(adj) % 2:
        raise ValueError("odd number of CSR entries: not a symmetric graph")
    has_vsize = graph.vsize is not None
    has_vwgt = graph.vwgt is not None
    has_ewgt = graph.adjwgt is not None
    fmt = f"{int(has_vsize)}{int(has_vwgt)}{int(has_ewgt)}".lstrip("0") or "0"
    out = io.StringIO()
    header = f"{n} {len(adj) // 2}"
    if fmt != "0" or graph.ncon != 1:
        header += f" {fmt}"
        if graph.ncon != 1:
            header += f" {graph.ncon}"
    out.write(header + "\n")
    for v in range(n):
        tok = []
        if has_vsize:
            tok.append(str(int(graph.vsize[v])))
        if has_vwgt:
            tok += [str(int(x)) for x in graph.vwgt[v * graph.ncon:(v + 1) * graph.ncon]]
        for j in range(xadj[v], xadj[v + 1]):
            tok.append(str(int(adj[j]) + 1))
            if has_ewgt:
                tok.append(str(int(graph.adjwgt[j])))
        out.write(" ".join(tok) + "\n")
    return out.getvalue()


def write_metis_graph(graph, path: str | os.PathLike) -> None:
    """Write `graph` as a `.graph` file."""
    with open(path, "w") as f:
        f.write(format_metis_graph(graph))
