"""METIS .graph files (DEVELOPMENT_GUIDE.md:844-866): the guide's example,
every fmt variant, comments, and the errors a reader must report."""
import numpy as np
import pytest

from rmetis_b200 import generators as G


def test_guide_example_is_the_reference_cycle(rmb):
    # The example of the guide: 4 vertices, 4 edges, no weights, 1-based.
    g = rmb.parse_metis_graph("% a 4-cycle\n4 4\n2 4\n1 3\n2 4\n1 3\n")
    assert g.nvtxs == 4 and g.nedges == 4
    assert list(g.xadj) == [0, 2, 4, 6, 8]
    assert list(g.adjncy) == [1, 3, 0, 2, 1, 3, 0, 2]   # the cycle of src/refine/greedy.rs:229-251
    assert g.vwgt is None and g.adjwgt is None


@pytest.mark.parametrize("vsize,vwgt,ewgt,ncon", [(0, 0, 0, 1), (0, 0, 1, 1), (0, 1, 0, 1), (0, 1, 1, 1),
                                                   (0, 1, 1, 3), (1, 0, 0, 1), (1, 1, 1, 2)])
def test_round_trip(rmb, tmp_path, vsize, vwgt, ewgt, ncon):
    x, a, w, _ = G.rgg2d(500, 3, 7.0)
    n = len(x) - 1
    rng = np.random.default_rng(1)
    g = rmb.Graph.new(n, ncon, x, a,
                      vwgt=rng.integers(1, 9, n * ncon).astype(np.int32) if vwgt else None,
                      adjwgt=w if ewgt else None,
                      vsize=rng.integers(1, 5, n).astype(np.int32) if vsize else None)
    p = tmp_path / "g.graph"
    rmb.write_metis_graph(g, p)
    h = rmb.read_metis_graph(p)
    assert (h.nvtxs, h.ncon) == (g.nvtxs, g.ncon)
    assert (h.xadj == g.xadj).all() and (h.adjncy == g.adjncy).all()
    for f in ("vwgt", "adjwgt", "vsize"):
        a_, b_ = getattr(g, f), getattr(h, f)
        assert (a_ is None) == (b_ is None)
        if a_ is not None:
            assert (a_ == b_).all()
    header = p.read_text().splitlines()[0].split()
    fmt = f"{vsize}{vwgt}{ewgt}".lstrip("0") or "0"
    assert header[:2] == [str(n), str(len(a) // 2)]
    if fmt != "0" or ncon != 1:
        assert header[2] == fmt


def test_comments_and_blank_lines(rmb):
    text = "% header comment\n\n3 2 1\n% vertex 1\n2 5\n1 5 3 7\n2 7\n"
    g = rmb.parse_metis_graph(text)
    assert list(g.adjncy) == [1, 0, 2, 1] and list(g.adjwgt) == [5, 5, 7, 7]


def test_isolated_vertex_lines(rmb):
    # An isolated vertex has an empty line.
    g = rmb.parse_metis_graph("3 1\n2\n1\n\n")
    assert list(g.xadj) == [0, 1, 2, 2]


@pytest.mark.parametrize("text,msg", [
    ("", "empty"),
    ("3 1\n2\n1\n", "vertex lines"),                 # one vertex line missing
    ("2 2\n2\n1\n", "neighbour entries"),            # edge count does not match
    ("2 1\n3\n1\n", "outside"),                      # 1-based id out of range
    ("2 1\n0\n1\n", "outside"),                      # 0 is not a 1-based id
    ("2 1 1\n2\n1 4\n", "edge weight"),              # neighbour without its weight
    ("2 1 10 2\n5\n5\n", "missing weights"),        # ncon=2 but one weight
    ("2 1 0 2\n2\n1\n", "ncon given"),
    ("2 1 7\n2\n1\n", "fmt"),
])
def test_errors(rmb, text, msg):
    with pytest.raises(rmb.InputError, match=msg):
        rmb.parse_metis_graph(text)


def test_asymmetric_file_fails_validation(rmb):
    # Vertex 1 lists 2 twice, vertex 2 lists 1 once and 3 once: the counts
    # match (2 edges) but the degree symmetry check of validate_csr fails.
    with pytest.raises(rmb.InputError):
        rmb.parse_metis_graph("3 2\n2 2\n1 3\n\n")


def test_grid_file_partitions_like_the_array(rmb, oracle, tmp_path):
    """A file written from a generated grid reads back to the same CSR, so the
    oracle gives it the same cut."""
    x, a, v, w = G.grid3d(8, weights_seed=2)
    g = rmb.Graph.new(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
    p = tmp_path / "grid.graph"
    rmb.write_metis_graph(g, p)
    h = rmb.read_metis_graph(p)
    part = np.random.default_rng(0).integers(0, 4, g.nvtxs).astype(np.int32)
    assert oracle.edge_cut(h.xadj, h.adjncy, h.adjwgt, part) == oracle.edge_cut(x, a, w, part)
