"""The reference's own known answers (tests/golden/known_answers.json, made by
tests/golden/make_known_answers.py from the reference's unit tests) checked on
the oracle (CPU) and through the GPU library's C ABI."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "known_answers.json")) as _f:
    GOLDEN = json.load(_f)
CASES = GOLDEN["cases"]


def _graph(name):
    g = GOLDEN["graphs"][name]
    w = g.get("adjwgt")
    return (np.array(g["xadj"], np.int32), np.array(g["adjncy"], np.int32),
            None if w is None else np.array(w, np.int32))


def _ids(cases):
    return [f"{c['kind']}:{c['ref']}" for c in cases]


def _coarse_ok(nvtxs, nedges, cmap, exp):
    return (nvtxs == exp["nvtxs"] and nedges == exp["nedges"]
            and all(cmap[a] == cmap[b] for a, b in exp["same"])
            and all(cmap[a] != cmap[b] for a, b in exp["different"]))


@pytest.mark.parametrize("case", CASES, ids=_ids(CASES))
def test_oracle_known_answers(oracle, case):
    kind = case["kind"]
    if kind == "validate":
        v = None if "vwgt" not in case else np.array(case["vwgt"], np.int32)
        rc = oracle.validate_csr(case["n"], 1, np.array(case["xadj"]), np.array(case["adjncy"]), vwgt=v)
        assert (rc == 0) == (case["expect"] == "ok")
        return
    x, a, w = _graph(case["graph"])
    n = len(x) - 1
    if kind == "edge_cut":
        assert oracle.edge_cut(x, a, w, case["part"]) == case["expect"]
    elif kind == "partition_weights":
        assert oracle.partition_weights(n, 1, None, case["part"], case["nparts"]).tolist() == case["expect"]
    elif kind == "total_weight":
        assert oracle.total_weight(n, 1, None).tolist() == case["expect"]
    elif kind == "boundary":
        assert sorted(oracle.boundary_vertices(x, a, case["part"]).tolist()) == case["expect"]
    elif kind == "coarse":
        r = oracle.build_coarse_graph(x, a, case["matching"])
        assert _coarse_ok(r["cn"], len(r["cadjncy"]) // 2, r["cmap"], case["expect"])
    elif kind == "matching":
        rng = oracle.SmallRng(case["seed"])
        m = oracle.shem_matching(x, a, w, rng) if case["mode"] == "shem" else oracle.random_matching(x, a, rng)
        assert all(m[m[v]] == v for v in range(n))
        assert sum(1 for v in range(n) if m[v] != v) >= case["min_matched"]
    elif kind == "refine_no_increase":
        before = oracle.edge_cut(x, a, w, case["part"])
        fn = oracle.greedy_refine if case["rtype"] == "greedy" else oracle.fm_kway_refine
        out = fn(x, a, case["part"], case["nparts"], case["tpwgts"], case["ubvec"], case["niter"], adjwgt=w)
        assert out[1] <= before and out[1] == oracle.edge_cut(x, a, w, out[0])
    else:
        raise AssertionError(f"unknown case kind {kind}")


GPU_KINDS = ("edge_cut", "partition_weights", "boundary", "coarse", "matching", "refine_no_increase")
GPU_CASES = [c for c in CASES if c["kind"] in GPU_KINDS]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_CASES, ids=_ids(GPU_CASES))
def test_gpu_known_answers(rmb, case):
    """The same answers from the GPU entry points. (The validation cases pass
    arrays whose lengths disagree with n, which raw C pointers cannot carry;
    the C ABI's rejections are tested on well-formed arrays in
    tests/test_gpu_kway.py.)"""
    from rmetis_b200 import functions as F
    x, a, w = _graph(case["graph"])
    n = len(x) - 1
    g = rmb.Graph(n, 1, x, a, adjwgt=w)
    kind = case["kind"]
    part = None if "part" not in case else np.array(case["part"], np.int32)
    if kind == "edge_cut":
        assert g.edge_cut(part) == case["expect"]
    elif kind == "partition_weights":
        assert g.partition_weights(part, case["nparts"]).tolist() == case["expect"]
    elif kind == "boundary":
        assert sorted(g.boundary_vertices(part).tolist()) == case["expect"]
    elif kind == "coarse":
        cg, cmap = g.build_coarse_graph(case["matching"])
        assert _coarse_ok(cg.nvtxs, cg.nedges, cmap, case["expect"])
    elif kind == "matching":
        m = F.match(g, mode=1 if case["mode"] == "shem" else 0, seed=case["seed"])
        assert all(m[m[v]] == v for v in range(n))
        assert sum(1 for v in range(n) if m[v] != v) >= case["min_matched"]
    elif kind == "refine_no_increase":
        before = g.edge_cut(part)
        fn = F.greedy_refine if case["rtype"] == "greedy" else F.fm_refine
        out_part, cut, _ = fn(g, part, case["nparts"], case["tpwgts"], case["ubvec"], case["niter"])
        assert cut <= before and cut == g.edge_cut(out_part)
