"""Debug invariant checks (RMETIS_B200_CHECKS=1) and the per-level JSON trace
(RMETIS_B200_TRACE_JSON=<path>), in a child process with both set.

With the checks on, every contraction is checked (cmap onto [0, cn), one or
two members per coarse vertex, coarse weights summing to the fine ones) and
every refined level (part ids in [0, k), part weights summing to the level's
total); a violation would fail the call with METIS_ERROR. The results must
equal those of a run without the checks, and the trace must hold one line
per attempt with every refined level.
"""
import json
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import json, sys
    sys.path.insert(0, {root!r})
    import rmetis_b200 as rmb
    from rmetis_b200 import generators as G
    out = []
    x, a, v, w = G.grid3d(48, 40, 30, weights_seed=3)
    g = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w)
    for rtype in (rmb.RType.Greedy, rmb.RType.Fm):
        r = rmb.part_graph_kway(g, 32, options=rmb.Options(rtype=rtype, seed=5))
        out.append([int(r.objval), r.part.tolist()])
    x, a = G.grid2d(70, 70)
    r = rmb.part_graph_kway(rmb.Graph(len(x) - 1, 1, x, a), 8, options=rmb.Options(rtype=rmb.RType.Greedy, seed=2))
    out.append([int(r.objval), r.part.tolist()])
    print("RESULT " + json.dumps(out))
""")


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    proc = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                          timeout=600)
    assert proc.returncode == 0, proc.stderr[-3000:]
    line = [ln for ln in proc.stdout.splitlines() if ln.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):]), proc.stderr


def test_checks_pass_and_trace_lists_every_level(tmp_path):
    trace = tmp_path / "trace.jsonl"
    checked, err = _run({"RMETIS_B200_CHECKS": "1", "RMETIS_B200_TRACE_JSON": str(trace)})
    assert "invariant violated" not in err
    plain, _ = _run({})
    assert checked == plain, "the checks and the trace change no result"
    lines = [json.loads(ln) for ln in trace.read_text().splitlines()]
    assert len(lines) == 3
    for rec, (obj, _) in zip(lines, checked):
        assert rec["cut"] == obj
        lv = rec["levels"]
        assert len(lv) >= 2 and lv[-1]["n"] == rec["n"]   # coarsest first, the input graph last
        assert all(x["passes"] >= 1 and x["refine_ms"] >= 0 for x in lv)
        assert [x["n"] for x in lv] == sorted(x["n"] for x in lv)
    assert lines[0]["rtype"] == "greedy" and lines[1]["rtype"] == "fm"
