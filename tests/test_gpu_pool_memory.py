"""The worker pool's out-of-memory path, exercised without driving a GPU out
of memory.

A child process runs with RMETIS_B200_ARENA_CAP set to 300 MiB: every device
workspace allocation of the library past that total fails on the host as a
cudaMalloc out of memory would (the arenas take 256 MiB chunks). With two
workers:

* two small requests submitted together cannot both hold a chunk, so one of
  them fails beside the other, is retried alone once every worker has freed
  its workspace, and succeeds; both results equal the plain call's;
* a request that needs more than the cap even alone returns
  METIS_ERROR_MEMORY (-3, src/ffi/c_api.rs:205-207 maps allocation failure to
  it) after its retry;
* the next small request succeeds again: the failed job released its space.
"""
import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import json, sys
    sys.path.insert(0, {root!r})
    import numpy as np
    import rmetis_b200 as rmb
    from rmetis_b200 import generators as G
    out = {{}}
    o = rmb.Options(rtype=rmb.RType.Greedy, seed=3)
    small = []
    for side in (30, 32):
        x, a, v, w = G.grid3d(side, weights_seed=side)
        small.append(rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w))
    reqs = [rmb.submit_kway(g, 16, options=o) for g in small]
    res = [r.wait() for r in reqs]
    out["small"] = [[int(r.objval), r.part.tolist()] for r in res]
    x, a, v, w = G.grid3d(128, weights_seed=7)
    big = rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w, validate=False)
    try:
        rmb.submit_kway(big, 64, options=o).wait()
        out["big"] = "ok"
    except rmb.OutOfMemoryError:
        out["big"] = "memory"
    r = rmb.submit_kway(small[0], 16, options=o).wait()
    out["again"] = [int(r.objval), r.part.tolist()]
    print("RESULT " + json.dumps(out))
""")


def test_out_of_memory_retry_and_release(rmb):
    env = dict(os.environ)
    env.update(RMETIS_B200_ARENA_CAP=str(300 << 20), RMETIS_B200_WORKERS="2", RMETIS_B200_VERBOSE="1")
    proc = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                          timeout=600)
    assert proc.returncode == 0, proc.stderr[-3000:]
    line = [ln for ln in proc.stdout.splitlines() if ln.startswith("RESULT ")][-1]
    out = json.loads(line[len("RESULT "):])
    assert "retrying it alone" in proc.stderr
    assert out["big"] == "memory"
    # the same requests in this process (no cap) through the plain call
    from rmetis_b200 import generators as G
    o = rmb.Options(rtype=rmb.RType.Greedy, seed=3)
    for side, (obj, part) in zip((30, 32), out["small"]):
        x, a, v, w = G.grid3d(side, weights_seed=side)
        ref = rmb.part_graph_kway(rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w), 16, options=o)
        assert obj == ref.objval and (np.array(part) == ref.part).all()
    assert out["again"] == out["small"][0]
