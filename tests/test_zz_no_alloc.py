"""The no-allocation entry point (RMETIS_GPU_EdgeCutWeightsNoAlloc).

It serves callers that cannot allocate device memory where they need an edge
cut and part weights (a host-owned fixed memory budget or pool that must not
grow, loops where cudaMalloc/cudaFree would synchronise the device): the
library keeps its scratch in a fixed device array instead. This test calls it
through the C ABI twice in a row on device buffers and compares both results
with the oracle's edge_cut and partition_weights (exact integer equality,
src/graph/mod.rs:123-149), then checks that out-of-range entries give
*d_cut = -1. The file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import numpy as np
import pytest

from rmetis_b200 import generators as G

pytestmark = pytest.mark.gpu


def _dev(torch, arr):
    return None if arr is None else torch.from_numpy(np.ascontiguousarray(arr, np.int32)).cuda()


def _call(lib, torch, n, ncon, x, a, w, v, part, k):
    ptr = lambda t: None if t is None else t.data_ptr()
    dx, da, dw, dv, dp = (_dev(torch, z) for z in (x, a, w, v, part))
    dcut = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    dpw = torch.full((k * ncon,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.RMETIS_GPU_EdgeCutWeightsNoAlloc(n, ncon, len(a), ptr(dx), ptr(da), ptr(dw), ptr(dv), ptr(dp), k,
                                              ptr(dcut), ptr(dpw), stream.cuda_stream)
    torch.cuda.synchronize()
    return rc, int(dcut.item()), dpw.cpu().numpy().reshape(k, ncon)


def test_no_alloc_matches_the_oracle(rmb, oracle):
    torch = pytest.importorskip("torch")
    lib = rmb._lib.load()
    cases = [
        (G.grid3d(30, 28, 26, weights_seed=11), 64, 1),
        (G.random_graph(20000, 9.0, seed=3), 37, 2),
        (G.grid3d(20, 20, 20, weights_seed=4), 2, 1),       # a bisection: part sums in shared memory
        (G.random_graph(30000, 6.0, seed=8), 5000, 1),      # nparts*ncon above the shared-memory sums
    ]
    for (x, a, v, w), k, ncon in cases:
        n = len(x) - 1
        if ncon == 2:
            v = np.random.default_rng(5).integers(1, 9, 2 * n).astype(np.int32)
        for call in range(2):  # two calls in a row: the shared scratch is cleared each time
            part = np.random.default_rng(100 + call).integers(0, k, n).astype(np.int32)
            rc, cut, pw = _call(lib, torch, n, ncon, x, a, w, v, part, k)
            assert rc == 1
            assert cut == oracle.edge_cut(x, a, w, part)
            assert (pw == oracle.partition_weights(n, ncon, v, part, k)).all()


def test_no_alloc_flags_out_of_range_entries(rmb, oracle):
    """The kernel checks every index before it follows it: a part id outside
    [0, nparts) or a neighbour id outside [0, n) is skipped and flagged."""
    torch = pytest.importorskip("torch")
    lib = rmb._lib.load()
    x, a, v, w = G.grid3d(12, 10, 8, weights_seed=2)
    n, k = len(x) - 1, 8
    part = np.random.default_rng(1).integers(0, k, n).astype(np.int32)
    bad_part = part.copy()
    bad_part[n // 2] = k
    assert _call(lib, torch, n, 1, x, a, w, v, bad_part, k)[:2] == (1, -1)
    bad_adj = a.copy()
    bad_adj[len(a) // 3] = n + 5
    assert _call(lib, torch, n, 1, x, bad_adj, w, v, part, k)[:2] == (1, -1)
    # the next well-formed call is unaffected by the flag of the one before
    rc, cut, pw = _call(lib, torch, n, 1, x, a, w, v, part, k)
    assert rc == 1 and cut == oracle.edge_cut(x, a, w, part)


def test_no_alloc_rejects_sizes_beyond_the_limit(rmb):
    torch = pytest.importorskip("torch")
    lib = rmb._lib.load()
    x, a = G.grid2d(8, 8)
    dx = torch.from_numpy(x).cuda()
    da = torch.from_numpy(a).cuda()
    dp = torch.zeros(64, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.RMETIS_GPU_EdgeCutWeightsNoAlloc(64, 2, len(a), dx.data_ptr(), da.data_ptr(), None, None,
                                                dp.data_ptr(), 9000, out.data_ptr(), out.data_ptr(), None) == -2
