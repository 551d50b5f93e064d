"""The no-allocation entry point (RMETIS_GPU_EdgeCutWeightsNoAlloc).

It serves callers that cannot allocate device memory where they need an edge
cut and part weights (recording a CUDA graph, a host-owned fixed memory
budget, loops that must not synchronise the device): the library keeps its
scratch in a fixed device array instead. This test calls it through the C ABI
twice in a row on device buffers and compares both results with the
allocating entry points RMETIS_GPU_EdgeCut and RMETIS_GPU_PartitionWeights
(exact integer equality). The file is collected last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from rmetis_b200 import generators as G

pytestmark = pytest.mark.gpu


def test_no_alloc_matches_allocating_entry_points(rmb):
    torch = pytest.importorskip("torch")
    lib = rmb._lib.load()
    cases = [
        (G.grid3d(30, 28, 26, weights_seed=11), 64, 1),
        (G.random_graph(20000, 9.0, seed=3), 37, 2),
    ]
    stream = torch.cuda.current_stream()
    for (x, a, v, w), k, ncon in cases:
        n = len(x) - 1
        if ncon == 2:
            v = np.random.default_rng(5).integers(1, 9, 2 * n).astype(np.int32)
        g = rmb.Graph(n, ncon, x, a, vwgt=v, adjwgt=w)
        dev = lambda arr: None if arr is None else torch.from_numpy(np.ascontiguousarray(arr, np.int32)).cuda()
        dx, da, dv, dw = dev(x), dev(a), dev(v), dev(w)
        ptr = lambda t: None if t is None else t.data_ptr()
        for call in range(2):  # two calls in a row: the shared scratch is cleared each time
            part = np.random.default_rng(100 + call).integers(0, k, n).astype(np.int32)
            dpart = dev(part)
            dcut = torch.full((1,), -7, dtype=torch.int32, device="cuda")
            dpw = torch.full((k * ncon,), -7, dtype=torch.int32, device="cuda")
            rc = lib.RMETIS_GPU_EdgeCutWeightsNoAlloc(n, ncon, len(a), ptr(dx), ptr(da), ptr(dw), ptr(dv),
                                                      ptr(dpart), k, ptr(dcut), ptr(dpw), stream.cuda_stream)
            assert rc == 1
            torch.cuda.synchronize()
            assert int(dcut.item()) == g.edge_cut(part)
            assert (dpw.cpu().numpy().reshape(k, ncon) == g.partition_weights(part, k)).all()


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
