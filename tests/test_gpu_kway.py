"""Full k-way partitions on the GPU through the drop-in C ABI: validity,
balance, determinism, objval, quality against the oracle's best-of-ncuts, and
the reference's error behaviour."""
import ctypes

import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests.conftest import greedy_options

pytestmark = pytest.mark.gpu


def call_c_abi(rmb, x, a, k, vwgt=None, adjwgt=None, ncon=1, options=None, tpwgts=None, ubvec=None):
    lib = rmb._lib.load()
    I32P = ctypes.POINTER(ctypes.c_int32)
    F32P = ctypes.POINTER(ctypes.c_float)
    n = len(x) - 1
    p = lambda arr: None if arr is None else np.ascontiguousarray(arr, np.int32).ctypes.data_as(I32P)
    keep = [np.ascontiguousarray(arr, np.int32) if arr is not None else None for arr in (x, a, vwgt, adjwgt, options)]
    part = np.full(n, -7, np.int32)
    obj = ctypes.c_int32(-1)
    nv, nc, npr = ctypes.c_int32(n), ctypes.c_int32(ncon), ctypes.c_int32(k)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, np.float32)
    ub = None if ubvec is None else np.ascontiguousarray(ubvec, np.float32)
    rc = lib.RMETIS_PartGraphKway(ctypes.byref(nv), ctypes.byref(nc), *(p(k_) for k_ in keep[:2]), p(keep[2]), None,
                                  p(keep[3]), ctypes.byref(npr), None if tp is None else tp.ctypes.data_as(F32P),
                                  None if ub is None else ub.ctypes.data_as(F32P), p(keep[4]), ctypes.byref(obj),
                                  part.ctypes.data_as(I32P))
    return rc, part, obj.value


def feasible_limit(oracle, n, ncon, vwgt, k, ub, tpwgts=None):
    t = oracle.compute_target_weights(n, ncon, vwgt, k, tpwgts).reshape(k, ncon)
    return np.floor(t * np.asarray(ub)[None, :])


def check_partition(oracle, x, a, v, w, part, k, obj, ncon=1, ufactor=30):
    n = len(x) - 1
    assert ((part >= 0) & (part < k)).all()
    assert obj == oracle.edge_cut(x, a, w, part)
    pw = oracle.partition_weights(n, ncon, v, part, k)
    total = oracle.total_weight(n, ncon, v).astype(np.float64)
    # the reference tests' balance rule (tests/correctness.rs:68-79), per constraint
    max_allowed = total * (1.0 + ufactor / 1000.0) / k + 1.0
    assert (pw <= max_allowed[None, :]).all(), (pw.max(axis=0), max_allowed)


CASES = [
    ("grid2d_64", lambda: G.grid2d(64, 64) + (None, None), 8),
    ("grid2d_50", lambda: G.grid2d(50, 50) + (None, None), 16),
    ("grid3d_24_w", lambda: G.grid3d(24, weights_seed=7), 32),
    ("rgg_8k", lambda: (lambda r: (r[0], r[1], None, r[2]))(G.rgg2d(8000, 4)), 12),
]


@pytest.mark.parametrize("name,make,k", CASES)
def test_kway_valid_balanced_and_close_to_reference(rmb, oracle, name, make, k):
    x, a, v, w = make()
    n = len(x) - 1
    seeds = range(1, 7)
    cuts = []
    for seed in seeds:
        opts = greedy_options(seed=seed)
        rc, part, obj = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, options=opts)
        assert rc == 1
        check_partition(oracle, x, a, v, w, part, k, obj)
        cuts.append(obj)
    ref = []
    for seed in seeds:
        rc, part, obj = oracle.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, options=greedy_options(seed=seed))
        assert rc == 1
        ref.append(obj)
    # quality gate: mean cut over the same seeds within 5% of the reference's
    assert np.mean(cuts) <= 1.05 * np.mean(ref), (cuts, ref)


def test_kway_best_of_ncuts(rmb, oracle):
    x, a = G.grid2d(64, 64)
    rc1, _, o1 = call_c_abi(rmb, x, a, 8, options=greedy_options(seed=42, ncuts=1))
    rc4, p4, o4 = call_c_abi(rmb, x, a, 8, options=greedy_options(seed=42, ncuts=4))
    assert rc1 == rc4 == 1 and o4 <= o1
    rcr, _, oref = oracle.part_graph_kway(x, a, 8, options=greedy_options(seed=42, ncuts=4))
    assert o4 <= 1.05 * oref


def test_kway_deterministic(rmb):
    x, a, v, w = G.grid3d(20, weights_seed=3)
    r1 = call_c_abi(rmb, x, a, 16, vwgt=v, adjwgt=w, options=greedy_options(seed=123))
    r2 = call_c_abi(rmb, x, a, 16, vwgt=v, adjwgt=w, options=greedy_options(seed=123))
    assert r1[0] == r2[0] == 1 and r1[2] == r2[2] and (r1[1] == r2[1]).all()


def test_kway_rm_and_random_initial(rmb, oracle):
    x, a = G.grid2d(40, 40)
    for ctype, iptype in ((0, 0), (1, 1), (1, 4)):
        rc, part, obj = call_c_abi(rmb, x, a, 6, options=greedy_options(seed=5, ctype=ctype, iptype=iptype))
        assert rc == 1
        assert ((part >= 0) & (part < 6)).all() and obj == oracle.edge_cut(x, a, None, part)


def test_kway_multiconstraint_tpwgts_ubvec(rmb, oracle):
    x, a, _, w = G.random_graph(5000, 8.0, seed=4)
    n = len(x) - 1
    v = np.random.default_rng(1).integers(1, 9, 2 * n).astype(np.int32)
    k = 8
    rc, part, obj = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, ncon=2, options=greedy_options(seed=3, ufactor=50),
                               ubvec=[1.05, 1.05])
    assert rc == 1
    check_partition(oracle, x, a, v, w, part, k, obj, ncon=2, ufactor=50)


def test_kway_reference_small_graphs(rmb, oracle):
    # tests/correctness.rs: cycle4 k=2, grid2x3 k=2, grid4x4 k=4 (ncuts 5), weighted cycle
    cyc = (np.array([0, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 2]))
    rc, part, obj = call_c_abi(rmb, *cyc, 2, options=greedy_options(seed=1))
    assert rc == 1 and obj <= 4
    rc, part, obj = call_c_abi(rmb, *cyc, 2, vwgt=[2, 1, 2, 1], adjwgt=[3, 1, 3, 1, 3, 1, 3, 1],
                               options=greedy_options(seed=5))
    assert rc == 1 and ((part >= 0) & (part < 2)).all()
    x, a = G.grid2d(4, 4)
    rc, part, obj = call_c_abi(rmb, x, a, 4, options=greedy_options(seed=1, ncuts=5))
    assert rc == 1
    check_partition(oracle, x, a, None, None, part, 4, obj)


def test_kway_errors(rmb):
    cyc = (np.array([0, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 2]))
    assert call_c_abi(rmb, *cyc, 10, options=greedy_options())[0] == -2        # nparts > n
    assert call_c_abi(rmb, *cyc, 1, options=greedy_options())[0] == -2         # nparts < 2
    assert call_c_abi(rmb, *cyc, 2, options=None)[0] == 1                      # default rtype = Fm runs
    bad = (np.array([0, 2, 4, 6, 8]), np.array([1, 3, 0, 2, 1, 3, 0, 0]))     # asymmetric
    assert call_c_abi(rmb, *bad, 2, options=greedy_options())[0] == -2
    loop = (np.array([0, 2, 4, 6, 8]), np.array([0, 3, 0, 2, 1, 3, 0, 2]))    # self-loop
    assert call_c_abi(rmb, *loop, 2, options=greedy_options())[0] == -2
    rng = (np.array([0, 2, 4, 6, 8]), np.array([1, 9, 0, 2, 1, 3, 0, 2]))     # out of range
    assert call_c_abi(rmb, *rng, 2, options=greedy_options())[0] == -2
    assert call_c_abi(rmb, *cyc, 2, vwgt=[1, 0, 1, 1], options=greedy_options())[0] == -2


def test_python_api_mirror(rmb, oracle):
    x, a = G.grid2d(32, 32)
    g = rmb.Graph.new_unweighted(len(x) - 1, x, a)
    res = rmb.part_graph_kway(g, 4, options=rmb.Options(rtype=rmb.RType.Greedy, seed=2))
    assert res.objval == g.edge_cut(res.part) == oracle.edge_cut(x, a, None, res.part)
    fm = rmb.part_graph_kway(g, 4, options=rmb.Options(seed=2))  # rtype Fm, the default
    assert fm.objval == g.edge_cut(fm.part) and ((fm.part >= 0) & (fm.part < 4)).all()
    with pytest.raises(rmb.InputError):
        rmb.part_graph_kway(g, 2000, options=rmb.Options(rtype=rmb.RType.Greedy))


def test_device_pointer_entry(rmb, oracle):
    torch = pytest.importorskip("torch")
    x, a, v, w = G.grid3d(16, weights_seed=1)
    n = len(x) - 1
    dev = lambda arr: torch.from_numpy(np.ascontiguousarray(arr, np.int32)).cuda()
    dx, da, dv, dw = dev(x), dev(a), dev(v), dev(w)
    dp = torch.empty(n, dtype=torch.int32, device="cuda")
    lib = rmb._lib.load()
    I32P = ctypes.POINTER(ctypes.c_int32)
    opts = greedy_options(seed=4)
    obj = ctypes.c_int32(0)
    rc = lib.RMETIS_GPU_PartGraphKwayDevice(ctypes.byref(ctypes.c_int32(n)), ctypes.byref(ctypes.c_int32(1)),
                                            dx.data_ptr(), da.data_ptr(), dv.data_ptr(), dw.data_ptr(),
                                            ctypes.byref(ctypes.c_int32(8)), None, None,
                                            opts.ctypes.data_as(I32P), ctypes.byref(obj), dp.data_ptr())
    assert rc == 1
    part = dp.cpu().numpy()
    rc2, part2, obj2 = call_c_abi(rmb, x, a, 8, vwgt=v, adjwgt=w, options=opts)
    assert obj.value == obj2 and (part == part2).all()
