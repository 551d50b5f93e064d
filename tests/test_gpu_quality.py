"""Full-partition acceptance on the benchmark workloads, against the oracle.

Every case partitions the same graph with the same seeds on the GPU (through
the drop-in C ABI) and in the oracle, and checks:

* validity and objval == the oracle's edge_cut of the returned part;
* balance by the reference's own feasibility rule, pw[p][c] <= floor(t[p][c] *
  ub[c]) on every part and constraint (src/refine/greedy.rs:85-88 tests moves
  with it). Where the oracle's own partitions break that rule (one repair pass
  cannot always fix a projected partition of an unweighted graph), the GPU's
  worst overshoot over the seed set may not exceed the oracle's worst;
* quality: the GPU's summed (or best-of-ncuts) cut at most 1.05x the oracle's
  on the same seeds (src/partition/kway.rs:94-98 keeps the best attempt).

The matchings of a full run differ by design (parallel handshake vs the
sequential visit), so cuts are compared by quality, not bit for bit. The
oracle's seeded random streams are a faithful restatement of rand 0.8.5's
SmallRng but not pinned by any reference test (parity of seeded streams is
unpinned), which is why quality is compared over several seeds.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from rmetis_b200 import generators as G
from tests.conftest import greedy_options
from tests.test_gpu_kway import call_c_abi

pytestmark = pytest.mark.gpu

THREADS = max(1, min(16, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else 4))


def overshoot(oracle, x, v, part, k, ncon, ufactor=30, ubvec=None, tpwgts=None):
    """max over (p, c) of pw[p][c] - floor(t[p][c] * ub[c]); <= 0 means every
    part is within the reference's feasibility limit."""
    n = len(x) - 1
    ub = np.asarray(ubvec, np.float64) if ubvec is not None else np.full(ncon, 1.0 + ufactor / 1000.0)
    t = oracle.compute_target_weights(n, ncon, v, k, tpwgts).reshape(k, ncon)
    lim = np.floor(t * ub[None, :])
    pw = oracle.partition_weights(n, ncon, v, part, k).astype(np.float64)
    return float((pw - lim).max())


def run_both(rmb, oracle, x, a, v, w, k, seeds, ncon=1, opts_fn=greedy_options, **okw):
    """GPU and oracle partitions for every seed: lists of (cut, overshoot)."""
    ufactor = okw.get("ufactor", 30)
    gpu = []
    for s in seeds:
        rc, part, obj = call_c_abi(rmb, x, a, k, vwgt=v, adjwgt=w, ncon=ncon, options=opts_fn(seed=s, **okw))
        assert rc == 1
        assert ((part >= 0) & (part < k)).all()
        assert obj == oracle.edge_cut(x, a, w, part)
        gpu.append((obj, overshoot(oracle, x, v, part, k, ncon, ufactor)))

    def one(s):
        rc, part, obj = oracle.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, ncon=ncon, options=opts_fn(seed=s, **okw))
        assert rc == 1
        return obj, overshoot(oracle, x, v, part, k, ncon, ufactor)

    with cf.ThreadPoolExecutor(THREADS) as ex:
        ref = list(ex.map(one, seeds))
    return gpu, ref


def assert_balance(gpu, ref, what):
    g_worst = max(o for _, o in gpu)
    r_worst = max(o for _, o in ref)
    assert g_worst <= max(0.0, r_worst), f"{what}: GPU overshoot {g_worst} vs oracle {r_worst}"


def test_c1_grid2d_64_k8(rmb, oracle):
    """64x64 grid, unit weights, k=8 (seed 1 is the workload; 16 seeds for the
    quality sum)."""
    x, a = G.grid2d(64, 64)
    gpu, ref = run_both(rmb, oracle, x, a, None, None, 8, range(1, 17))
    assert sum(c for c, _ in gpu) <= 1.05 * sum(c for c, _ in ref), (gpu, ref)
    assert_balance(gpu, ref, "C1")


def test_c2_grid3d_128_k64(rmb, oracle):
    """128^3 grid, vwgt U{1..4}, adjwgt U{1..10}, k=64, seed 7 (the benchmark
    workload) and seed 8."""
    x, a, v, w = G.grid3d(128, weights_seed=7)
    gpu, ref = run_both(rmb, oracle, x, a, v, w, 64, [7, 8])
    for (gc, go), (rc_, ro) in zip(gpu, ref):
        assert gc <= 1.05 * rc_, (gpu, ref)
    # vertex weights are summed through coarsening: the strict rule holds
    assert_balance(gpu, ref, "C2")


def _c4_graphs(count=8):
    """C4's law: 2D RGGs, n log-uniform in [1e3, 2e5] (here capped at 5e4 so
    the oracle stays fast), ncon=2 vwgt U{1..8}, k from {2..64}."""
    out = []
    for i in range(count):
        rng = np.random.default_rng([4, 1000 + i])
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(5e4))))
        k = int(rng.choice([2, 4, 8, 16, 32, 64]))
        x, a, w, _ = G.rgg2d(n, int(rng.integers(1 << 31)))
        v = rng.integers(1, 9, size=2 * n).astype(np.int32)
        out.append((x, a, v, w, k))
    return out


def test_c4_rgg_ncon2_ufactor50(rmb, oracle):
    tot_g = tot_r = 0
    for x, a, v, w, k in _c4_graphs():
        gpu, ref = run_both(rmb, oracle, x, a, v, w, k, [1, 2], ncon=2, ufactor=50)
        tot_g += sum(c for c, _ in gpu)
        tot_r += sum(c for c, _ in ref)
        assert_balance(gpu, ref, f"C4 n={len(x) - 1} k={k}")
    assert tot_g <= 1.05 * tot_r, (tot_g, tot_r)


def test_c3_law_rmat14_k256_best_of_16(rmb, oracle):
    """C3's law at a size the oracle finishes: R-MAT scale 14, unit weights,
    k=256, best of 16 attempts (seed 1 + attempt) on both sides."""
    x, a = G.rmat(14, seed=22)
    k = 256
    rc, part, obj = call_c_abi(rmb, x, a, k, options=greedy_options(seed=1, ncuts=16))
    assert rc == 1 and obj == oracle.edge_cut(x, a, None, part)
    g_over = overshoot(oracle, x, None, part, k, 1)

    def one(s):
        rc_, p_, o_ = oracle.part_graph_kway(x, a, k, options=greedy_options(seed=s))
        assert rc_ == 1
        return o_, overshoot(oracle, x, None, p_, k, 1)

    with cf.ThreadPoolExecutor(THREADS) as ex:
        ref = list(ex.map(one, range(1, 17)))
    best = min(ref, key=lambda r: r[0])  # first strict minimum, kway.rs:96-98
    assert obj <= 1.05 * best[0], (obj, ref)
    assert g_over <= max(0.0, max(o for _, o in ref)), (g_over, ref)


@pytest.mark.parametrize("name", ["grid3d_24_w", "rgg_20k"])
def test_rm_coarsening_quality(rmb, oracle, name):
    """CType::Rm (random matching, src/coarsen/rm.rs:13-43) end to end."""
    if name == "grid3d_24_w":
        x, a, v, w = G.grid3d(24, weights_seed=7)
        k = 16
    else:
        x, a, w, _ = G.rgg2d(20000, 3)
        v, k = None, 16
    gpu, ref = run_both(rmb, oracle, x, a, v, w, k, range(1, 9), ctype=0)
    assert sum(c for c, _ in gpu) <= 1.05 * sum(c for c, _ in ref), (gpu, ref)
    assert_balance(gpu, ref, f"Rm {name}")


@pytest.mark.parametrize("name", ["grid2d_64", "grid3d_24_w"])
def test_random_initial_quality(rmb, oracle, name):
    """IpType::Random (src/initial/random.rs:8-10) end to end."""
    if name == "grid2d_64":
        x, a = G.grid2d(64, 64)
        v = w = None
        k = 8
    else:
        x, a, v, w = G.grid3d(24, weights_seed=7)
        k = 16
    # A random start leaves much to the refinement, so single cuts vary
    # widely; the sum over 32 seeds is compared.
    gpu, ref = run_both(rmb, oracle, x, a, v, w, k, range(1, 33), iptype=1)
    assert sum(c for c, _ in gpu) <= 1.05 * sum(c for c, _ in ref), (gpu, ref)
    assert_balance(gpu, ref, f"Random {name}")
