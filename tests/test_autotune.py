"""The autotuner of the launch-shape knobs (rmetis_b200/autotune.py): the
search and its result-neutrality guard on a fake runner (CPU), the tuning
table, and on the GPU a small sweep of both modes through the library."""
import json
import types

import numpy as np
import pytest

from rmetis_b200 import autotune as A


def _res(obj, part):
    return types.SimpleNamespace(objval=obj, part=np.asarray(part, np.int32))


def test_candidates_start_with_the_engine_defaults():
    c = A.candidates()
    assert c[0] == A.DEFAULTS
    assert len(c) == len({tuple(sorted(s.items())) for s in c})
    assert len(c) == len(A.FUSED_CANDIDATES) * len(A.TAIL_CANDIDATES)


def test_tune_picks_the_fastest_and_sorts(monkeypatch):
    cost = {0: 0.30, 1024: 0.10, 4096: 0.20}
    clock = [0.0]

    def fake_counter():
        return clock[0]

    def run(s):
        clock[0] += cost[s["fused_max_n"]]
        return [_res(5, [0, 1, 1, 0])]

    monkeypatch.setattr(A.time, "perf_counter", fake_counter)
    settings = [{"fused_max_n": f, "tail_max_n": 0} for f in (4096, 0, 1024)]
    trials = A.tune(run, settings, repeats=2)
    assert [t.setting["fused_max_n"] for t in trials] == [1024, 4096, 0]
    assert trials[0].seconds == pytest.approx(0.10)
    assert len(trials[0].times) == 2


def test_tune_raises_when_a_knob_changes_a_result():
    def run(s):
        return [_res(5, [0, 1]), _res(7, [1, 0] if s["fused_max_n"] == 0 else [0, 1])]

    settings = [{"fused_max_n": 4096, "tail_max_n": 0}, {"fused_max_n": 0, "tail_max_n": 0}]
    with pytest.raises(A.TuningMismatch, match="changed result 1"):
        A.tune(run, settings, repeats=1)


def test_tune_raises_when_a_setting_is_not_reproducible():
    calls = [0]

    def run(s):
        calls[0] += 1
        return [_res(3 if calls[0] < 3 else 4, [0])]

    with pytest.raises(A.TuningMismatch, match="not reproducible"):
        A.tune(run, [{"fused_max_n": 1, "tail_max_n": 1}], repeats=3)


def test_table_round_trip_and_apply(tmp_path):
    path = str(tmp_path / "t.json")
    assert A.apply(path, device="X") == {}
    plain = [A.Trial({"fused_max_n": 2048, "tail_max_n": 1024}, 0.01), A.Trial(dict(A.DEFAULTS), 0.02)]
    pool = [A.Trial({"fused_max_n": 8192, "tail_max_n": 16384}, 0.5)]
    A.save_entry(path, "Dev A", "plain", plain, note="n")
    A.save_entry(path, "Dev A", "pool", pool)
    A.save_entry(path, "Dev B", "plain", pool)
    t = json.load(open(path))
    assert t["Dev A"]["plain"]["setting"] == {"fused_max_n": 2048, "tail_max_n": 1024}
    assert [x["ms"] for x in t["Dev A"]["plain"]["trials"]] == [10.0, 20.0]
    got = {}
    setters = {"plain": lambda **kw: got.__setitem__("plain", kw), "pool": lambda **kw: got.__setitem__("pool", kw)}
    applied = A.apply(path, device="Dev A", setters=setters)
    assert applied == {"plain": {"fused_max_n": 2048, "tail_max_n": 1024},
                       "pool": {"fused_max_n": 8192, "tail_max_n": 16384}}
    assert got == applied
    got.clear()
    assert A.apply(path, device="Dev C", setters=setters) == {} and got == {}


def test_committed_table_is_well_formed():
    t = A.load_table()
    for dev, entry in t.items():
        assert set(entry) <= {"plain", "pool", "shapes", "refine"}
        for name, mode in entry.items():
            s = mode["setting"]
            if name in ("plain", "pool"):
                assert set(s) == {"fused_max_n", "tail_max_n"}
                assert all(isinstance(v, int) and v >= 0 for v in s.values())
            elif name == "shapes":
                assert s["contract_thread_max"] in (16, 32) and s["gain_block"] in (128, 256, 512)
            else:
                assert s["exact_max_n"] in A.EXACT_CANDIDATES
                assert s["cut_ratio"] <= 1.0 + A.QUALITY_TOL or s["exact_max_n"] == A.EXACT_DEFAULT


def test_tune_scores_items_relative_to_the_first_setting():
    """With per-item times, a setting that halves a small item's time beats
    one that saves the same absolute time on a large item."""
    items = {"a": [1.0, 0.010], "b": [0.99, 0.005], "c": [0.985, 0.010]}

    def run(s):
        run.item_times = list(items[s["name"]])
        return [_res(1, [0])]
    run.item_times = []
    trials = A.tune(run, [{"name": "a"}, {"name": "b"}, {"name": "c"}], repeats=1)
    assert [t.setting["name"] for t in trials] == ["b", "c", "a"]


def test_shape_candidates_start_with_the_defaults():
    c = A.shape_candidates()
    assert c[0] == A.SHAPE_DEFAULTS
    assert len(c) == 6 and len({tuple(sorted(x.items())) for x in c}) == 6


def test_quality_gated_refine_mode(monkeypatch):
    """The result-changing knob: the fastest setting whose summed cut stays
    within the tolerance of sequential passes everywhere wins."""
    cut = {-1: 1000, 4096: 1030, 8192: 1004, 16384: 1001}
    cost = {-1: 0.9, 4096: 0.1, 8192: 0.2, 16384: 0.3}
    clock = [0.0]
    monkeypatch.setattr(A.time, "perf_counter", lambda: clock[0])

    def run(v):
        clock[0] += cost[v]
        return [_res(cut[v], [0])]

    elig, trials = A.tune_quality(run, (4096, 8192, 16384), repeats=2, tol=0.005)
    assert [t.setting["exact_max_n"] for t in elig] == [8192, 16384]
    assert {t.setting["exact_max_n"]: t.setting["cut_ratio"] for t in trials}[4096] == 1.03


def test_apply_sets_shapes_and_refine_mode(tmp_path):
    path = str(tmp_path / "t.json")
    A.save_entry(path, "Dev", "shapes", [A.Trial({"contract_thread_max": 16, "gain_block": 512}, 0.1)])
    A.save_entry(path, "Dev", "refine", [A.Trial({"exact_max_n": 8192, "cut_ratio": 1.001}, 0.1)])
    got = {}
    setters = {"shapes": lambda c, b: got.__setitem__("shapes", (c, b)),
               "refine": lambda v: got.__setitem__("refine", v)}
    applied = A.apply(path, device="Dev", setters=setters)
    assert got == {"shapes": (16, 512), "refine": 8192}
    assert applied == {"shapes": {"contract_thread_max": 16, "gain_block": 512}, "refine": {"exact_max_n": 8192}}


@pytest.mark.gpu
def test_gpu_sweep_is_result_neutral_in_both_modes():
    import rmetis_b200 as rmb
    from rmetis_b200 import generators as G
    graphs = []
    x, a = G.grid2d(40, 40)
    graphs.append((rmb.Graph(len(x) - 1, 1, x, a), 8))
    x, a, v, w = G.grid3d(24, 20, 16, weights_seed=3)
    graphs.append((rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w), 16))
    rggs = []
    for n, seed, k in ((6000, 5, 8), (2500, 6, 4), (9000, 7, 16)):
        x, a, w, _ = G.rgg2d(n, seed)
        v = np.random.default_rng(seed).integers(1, 9, size=2 * (len(x) - 1)).astype(np.int32)
        rggs.append((rmb.Graph(len(x) - 1, 2, x, a, vwgt=v, adjwgt=w), k))
    settings = A.candidates(fused=(0, 8192), tail=(0, 16384))
    try:
        trials = A.tune(A.plain_runner(graphs), settings, repeats=1)
        assert len(trials) == len(settings)
        batch = rggs
        o = rmb.Options(rtype=rmb.RType.Greedy, seed=3)
        ptrials = A.tune(A.pool_runner([g for g, _ in batch], [k for _, k in batch], options=o), settings, repeats=1)
        assert len(ptrials) == len(settings)
        # A pooled job gives what a single call gives, whatever the pool knobs.
        rmb.set_pool_tuning(0, 16384)
        res = rmb.part_graph_kway_batch([g for g, _ in batch], [k for _, k in batch], options=o)
        rmb.set_tuning(fused_max_n=8192, tail_max_n=0)
        for r, (g, k) in zip(res, batch):
            s = rmb.part_graph_kway(g, k, options=o)
            assert s.objval == r.objval
            np.testing.assert_array_equal(s.part, r.part)
    finally:
        rmb.set_tuning(**A.DEFAULTS)
        rmb.set_pool_tuning(-1, -1)
