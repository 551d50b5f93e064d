"""Autotuner for the engine's launch-shape, kernel-shape and refinement knobs.

Result-neutral knobs (the same kernel bodies run either way; tested
bit-identical in tests/test_gpu_fused.py, tests/test_gpu_tail.py and the
contraction parity tests):

* ``fused_max_n``: a level of at most this many vertices (and at most 4 times
  as many adjacency entries) is refined by one single-block launch instead of
  a sequence of grid-wide kernels per pass;
* ``tail_max_n``: from a level of at most this many vertices (and at most 64
  times as many adjacency entries) on, every remaining coarsening level runs
  in one single-block launch;
* ``contract_thread_max`` (16 or 32): the degree bucket of contraction, the
  longest merged-row bound one thread merges in registers; longer rows go to
  a warp each (thread-vs-warp per coarse vertex);
* ``gain_block`` (128, 256, 512): the block size of the gain-table kernel.

A single-block launch saves launches and host round trips but runs on one SM.
In a lone call the rest of the device idles meanwhile; jobs that share the
device (the graphs of a batch, served requests) fill it. The best sizes
therefore depend on the device and on the concurrency, and the launch shapes
are tuned separately for ``plain`` (single calls, ``set_tuning``) and
``pool`` (batch graphs and submitted requests, ``set_pool_tuning``); the
kernel shapes are device-wide (``set_kernel_shapes``) and tuned in plain
mode.

One knob changes results: ``exact_max_n``, the largest level whose greedy
cut passes decide sequentially (larger levels decide by parallel admission,
``set_refine_mode``). It is tuned for speed under a quality gate: a setting
is eligible when its summed cut over the plain workload is within
``QUALITY_TOL`` of the summed cut with sequential passes everywhere.

For each result-neutral candidate the tuner runs a workload, checks that
every result (objval and part vector) equals the first candidate's -- a
difference means a knob is not neutral and raises ``TuningMismatch`` -- and
keeps the best of ``repeats`` wall-clock times. The fastest candidate wins; a
table maps the device name to the winner of each mode, and ``apply()`` sets
them for the current device when the table has an entry for it.

    python -m rmetis_b200.autotune --mode both --out rmetis_b200/tuning.json
"""
from __future__ import annotations

import argparse
import hashlib
import itertools
import json
import os
import time
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning.json")

FUSED_CANDIDATES = (0, 1024, 2048, 4096, 8192)
TAIL_CANDIDATES = (0, 1024, 4096, 16384)
DEFAULTS = {"fused_max_n": 4096, "tail_max_n": 4096}
SHAPE_CANDIDATES = {"contract_thread_max": (16, 32), "gain_block": (128, 256, 512)}
SHAPE_DEFAULTS = {"contract_thread_max": 32, "gain_block": 256}
EXACT_CANDIDATES = (4096, 8192, 16384, 32768, 65536)
EXACT_DEFAULT = 16384
QUALITY_TOL = 0.02


class TuningMismatch(RuntimeError):
    """A knob that must not change results changed one."""


@dataclass
class Trial:
    setting: dict
    seconds: float
    times: list = field(default_factory=list)


def candidates(fused=FUSED_CANDIDATES, tail=TAIL_CANDIDATES):
    """Every (fused_max_n, tail_max_n) pair, the engine defaults first so that
    they are the reference the other results are compared against."""
    out = [dict(DEFAULTS)]
    for f, t in itertools.product(fused, tail):
        s = {"fused_max_n": int(f), "tail_max_n": int(t)}
        if s != out[0]:
            out.append(s)
    return out


def shape_candidates():
    """Every kernel-shape pair, the engine defaults first."""
    out = [dict(SHAPE_DEFAULTS)]
    for c, b in itertools.product(SHAPE_CANDIDATES["contract_thread_max"], SHAPE_CANDIDATES["gain_block"]):
        s = {"contract_thread_max": int(c), "gain_block": int(b)}
        if s != out[0]:
            out.append(s)
    return out


def tune_quality(run, values, repeats: int = 3, tol: float = QUALITY_TOL, log=None):
    """The result-changing knob: run(value) for the reference value -1 (every
    pass sequential) and each candidate; a candidate whose summed objval is
    within `tol` of the reference's is eligible. Returns (eligible trials
    fastest first, all trials with their cut ratios)."""
    ref = sum(int(r.objval) for r in run(-1))
    trials, eligible = [], []
    for v in values:
        out = run(v)  # warm-up; the cut of this setting
        cut = sum(int(r.objval) for r in out)
        times = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            run(v)
            times.append(time.perf_counter() - t0)
        tr = Trial({"exact_max_n": int(v), "cut_ratio": round(cut / max(1, ref), 5)}, min(times), times)
        trials.append(tr)
        if cut <= (1.0 + tol) * ref:
            eligible.append(tr)
        if log:
            log(f"  exact_max_n={v}: {tr.seconds * 1e3:.2f} ms, cut {cut} ({cut / max(1, ref):.4f} of sequential)")
    return sorted(eligible, key=lambda t: t.seconds), trials


def digest(results) -> list:
    """(objval, sha1 of the part vector) per result: what must not change."""
    return [(int(r.objval), hashlib.sha1(np.ascontiguousarray(r.part, dtype=np.int32).tobytes()).hexdigest())
            for r in results]


def tune(run, settings, repeats: int = 3, log=None):
    """Run `run(setting) -> results` `repeats` times per setting (plus one
    untimed warm-up), check every result against the first setting's, and
    return the trials sorted fastest first. A runner that records the time of
    each item of a run (`run.item_times`, a list) is scored by the sum of its
    items' times relative to the first setting's, so that a small graph
    counts as much as a large one; otherwise by the run's wall time."""
    ref = None
    base = None
    trials = []
    for s in settings:
        first = digest(run(s))  # warm-up, and the results to compare
        if ref is None:
            ref = first
        elif first != ref:
            bad = next(i for i, (a, b) in enumerate(zip(first, ref)) if a != b) if len(first) == len(ref) else -1
            raise TuningMismatch(f"setting {s} changed result {bad}: {first[bad] if bad >= 0 else len(first)} "
                                 f"vs {ref[bad] if bad >= 0 else len(ref)}")
        times, items = [], None
        for _ in range(repeats):
            t0 = time.perf_counter()
            out = run(s)
            times.append(time.perf_counter() - t0)
            it = getattr(run, "item_times", None)
            if it:
                items = list(it) if items is None else [min(a, b) for a, b in zip(items, it)]
            if digest(out) != ref:
                raise TuningMismatch(f"setting {s} is not reproducible")
        score = min(times)
        if items:
            if base is None:
                base = items
            score = sum(a / b for a, b in zip(items, base) if b > 0) / len(items) * sum(base)
        tr = Trial(dict(s), score, times)
        trials.append(tr)
        if log:
            log(f"  {s}: {tr.seconds * 1e3:.2f} ms (best of {repeats})")
    return sorted(trials, key=lambda t: t.seconds)


# ---------------------------------------------------------------------------
# Workloads (the GPU library; only the tuner's CLI and the GPU tests use them)
# ---------------------------------------------------------------------------

def plain_workload(large: bool = True):
    """Single graphs of the sizes the plain path serves: the 64x64 grid (k=8),
    a weighted 64^3 grid (k=64), a 20,000-vertex RGG with two constraints
    (k=16) and, when `large`, the weighted 128^3 grid (k=64)."""
    import rmetis_b200 as rmb
    from rmetis_b200 import generators as G
    out = []
    x, a = G.grid2d(64, 64)
    out.append((rmb.Graph(len(x) - 1, 1, x, a), 8))
    x, a, v, w = G.grid3d(64, weights_seed=7)
    out.append((rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w), 64))
    x, a, w, _ = G.rgg2d(20000, 11)
    v = np.random.default_rng(11).integers(1, 9, size=2 * (len(x) - 1)).astype(np.int32)
    out.append((rmb.Graph(len(x) - 1, 2, x, a, vwgt=v, adjwgt=w), 16))
    if large:
        x, a, v, w = G.grid3d(128, weights_seed=7)
        out.append((rmb.Graph(len(x) - 1, 1, x, a, vwgt=v, adjwgt=w), 64))
    return out


def pool_workload(count: int = 64, seed: int = 4):
    """A batch of `count` 2D RGGs of uneven sizes (n log-uniform in
    [1e3, 2e5]), two constraints, k from {2,...,64}: the batched shape."""
    import rmetis_b200 as rmb
    from rmetis_b200 import generators as G
    graphs, ks = [], []
    for i in range(count):
        rng = np.random.default_rng([seed, i])
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
        k = int(rng.choice([2, 4, 8, 16, 32, 64]))
        x, a, w, _ = G.rgg2d(n, int(rng.integers(1 << 31)))
        v = rng.integers(1, 9, size=2 * (len(x) - 1)).astype(np.int32)
        graphs.append(rmb.Graph(len(x) - 1, 2, x, a, vwgt=v, adjwgt=w, validate=False))
        ks.append(k)
    return graphs, ks


def plain_runner(graphs, options=None):
    import rmetis_b200 as rmb
    o = options or rmb.Options(rtype=rmb.RType.Greedy, seed=7)

    def run(s):
        if "fused_max_n" in s:
            rmb.set_tuning(fused_max_n=s["fused_max_n"], tail_max_n=s["tail_max_n"])
        if "contract_thread_max" in s:
            rmb.set_kernel_shapes(s["contract_thread_max"], s["gain_block"])
        out, run.item_times = [], []
        for g, k in graphs:
            t0 = time.perf_counter()
            out.append(rmb.part_graph_kway(g, k, options=o))
            run.item_times.append(time.perf_counter() - t0)
        return out
    run.item_times = []
    return run


def exact_runner(graphs, options=None):
    import rmetis_b200 as rmb
    inner = plain_runner(graphs, options)

    def run(v):
        rmb.set_refine_mode(v)
        return inner({})
    return run


def pool_runner(graphs, ks, options=None):
    import rmetis_b200 as rmb
    o = options or rmb.Options(rtype=rmb.RType.Greedy, seed=1, ufactor=50)

    def run(s):
        rmb.set_pool_tuning(fused_max_n=s["fused_max_n"], tail_max_n=s["tail_max_n"])
        return rmb.part_graph_kway_batch(graphs, ks, options=o)
    return run


# ---------------------------------------------------------------------------
# The table
# ---------------------------------------------------------------------------

def device_name(index: int | None = None) -> str:
    """Name of CUDA device `index` (default: the current device)."""
    import torch
    return torch.cuda.get_device_name(index)


def load_table(path: str = DEFAULT_TABLE) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save_entry(path: str, device: str, mode: str, trials, note: str = ""):
    """Record the winner of `mode` for `device` (and every trial's time)."""
    table = load_table(path)
    dev = table.setdefault(device, {})
    dev[mode] = {"setting": trials[0].setting,
                 "ms": round(trials[0].seconds * 1e3, 3),
                 "trials": [{**t.setting, "ms": round(t.seconds * 1e3, 3)} for t in trials],
                 "note": note}
    with open(path, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
        f.write("\n")
    return table


def apply(path: str = DEFAULT_TABLE, device: str | None = None, setters=None) -> dict:
    """Set the tuned knobs of every mode the table holds for `device` (the
    current CUDA device by default). Returns what was applied ({} when the
    table has no entry for the device: the engine defaults stay)."""
    table = load_table(path)
    if not table:
        return {}
    if device is None:
        device = device_name()
    entry = table.get(device)
    if not entry:
        return {}
    if setters is None:
        import rmetis_b200 as rmb
        setters = {"plain": rmb.set_tuning, "pool": rmb.set_pool_tuning, "shapes": rmb.set_kernel_shapes,
                   "refine": rmb.set_refine_mode}
    applied = {}
    for mode in ("plain", "pool"):
        if mode in entry and mode in setters:
            s = entry[mode]["setting"]
            setters[mode](fused_max_n=int(s["fused_max_n"]), tail_max_n=int(s["tail_max_n"]))
            applied[mode] = {"fused_max_n": int(s["fused_max_n"]), "tail_max_n": int(s["tail_max_n"])}
    if "shapes" in entry and "shapes" in setters:
        s = entry["shapes"]["setting"]
        setters["shapes"](int(s["contract_thread_max"]), int(s["gain_block"]))
        applied["shapes"] = {"contract_thread_max": int(s["contract_thread_max"]), "gain_block": int(s["gain_block"])}
    if "refine" in entry and "refine" in setters:
        v = int(entry["refine"]["setting"]["exact_max_n"])
        setters["refine"](v)
        applied["refine"] = {"exact_max_n": v}
    return applied


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--mode", choices=["plain", "pool", "both"], default="both")
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--graphs", type=int, default=64, help="pool mode: graphs in the batch")
    ap.add_argument("--small", action="store_true", help="plain mode without the 128^3 grid")
    args = ap.parse_args(argv)
    dev = device_name()
    settings = candidates()
    if args.mode in ("plain", "both"):
        print(f"plain ({len(settings)} settings) on {dev}", flush=True)
        wl = plain_workload(large=not args.small)
        trials = tune(plain_runner(wl), settings, args.repeats, log=print)
        import rmetis_b200 as rmb
        rmb.set_tuning(**DEFAULTS)
        save_entry(args.out, dev, "plain", trials,
                   note="sum over: 64x64 grid k=8, weighted 64^3 grid k=64, RGG n=20000 ncon=2 k=16"
                        + ("" if args.small else ", weighted 128^3 grid k=64") + "; host-buffer calls")
        print(f"plain winner {trials[0].setting} {trials[0].seconds * 1e3:.2f} ms", flush=True)
        rmb.set_tuning(**trials[0].setting)
        shapes = shape_candidates()
        print(f"kernel shapes ({len(shapes)} settings)", flush=True)
        st = tune(plain_runner(wl), shapes, args.repeats, log=print)
        save_entry(args.out, dev, "shapes", st, note="plain workload, launch shapes of the plain winner")
        rmb.set_kernel_shapes(**st[0].setting)
        print(f"shapes winner {st[0].setting} {st[0].seconds * 1e3:.2f} ms", flush=True)
        elig, all_trials = tune_quality(exact_runner(wl), EXACT_CANDIDATES, args.repeats, log=print)
        best = elig if elig else [t for t in all_trials if t.setting["exact_max_n"] == EXACT_DEFAULT]
        rest = [t for t in sorted(all_trials, key=lambda t: t.seconds) if t is not best[0]]
        save_entry(args.out, dev, "refine", [best[0]] + rest,
                   note=f"fastest exact_max_n whose summed cut is within {QUALITY_TOL:.1%} of sequential passes "
                        "everywhere (cut_ratio)")
        rmb.set_refine_mode(EXACT_DEFAULT)
        rmb.set_kernel_shapes(**SHAPE_DEFAULTS)
        rmb.set_tuning(**DEFAULTS)
        print(f"refine winner {best[0].setting} {best[0].seconds * 1e3:.2f} ms", flush=True)
    if args.mode in ("pool", "both"):
        print(f"pool ({len(settings)} settings, {args.graphs} graphs) on {dev}", flush=True)
        graphs, ks = pool_workload(args.graphs)
        trials = tune(pool_runner(graphs, ks), settings, args.repeats, log=print)
        import rmetis_b200 as rmb
        rmb.set_pool_tuning(-1, -1)
        save_entry(args.out, dev, "pool", trials,
                   note=f"one batch of {args.graphs} RGGs, n log-uniform [1e3, 2e5], ncon=2, k in {{2..64}}")
        print(f"pool winner {trials[0].setting} {trials[0].seconds * 1e3:.2f} ms", flush=True)


if __name__ == "__main__":
    main()
