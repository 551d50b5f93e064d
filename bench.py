"""Benchmark: multilevel k-way partitioning, edges/s, on N GPUs of one node.

Workload (one step): the plain k-way path on a 3D 7-point grid 128^3
(2,097,152 vertices, 12,484,608 directed CSR entries), vertex weights U{1..4},
symmetric edge weights U{1..10} (numpy default_rng(7)), nparts=64, Shem +
Greedy, ufactor=30, ncuts=1, seed=7. Synthetic input of that shape.

value: edges/s with the graph resident in HBM (RMETIS_GPU_PartGraphKwayDevice),
timed with CUDA events on the launching stream, L2 flushed before each step.
e2e:   the same metric through the drop-in RMETIS_PartGraphKway with pinned
host buffers (host->device inputs and device->host part inside every step).
With --gpus N > 1 every rank partitions its own replica (the path does not
shard within one graph); value = N * m / max-over-ranks step time.

--impl reference times the oracle (CPU restatement of the reference) on the
host cores instead; rank 0 only.

Further workloads (one JSON line each, same keys):
  --workload rmat_seeds  R-MAT scale 22 (--scale), k=256, ncuts=16: the 16
                         attempts concurrently on the device's worker pool vs
                         one after another (the plain path), attempts/s.
  --workload rgg_batch   512 uneven 2D RGGs (--graphs), ncon=2, k in
                         {2..64}, ufactor=50: one batched call vs plain calls
                         one graph at a time, graphs/s.
  --workload serving     Poisson arrivals (--rates, --requests) of 2D grid /
                         3D grid / RGG requests, n log-uniform in [1e4, 2e6],
                         k in {2..128}, through the asynchronous API; p50/p99
                         latency and throughput vs the plain path serving the
                         same arrivals one request at a time. Defaults: the
                         configured stream of 10,000 requests per rate at
                         50..2,000 req/s (about 12 minutes, the plain pass included).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from rmetis_b200 import generators as G  # noqa: E402

METRIC = "k-way edges/s (plain path)"
UNIT = "edges/s"
WORKLOADS = {
    # name: (builder, nparts, seed, description)
    "grid3d_128": (lambda: G.grid3d(128, weights_seed=7), 64, 7,
                   "3D 7-point grid 128^3, vwgt U{1..4}, adjwgt U{1..10}, nparts=64, Shem+Greedy, "
                   "ufactor=30, ncuts=1, seed=7"),
    "grid2d_64": (lambda: G.grid2d(64, 64) + (None, None), 8, 1,
                  "2D 5-point grid 64x64, unit weights, nparts=8, Shem+Greedy, ufactor=30, ncuts=1, seed=1"),
    # a smaller case of the 128^3 workload for profiler captures
    "grid3d_64": (lambda: G.grid3d(64, weights_seed=7), 64, 7,
                  "3D 7-point grid 64^3, vwgt U{1..4}, adjwgt U{1..10}, nparts=64, Shem+Greedy, "
                  "ufactor=30, ncuts=1, seed=7"),
}
EXTRA_WORKLOADS = ("rmat_seeds", "rgg_batch", "serving")
# Kernel families of RMETIS_GPU_GetProfile, in its slot order.
PROF_NAMES = ["k_gain", "k_walk", "k_match_propose", "k_contract_thread", "k_cut", "k_grow", "k_refine_level",
              "k_coarsen_tail", "k_admit"]
CPU_SAMPLE = {
    "grid3d_128": (lambda: G.grid3d(64, weights_seed=7), "3D 7-point grid 64^3 (same weight laws), nparts=64"),
    "grid2d_64": (lambda: G.grid2d(64, 64) + (None, None), "2D grid 64x64, nparts=8"),
    "grid3d_64": (lambda: G.grid3d(64, weights_seed=7), "3D 7-point grid 64^3 (the workload itself), nparts=64"),
}


RTYPE = {"code": 1, "name": "greedy"}  # --rtype: 1 = Greedy (default), 0 = Fm


def kway_options(seed, ncuts=1, niter=10, ufactor=30):
    a = np.full(40, -1, dtype=np.int32)
    a[0] = 0; a[1] = 0; a[2] = 1; a[3] = 0; a[4] = RTYPE["code"]; a[5] = 0
    a[6] = niter; a[7] = ncuts; a[8] = seed; a[9] = 0; a[10] = 0; a[11] = 0
    a[16] = ufactor; a[17] = 0
    return a


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", self.gpu_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self, t0, t1):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, line in self.lines:
            if ts < t0 - 0.05 or ts > t1 + 0.25:
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_id_for(local_rank: int) -> str:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


def cpu_baseline(workload: str, graph=None):
    """The oracle on one core: one partition of the full workload (about
    16 s for the 128^3 grid), or of the bounded sample when no graph is given."""
    from oracle import oracle as O
    if graph is None:
        build, desc = CPU_SAMPLE[workload]
        x, a, v, w = build()
    else:
        (x, a, v, w), desc = graph, "the full workload"
    k, seed = WORKLOADS[workload][1], WORKLOADS[workload][2]
    t0 = time.perf_counter()
    rc, part, obj = O.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, options=kway_options(seed))
    dt = time.perf_counter() - t0
    assert rc == 1
    return {"value": len(a) / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{desc} (n={len(x) - 1}, m={len(a)}), 1 partition, {dt:.2f} s, cut {obj}", "objval": obj}


def run_reference(args):
    """--impl reference: the oracle (CPU restatement of the reference's path)
    on all host cores. The reference has no parallelism inside one partition
    (rayon is declared but unused); its only parallel axis is independent
    attempts (src/partition/kway.rs:54). So every timed step runs one
    partition of the configured workload itself (the full graph, same k,
    options and seed) in each of `cores` threads, and value = cores * m /
    step time. Warm-up steps (untimed) run one partition of the bounded
    sample per thread, so that the whole run stays within a few minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    build, k, seed, desc = WORKLOADS[args.workload]
    x, a, v, w = build()
    wx, wa, wv, ww = CPU_SAMPLE[args.workload][0]()
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    O.lib()
    objs = []

    def one(graph):
        gx, ga, gv, gw = graph
        rc, _, obj = O.part_graph_kway(gx, ga, k, vwgt=gv, adjwgt=gw, options=kway_options(seed))
        assert rc == 1
        return obj

    times = []
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        for step in range(args.warmup + args.steps):
            graph = (wx, wa, wv, ww) if step < args.warmup else (x, a, v, w)
            t0 = time.perf_counter()
            res = list(ex.map(one, [graph] * threads))
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append(dt)
                objs.append(res[0])
    ms = 1000.0 * statistics.mean(times)
    value = threads * len(a) / (ms / 1000.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": _config(args.workload, len(x) - 1, len(a), k, args.gpus),
            "objval": int(objs[0]),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"the workload itself (n={len(x) - 1}, m={len(a)}): {threads} independent "
                                       f"partitions (same seed) per step in {threads} threads; warm-up steps on "
                                       f"{CPU_SAMPLE[args.workload][1]}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line["repro"] = _repro()
    print(json.dumps(line))


def _config(workload, n, m, k, world):
    """The config object both arms print (identical for the same workload)."""
    desc = WORKLOADS[workload][3]
    if RTYPE["name"] == "fm":
        desc = desc.replace("Greedy", "Fm")
    return {"workload": desc, "name": workload, "n": n, "m": m, "nparts": k, "rtype": RTYPE["name"],
            "parallelism": "replicas" if world > 1 else "single"}


def balance_summary(x, v, part, k, ufactor=30):
    """max over parts of pw / t (1.0 = exactly on target) and the largest
    pw - floor(t * ub), the reference's feasibility limit (<= 0: within),
    ncon = 1, computed with numpy."""
    n = len(x) - 1
    vw = np.ones(n, np.int64) if v is None else np.asarray(v, np.int64)
    pw = np.bincount(np.asarray(part, np.int64), weights=vw, minlength=k).astype(np.int64)
    t = float(vw.sum()) / k
    lim = np.floor(t * (1.0 + ufactor / 1000.0))
    return {"max_imbalance": float(pw.max() / t), "max_overshoot": int(pw.max() - lim),
            "within_ufactor": bool(pw.max() <= lim)}


# ---------------------------------------------------------------------------
# Batched seeds, batched graphs and the serving stream
# ---------------------------------------------------------------------------
TUNING = {}


def _repro():
    """What a rerun needs to know: device, driver, CUDA runtime, host cores,
    source revision (when the tree has its git metadata)."""
    out = {"host_cores": len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()}
    try:
        import torch
        out["cuda_runtime"] = torch.version.cuda
        if torch.cuda.is_available():
            out["gpu"] = torch.cuda.get_device_name()
    except Exception:
        pass
    try:
        q = subprocess.run(["nvidia-smi", "--query-gpu=driver_version", "--format=csv,noheader"],
                           capture_output=True, text=True, timeout=20)
        if q.returncode == 0 and q.stdout.strip():
            out["driver"] = q.stdout.strip().splitlines()[0]
    except Exception:
        pass
    try:
        q = subprocess.run(["git", "rev-parse", "--short", "HEAD"], cwd=os.path.dirname(os.path.abspath(__file__)),
                           capture_output=True, text=True, timeout=20)
        out["git"] = q.stdout.strip() if q.returncode == 0 else "not a git checkout"
    except Exception:
        out["git"] = "not a git checkout"
    return out


def _apply_tuning():
    """Set the launch-shape knobs the autotuner recorded for this device in
    rmetis_b200/tuning.json (none recorded: the engine defaults stay)."""
    from rmetis_b200 import autotune
    dev = autotune.device_name(int(os.environ.get("LOCAL_RANK", "0")))
    TUNING.update(autotune.apply(device=dev) or {"engine defaults": dict(autotune.DEFAULTS)})


def _setup_device():
    import torch
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    return torch, torch.device("cuda", local_rank), local_rank


def _device_call(lib, torch, dev, x, a, v, w, k, opts, ncon=1):
    """A closure running one RMETIS_GPU_PartGraphKwayDevice call on
    device-resident copies of the graph; returns (call, part tensor, objval)."""
    I32P = ctypes.POINTER(ctypes.c_int32)
    t = lambda arr: None if arr is None else torch.from_numpy(np.ascontiguousarray(arr, np.int32)).to(dev)
    dx, da, dv, dw = t(x), t(a), t(v), t(w)
    n = len(x) - 1
    dpart = torch.empty(n, dtype=torch.int32, device=dev)
    nv, nc, npr = ctypes.c_int32(n), ctypes.c_int32(ncon), ctypes.c_int32(k)
    obj = ctypes.c_int32(0)
    op = opts.ctypes.data_as(I32P)
    ptr = lambda tt: None if tt is None else tt.data_ptr()

    def call():
        rc = lib.RMETIS_GPU_PartGraphKwayDevice(ctypes.byref(nv), ctypes.byref(nc), ptr(dx), ptr(da), ptr(dv),
                                                ptr(dw), ctypes.byref(npr), None, None, op, ctypes.byref(obj),
                                                ptr(dpart))
        if rc != 1:
            raise RuntimeError(f"RMETIS_GPU_PartGraphKwayDevice returned {rc}")
    return call, dpart, obj


def _timed(torch, stream, fn, reps):
    """Device time of fn() per call (CUDA events on the caller's stream; the
    call returns only when all its work, on any stream, is done)."""
    out = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def run_rmat_seeds(args):
    """R-MAT, k=256, 16 attempts (seed 1+attempt), best cut kept."""
    torch, dev, local_rank = _setup_device()
    import rmetis_b200 as rmb
    lib = rmb._lib.load()
    k, ncuts, seed = 256, 16, 1
    t0 = time.perf_counter()
    x, a = G.rmat_device(args.scale, seed=22)
    gen_s = time.perf_counter() - t0
    n, m = len(x) - 1, len(a)
    stream = torch.cuda.current_stream(dev)
    assert lib.RMETIS_GPU_SetStream(stream.cuda_stream) == 1
    call16, dpart16, obj16 = _device_call(lib, torch, dev, x, a, None, None, k, kway_options(seed, ncuts=ncuts))
    warm = args.warmup
    reps = max(1, min(args.steps, 3))
    rmb.set_tuning(parallel_attempts=1)
    for _ in range(warm):
        call16()
    sampler = ClockSampler(gpu_id_for(local_rank))
    sampler.start()
    tw0 = time.time()
    batched = _timed(torch, stream, call16, reps)
    tw1 = time.time()
    sampler.stop()
    best_batched = (int(obj16.value), dpart16.cpu().numpy().copy())
    # The plain path: the same 16 attempts one after another.
    rmb.set_tuning(parallel_attempts=0)
    plain = _timed(torch, stream, call16, 1)
    rmb.set_tuning(parallel_attempts=1)
    same = int(obj16.value) == best_batched[0] and bool((dpart16.cpu().numpy() == best_batched[1]).all())
    # One attempt, profiled, for the roofline of the dominant kernel.
    call1, _, obj1 = _device_call(lib, torch, dev, x, a, None, None, k, kway_options(seed, ncuts=1))
    call1()
    prof = _profile_one(lib, torch, call1)
    # e2e: the drop-in C ABI with pinned host buffers, 16 attempts.
    e2e_ms = _host_call_ms(lib, torch, x, a, None, None, k, kway_options(seed, ncuts=ncuts))
    ms = float(np.mean(batched))
    line = {
        "metric": "k-way attempt-edges/s (batched seeds, best of 16)", "value": ncuts * m / (ms / 1e3),
        "unit": "edges/s", "n_gpus": 1, "steps": reps, "warmup": warm, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"R-MAT scale {args.scale} (a,b,c=.57,.19,.19, edge factor 16, torch seed 22, "
                               "symmetrised, deduplicated), unit weights, nparts=256, ncuts=16 (seed 1+attempt), "
                               "Shem+Greedy, ufactor=30", "name": "rmat_seeds", "n": n, "m": m,
                   "generation_s": round(gen_s, 1), "tuning": TUNING, "l2": "inputs larger than L2"},
        "objval": int(obj16.value), "objval_first_attempt": int(obj1.value),
        "attempts_per_s": ncuts / (ms / 1e3),
        "plain_gpu": {"ms": plain[0], "attempts_per_s": ncuts / (plain[0] / 1e3), "same_result": same},
        "speedup_vs_plain_gpu": plain[0] / ms,
        "e2e": {"value": ncuts * m / (e2e_ms / 1e3), "unit": "edges/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(4 * (len(x) + len(a))), "d2h_bytes_per_step": int(4 * n + 4)},
        "roofline": prof["roofline"], "kernels_one_attempt": prof["kernels"],
        "gpu_launches": prof["launches"],
        "clocks": sampler.summary(tw0, tw1),
    }
    if not args.no_cpu_baseline:
        # The oracle's cost on R-MAT grows with sum(deg^2) (row merges) and
        # k*deg (gains); one attempt on a scale-16 graph of the same law.
        from oracle import oracle as O
        xs, as_ = G.rmat_device(16, seed=22)
        t0 = time.perf_counter()
        rc, _, cobj = O.part_graph_kway(xs, as_, k, options=kway_options(seed))
        dt = time.perf_counter() - t0
        assert rc == 1
        line["cpu_baseline"] = {"value": len(as_) / dt, "unit": "edges/s (attempt-edges)", "cores": 1,
                                "kind": "port", "sample": f"R-MAT scale 16 (n={len(xs) - 1}, m={len(as_)}), "
                                f"k=256, 1 attempt, {dt:.2f} s, cut {cobj}"}
    line["repro"] = _repro()
    print(json.dumps(line))


def _profile_one(lib, torch, call):
    """Per-kernel CUDA-event totals of one call, and the roofline of the kernel
    with the most device time among those with counted bytes."""
    nprof = len(PROF_NAMES)
    launches = (ctypes.c_int64 * (nprof + 1))()
    ms_k = (ctypes.c_double * nprof)()
    bytes_k = (ctypes.c_double * nprof)()
    lib.RMETIS_GPU_GetProfile(launches, ms_k, bytes_k, nprof + 1)
    l0 = [launches[i] for i in range(nprof + 1)]
    m0 = [ms_k[i] for i in range(nprof)]
    b0 = [bytes_k[i] for i in range(nprof)]
    lib.RMETIS_GPU_SetProfiling(1)
    call()
    torch.cuda.synchronize()
    lib.RMETIS_GPU_GetProfile(launches, ms_k, bytes_k, nprof + 1)
    lib.RMETIS_GPU_SetProfiling(0)
    names = PROF_NAMES
    L = [launches[i] - l0[i] for i in range(nprof)]
    M = [ms_k[i] - m0[i] for i in range(nprof)]
    B = [bytes_k[i] - b0[i] for i in range(nprof)]
    dom = max(range(nprof), key=lambda i: M[i] if B[i] > 0 else -1.0)
    avg_ms = M[dom] / max(1, L[dom])
    avg_b = B[dom] / max(1, L[dom])
    peak, kind = load_peaks()
    ach = (avg_b / (avg_ms / 1e3)) / 1e9 if avg_ms > 0 else 0.0
    return {"roofline": {"bound": "hbm", "kernel": names[dom], "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_source": kind, "traffic": None, "bytes_per_launch": avg_b,
                         "ms_per_launch": avg_ms},
            "kernels": {names[i]: {"launches": int(L[i]), "ms": round(M[i], 3)} for i in range(nprof)},
            "launches": int(launches[nprof] - l0[nprof])}


def _host_call_ms(lib, torch, x, a, v, w, k, opts, ncon=1, reps=1):
    I32P = ctypes.POINTER(ctypes.c_int32)
    pin = lambda arr: None if arr is None else torch.from_numpy(np.ascontiguousarray(arr, np.int32)).pin_memory()
    hx, ha, hv, hw = pin(x), pin(a), pin(v), pin(w)
    n = len(x) - 1
    hpart = torch.empty(n, dtype=torch.int32).pin_memory()
    hp = lambda tt: None if tt is None else ctypes.cast(tt.data_ptr(), I32P)
    nv, nc, npr, obj = ctypes.c_int32(n), ctypes.c_int32(ncon), ctypes.c_int32(k), ctypes.c_int32(0)
    op = opts.ctypes.data_as(I32P)
    out = []
    for _ in range(reps):
        t0 = time.perf_counter()
        rc = lib.RMETIS_PartGraphKway(ctypes.byref(nv), ctypes.byref(nc), hp(hx), hp(ha), hp(hv), None, hp(hw),
                                      ctypes.byref(npr), None, None, op, ctypes.byref(obj), hp(hpart))
        out.append((time.perf_counter() - t0) * 1e3)
        if rc != 1:
            raise RuntimeError(f"RMETIS_PartGraphKway returned {rc}")
    return float(np.mean(out))


def _rgg_batch_graphs(count):
    """Graph i: n log-uniform in [1e3, 2e5], k from {2,4,...,64}, vertex
    weights U{1..8} on 2 constraints (numpy default_rng([4, i])), points and
    edges from the device generator seeded by the same stream."""
    out = []
    for i in range(count):
        rng = np.random.default_rng([4, i])
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
        k = int(rng.choice([2, 4, 8, 16, 32, 64]))
        x, a, w = G.rgg2d_device(n, int(rng.integers(1 << 31)), 10.0)
        v = rng.integers(1, 9, size=2 * n).astype(np.int32)
        out.append((x, a, v, w, k))
    return out


def run_rgg_batch(args):
    torch, dev, local_rank = _setup_device()
    import rmetis_b200 as rmb
    t0 = time.perf_counter()
    specs = _rgg_batch_graphs(args.graphs)
    gen_s = time.perf_counter() - t0
    graphs = [rmb.Graph(len(x) - 1, 2, x, a, vwgt=v, adjwgt=w, validate=False) for x, a, v, w, _ in specs]
    ks = [k for *_, k in specs]
    n_tot = sum(g.nvtxs for g in graphs)
    m_tot = sum(len(g.adjncy) for g in graphs)
    o = rmb.Options(rtype=rmb.RType.Greedy, seed=1, ufactor=50)
    warm = args.warmup
    reps = max(1, min(args.steps, 3))
    # The batch as a caller of the C ABI holds it: concatenated CSR arrays in
    # pinned host memory, built once (outside the timed region).
    lib = rmb._lib.load()
    I32P, I64P = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)
    pin = lambda arr, dt=torch.int32: torch.from_numpy(np.ascontiguousarray(arr)).to(dt).pin_memory()
    G_ = len(graphs)
    vtx_off = np.zeros(G_ + 1, np.int64)
    edge_off = np.zeros(G_ + 1, np.int64)
    vtx_off[1:] = np.cumsum([g.nvtxs for g in graphs])
    edge_off[1:] = np.cumsum([len(g.adjncy) for g in graphs])
    h_vo, h_eo = pin(vtx_off, torch.int64), pin(edge_off, torch.int64)
    h_x = pin(np.concatenate([g.xadj for g in graphs]).astype(np.int32))
    h_a = pin(np.concatenate([g.adjncy for g in graphs]).astype(np.int32))
    h_v = pin(np.concatenate([g.vwgt for g in graphs]).astype(np.int32))
    h_w = pin(np.concatenate([g.adjwgt for g in graphs]).astype(np.int32))
    h_k = pin(np.asarray(ks, np.int32))
    h_part = torch.empty(int(vtx_off[-1]), dtype=torch.int32).pin_memory()
    h_obj = torch.zeros(G_, dtype=torch.int32).pin_memory()
    h_st = torch.zeros(G_, dtype=torch.int32).pin_memory()
    opts = o.c_array()
    ptr = lambda t, ty=I32P: ctypes.cast(t.data_ptr(), ty)

    def batch_call():
        rc = lib.RMETIS_GPU_PartGraphKwayBatch(G_, 2, ptr(h_vo, I64P), ptr(h_eo, I64P), ptr(h_x), ptr(h_a),
                                               ptr(h_v), ptr(h_w), ptr(h_k), None, opts.ctypes.data_as(I32P),
                                               ptr(h_obj), ptr(h_part), ptr(h_st))
        if rc != 1:
            raise RuntimeError(f"RMETIS_GPU_PartGraphKwayBatch returned {rc}")

    for _ in range(warm):
        batch_call()
    sampler = ClockSampler(gpu_id_for(local_rank))
    sampler.start()
    tw0 = time.time()
    bt = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batch_call()
        bt.append(time.perf_counter() - t0)
    tw1 = time.time()
    sampler.stop()
    res_part = h_part.numpy().copy()
    res_obj = h_obj.numpy().copy()
    # The plain path: the same graphs one RMETIS_PartGraphKway call after
    # another, from the same pinned buffers.
    nv, nc, npr, obj = ctypes.c_int32(0), ctypes.c_int32(2), ctypes.c_int32(0), ctypes.c_int32(0)
    h_plain = torch.empty(int(vtx_off[-1]), dtype=torch.int32).pin_memory()
    same = True
    t0 = time.perf_counter()
    for i in range(0 if args.no_plain else G_):
        v0, e0 = int(vtx_off[i]), int(edge_off[i])
        nv.value = int(vtx_off[i + 1] - v0)
        npr.value = ks[i]
        off = lambda t, e: ctypes.cast(t.data_ptr() + 4 * e, I32P)
        rc = lib.RMETIS_PartGraphKway(ctypes.byref(nv), ctypes.byref(nc), off(h_x, v0 + i), off(h_a, e0),
                                      off(h_v, 2 * v0), None, off(h_w, e0), ctypes.byref(npr), None, None,
                                      opts.ctypes.data_as(I32P), ctypes.byref(obj), off(h_plain, v0))
        if rc != 1:
            raise RuntimeError(f"RMETIS_PartGraphKway returned {rc}")
        same = same and obj.value == int(res_obj[i])
    pt = time.perf_counter() - t0
    same = same and bool((h_plain.numpy() == res_part).all()) if not args.no_plain else None
    b = float(np.mean(bt))
    line = {
        "metric": "k-way graphs/s (batched uneven graphs)", "value": args.graphs / b, "unit": "graphs/s",
        "n_gpus": 1, "steps": reps, "warmup": warm, "ms_per_step": b * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"{args.graphs} 2D RGGs, n log-uniform [1e3, 2e5], mean degree 10, "
                               "edge w = 1+floor(10(1-d/r)), ncon=2 vwgt U{1..8}, k from {2,..,64}, ufactor=50, "
                               "Shem+Greedy, seed 1", "name": "rgg_batch", "n_total": n_tot, "m_total": m_tot,
                   "generation_s": round(gen_s, 1), "tuning": TUNING,
                   "timing": "host wall clock around the whole RMETIS_GPU_PartGraphKwayBatch call from pinned "
                             "host buffers (one upload, all graphs, results back on the host)",
                   "l2": "inputs larger than L2"},
        "edges_per_s": m_tot / b,
        "plain_gpu": None if args.no_plain else {"s": pt, "graphs_per_s": args.graphs / pt, "same_result": same},
        "speedup_vs_plain_gpu": None if args.no_plain else pt / b,
        "e2e": {"value": args.graphs / b, "unit": "graphs/s", "ms_per_step": b * 1e3,
                "h2d_bytes_per_step": int(4 * (sum(len(s[0]) + len(s[1]) + len(s[2]) + len(s[3]) for s in specs))),
                "d2h_bytes_per_step": int(4 * n_tot + 8 * args.graphs)},
        "clocks": sampler.summary(tw0, tw1),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        sample = specs[:32]
        t0 = time.perf_counter()
        for x, a, v, w, kk in sample:
            rc, _, _ = O.part_graph_kway(x, a, kk, vwgt=v, adjwgt=w, ncon=2, options=kway_options(1, ufactor=50))
            assert rc == 1
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": len(sample) / dt, "unit": "graphs/s", "cores": 1, "kind": "port",
                                "sample": f"the first {len(sample)} graphs of the batch, 1 thread, {dt:.2f} s"}
    line["repro"] = _repro()
    print(json.dumps(line))


def _serving_templates(count=24):
    """Graph templates of the serving stream: 2D grid, 3D grid, 2D RGG (1:1:1),
    n log-uniform in [1e4, 2e6], unit or U{1..10} edge weights
    (numpy default_rng(5))."""
    rng = np.random.default_rng(5)
    out = []
    for i in range(count):
        kind = i % 3
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        weighted = bool(rng.integers(2))
        if kind == 0:
            side = max(2, int(round(np.sqrt(n))))
            x, a = G.grid2d(side, side)
            w = G.grid_weighted((side, side), seed=int(rng.integers(1 << 30)), wmax=10)[2] if weighted else None
            name = f"grid2d {side}x{side}"
        elif kind == 1:
            side = max(2, int(round(n ** (1 / 3))))
            x, a, _, w = G.grid3d(side, weights_seed=int(rng.integers(1 << 30)))
            w = w if weighted else None
            name = f"grid3d {side}^3"
        else:
            x, a, w = G.rgg2d_device(n, int(rng.integers(1 << 31)), 10.0)
            w = w if weighted else None
            name = f"rgg n={n}"
        out.append((name, x, a, w))
    return out


def run_serving(args):
    torch, dev, local_rank = _setup_device()
    import rmetis_b200 as rmb
    t0 = time.perf_counter()
    templates = _serving_templates()
    gen_s = time.perf_counter() - t0
    graphs = [rmb.Graph(len(x) - 1, 1, x, a, adjwgt=w, validate=False) for _, x, a, w in templates]
    rates = [float(r) for r in args.rates.split(",")]
    R = args.requests
    rng = np.random.default_rng(55)
    # Requests: template, k in {2..128}, seed; the same list for every rate.
    req_t = rng.integers(0, len(graphs), R)
    req_k = rng.integers(2, 129, R)
    req_s = rng.integers(1, 1 << 30, R)
    opts = [rmb.Options(rtype=rmb.RType.Greedy, seed=int(s)) for s in req_s]
    # Plain path service times: one request at a time.
    for g in graphs[:3]:
        rmb.part_graph_kway(g, 8, options=opts[0])
    service = np.zeros(R)
    plain_obj = {}
    for i in range(R):
        t0 = time.perf_counter()
        r = rmb.part_graph_kway(graphs[req_t[i]], int(req_k[i]), options=opts[i])
        service[i] = time.perf_counter() - t0
        plain_obj[i] = r.objval
    results = []
    sampler = ClockSampler(gpu_id_for(local_rank))
    sampler.start()
    tw0 = time.time()
    for rate in rates:
        arrivals = np.cumsum(rng.exponential(1.0 / rate, R))
        # Continuous batching: requests are submitted as they arrive and run
        # concurrently on the worker pool.
        done_at = np.zeros(R)
        pending = {}
        mismatches = 0
        start = time.perf_counter()
        nxt = 0
        while nxt < R or pending:
            now = time.perf_counter() - start
            while nxt < R and arrivals[nxt] <= now:
                pending[nxt] = rmb.submit_kway(graphs[req_t[nxt]], int(req_k[nxt]), options=opts[nxt])
                nxt += 1
            for i in [i for i, q in pending.items() if q.done()]:
                done_at[i] = time.perf_counter() - start
                res = pending.pop(i).wait()
                mismatches += int(res.objval != plain_obj[i])
            if nxt < R and not pending:
                time.sleep(max(0.0, min(0.002, arrivals[nxt] - (time.perf_counter() - start))))
            else:
                time.sleep(0.0002)
        lat = (done_at - arrivals) * 1e3
        # The plain path on the same arrivals: FIFO, one request at a time.
        finish = np.zeros(R)
        prev = 0.0
        for i in range(R):
            prev = max(prev, arrivals[i]) + service[i]
            finish[i] = prev
        plat = (finish - arrivals) * 1e3
        results.append({"rate": rate, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "throughput": R / (done_at.max() - arrivals[0]),
                        "plain_p50_ms": float(np.percentile(plat, 50)),
                        "plain_p99_ms": float(np.percentile(plat, 99)),
                        "plain_throughput": R / (finish.max() - arrivals[0]),
                        "results_equal_plain": mismatches == 0})
    tw1 = time.time()
    sampler.stop()
    best = max(results, key=lambda r: r["throughput"])
    line = {
        "metric": "serving throughput (req/s) and p50/p99 latency (ms)", "value": best["throughput"],
        "unit": "requests/s", "n_gpus": 1, "steps": len(rates), "warmup": 1,
        "ms_per_step": float(np.mean(service)) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"{R} requests per rate, Poisson arrivals at {args.rates} req/s, 24 graph "
                               "templates (2D grid / 3D grid / RGG 1:1:1, n log-uniform [1e4, 2e6], unit or "
                               "U{1..10} edge weights), k U{2..128}, ncuts=1, Shem+Greedy",
                   "name": "serving", "generation_s": round(gen_s, 1), "tuning": TUNING,
                   "pool": {"workers": int(os.environ.get("RMETIS_B200_WORKERS", "8")),
                            "budget_bytes": int(os.environ.get("RMETIS_B200_POOL_BYTES", str(150 << 30)))}},
        "rates": results,
        "plain_mean_service_ms": float(np.mean(service)) * 1e3,
        "e2e": {"value": best["throughput"], "unit": "requests/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None},
        "clocks": sampler.summary(tw0, tw1),
    }
    line["repro"] = _repro()
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="grid3d_128", choices=list(WORKLOADS) + list(EXTRA_WORKLOADS))
    ap.add_argument("--scale", type=int, default=22, help="rmat_seeds: R-MAT scale")
    ap.add_argument("--graphs", type=int, default=512, help="rgg_batch: number of graphs")
    ap.add_argument("--requests", type=int, default=10000, help="serving: requests per arrival rate")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="serving: arrival rates, requests/s")
    ap.add_argument("--rtype", default="greedy", choices=["greedy", "fm"],
                    help="refinement: greedy (the measured path) or fm (the reference's default rtype)")
    ap.add_argument("--exact-max-n", type=int, default=None,
                    help="largest level whose greedy cut passes decide sequentially (engine default 16384; "
                         "-1 = every level)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-plain", action="store_true",
                    help="rgg_batch: skip the one-graph-at-a-time leg (profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    RTYPE.update(code=0 if args.rtype == "fm" else 1, name=args.rtype)

    if args.impl == "reference":
        run_reference(args)
        return
    _apply_tuning()
    if args.exact_max_n is not None:
        import rmetis_b200 as rmb
        rmb.set_refine_mode(args.exact_max_n)
        TUNING["exact_max_n"] = args.exact_max_n
    if args.workload in EXTRA_WORKLOADS:
        {"rmat_seeds": run_rmat_seeds, "rgg_batch": run_rgg_batch, "serving": run_serving}[args.workload](args)
        return

    import torch
    import torch.distributed as dist
    import rmetis_b200 as rmb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    build, k, seed, desc = WORKLOADS[args.workload]
    if RTYPE["name"] == "fm":
        desc = desc.replace("Greedy", "Fm")
    x, a, v, w = build()
    n, m = len(x) - 1, len(a)
    lib = rmb._lib.load()
    I32P = ctypes.POINTER(ctypes.c_int32)
    opts = kway_options(seed)
    opts_p = opts.ctypes.data_as(I32P)
    nv, nc, npr = ctypes.c_int32(n), ctypes.c_int32(1), ctypes.c_int32(k)
    obj = ctypes.c_int32(0)

    dev = torch.device("cuda", local_rank)
    t = lambda arr: None if arr is None else torch.from_numpy(np.ascontiguousarray(arr, np.int32)).to(dev)
    dx, da, dv, dw = t(x), t(a), t(v), t(w)
    dpart = torch.empty(n, dtype=torch.int32, device=dev)
    ptr = lambda tt: None if tt is None else tt.data_ptr()
    stream = torch.cuda.current_stream(dev)
    assert lib.RMETIS_GPU_SetStream(stream.cuda_stream) == 1
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def step_device():
        rc = lib.RMETIS_GPU_PartGraphKwayDevice(ctypes.byref(nv), ctypes.byref(nc), ptr(dx), ptr(da), ptr(dv),
                                                ptr(dw), ctypes.byref(npr), None, None, opts_p, ctypes.byref(obj),
                                                ptr(dpart))
        if rc != 1:
            raise RuntimeError(f"RMETIS_GPU_PartGraphKwayDevice returned {rc}")

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    nprof = len(PROF_NAMES)
    launches = (ctypes.c_int64 * (nprof + 1))()
    ms_k = (ctypes.c_double * nprof)()
    bytes_k = (ctypes.c_double * nprof)()
    lib.RMETIS_GPU_GetProfile(launches, ms_k, bytes_k, nprof + 1)
    launches_before = launches[nprof]

    # Timed steps: per-launch profiling off, so the step time carries no
    # profiler events.
    sampler = ClockSampler(gpu_id_for(local_rank))
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_wall0 = time.time()
    for i in range(args.steps):
        flush.zero_()  # L2 flush, outside the timed interval of the step
        starts[i].record(stream)
        step_device()
        ends[i].record(stream)
    torch.cuda.synchronize()
    t_wall1 = time.time()
    if world > 1:
        dist.barrier()
    time.sleep(0.3)
    sampler.stop()
    clocks = sampler.summary(t_wall0, t_wall1)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms_local = float(np.mean(step_ms))
    lib.RMETIS_GPU_GetProfile(launches, ms_k, bytes_k, nprof + 1)
    gpu_launches = int(launches[nprof] - launches_before)
    cut_val = int(obj.value)
    part_host = dpart.cpu().numpy().copy()

    # Separate profiled steps: CUDA events around every profiled launch on
    # the engine's stream give the per-kernel breakdown and the roofline.
    prof_steps = 2
    l0 = [launches[i] for i in range(nprof)]
    m0 = [ms_k[i] for i in range(nprof)]
    b0 = [bytes_k[i] for i in range(nprof)]
    lib.RMETIS_GPU_SetProfiling(1)
    prof_ms = []
    for i in range(prof_steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_device()
        e1.record(stream)
        torch.cuda.synchronize()
        prof_ms.append(e0.elapsed_time(e1))
    lib.RMETIS_GPU_GetProfile(launches, ms_k, bytes_k, nprof + 1)
    lib.RMETIS_GPU_SetProfiling(0)
    P_L = [launches[i] - l0[i] for i in range(nprof)]
    P_M = [ms_k[i] - m0[i] for i in range(nprof)]
    P_B = [bytes_k[i] - b0[i] for i in range(nprof)]

    # e2e through the drop-in C ABI with pinned host buffers
    pin = lambda arr: None if arr is None else torch.from_numpy(np.ascontiguousarray(arr, np.int32)).pin_memory()
    hx, ha, hv, hw = pin(x), pin(a), pin(v), pin(w)
    hpart = torch.empty(n, dtype=torch.int32).pin_memory()
    hp = lambda tt: None if tt is None else ctypes.cast(tt.data_ptr(), I32P)

    def step_host():
        rc = lib.RMETIS_PartGraphKway(ctypes.byref(nv), ctypes.byref(nc), hp(hx), hp(ha), hp(hv), None, hp(hw),
                                      ctypes.byref(npr), None, None, opts_p, ctypes.byref(obj), hp(hpart))
        if rc != 1:
            raise RuntimeError(f"RMETIS_PartGraphKway returned {rc}")

    e2e_steps = args.e2e_steps or max(3, args.steps // 2)
    e2e_local = float("nan")
    if not args.no_e2e:
        for _ in range(2):
            step_host()
        e2e_times = []
        for _ in range(e2e_steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step_host()
            e2e_times.append(time.perf_counter() - t0)
        e2e_local = float(np.mean(e2e_times))
        assert int(obj.value) == cut_val and bool((hpart.numpy() == dpart.cpu().numpy()).all()), \
            "host and device entry points disagree"

    if world > 1:
        tt = torch.tensor([ms_local, e2e_local], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max, e2e_max = float(tt[0]), float(tt[1])
    else:
        ms_max, e2e_max = ms_local, e2e_local

    if rank == 0:
        value = world * m / (ms_max / 1000.0)
        e2e_value = world * m / e2e_max
        peak, peak_kind = load_peaks()
        names = PROF_NAMES
        dom = max(range(nprof), key=lambda i: P_M[i] if P_B[i] > 0 else -1.0)
        avg_ms = P_M[dom] / max(1, P_L[dom])
        avg_bytes = P_B[dom] / max(1, P_L[dom])
        achieved = (avg_bytes / (avg_ms / 1000.0)) / 1e9 if avg_ms > 0 else 0.0
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            try:
                traffic = json.load(open(tpath)).get(args.workload, {}).get(names[dom])
            except Exception:
                traffic = None
        kernels = {names[i]: {"launches": int(P_L[i]) // prof_steps, "ms": round(P_M[i] / prof_steps, 4),
                              "GBps": round(P_B[i] / (P_M[i] / 1000.0) / 1e9, 1) if P_M[i] > 0 and P_B[i] > 0
                              else None} for i in range(nprof)}
        step_bytes = sum(P_B) / prof_steps
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": _config(args.workload, n, m, k, world),
            "l2": "flushed before every timed step (256 MiB write)",
            "tuning": TUNING,
            "objval": cut_val,
            "balance": balance_summary(x, v, part_host, k),
            "gpu_launches": gpu_launches,
            "gpu_launches_per_step": gpu_launches / args.steps,
            "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": e2e_max * 1000.0,
                    "h2d_bytes_per_step": int(4 * (len(x) + len(a) + (0 if v is None else len(v)) +
                                                   (0 if w is None else len(w)))),
                    "d2h_bytes_per_step": int(4 * n + 4)},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic, "bytes_per_launch": avg_bytes, "ms_per_launch": avg_ms,
                         "timing": f"CUDA events around each launch in {prof_steps} profiled steps after the "
                                   "timed ones"},
            "roofline_step": {"bound": "hbm", "bytes_per_step": step_bytes,
                              "achieved": step_bytes / (ms_max / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                              "frac": step_bytes / (ms_max / 1000.0) / 1e9 / peak, "peak_source": peak_kind,
                              "bytes": "algorithmic bytes of the profiled kernel families (gain tables, "
                                       "matching round 0, contraction, grow, single-block levels, coarse "
                                       "tail, cut), per step"},
            "profiled_ms_per_step": float(np.mean(prof_ms)),
            "kernels_per_step": kernels,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload, graph=(x, a, v, w))
            ref_cut = int(line["cpu_baseline"].pop("objval"))
            line["quality"] = {"objval": cut_val, "oracle_objval": ref_cut, "ratio": cut_val / max(1, ref_cut),
                               "seed": seed}
        line["repro"] = _repro()
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
