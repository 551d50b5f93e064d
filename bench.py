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
}
CPU_SAMPLE = {
    "grid3d_128": (lambda: G.grid3d(64, weights_seed=7), "3D 7-point grid 64^3 (same weight laws), nparts=64"),
    "grid2d_64": (lambda: G.grid2d(64, 64) + (None, None), "2D grid 64x64, nparts=8"),
}


def kway_options(seed, ncuts=1, niter=10, ufactor=30):
    a = np.full(40, -1, dtype=np.int32)
    a[0] = 0; a[1] = 0; a[2] = 1; a[3] = 0; a[4] = 1; a[5] = 0
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
            "sample": f"{desc} (n={len(x) - 1}, m={len(a)}), 1 partition, {dt:.2f} s, cut {obj}"}


def run_reference(args):
    """--impl reference: the oracle on all host cores (independent partitions
    of a bounded sample in parallel threads; the reference's only parallel
    axis is independent attempts)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    build, desc = CPU_SAMPLE[args.workload]
    x, a, v, w = build()
    k, seed = WORKLOADS[args.workload][1], WORKLOADS[args.workload][2]
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    O.lib()

    def one(i):
        rc, _, obj = O.part_graph_kway(x, a, k, vwgt=v, adjwgt=w, options=kway_options(seed + i))
        assert rc == 1
        return obj

    times = []
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            list(ex.map(one, range(threads)))
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append(dt)
    ms = 1000.0 * statistics.mean(times)
    value = threads * len(a) / (ms / 1000.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload][3], "sample": desc, "n": len(x) - 1, "m": len(a)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{desc}: {threads} independent partitions per step in {threads} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="grid3d_128", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
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

    nprof = 6
    launches = (ctypes.c_int64 * (nprof + 1))()
    ms_k = (ctypes.c_double * nprof)()
    bytes_k = (ctypes.c_double * nprof)()
    lib.RMETIS_GPU_GetProfile(launches, ms_k, bytes_k, nprof + 1)
    launches_before = launches[nprof]
    lib.RMETIS_GPU_SetProfiling(1)

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
    lib.RMETIS_GPU_SetProfiling(0)
    gpu_launches = int(launches[nprof] - launches_before)
    cut_val = int(obj.value)

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
        names = ["k_gain", "k_walk", "k_match_propose", "k_contract_thread", "k_cut", "k_grow"]
        dom = max(range(nprof), key=lambda i: ms_k[i] if bytes_k[i] > 0 else -1.0)
        avg_ms = ms_k[dom] / max(1, launches[dom])
        avg_bytes = bytes_k[dom] / max(1, launches[dom])
        achieved = (avg_bytes / (avg_ms / 1000.0)) / 1e9 if avg_ms > 0 else 0.0
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            try:
                traffic = json.load(open(tpath)).get(args.workload, {}).get(names[dom])
            except Exception:
                traffic = None
        kernels = {names[i]: {"launches": int(launches[i]), "ms": round(ms_k[i] / args.steps, 4),
                              "GBps": round(bytes_k[i] / (ms_k[i] / 1000.0) / 1e9, 1) if ms_k[i] > 0 and bytes_k[i] > 0
                              else None} for i in range(nprof)}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": desc, "name": args.workload, "n": n, "m": m, "nparts": k,
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "objval": cut_val,
            "gpu_launches": gpu_launches,
            "gpu_launches_per_step": gpu_launches / args.steps,
            "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": e2e_max * 1000.0,
                    "h2d_bytes_per_step": int(4 * (len(x) + len(a) + (0 if v is None else len(v)) +
                                                   (0 if w is None else len(w)))),
                    "d2h_bytes_per_step": int(4 * n + 4)},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic, "bytes_per_launch": avg_bytes, "ms_per_launch": avg_ms},
            "kernels_per_step": kernels,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload, graph=(x, a, v, w))
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
