"""The benchmark's command-line contract, checked on the CPU.

The reference arm (`--impl reference`) runs the oracle on the host cores, so
it runs here: one JSON line with the arm's metric, unit and config, a
`cpu_baseline` describing the run and an `e2e` with no host-device traffic;
under a multi-rank launch only rank 0 works and prints. The library's own arm
needs a GPU and must fail loudly without one (no CPU fallback)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None, timeout=300):
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, "bench.py"] + args, cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=timeout)


def test_reference_arm_line_on_small_grid():
    r = _run(["--impl", "reference", "--workload", "grid2d_64", "--steps", "1", "--warmup", "3"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "k-way edges/s (plain path)" and d["unit"] == "edges/s"
    assert d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] >= 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["name"] == "grid2d_64" and d["config"]["n"] == 4096 and d["config"]["m"] == 16128
    assert "workload" in d["config"] and d["config"]["nparts"] == 8
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert isinstance(d["objval"], int) and d["objval"] > 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run(["--impl", "reference", "--workload", "grid2d_64", "--steps", "1", "--warmup", "3"],
             {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_library_arm_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the GPU tests cover this arm")
    r = _run(["--workload", "grid2d_64", "--steps", "1", "--warmup", "3"], timeout=120)
    assert r.returncode != 0
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
