"""The JSON line of ``bench.py --impl reference`` (GLU's own solver on the host
cores), run as a short subprocess on the CPU for every workload (Landau FACG,
the FASD ensemble, Coulomb 64^3x128, gluon propagators, heatbath): every key
of the bench line, a positive throughput, the reference arm's own
``cpu_baseline`` and a zero-copy ``e2e``.  A non-zero rank of a multi-rank
launch exits 0 without a line.  Without a CUDA device the GPU arm of every
workload fails with no line printed (no CPU fallback).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT, _ensure_oracle

ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "0",
        "--cpu-sample-s", "0.5"]


def _run(extra=(), env_extra=None):
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *ARGS, *extra],
                          cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=240)


def _lines(out: str):
    return [json.loads(s) for s in out.splitlines() if s.startswith("{")]


# configurations fixed per step, from the line's config
def _landau_n(cfg):
    return len(cfg["full_fix_iters"])


def _one(cfg):
    return 1


def _coulomb_n(cfg):
    assert cfg["slice_steps"] > 0
    return 1


def _ensemble_n(cfg):
    assert cfg["configs"] == 48 + 16
    return cfg["configs"]


@pytest.mark.parametrize("extra, configs_per_step", [
    ((), _landau_n),
    (("--workload", "ensemble"), _ensemble_n),
    (("--workload", "coulomb"), _coulomb_n),
    (("--workload", "gluonprop"), _one),
    (("--workload", "heatbath"), _one),
], ids=["landau", "ensemble", "coulomb", "gluonprop", "heatbath"])
def test_reference_arm_line(extra, configs_per_step):
    _ensure_oracle()
    r = _run(extra)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup",
              "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
              "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["unit"].endswith("/hour") and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # configs/hour and ms per step describe the same step of E configurations
    n = configs_per_step(d["config"])
    assert abs(d["value"] * d["ms_per_step"] / 3.6e6 - n) < 1e-6 * n


def test_reference_arm_other_ranks_silent():
    r = _run((), {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert _lines(r.stdout) == []


@pytest.mark.parametrize("workload", ["landau", "coulomb", "ensemble", "gluonprop",
                                      "heatbath"])
def test_gpu_arm_fails_loudly_without_cuda(workload):
    # no CPU fallback: without a CUDA device the GPU arm exits with an error
    # and prints no bench line
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--workload", workload,
                        "--steps", "1", "--warmup", "3", "--no-cpu-baseline"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=240)
    assert r.returncode != 0
    assert _lines(r.stdout) == []


def _bench_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_other_workloads_are_bounded(monkeypatch):
    """The default run's section for the benchmark table's other
    configurations: off at a budget of 0, and every workload listed as
    skipped (none started) when the budget cannot hold one."""
    b = _bench_module()
    monkeypatch.setenv("GLU_GFIX_BENCH_OTHERS_S", "0")
    assert b.other_workloads() == []
    monkeypatch.setenv("GLU_GFIX_BENCH_OTHERS_S", "30")
    recs = b.other_workloads()
    assert [r["workload"] for r in recs] == [w[0] for w in b.OTHER_WORKLOADS]
    assert all("time budget" in r["skipped"] for r in recs)


def test_compact_line_keeps_the_figures():
    b = _bench_module()
    line = {"metric": "m", "value": 2.0, "unit": "configs/hour", "steps": 1, "warmup": 3,
            "ms_per_step": 5.0, "dtype": "f32+f64", "data": "d",
            "e2e": {"value": 1.5, "unit": "configs/hour"},
            "config": {"workload": "w", "iters_total": 10, "iters_min_max": [1, 9],
                       "fp64_only": {"value": 1.0, "e2e": 0.9, "ms_per_step": 9.0}},
            "roofline": {"kernel": "k", "frac": 0.5, "unit": "GB/s", "achieved": 3.0,
                         "per_kernel": {}},
            "clocks": {"sm_mhz": 1800.0}}
    c = b.compact_line(line)
    assert (c["metric"], c["value"], c["e2e"], c["workload"]) == ("m", 2.0, 1.5, "w")
    assert c["iters_total"] == 10 and c["iters_min_max"] == [1, 9]
    assert c["fp64_only"] == {"value": 1.0, "e2e": 0.9}
    assert c["roofline"] == {"kernel": "k", "frac": 0.5, "unit": "GB/s", "achieved": 3.0}
    assert c["clocks"] == {"sm_mhz": 1800.0}
