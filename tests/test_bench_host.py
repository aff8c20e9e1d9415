"""Host-side helpers of bench.py that need no GPU: where the end-to-end job places its host
threads (NVML's CPU affinity of the device, narrowed to what the process may use), read
through a stand-in NVML module."""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _fake_nvml(mask_words):
    m = types.ModuleType("pynvml")
    m.nvmlInit = lambda: None
    m.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    m.nvmlDeviceGetCpuAffinity = lambda h, n: list(mask_words)[:n]
    return m


@pytest.fixture
def allowed():
    return sorted(os.sched_getaffinity(0))


def test_local_cpus_narrow_to_the_gpu_node(monkeypatch, allowed):
    if len(allowed) < 2:
        pytest.skip("needs two CPUs")
    first = allowed[0]
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml([1 << first] + [0] * 15))
    assert bench.gpu_local_cpus(0) == {first}


def test_local_cpus_none_when_not_narrower_or_unknown(monkeypatch, allowed):
    words = [0] * 16
    for c in allowed:
        words[c // 64] |= 1 << (c % 64)
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml(words))
    assert bench.gpu_local_cpus(0) is None  # every allowed CPU: nothing to narrow
    bad = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no NVML")
    bad.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", bad)
    assert bench.gpu_local_cpus(0) is None
    # CPUs outside the process's set are dropped; none left means no binding
    outside = max(allowed) + 1
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml([1 << outside if outside < 64 else 0] + [0] * 15))
    assert bench.gpu_local_cpus(0) is None
