"""bench.py's host logic on the CPU (no GPU, no oracle run): both arms
describe the same workload, and the CPU-baseline sample grows until it fills
its target time (whole-image passes up to 64 spp)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import bench  # noqa: E402
from colvillea_b200 import scenes  # noqa: E402


@pytest.mark.parametrize("spp_per_step", [0, 8])
def test_both_arms_describe_the_same_workload(spp_per_step):
    """Our arm passes the step's spp, the reference arm the command-line value: the config objects are equal."""
    s = scenes.config1(0, 64, 48)
    ours = bench.workload_desc(s, bench.step_spp(s, spp_per_step))
    ref = bench.workload_desc(s, spp_per_step)
    assert ours == ref
    assert ours["spp_per_step"] == (spp_per_step or min(s.spp, 64))


class _FakeOracle:
    """Renders nothing; each call advances a fake clock by paths / rate plus a fixed start-up cost."""

    def __init__(self, rate, startup, clock):
        self.rate, self.startup, self.clock, self.calls = rate, startup, clock, []

    def render(self, spp, max_depth, rr_start, flags, pixels, threads):
        n = len(pixels) * spp
        self.calls.append((len(pixels), spp))
        self.clock[0] += self.startup + n / self.rate
        return None, None, np.array([n, n // 2], np.uint64)


@pytest.mark.parametrize("rate,seconds,expect_spp", [(3.0e6, 15.0, None), (1.0e5, 8.0, 1), (1.0e9, 15.0, 64)])
def test_cpu_sample_fills_its_target_time(monkeypatch, rate, seconds, expect_spp):
    clock = [0.0]
    monkeypatch.setattr(bench.time, "perf_counter", lambda: clock[0])
    w, h = 1920, 1080
    fake_scene = type("S", (), {"width": w, "height": h, "max_depth": 8, "rr_start": 3})()
    o = _FakeOracle(rate, 0.01, clock)
    value, sample = bench._oracle_rate(o, fake_scene, seconds, threads=16)
    npix, spp = o.calls[-1]
    dt = o.startup + npix * spp / rate
    assert dt >= 0.5 * seconds or (npix == w * h and spp == 64)
    assert dt <= 2.0 * seconds
    assert abs(value - npix * spp / dt / 1e6) < 1e-6 * max(1.0, value)
    if expect_spp is not None:
        assert spp == expect_spp
    if spp > 1:
        assert npix == w * h                   # several spp only over the whole image
    assert f"{spp} spp" in sample
