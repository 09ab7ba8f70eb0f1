"""Host-side arithmetic of bench.py (no GPU): the work and real-time-channel
conversions, the roofline denominator, the DRAM traffic read from the committed
ncu summaries, and the rule that the product package never reaches the CPU
oracle."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_exact_ops_and_realtime_channel():
    # 8 ops (4 int8 MACs) per upper-triangle complex visibility per sample
    assert bench.vis_ops(2048, 1, 1) == 8 * 2048 * 2049 / 2
    assert bench.vis_ops(256, 10, 3) == 3 * 10 * bench.vis_ops(256, 1, 1)
    # one real-time E=2048 channel is 390625 samples/s of that work: 6.557 TOPS
    assert bench.E2048_RT_TOPS == pytest.approx(bench.vis_ops(2048, 390625, 1) / 1e12)
    assert bench.E2048_RT_TOPS == pytest.approx(6.557, abs=1e-3)


def test_int8_peak_is_twice_the_measured_bf16_burst():
    peak, src = bench.int8_peak({"bf16_tflops": 1691.3, "hbm_gbs": 6452.8})
    assert peak == pytest.approx(3382.6)
    assert "measured" in src
    peak, src = bench.int8_peak(None)
    assert peak == pytest.approx(3180.0)
    assert "fallback" in src


def test_traffic_comes_from_the_committed_summaries():
    plain = bench.profile_traffic("tc_pair_correlate_E2048_F8_T16384.md")
    batched = bench.profile_traffic("tc_pair_correlate_batched64.md")
    # both captures moved about the algorithmic bytes (input once, blocks once)
    assert plain is not None and 0.9 < plain / (268435456 + 136314880) < 1.2
    assert batched is not None and 0.9 < batched / (314327040 + 1816395776) < 1.1
    assert bench.profile_traffic("no_such_summary.md") is None


def test_product_package_does_not_reach_the_oracle():
    pkg = os.path.join(ROOT, "chime-x_b200")
    offenders = []
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if not f.endswith((".py", ".cu", ".cuh", ".h", ".c", ".cpp")):
                continue
            with open(os.path.join(dirpath, f), errors="replace") as fh:
                text = fh.read()
            if "oracle" in text or "pyoracle" in text or "chx_oracle" in text:
                offenders.append(os.path.relpath(os.path.join(dirpath, f), ROOT))
    assert offenders == []


def test_channel_shards_balance_cost():
    """Largest-first assignment: disjoint shards covering every channel, the
    same on every rank, with per-rank cost within one channel of the mean."""
    costs = [5, 1, 9, 3, 3, 7, 2, 8, 4, 6]
    for world in (1, 2, 3, 4):
        shards = [bench.shard_channels(costs, world, r) for r in range(world)]
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in sh) for sh in shards]
        assert max(loads) - min(loads) <= max(costs)
    assert bench.shard_channels(costs, 1, 0) == list(range(len(costs)))


def test_clock_records_that_reject_a_number():
    ok = {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": []}
    assert not bench.clocks_rejected(ok)
    assert not bench.clocks_rejected(dict(ok, sm_mhz=1400.0, reasons=["sw_power_cap"]))
    assert bench.clocks_rejected(dict(ok, reasons=["hw_slowdown"]))
    assert bench.clocks_rejected(dict(ok, reasons=["sw_thermal_slowdown"]))
    assert bench.clocks_rejected(dict(ok, sm_mhz=900.0))   # stuck low, no reason: a lock


def test_default_run_is_bounded():
    """The driver's default invocation (no flags) runs the headline, sustained,
    peak, batched and stream legs with a small K and W."""
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert 'default="all"' in src
    assert '"--steps", type=int, default=20' in src
    assert '"--warmup", type=int, default=5' in src
