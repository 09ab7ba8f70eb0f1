"""Benchmark of the CHIME X-engine hot path on B200.

Headline workload (N=1): the plain correlator at full CHIME size, E=2048
elements, F=8 channels, T=16384 samples (64 integrations of time_accum=256),
one fused chx_correlate launch per step over inputs already resident in HBM.
Metric: exact INT8 tensor-core TOPS = 8 * E(E+1)/2 * T * F / seconds (4 int8
MACs per upper-triangle complex visibility per sample; diagonal-tile waste
not credited).

The default run prints ONE JSON line holding, besides the headline value:
  sustained         >= 5 s of back-to-back launches of the same workload with
                    the SM clock sampled, binned by clock; real-time channels
  int8_peak_in_run  a cuBLAS int8 GEMM (torch._int_mm, 8192^3) timed in the
                    same process, with its median SM clock
  batched           the 64-channel ragged batch in one CUDA-graph
                    launch against the plain per-channel launches
  stream            the 1024-channel streaming loop, real-time
                    channels sustained, p50/p99 frame-to-visibility latency
  e2e, cpu_baseline, roofline, clocks, gpu_launches

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--config all|plain|batched|stream|helpers] [--algo auto|simt|tc]

Multi-GPU: one process per GPU.  `--gpus N` without a torchrun environment
relaunches itself under torch.distributed.run.  Each rank correlates its own
plain-workload channels (weak scaling) and its share of the batched and
streamed channel lists (largest-first assignment, strong scaling); there is
no data-path collective, the job time is the max over ranks and the work the
sum over ranks.  `--impl reference` times the reference's own CPU correlator
(cpu_corr_test.c, built from the reference sources into oracle/_ref) on the
host cores instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "chime-x_b200"))

OPS_PER_VIS_SAMPLE = 8  # 4 int8 MACs per complex visibility per sample
REALTIME_SPS = 390625   # CHIME samples/s per channel
E2048_RT_TOPS = OPS_PER_VIS_SAMPLE * 2048 * 2049 / 2 * REALTIME_SPS / 1e12
NOMINAL_INT8_TOPS = 4500.0


def vis_ops(E, T, F):
    return OPS_PER_VIS_SAMPLE * E * (E + 1) / 2 * T * F


def max_over_ranks(value, dist, device):
    """The maximum of `value` over all ranks (the job's time is the slowest
    rank's); `value` itself when there is no process group.  `device` is where
    the collective's tensor lives (the rank's GPU for NCCL, CPU for gloo)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist, device):
    """The sum of `value` over all ranks; `value` itself when there is no
    process group."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def shard_channels(costs, world, rank):
    """Indices of the channels rank `rank` owns out of `world` ranks: the
    channels, costliest first (ties by index), each go to the rank with the
    least cost so far (ties to the lowest rank).  Deterministic, so every rank
    computes the same partition without communicating: the shards are
    disjoint and cover every channel."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += costs[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


# ----------------------------------------------------------------- peaks
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return json.load(fh)
    except Exception:
        return None


def int8_peak(peaks):
    """Dense INT8 tensor peak used as the roofline denominator.

    MEASURED_PEAKS.json holds cuBLAS bf16 figures; B200's dense INT8 rate is
    twice its dense BF16 rate, so the INT8 denominator is 2 x the measured
    bf16 burst figure (the kernel is timed alone in a burst of launches).
    Fallback: 2 x 1590 TFLOP/s, an earlier measurement on this pool."""
    if peaks and peaks.get("bf16_tflops"):
        return 2.0 * float(peaks["bf16_tflops"]), "2 x measured bf16 burst (MEASURED_PEAKS.json)"
    return 2.0 * 1590.0, "2 x fallback bf16 1.59 PF/s"


def profile_traffic(name):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    recorded from one ncu capture of this workload in profiles/<name>; None
    when there is no summary."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ----------------------------------------------------------------- clocks
# NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*).
_REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}
REJECT_REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                  "hw_power_brake_slowdown")


class ClockSampler:
    """Samples the SM clock, power and clock-event reasons of one GPU through
    NVML from a background thread every `period_s` (2 ms by default: fine
    enough to see a 20 ms timed region).  Reading only: nothing is set."""

    def __init__(self, torch_device, period_s=0.002):
        self.dev = torch_device
        self.period = period_s
        self.samples = []  # (time, sm MHz, power W, reasons bits)
        self.handle = None
        self.nvml = None
        self.sm_max = None
        self._stop = threading.Event()
        self._thread = None
        self.t0 = self.t1 = None
        self.error = None

    def _open(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.dev)
        h = None
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))
        except Exception:
            h = None
        if h is None:
            try:
                h = pynvml.nvmlDeviceGetHandleByPciBusId(
                    "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id,
                                          props.pci_device_id))
            except Exception:
                h = None
        if h is None:
            h = pynvml.nvmlDeviceGetHandleByIndex(int(self.dev.index or 0))
        self.nvml, self.handle = pynvml, h
        self.sm_max = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

    def _run(self):
        nv, h = self.nvml, self.handle
        while not self._stop.is_set():
            try:
                t = time.time()
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((t, sm, pw, rs))
            except Exception as e:  # keep the benchmark running without clocks
                self.error = str(e)
                return
            time.sleep(self.period)

    def __enter__(self):
        try:
            self._open()
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        except Exception as e:
            self.error = "nvml unavailable: %s" % e
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=5)
        try:
            if self.nvml is not None:
                self.nvml.nvmlShutdown()
        except Exception:
            pass

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def window(self, t0=None, t1=None):
        t0 = self.t0 if t0 is None else t0
        t1 = self.t1 if t1 is None else t1
        if t0 is None or t1 is None:
            return list(self.samples)
        return [s for s in self.samples if t0 <= s[0] <= t1]

    def summary(self, t0=None, t1=None):
        rows = self.window(t0, t1)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": self.sm_max,
                    "reasons": [self.error or "no samples"], "samples": 0}
        sm = [r[1] for r in rows]
        reasons = [n for n, bit in _REASONS.items() if any(r[3] & bit for r in rows)]
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm),
                "sm_max_mhz": self.sm_max, "power_w_max": max(r[2] for r in rows),
                "samples": len(rows), "reasons": reasons, "source": "NVML, 2 ms"}


def clocks_rejected(summary):
    """True when a clock record shows a throttle that invalidates a number
    (hardware or thermal slowdown), or SM clocks stuck well below the maximum
    with no reason (a leftover clock lock)."""
    if any(r in REJECT_REASONS for r in summary.get("reasons", [])):
        return True
    sm, smax = summary.get("sm_mhz"), summary.get("sm_max_mhz")
    if sm and smax and sm < 0.8 * smax and not summary.get("reasons"):
        return True
    return False


# ------------------------------------------------------------ cpu baseline
def _ref_driver():
    p = os.path.join(ROOT, "oracle", "_ref", "cpu_corr_ref")
    return p if os.path.exists(p) else None


def cpu_reference_rate(E, T_sample, max_procs=None, no_repeat=1, seed0=42):
    """Times the reference's own CPU correlator (oracle/_ref/cpu_corr_ref,
    built from cpu_corr_test.c) on the host cores: one process per core, each
    correlating one E-element channel over T_sample samples.  Returns
    (ops_per_s, cores, sample description, kind, wall seconds) or None."""
    driver = _ref_driver()
    if driver is None:
        return None
    cores = max_procs or os.cpu_count() or 1
    t0 = time.time()
    procs = [subprocess.Popen([driver, str(T_sample), "1", str(E), "4", str(seed0 + i),
                               str(no_repeat), "1"], stdout=subprocess.PIPE, text=True)
             for i in range(cores)]
    outs = [p.communicate()[0] for p in procs]
    wall = time.time() - t0
    total_ops = 0.0
    for o in outs:
        rec = json.loads(o.strip().splitlines()[-1])
        total_ops += OPS_PER_VIS_SAMPLE * rec["updates"]
    sample = ("%d concurrent processes x (E=%d, F=1, T=%d, seeded random) of the "
              "reference cpu_data_generate_and_correlate_upper_triangle_only" % (cores, E, T_sample))
    return total_ops / wall, cores, sample, "reference", wall


def cpu_single_core():
    """The reference CPU correlator on ONE core: the small plain case in full
    (E=256, F=1, T=256, seed 42, repeating generator), repeated for about a
    second, and a bounded sample of the full-size plain workload (E=2048, F=1, T=512,
    no repeat).
    Each figure is the reference's own timing of its correlation loop."""
    driver = _ref_driver()
    if driver is None:
        return None
    out = {"cores": 1, "cpu_model": cpu_model(), "kind": "reference"}

    def run(T, E, no_repeat):
        r = subprocess.run([driver, str(T), "1", str(E), "4", "42", str(no_repeat), "1"],
                           capture_output=True, text=True, check=True)
        return json.loads(r.stdout.strip().splitlines()[-1])

    recs, t_end = [], time.time() + 1.0
    while time.time() < t_end or not recs:
        recs.append(run(256, 256, 0))
    secs = statistics.median(r["seconds"] for r in recs)
    out["config1"] = {"value": OPS_PER_VIS_SAMPLE * recs[0]["updates"] / secs / 1e12,
                      "unit": "TOPS", "seconds": secs, "runs": len(recs),
                      "sample": "E=256 F=1 T=256 seed 42 repeat (the small plain case in full)",
                      "triangle_fnv": recs[0]["hash"]}
    r2 = run(512, 2048, 1)
    out["config2_sample"] = {"value": OPS_PER_VIS_SAMPLE * r2["updates"] / r2["seconds"] / 1e12,
                             "unit": "TOPS", "seconds": r2["seconds"],
                             "sample": "E=2048 F=1 T=512 seed 42 no repeat (1/256 of the full-size plain workload)"}
    return out


def run_reference_arm(args):
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    E, F, T = 2048, 8, 16384
    if _ref_driver() is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/cpu_corr_ref not built (needs the reference sources)"}))
        return 0
    cores = os.cpu_count() or 1
    # Samples per process per step: 384 is ~2 s of CPU work per core; by
    # default the sample shrinks so that all the timed steps take ~2.5 min.
    if args.ref_sample:
        t_sample = args.ref_sample
    else:
        t_sample = max(8, min(384, int(384 * (150.0 / max(1, args.steps)) / 2.0)))
    for _ in range(args.warmup):
        cpu_reference_rate(E, 8, max_procs=cores)
    rates, walls = [], []
    for _ in range(args.steps):
        r = cpu_reference_rate(E, t_sample, max_procs=cores)
        rates.append(r[0])
        walls.append(r[4])
    ops_s = sum(rates) / len(rates)
    value = ops_s / 1e12
    line = {
        "impl": "reference", "metric": "exact INT8-TC TOPS", "value": value, "unit": "TOPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(walls) / len(walls), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32 (reference CPU)",
        "data": "synthetic: reference generator, seeded random, no_repeat",
        "config": {"workload": "plain correlator E=2048 F=8 T=16384 time_accum=256; each step "
                               "a bounded sample of it on the host cores", "E": E, "F": F, "T": T},
        "cpu_baseline": {"value": value, "unit": "TOPS", "cores": cores, "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": "%d processes x (E=%d, T=%d) per step" % (cores, E, t_sample)},
        "e2e": {"value": value, "unit": "TOPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "realtime_channels_e2048": ops_s / (E2048_RT_TOPS * 1e12),
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------- our arm
def make_plain_plan(args, cx, local_rank):
    plan = cx.Plan(args.E, args.F, args.T, 256, 1, 0, local_rank)
    if args.algo == "simt":
        plan.set_option(cx.OPT_ALGO, cx.ALGO_SIMT)
    elif args.algo == "tc":
        plan.set_option(cx.OPT_ALGO, cx.ALGO_TC)
    if args.tsplit:
        plan.set_option(cx.OPT_TSPLIT, args.tsplit)
    if args.tile:
        plan.set_option(cx.OPT_TILE, args.tile)
    return plan


def run_plain(args, torch, cx, dist, clk):
    """The headline leg: one chx_correlate launch of E=2048 F=8 T=16384 per step."""
    rank, local_rank, world = env_rank()
    E, F, T, TA = args.E, args.F, args.T, 256
    dev = torch.device("cuda", local_rank)
    plan = make_plain_plan(args, cx, local_rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(42 + rank)
    packed = torch.randint(0, 256, (plan.input_bytes,), dtype=torch.uint8, device=dev,
                           generator=gen)
    blocks = torch.empty(plan.block_words, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ops_step = vis_ops(E, T, F)

    def step():
        plan.correlate(packed, blocks, stream=stream)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for _ in range(max(args.warmup, 3)):
        step()
    plan.check_device()
    torch.cuda.synchronize(dev)
    # device-timed region: inputs larger than L2 (see config["l2"])
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    clk.mark_start()
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    clk.mark_end()
    if dist is not None:
        dist.barrier()
    plan.check_device()
    clocks = clk.summary()
    total_ms = max_over_ranks(t_start.elapsed_time(t_end), dist, dev)
    per_launch = [a.elapsed_time(b) for a, b in ev]
    job_ops = sum_over_ranks(ops_step * args.steps, dist, dev)
    value = job_ops / (total_ms * 1e-3) / 1e12

    peak, peak_src = int8_peak(load_peaks())
    traffic = None
    if (E, F, T) == (2048, 8, 16384) and args.algo != "simt" and args.tile in (0, 2):
        traffic = profile_traffic("tc_pair_correlate_E2048_F8_T16384.md")
    achieved = ops_step / (sum(per_launch) / len(per_launch) * 1e-3) / 1e12
    line = {
        "metric": "exact INT8-TC TOPS", "value": value, "unit": "TOPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: seeded uniform 4-bit complex (re, im uniform in [-8, 7]), "
                "device-generated",
        "config": {"workload": "Plain correlator at full CHIME size: E=2048, F=8, T=16384 "
                               "(64 integrations of time_accum=256), random uniform [-8,7] "
                               "re/im; one chx_correlate launch per step per GPU",
                   "E": E, "F": F, "T": T, "time_accum": TA, "algo": args.algo, "tile": args.tile,
                   "l2": "inputs (%d MiB) %s L2 (126 MB); no flush" % (
                       E * F * T >> 20, "larger than" if E * F * T > 126e6 else "SMALLER than"),
                   "parallelism": "channel shards, %d GPU(s), no collective" % world},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOPS",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                     "kernel": "tc_pair_kernel (correlator)",
                     "median_launch_ms": sorted(per_launch)[len(per_launch) // 2],
                     "nominal_peak": NOMINAL_INT8_TOPS,
                     "frac_of_nominal": achieved / NOMINAL_INT8_TOPS},
        "pct_of_int8_peak": 100.0 * value / world / peak,
        "realtime_channels_e2048_burst": value / E2048_RT_TOPS,
        "gpu_launches": args.steps,
        "clocks": clocks,
    }
    if clocks_rejected(clocks):
        line["clocks_rejected"] = True
    return line, plan, packed, blocks, ops_step


def run_sustained(args, torch, plan, packed, blocks, ops_step, dist, dev, clk, seconds=5.0):
    """Back-to-back launches of the headline workload for `seconds`, in chunks
    of launches each timed with CUDA events, with the NVML clock samples of
    each chunk's window: sustained TOPS, the median SM clock under load and
    TOPS per MHz (the kernel's speed at the clock it actually ran at)."""
    stream = torch.cuda.current_stream(dev)
    # chunk of about 0.2 s of launches
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(10):
        plan.correlate(packed, blocks, stream=stream)
    b.record(stream)
    torch.cuda.synchronize(dev)
    per_ms = a.elapsed_time(b) / 10
    chunk = max(10, int(200.0 / max(per_ms, 1e-3)))
    nchunks = max(5, int(seconds * 1000.0 / (chunk * per_ms)))
    if dist is not None:
        dist.barrier()
    rows = []
    t_all0 = time.time()
    for _ in range(nchunks):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0 = time.time()
        e0.record(stream)
        for _ in range(chunk):
            plan.correlate(packed, blocks, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        h1 = time.time()
        ms = e0.elapsed_time(e1)
        win = clk.window(h0, h1)
        mhz = statistics.median([s[1] for s in win]) if win else None
        rows.append((ms, mhz))
    t_all1 = time.time()
    plan.check_device()
    total_ms = sum(r[0] for r in rows)
    total_ms = max_over_ranks(total_ms, dist, dev)
    launches = chunk * nchunks
    job_ops = sum_over_ranks(ops_step * launches, dist, dev)
    tops = job_ops / (total_ms * 1e-3) / 1e12
    per_chunk = [(ops_step * chunk / (ms * 1e-3) / 1e12, mhz) for ms, mhz in rows]
    ratios = [t / m for t, m in per_chunk if m]
    bins = {}
    for t, m in per_chunk:
        if m:
            key = int(round(m / 50.0) * 50)
            bins.setdefault(key, []).append(t)
    peak, _ = int8_peak(load_peaks())
    clocks = clk.summary(t_all0, t_all1)
    return {
        "value": tops, "unit": "TOPS", "seconds": total_ms / 1e3, "launches": launches,
        "chunks": nchunks, "pct_of_int8_peak": 100.0 * tops / (peak * (dist.get_world_size()
                                                                       if dist else 1)),
        "sm_mhz_median": clocks.get("sm_mhz"),
        "tops_per_mhz": statistics.median(ratios) if ratios else None,
        "tops_by_sm_mhz": {str(k): statistics.median(v) for k, v in sorted(bins.items())},
        "realtime_channels_e2048": tops / E2048_RT_TOPS,
        "clocks": clocks,
        "note": "back-to-back chx_correlate launches of the headline workload; real-time "
                "channels = sustained TOPS / 6.557 TOPS per E=2048 channel",
    }


def measure_int8_peak(torch, dev, clk, seconds=2.0):
    """Dense int8 GEMM rate on this GPU in this process: torch._int_mm (cuBLAS)
    on 8192 x 8192 x 8192 int8 operands resident in HBM, timed with CUDA events
    over about `seconds`, with the median SM clock of the timed window.  A
    library GEMM used only as a reference figure for the roofline."""
    n = 8192
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device=dev, generator=g)
    b = torch.randint(-128, 128, (n, n), dtype=torch.int8, device=dev, generator=g)
    best = None
    for name, bb in (("B row-major", b), ("B column-major", b.t().contiguous().t())):
        try:
            for _ in range(3):
                torch._int_mm(a, bb)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(5):
                torch._int_mm(a, bb)
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / 5
            if best is None or ms < best[1]:
                best = (name, ms, bb)
        except Exception as e:  # noqa: BLE001
            err = str(e)
    if best is None:
        return {"tops": None, "error": err[:200]}
    name, ms, bb = best
    reps = max(10, int(seconds * 1000.0 / ms))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0 = time.time()
    e0.record()
    for _ in range(reps):
        torch._int_mm(a, bb)
    e1.record()
    torch.cuda.synchronize(dev)
    h1 = time.time()
    ms = e0.elapsed_time(e1) / reps
    tops = 2.0 * n ** 3 / (ms * 1e-3) / 1e12
    return {"tops": tops, "ms_per_gemm": ms, "reps": reps, "layout": name,
            "clocks": clk.summary(h0, h1),
            "what": "torch._int_mm (cuBLAS int8 GEMM, int32 out), 8192^3, operands in HBM"}


def run_e2e(args, torch, cx, plan, dev, ops_step, world, dist):
    """Same metric through the public API with host buffers: every step copies
    its pinned input H2D, correlates, and copies the whole block buffer D2H.
    Two stages are double-buffered on three streams (H2D / kernel / D2H), the
    transfer pipeline of main_wrapper.c:614-785."""
    nin = plan.input_bytes
    nout = plan.block_words
    host_in = [torch.randint(0, 256, (nin,), dtype=torch.uint8).pin_memory() for _ in range(2)]
    host_out = [torch.empty(nout, dtype=torch.int32).pin_memory() for _ in range(2)]
    d_in = [torch.empty(nin, dtype=torch.uint8, device=dev) for _ in range(2)]
    d_out = [torch.empty(nout, dtype=torch.int32, device=dev) for _ in range(2)]
    h2d = torch.cuda.Stream(dev)
    comp = torch.cuda.Stream(dev)
    d2h = torch.cuda.Stream(dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_comp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def run(nsteps):
        for k in range(nsteps):
            s = k % 2
            if k >= 2:
                h2d.wait_event(ev_comp[s])      # d_in[s] no longer read
            with torch.cuda.stream(h2d):
                d_in[s].copy_(host_in[s], non_blocking=True)
            ev_in[s].record(h2d)
            comp.wait_event(ev_in[s])
            if k >= 2:
                comp.wait_event(ev_out[s])      # d_out[s] already copied out
            plan.correlate(d_in[s], d_out[s], stream=comp)
            ev_comp[s].record(comp)
            d2h.wait_event(ev_comp[s])
            with torch.cuda.stream(d2h):
                host_out[s].copy_(d_out[s], non_blocking=True)
            ev_out[s].record(d2h)

    run(max(args.warmup, 3))
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    # as many steps as the headline leg: the pipeline's fill (the first input's
    # H2D copy) and drain (the last D2H copy) are paid once per timed region
    steps = max(4, args.steps)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(h2d)
    comp.wait_event(t0)
    d2h.wait_event(t0)
    run(steps)
    d2h.wait_stream(comp)
    d2h.wait_stream(h2d)
    t1.record(d2h)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(t0.elapsed_time(t1), dist, dev)
    job_ops = sum_over_ranks(ops_step * steps, dist, dev)
    return {"value": job_ops / (ms * 1e-3) / 1e12, "unit": "TOPS",
            "h2d_bytes_per_step": nin, "d2h_bytes_per_step": nout * 4,
            "ms_per_step": ms / steps, "steps": steps,
            "pipeline": "2-stage pinned double buffer; H2D, kernel, D2H on three streams"}


def cpu_baselines(args):
    """The reference's CPU correlator on the host cores: all cores on a
    bounded sample of the full-size plain workload (the line's cpu_baseline),
    plus one core on the small plain case (E=256, T=256) in full and on a
    sample of the full-size workload, with the CPU model."""
    if args.no_cpu:
        return None
    r = cpu_reference_rate(2048, 3072)
    if r is None:
        return None
    out = {"value": r[0] / 1e12, "unit": "TOPS", "cores": r[1], "kind": r[3],
           "sample": r[2], "seconds": round(r[4], 2), "cpu_model": cpu_model()}
    single = cpu_single_core()
    if single is not None:
        out["single_core"] = single
    return out


def relaunch_under_torchrun(args):
    """`--gpus N` (N > 1) started as a plain process: run N ranks of this
    script under torch.distributed.run, one per GPU, and return its status."""
    port = os.environ.get("MASTER_PORT", "29571")
    argv = [a for a in sys.argv[1:]]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(args.gpus), "--master-addr", "127.0.0.1",
           "--master-port", port, os.path.abspath(__file__)] + argv
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--E", type=int, default=2048, help="elements (profiling cases)")
    ap.add_argument("--F", type=int, default=8, help="channels per GPU (profiling cases)")
    ap.add_argument("--T", type=int, default=16384, help="samples (profiling cases)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="all",
                    choices=["all", "plain", "batched", "stream", "helpers"])
    ap.add_argument("--algo", default="auto", choices=["auto", "simt", "tc"])
    ap.add_argument("--tsplit", type=int, default=0)
    ap.add_argument("--tile", type=int, default=0, help="tensor-core tile: 0 auto, 1 one SM, 2 SM pair")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--sustain-s", type=float, default=5.0,
                    help="seconds of back-to-back launches for the sustained figure (0: skip)")
    ap.add_argument("--no-peak", action="store_true",
                    help="skip the in-run int8 GEMM reference (profiling runs)")
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="reference arm: samples per process per step (0: sized so the "
                         "timed steps take ~2.5 min)")
    ap.add_argument("--no-tune", action="store_true",
                    help="batched: skip the autotuner (default tiles; profiling cases)")
    ap.add_argument("--no-plain", action="store_true",
                    help="batched: skip the plain per-channel comparison and e2e (profiling cases)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_under_torchrun(args)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import chimex as cx
    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=dev)
        dist = tdist
    import bench_workloads as W
    try:
        with ClockSampler(dev) as clk:
            if args.config in ("all", "plain"):
                line, plan, packed, blocks, ops_step = run_plain(args, torch, cx, dist, clk)
                if not args.no_e2e:
                    line["e2e"] = run_e2e(args, torch, cx, plan, dev, ops_step, world, dist)
                if args.sustain_s > 0:
                    sus = run_sustained(args, torch, plan, packed, blocks, ops_step, dist, dev,
                                        clk, args.sustain_s)
                    line["sustained"] = sus
                    line["realtime_channels_e2048"] = sus["realtime_channels_e2048"]
                del packed, blocks
                plan.close()
                torch.cuda.empty_cache()
                pk = {"skipped": True} if args.no_peak else measure_int8_peak(torch, dev, clk)
                if pk.get("tops"):
                    pk["kernel_frac_of_this"] = line["roofline"]["achieved"] / pk["tops"]
                    if "sustained" in line:
                        pk["sustained_frac_of_this"] = line["sustained"]["value"] / world / pk["tops"]
                line["int8_peak_in_run"] = pk
                torch.cuda.empty_cache()
                if args.config == "all":
                    line["batched"] = W.run_batched(args, torch, cx, dist, clk)
                    torch.cuda.empty_cache()
                    line["stream"] = W.run_stream(args, torch, cx, dist, clk)
                    torch.cuda.empty_cache()
                if rank == 0 and world == 1:
                    cpu = cpu_baselines(args)
                    if cpu is not None:
                        line["cpu_baseline"] = cpu
                if rank == 0:
                    print(json.dumps(line))
            elif args.config == "batched":
                out = W.run_batched(args, torch, cx, dist, clk)
                if rank == 0:
                    print(json.dumps(out))
            elif args.config == "stream":
                out = W.run_stream(args, torch, cx, dist, clk)
                if rank == 0:
                    print(json.dumps(out))
            else:
                W.run_helpers(args, torch, cx, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
