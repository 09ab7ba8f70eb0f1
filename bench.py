"""Benchmark of the CHIME X-engine hot path on B200.

Default workload (N=1): the plain correlator at full CHIME size, E=2048
elements, F=8 channels, T=16384 samples (64 integrations of time_accum=256),
one fused chx_correlate launch per step over inputs already resident in HBM.
Metric: exact INT8 tensor-core TOPS = 8 * E(E+1)/2 * T * F / seconds (4 int8
MACs per upper-triangle complex visibility per sample; diagonal-tile waste
not credited).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--config plain|batched|stream|helpers] [--algo auto|simt|tc]

Under torchrun each rank correlates its own F channels (weak scaling, no
data-path collective); the time is the max over ranks.  `--impl reference`
times the reference's own CPU correlator (cpu_corr_test.c, built from the
reference sources into oracle/_ref) on the host cores instead.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
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


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def summary(self):
        if self.proc is None or self.tmp is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.tmp.name)
        import datetime
        t0, t1 = getattr(self, "t0", None), getattr(self, "t1", None)
        if t0 is not None and t1 is not None:
            keep = []
            for r in rows:
                try:
                    ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    continue
                if t0 - 0.05 <= ts <= t1 + 0.05:
                    keep.append(r)
            rows = keep
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, n in enumerate(names):
            if any(r[5 + k].lower().startswith("active") for r in rows):
                reasons.append(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max((num(r[3]) or 0.0) for r in rows),
                "samples": len(rows), "reasons": reasons}


# ------------------------------------------------------------ cpu baseline
def cpu_reference_rate(E, T_sample, seconds_target=12.0, max_procs=None):
    """Times the reference's own CPU correlator (oracle/_ref/cpu_corr_ref,
    built from cpu_corr_test.c) on the host cores: one process per core, each
    correlating one E-element channel over T_sample samples.  Returns
    (ops_per_s, cores, sample description, kind)."""
    driver = os.path.join(ROOT, "oracle", "_ref", "cpu_corr_ref")
    kind = "reference"
    if not os.path.exists(driver):
        return None
    cores = max_procs or os.cpu_count() or 1
    t0 = time.time()
    procs = [subprocess.Popen([driver, str(T_sample), "1", str(E), "4", str(42 + i), "1", "1"],
                              stdout=subprocess.PIPE, text=True) for i in range(cores)]
    outs = [p.communicate()[0] for p in procs]
    wall = time.time() - t0
    total_ops = 0.0
    for o in outs:
        rec = json.loads(o.strip().splitlines()[-1])
        total_ops += OPS_PER_VIS_SAMPLE * rec["updates"]
    sample = ("%d concurrent processes x (E=%d, F=1, T=%d, seeded random) of the "
              "reference cpu_data_generate_and_correlate_upper_triangle_only" % (cores, E, T_sample))
    return total_ops / wall, cores, sample, kind, wall


def run_reference_arm(args):
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    E, F, T = 2048, 8, 16384
    driver = os.path.join(ROOT, "oracle", "_ref", "cpu_corr_ref")
    if not os.path.exists(driver):
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
                         "sample": "%d processes x (E=%d, T=%d) per step" % (cores, E, t_sample)},
        "e2e": {"value": value, "unit": "TOPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "realtime_channels_e2048": ops_s / (E2048_RT_TOPS * 1e12),
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------- our arm
def run_plain(args, torch, cx, dist):
    rank, local_rank, world = env_rank()
    E, F, T, TA = args.E, args.F, args.T, 256
    dev = torch.device("cuda", local_rank)
    plan = cx.Plan(E, F, T, TA, 1, 0, local_rank)
    if args.algo == "simt":
        plan.set_option(cx.OPT_ALGO, cx.ALGO_SIMT)
    elif args.algo == "tc":
        plan.set_option(cx.OPT_ALGO, cx.ALGO_TC)
    if args.tsplit:
        plan.set_option(cx.OPT_TSPLIT, args.tsplit)
    if args.tile:
        plan.set_option(cx.OPT_TILE, args.tile)
    gen = torch.Generator(device=dev)
    gen.manual_seed(42 + rank)
    packed = torch.randint(0, 256, (plan.input_bytes,), dtype=torch.uint8, device=dev,
                           generator=gen)
    blocks = torch.empty(plan.block_words, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ops_step = vis_ops(E, T, F)

    def step():
        plan.correlate(packed, blocks, stream=stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local_rank) as clk:
        for _ in range(max(args.warmup, 3)):
            step()
        plan.check_device()
        torch.cuda.synchronize(dev)
        # device-timed region: inputs larger than L2 (see config["l2"])
        barrier()
        torch.cuda.synchronize(dev)
        clk.mark_start()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize(dev)
        clk.mark_end()
    barrier()
    plan.check_device()
    total_ms = t_start.elapsed_time(t_end)
    per_launch = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(total_ms, dist, dev)
    value = ops_step * world * args.steps / (total_ms * 1e-3) / 1e12
    clocks = clk.summary()

    # end to end through the public API with host buffers: pinned input
    # copied H2D and the block buffer copied D2H every step, two stages
    # double-buffered on two streams (main_wrapper.c:614-785 style).
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, torch, cx, plan, dev, ops_step, world, dist)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        r = cpu_reference_rate(E, 3072)
        if r is not None:
            cpu = {"value": r[0] / 1e12, "unit": "TOPS", "cores": r[1], "kind": r[3],
                   "sample": r[2], "seconds": round(r[4], 2)}

    peak, peak_src = int8_peak(load_peaks())
    traffic = None
    if (E, F, T) == (2048, 8, 16384) and args.algo != "simt" and args.tile in (0, 2):
        traffic = profile_traffic("tc_pair_correlate_E2048_F8_T16384.md")
    kernel_ms = sorted(per_launch)[len(per_launch) // 2]
    achieved = ops_step / (sum(per_launch) / len(per_launch) * 1e-3) / 1e12
    line = {
        "metric": "exact INT8-TC TOPS", "value": value, "unit": "TOPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: seeded uniform 4-bit complex (re, im uniform in [-8, 7]), "
                "device-generated",
        "config": {"workload": "plain correlator E=%d F=%d T=%d time_accum=256 per GPU, "
                               "one chx_correlate launch per step" % (E, F, T),
                   "E": E, "F": F, "T": T, "time_accum": TA, "algo": args.algo, "tile": args.tile,
                   "l2": "inputs (%d MiB) %s L2 (126 MB); no flush" % (
                       E * F * T >> 20, "larger than" if E * F * T > 126e6 else "SMALLER than"),
                   "parallelism": "channel shards, %d GPU(s), no collective" % world},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOPS",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                     "kernel": "correlator", "median_launch_ms": kernel_ms,
                     "nominal_peak": NOMINAL_INT8_TOPS},
        "pct_of_int8_peak": 100.0 * value / world / peak,
        "realtime_channels_e2048": value * 1e12 / (E2048_RT_TOPS * 1e12),
        "gpu_launches": args.steps * launches_per_step(cx, plan),
        "clocks": clocks,
    }
    if e2e is not None:
        line["e2e"] = e2e
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line))


def launches_per_step(cx, plan):
    return 1


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
    steps = max(4, args.steps // 2)
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
    ms = t0.elapsed_time(t1)
    ms = max_over_ranks(ms, dist, dev)
    return {"value": ops_step * world * steps / (ms * 1e-3) / 1e12, "unit": "TOPS",
            "h2d_bytes_per_step": nin, "d2h_bytes_per_step": nout * 4,
            "ms_per_step": ms / steps, "steps": steps,
            "pipeline": "2-stage pinned double buffer; H2D, kernel, D2H on three streams"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--E", type=int, default=2048, help="elements (profiling cases)")
    ap.add_argument("--F", type=int, default=8, help="channels per GPU (profiling cases)")
    ap.add_argument("--T", type=int, default=16384, help="samples (profiling cases)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="plain", choices=["plain", "batched", "stream", "helpers"])
    ap.add_argument("--algo", default="auto", choices=["auto", "simt", "tc"])
    ap.add_argument("--tsplit", type=int, default=0)
    ap.add_argument("--tile", type=int, default=0, help="tensor-core tile: 0 auto, 1 one SM, 2 SM pair")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
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
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import chimex as cx
    rank, local_rank, world = env_rank()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local_rank))
        dist = tdist
    try:
        if args.config == "plain":
            run_plain(args, torch, cx, dist)
        elif args.config == "batched":
            import bench_workloads
            bench_workloads.run_batched(args, torch, cx, dist)
        elif args.config == "helpers":
            import bench_workloads
            bench_workloads.run_helpers(args, torch, cx, dist)
        else:
            import bench_workloads
            bench_workloads.run_stream(args, torch, cx, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
