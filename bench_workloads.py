"""Batched and streaming legs of bench.py (sub-objects of the default line,
or one line each with --config batched|stream).

batched: 64 channels with element counts drawn from
{256, 512, 1024, 1536, 2048} and time_accum uniform in [64, 1912] (seed 42),
4 integrations each, all in one persistent launch replayed from a CUDA graph
(chx_batch_run), against the plain per-channel path: one chx_correlate
launch per channel and integration.

stream: 1024 channels (70% E=2048, 30% E=1024, seed 42),
frames of 256 samples, time_accum 1024, admitted by free HBM.  Channels start
a quarter integration apart so that a quarter of them complete per frame
tick.  Phases: flat out (ticks back to back: sustained real-time channels);
the plain per-channel path for one tick's completions (one chx_correlate per
completing integration); paced at the CHIME frame rate (256 samples per
655.36 us) for the number of channels the GPU sustains with 20% headroom,
frames already in the rings (p50/p99 latency from the last frame of an
integration to its completed dump); and the same paced loop end to end,
every frame crossing PCIe from pinned host memory, for the channels 70% of
the measured H2D bandwidth carries.

Under torchrun each rank takes its share of the channel list
(bench.shard_channels, costliest first to the least-loaded rank): the work
is summed over ranks and the time is the slowest rank's.
"""
import gc
import json
import time

import bench as B

CONFIG4_TEXT = ("Batched ragged launch: 64 frequency channels in one persistent CUDA-graph "
                "launch. Element counts are drawn from {256, 512, 1024, 1536, 2048} and "
                "per-channel time_accum from uniform integers in [64,1912]. T is 4 integrations "
                "per channel, and values are seeded uniform [-8,7] 4-bit complex. The autotuner "
                "picks tile shape and split-T, and the run is compared against 64 plain launches.")
CONFIG5_TEXT = ("Streaming serving loop: 1024 channels. Frames of 256 time samples per channel "
                "arrive at 390625 samples/s per channel; 70% of channels have E=2048 and 30% have "
                "E=1024. time_accum is 1024, accumulators stay device-resident, and admission is "
                "by free HBM. Inputs are seeded uniform [-8,7] 4-bit complex. Reports real-time "
                "channels sustained and p50/p99 frame-to-visibility latency.")


def _peak():
    return B.int8_peak(B.load_peaks())


def config4_channels():
    """(E, time_accum) of the ragged batch's 64 channels (seed 42)."""
    import numpy as np
    rng = np.random.default_rng(42)
    Es = [int(e) for e in rng.choice([256, 512, 1024, 1536, 2048], size=64)]
    TAs = [int(t) for t in rng.integers(64, 1913, size=64)]
    return Es, TAs


def config5_channels():
    """Element counts of the streaming workload's 1024 channels: 717 with E=2048,
    307 with E=1024, order shuffled with seed 42."""
    import numpy as np
    Es = [2048] * 717 + [1024] * 307
    np.random.default_rng(42).shuffle(Es)
    return [int(e) for e in Es]


def run_batched(args, torch, cx, dist, clk):
    rank, local_rank, world = B.env_rank()
    dev = torch.device("cuda", local_rank)
    nint = 4
    Es_all, TAs_all = config4_channels()
    mine = B.shard_channels([B.vis_ops(E, nint * T, 1) for E, T in zip(Es_all, TAs_all)],
                            world, rank)
    Es = [Es_all[i] for i in mine]
    TAs = [TAs_all[i] for i in mine]
    nchan = len(Es)
    in_off, out_off = [0], [0]
    for E, T in zip(Es, TAs):
        in_off.append(in_off[-1] + nint * T * E)
        out_off.append(out_off[-1] + nint * cx.num_blocks(E) * 2048)
    gen = torch.Generator(device=dev)
    gen.manual_seed(42 + rank)
    packed = torch.randint(0, 256, (max(1, in_off[-1]),), dtype=torch.uint8, device=dev,
                           generator=gen)
    blocks = torch.empty(max(1, out_off[-1]), dtype=torch.int32, device=dev)
    chans = [(packed[in_off[c]:in_off[c + 1]], blocks[out_off[c]:out_off[c + 1]], Es[c], TAs[c],
              nint) for c in range(nchan)]
    stream = torch.cuda.current_stream(dev)

    # autotune every distinct (E, time_accum) shape class: the tuner caches
    # per (E, T) and batches look up the nearest T within a factor 2
    tuned = {}
    t_tune = time.time()
    if not args.no_tune and nchan:
        scratch_in = torch.randint(0, 256, (2048 * 2048,), dtype=torch.uint8, device=dev)
        scratch_out = torch.empty(cx.num_blocks(2048) * 2048, dtype=torch.int32, device=dev)
        for E in sorted(set(Es)):
            for T in (128, 512, 1536):
                tuned["%d/%d" % (E, T)] = cx.autotune(E, T, scratch_in, scratch_out, stream)[:2]
        del scratch_in, scratch_out
    t_tune = time.time() - t_tune
    batch = cx.Batch(chans, 1, local_rank) if nchan else None
    ops = batch.ops if batch else 0.0

    plans = {}
    for E, T in zip(Es, TAs):
        if (E, T) not in plans:
            plans[(E, T)] = cx.Plan(E, 1, T, T, 1, 0, local_rank)
    nbw = [cx.num_blocks(E) * 2048 for E in Es]

    def plain_step():
        for c in range(nchan):
            p = plans[(Es[c], TAs[c])]
            x, y = chans[c][0], chans[c][1]
            span, ow = TAs[c] * Es[c], nbw[c]
            for i in range(nint):
                p.correlate(x[i * span:(i + 1) * span], y[i * ow:(i + 1) * ow], stream=stream)

    def batch_step():
        if batch:
            batch.run(stream=stream)

    def timed(step, steps, mark=False):
        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        h0 = time.time()
        a.record(stream)
        for _ in range(steps):
            step()
        b.record(stream)
        torch.cuda.synchronize(dev)
        h1 = time.time()
        ms = a.elapsed_time(b)
        return B.max_over_ranks(ms, dist, dev) / steps, (h0, h1)

    steps = args.steps
    ms_batch, win = timed(batch_step, steps)
    clocks = clk.summary(*win)
    if batch:
        batch.check_device(stream)
    job_ops = B.sum_over_ranks(ops, dist, dev)
    value = job_ops / (ms_batch * 1e-3) / 1e12
    peak, peak_src = _peak()
    out = {
        "metric": "exact INT8-TC TOPS (batched ragged, 64 channels)", "value": value,
        "unit": "TOPS", "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms_batch, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "n/a (one GPU)",
        "pct_of_int8_peak": 100.0 * value / world / peak,
        "config": {"workload": CONFIG4_TEXT, "channels_this_rank": nchan,
                   "work_units": batch.work_units if batch else 0, "autotuned": tuned,
                   "autotune_s": round(t_tune, 2),
                   "l2": "inputs %d MiB + dumps %d MiB per step, larger than L2; no flush" % (
                       in_off[-1] >> 20, (out_off[-1] * 4) >> 20)},
        "clocks": clocks,
        "gpu_launches": steps,
    }
    if B.clocks_rejected(clocks):
        out["clocks_rejected"] = True
    if args.no_plain:
        out["note"] = "profiling case: no plain comparison, no e2e"
        if batch:
            batch.close()
        return out
    ms_plain, _ = timed(plain_step, max(5, steps // 4))
    # the batch and the plain path write the same buffers: check they agree
    ref = blocks.clone()
    batch_step()
    torch.cuda.synchronize(dev)
    identical = bool(torch.equal(ref, blocks))
    del ref

    # end to end: pinned host input H2D, the graph, all dumps D2H, one stream
    h_in = torch.randint(0, 256, (max(1, in_off[-1]),), dtype=torch.uint8).pin_memory()
    h_out = torch.empty(max(1, out_off[-1]), dtype=torch.int32).pin_memory()

    def e2e_step():
        packed.copy_(h_in, non_blocking=True)
        batch_step()
        h_out.copy_(blocks, non_blocking=True)

    e2e_steps = max(4, steps // 4)
    ms_e2e, _ = timed(e2e_step, e2e_steps)
    if batch:
        batch.check_device(stream)
        batch.close()
    out.update({
        "plain_ms_per_step": ms_plain,
        "plain_value": job_ops / (ms_plain * 1e-3) / 1e12,
        "plain_launches_per_step": nchan * nint,
        "speedup_vs_plain": ms_plain / ms_batch,
        "batch_equals_plain": identical,
        "roofline": {"bound": "tensor", "achieved": ops / (ms_batch * 1e-3) / 1e12, "peak": peak,
                     "unit": "TOPS", "frac": ops / (ms_batch * 1e-3) / 1e12 / peak,
                     "traffic": B.profile_traffic("tc_pair_correlate_batched64.md"),
                     "peak_source": peak_src, "kernel": "tc_pair_kernel (batched)"},
        "e2e": {"value": job_ops / (ms_e2e * 1e-3) / 1e12, "unit": "TOPS",
                "h2d_bytes_per_step": in_off[-1], "d2h_bytes_per_step": out_off[-1] * 4,
                "ms_per_step": ms_e2e, "steps": e2e_steps,
                "pipeline": "one stream: H2D of all inputs, graph launch, D2H of all dumps"},
    })
    for p in plans.values():
        p.close()
    return out


def run_stream(args, torch, cx, dist, clk):
    import ctypes

    rank, local_rank, world = B.env_rank()
    dev = torch.device("cuda", local_rank)
    frame, ta = 256, 1024
    per = ta // frame
    Es_all = config5_channels()
    mine = B.shard_channels([B.vis_ops(E, 1, 1) for E in Es_all], world, rank)
    Es_mine = [Es_all[i] for i in mine]
    stream = torch.cuda.current_stream(dev)

    # plain per-channel path for one tick's completions: one chx_correlate
    # launch per completing integration (a quarter of the channels, each on
    # its own input and dump buffer)
    tick_sel = Es_mine[::per]
    plans = {E: cx.Plan(E, 1, ta, ta, 1, 0, local_rank) for E in set(tick_sel)}
    g0 = torch.Generator(device=dev)
    g0.manual_seed(4242 + rank)
    pl_in = [torch.randint(0, 256, (ta * E,), dtype=torch.uint8, device=dev, generator=g0)
             for E in tick_sel]
    pl_out = [torch.empty(cx.num_blocks(E) * 2048, dtype=torch.int32, device=dev)
              for E in tick_sel]

    def plain_tick():
        for E, x, y in zip(tick_sel, pl_in, pl_out):
            plans[E].correlate(x, y, stream=stream)

    for _ in range(max(args.warmup, 3)):
        plain_tick()
    torch.cuda.synchronize(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    reps = 8
    a.record(stream)
    for _ in range(reps):
        plain_tick()
    b.record(stream)
    torch.cuda.synchronize(dev)
    plain_ms_tick = B.max_over_ranks(a.elapsed_time(b) / reps, dist, dev)
    for p in plans.values():
        p.check_device()
        p.close()
    del pl_in, pl_out
    torch.cuda.empty_cache()

    s = cx.Stream(max(1, len(Es_mine)), frame, 1, 0, local_rank)
    ids, refused = [], 0
    for E in Es_mine:
        try:
            ids.append(s.admit(int(E), ta))
        except cx.ChimexError as e:
            if e.code != cx.E_ADMISSION:
                raise
            refused += 1
    n = len(ids)
    Es = [int(E) for E in Es_mine[:n]]
    # each ring (two integrations) gets seeded random samples once; frames are
    # then submitted in place (the producer wrote them into the ring)
    g = torch.Generator(device=dev)
    g.manual_seed(42 + rank)
    for c, E in zip(ids, Es):
        view = cx.device_view(s.frame_slot(c), 2 * ta * E, "uint8", local_rank)
        view.copy_(torch.randint(0, 256, (2 * ta * E,), dtype=torch.uint8, device=dev,
                                 generator=g))
    torch.cuda.synchronize(dev)
    # stagger: channel c starts (c mod per) frames into its first integration
    for k in range(1, per):
        sub = [c for c in ids if c % per >= per - k]
        if sub:
            s.submit(sub, None, None, stream)
    ops_frame = [B.vis_ops(E, frame, 1) for E in Es]
    all_ids = (ctypes.c_int * n)(*ids)

    # phase 1: flat out
    warm = max(args.warmup, 3) * per
    for _ in range(warm):
        s.submit(all_ids, None, None, stream)
    torch.cuda.synchronize(dev)
    ticks = max(8 * per, (args.steps // per) * per)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    s.sync()
    dumps0 = s.stats()["dumps"]
    if dist is not None:
        dist.barrier()
    h0 = time.time()
    a.record(stream)
    t0 = time.perf_counter()
    for _ in range(ticks):
        s.submit(all_ids, None, None, stream)
    host_s = time.perf_counter() - t0
    b.record(stream)
    torch.cuda.synchronize(dev)
    h1 = time.time()
    clocks = clk.summary(h0, h1)
    ms_local = a.elapsed_time(b)
    s.check_device()
    ms = B.max_over_ranks(ms_local, dist, dev)
    dumps_flat = s.stats()["dumps"] - dumps0
    sps = ticks * frame / (ms * 1e-3)        # samples/s per channel sustained
    rt_channels = B.sum_over_ranks(n * sps / B.REALTIME_SPS, dist, dev)
    ops_s = B.sum_over_ranks(sum(ops_frame) * ticks, dist, dev) / (ms * 1e-3)
    tops = ops_s / 1e12

    period_ns = int(round(frame / B.REALTIME_SPS * 1e9))

    def paced(sel, nticks, before_submit=None, after_submit=None):
        """Submits one frame per channel in `sel` every frame period (arrival
        = the tick's due time); returns (stats, late ticks)."""
        sel_ids = (ctypes.c_int * len(sel))(*sel)
        arr = (ctypes.c_int64 * len(sel))()
        torch.cuda.synchronize(dev)
        s.sync()
        s.reset_stats()
        late = 0
        # the frame schedule is kept by this Python loop: no garbage
        # collection pauses inside it
        gc.collect()
        gc.disable()
        try:
            t0 = time.monotonic_ns() + 2 * period_ns
            for k in range(nticks):
                due = t0 + k * period_ns
                while True:
                    now = time.monotonic_ns()
                    if now >= due:
                        break
                    if due - now > 200000:
                        time.sleep((due - now - 150000) * 1e-9)
                if now - due > period_ns:
                    late += 1
                for i in range(len(sel)):
                    arr[i] = due
                frames = before_submit(k) if before_submit else None
                s.submit(sel_ids, frames, arr, stream)
                if after_submit:
                    after_submit(k)
        finally:
            gc.enable()
        torch.cuda.synchronize(dev)
        s.check_device()
        return s.stats(), late

    # phase 2: paced at the real frame rate for 80% of the sustained channels,
    # frames already in the rings (device-side ingest)
    n_rt = max(per, min(n, int(0.8 * n * sps / B.REALTIME_SPS)))
    paced_ticks = max(4 * per, int(2.0e9 / period_ns))  # about two seconds
    st, late = paced(ids[:n_rt], paced_ticks)

    # phase 3 (end to end): frames arrive in pinned host memory and cross PCIe
    # every tick (one H2D copy per tick on a copy stream, double-buffered
    # staging, one gather launch into the rings inside chx_stream_submit) for
    # as many channels as 70% of the measured H2D bandwidth carries.
    probe = torch.empty(256 << 20, dtype=torch.uint8).pin_memory()
    dprobe = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dprobe.copy_(probe, non_blocking=True)
    e0.record(stream)
    for _ in range(4):
        dprobe.copy_(probe, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    h2d_gbs = 4 * (256 << 20) / (e0.elapsed_time(e1) * 1e-3) / 1e9
    del probe, dprobe
    budget = 0.7 * h2d_gbs * 1e9 * period_ns * 1e-9
    sel, tick_bytes = [], 0
    for c, E in zip(ids, Es):
        if len(sel) >= n_rt or tick_bytes + frame * E > budget:
            break
        sel.append(c)
        tick_bytes += frame * E
    offs, o = [], 0
    for c in sel:
        offs.append(o)
        o += frame * Es[c]
    nbuf = 8  # distinct host frames per channel, reused round robin
    host = torch.randint(0, 256, (nbuf, tick_bytes), dtype=torch.uint8,
                         generator=torch.Generator().manual_seed(43 + rank)).pin_memory()
    staging = [torch.empty(tick_bytes, dtype=torch.uint8, device=dev) for _ in range(2)]
    fptr = [[st_.data_ptr() + off for off in offs] for st_ in staging]
    copy_stream = torch.cuda.Stream(dev)
    ev_copied = [torch.cuda.Event() for _ in range(2)]
    ev_used = [torch.cuda.Event() for _ in range(2)]

    def before(k):
        b = k % 2
        if k >= 2:
            copy_stream.wait_event(ev_used[b])
        with torch.cuda.stream(copy_stream):
            staging[b].copy_(host[k % nbuf], non_blocking=True)
        ev_copied[b].record(copy_stream)
        stream.wait_event(ev_copied[b])
        return fptr[b]

    def after_submit(k):
        ev_used[k % 2].record(stream)

    st_e2e, late_e2e = paced(sel, paced_ticks, before, after_submit)
    # whole job: the channels of every rank, valid when every rank kept the
    # frame schedule (<= 0.5% of ticks late)
    e2e_late_any = B.max_over_ranks(1.0 if late_e2e * 200 > paced_ticks else 0.0, dist, dev)
    e2e_channels = int(round(B.sum_over_ranks(len(sel), dist, dev)))

    peak, peak_src = _peak()
    stream_ms_tick = ms / ticks
    out = {
        "metric": "real-time channels sustained (stream, 1024 channels)",
        "value": rt_channels, "unit": "channels", "n_gpus": world, "steps": ticks, "warmup": warm,
        "ms_per_step": stream_ms_tick, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "n/a (one GPU)",
        "config": {"workload": CONFIG5_TEXT, "admitted": n, "refused": refused,
                   "frame_len": frame, "time_accum": ta,
                   "resident_gb": st["resident_bytes"] / 1e9,
                   "l2": "rings %d MiB resident, larger than L2; no flush" % (
                       sum(2 * ta * E for E in Es) >> 20)},
        "samples_per_s_per_channel": sps,
        "realtime_channels_e2048": ops_s / (B.E2048_RT_TOPS * 1e12),
        "tops": tops, "pct_of_int8_peak": 100.0 * tops / world / peak,
        "plain_ms_per_tick": plain_ms_tick,
        "speedup_vs_plain": plain_ms_tick / stream_ms_tick,
        "plain_note": "one chx_correlate launch per integration completing in a tick "
                      "(%d of this rank's channels), each on its own input and dump" % len(tick_sel),
        "host_submit_ms_per_tick": 1e3 * host_s / ticks,
        "paced": {"channels": n_rt * world, "ticks": paced_ticks, "period_us": period_ns / 1e3,
                  "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
                  "dumps": st["dumps"], "late_ticks": late,
                  "ingest": "frames already in the device rings"},
        "e2e": {"value": e2e_channels if e2e_late_any == 0 else None, "unit": "channels",
                "h2d_bytes_per_step": tick_bytes, "d2h_bytes_per_step": 0,
                "channels": len(sel), "p50_ms": st_e2e["p50_ms"], "p99_ms": st_e2e["p99_ms"],
                "max_ms": st_e2e["max_ms"], "late_ticks": late_e2e, "ticks": paced_ticks,
                "h2d_gbs_measured": h2d_gbs,
                "pipeline": "paced at 256 samples per 655.36 us; every tick one pinned H2D "
                            "copy of all frames (copy stream, double-buffered staging) and "
                            "chx_stream_submit gathering them into the rings; channels "
                            "limited to 70% of the measured H2D bandwidth; the dumps stay "
                            "in HBM (an E=2048 dump is 17 MB)"},
        "roofline": {"bound": "tensor", "achieved": tops / world, "peak": peak, "unit": "TOPS",
                     "frac": tops / world / peak, "traffic": None, "peak_source": peak_src,
                     "kernel": "tc_pair_kernel (stream launches)"},
        "gpu_launches": ticks,
        "dump_launch_integrations": dumps_flat,
        "clocks": clocks,
    }
    if B.clocks_rejected(clocks):
        out["clocks_rejected"] = True
    s.close()
    return out


def run_helpers(args, torch, cx, dist):
    """The HBM-bound kernels of the path on the plain workload (E=2048, F=8,
    T=16384): offset sums, preseed, block -> triangle and block -> full-matrix
    reorganisation, each timed with CUDA events over its algorithmic bytes
    (bytes the kernel must read plus bytes it must write) against the measured
    HBM copy bandwidth."""
    rank, local_rank, world = B.env_rank()
    dev = torch.device("cuda", local_rank)
    E, F, T = args.E, args.F, args.T
    p = cx.Plan(E, F, T, 256, 1, 0, local_rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(42 + rank)
    packed = torch.randint(0, 256, (p.input_bytes,), dtype=torch.uint8, device=dev, generator=gen)
    blocks = p.correlate(packed)
    sums = torch.empty(p.sum_words, dtype=torch.int32, device=dev)
    tri = torch.empty(p.triangle_words, dtype=torch.int32, device=dev)
    full = torch.empty(F * E * E * 2, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    nb_bytes = p.block_words * 4
    cases = {
        "offset_accumulate": (lambda: p.offset_accumulate(packed, sums, stream=stream),
                              p.input_bytes + p.sum_words * 4),
        "preseed": (lambda: p.preseed(sums, blocks, stream=stream), nb_bytes + p.sum_words * 4),
        "blocks_to_triangle": (lambda: p.blocks_to_triangle(blocks, tri, stream=stream),
                               nb_bytes + p.triangle_words * 4),
        "blocks_to_full": (lambda: p.blocks_to_full(blocks, full, stream=stream),
                           nb_bytes + full.numel() * 4),
    }
    peaks = B.load_peaks() or {}
    hbm = float(peaks.get("hbm_gbs") or 6650.0)
    out = {}
    reps = max(10, min(args.steps, 100))
    for name, (fn, nbytes) in cases.items():
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize(dev)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms = B.max_over_ranks(a.elapsed_time(b) / reps, dist, dev)
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "bytes": nbytes, "gbs": gbs, "frac_of_hbm": gbs / hbm}
    p.check_device()
    if rank == 0:
        print(json.dumps({"metric": "HBM GB/s of the helper kernels", "unit": "GB/s",
                          "config": {"E": E, "F": F, "T": T}, "reps": reps,
                          "hbm_peak_gbs": hbm,
                          "peak_source": "measured copy bandwidth (MEASURED_PEAKS.json)"
                          if peaks.get("hbm_gbs") else "fallback 6650 GB/s",
                          "kernels": out}))
