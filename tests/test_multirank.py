"""Multi-process logic of bench.py on CPU (gloo, world size 2): channels are
independent, so ranks share nothing on the data path; the only cross-rank
steps are the barrier around the timed region, the max-over-ranks of the
device times and the sum of per-rank counts, and only rank 0 prints.  The
batched and streamed channel lists are split between the ranks by
bench.shard_channels, which every rank computes on its own."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

torch = pytest.importorskip("torch")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r, lr, w = bench.env_rank()
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        dist.barrier()
        job_ms = bench.max_over_ranks(local_ms, dist, "cpu")
        job_channels = bench.sum_over_ranks(100 + rank, dist, "cpu")  # per-rank counts add up
        # the ragged-batch and streaming channel lists, each rank taking its share
        import bench_workloads as W
        Es, TAs = W.config4_channels()
        costs4 = [bench.vis_ops(E, 4 * T, 1) for E, T in zip(Es, TAs)]
        mine4 = bench.shard_channels(costs4, w, r)
        ops4 = bench.sum_over_ranks(sum(costs4[i] for i in mine4), dist, "cpu")
        E5 = W.config5_channels()
        costs5 = [bench.vis_ops(E, 1, 1) for E in E5]
        mine5 = bench.shard_channels(costs5, w, r)
        ops5 = bench.sum_over_ranks(sum(costs5[i] for i in mine5), dist, "cpu")
        with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as fh:
            json.dump({"env": [r, lr, w], "job_ms": job_ms, "job_channels": job_channels,
                       "mine4": mine4, "ops4": ops4, "total4": sum(costs4),
                       "mine5": mine5, "ops5": ops5, "total5": sum(costs5)}, fh)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    recs = [json.load(open(tmp_path / ("rank%d.json" % rank))) for rank in range(2)]
    for rank, rec in enumerate(recs):
        assert rec["env"] == [rank, rank, 2]
        assert rec["job_ms"] == 15.0
        assert rec["job_channels"] == 201.0
        # the summed per-rank work is the whole list's work
        assert rec["ops4"] == pytest.approx(rec["total4"])
        assert rec["ops5"] == pytest.approx(rec["total5"])
    # the shards are disjoint and cover every channel
    for key, n in (("mine4", 64), ("mine5", 1024)):
        a, b = set(recs[0][key]), set(recs[1][key])
        assert not (a & b) and (a | b) == set(range(n)), key
        assert abs(len(a) - len(b)) <= n // 4


def test_max_over_ranks_without_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.sum_over_ranks(7.0, None, "cpu") == 7.0


def test_reference_arm_under_torchrun_prints_once():
    """`bench.py --impl reference` launched as two ranks: rank 0 alone times
    the reference CPU code and prints one JSON line, rank 1 exits 0."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "cpu_corr_ref")
    if not os.path.exists(ref_bin):
        pytest.skip("reference CPU build absent")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "3", "--ref-sample", "16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference"
    assert rec["n_gpus"] == 2
    assert rec["cpu_baseline"]["kind"] == "reference"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0


def test_gpus_flag_relaunches_under_torchrun():
    """`bench.py --gpus 2` started as a plain process relaunches itself as two
    torchrun ranks (here on the reference arm, which needs no GPU): one JSON
    line, from rank 0, reporting both ranks."""
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "cpu_corr_ref")
    if not os.path.exists(ref_bin):
        pytest.skip("reference CPU build absent")
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT")}
    env.update(OMP_NUM_THREADS="1", MASTER_PORT=str(free_port()))
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "3", "--ref-sample", "16"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2
