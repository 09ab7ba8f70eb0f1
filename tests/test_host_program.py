"""The C host program (chime-x_b200/host/correlator_test.c): the reference
harness's command line over the C ABI.  CPU tests cover argument handling;
GPU tests run each path with --check_results, which compares every
visibility with a direct CPU sum inside the program."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "chime-x_b200", "correlator_test")


def run(*args, timeout=300):
    if not os.path.exists(BIN):
        pytest.skip("correlator_test not built")
    return subprocess.run([BIN, *map(str, args)], capture_output=True, text=True,
                          timeout=timeout)


def test_help_lists_the_reference_options():
    r = run("-h")
    assert r.returncode == 0
    for opt in ("--device", "--iterations", "--time_accum", "--time_steps", "--num_freq",
                "--num_elements", "--timer_without_copies", "--upper_triangle_convention",
                "--check_results", "--gen_type", "--random_seed", "--no_repeat_random",
                "--generate_frequency", "--kernel_batch"):
        assert opt in r.stdout


@pytest.mark.parametrize("args", [("-g", 0), ("-g", 5), ("-k", 2), ("-U", 3), ("--bogus",)])
def test_invalid_options_are_rejected(args):
    r = run(*args)
    assert r.returncode == 1
    assert "Usage" in r.stdout


def test_plan_validation_reaches_the_user():
    r = run("-e", 33, "-T", 64, "-i", 1)
    assert r.returncode == 1
    assert "num_elements=33" in r.stderr


GPU_CASES = [
    ("fused", ["-e", 256, "-f", 2, "-T", 512, "-t", 256, "-i", 3, "-p"]),
    ("fused_pair_tile", ["-e", 640, "-f", 1, "-T", 777, "-t", 259, "-i", 2, "-p"]),
    ("fused_nonUT", ["-e", 128, "-f", 3, "-T", 300, "-t", 100, "-i", 2, "-p", "-U", 0]),
    ("fused_no_copies", ["-e", 256, "-f", 1, "-T", 1024, "-t", 256, "-i", 4, "-w", "-p"]),
    ("constant_minus8", ["-e", 256, "-f", 1, "-T", 512, "-t", 256, "-i", 1, "-g", 1,
                         "-X", -8, "-Y", -8]),
    ("ramp_up", ["-e", 96, "-f", 2, "-T", 64, "-t", 64, "-i", 1, "-g", 2]),
    ("ramp_down", ["-e", 96, "-f", 2, "-T", 64, "-t", 64, "-i", 1, "-g", 3, "-X", 3]),
    ("single_freq", ["-e", 64, "-f", 3, "-T", 128, "-t", 128, "-i", 1, "-q", 1, "-x", 7,
                     "-y", -8, "-p"]),
    ("pipeline_conference", ["-e", 256, "-f", 2, "-T", 512, "-t", 256, "-i", 2, "-p", "-P"]),
    ("pipeline_packed", ["-e", 256, "-f", 1, "-T", 2048, "-t", 1024, "-i", 2, "-p", "-P",
                         "-k", 1]),
    ("pipeline_nonUT", ["-e", 128, "-f", 1, "-T", 256, "-t", 128, "-i", 1, "-p", "-P",
                        "-U", 0]),
    ("noalloc", ["-e", 512, "-f", 2, "-T", 600, "-t", 200, "-i", 2, "-p", "-n"]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,args", GPU_CASES, ids=[c[0] for c in GPU_CASES])
def test_paths_check_against_cpu(name, args):
    r = run(*args, "-c")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "CPU matches GPU" in r.stdout
    assert "TOPS exact int8" in r.stdout
