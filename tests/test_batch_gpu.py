"""Batched ragged launch and autotuner: every channel of a batch (own E,
integration length, integration count, input stride) must equal the oracle's
blocks for each of its integrations, bit for bit."""
import numpy as np
import pytest

import pyoracle as orc

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def chimex():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chimex as cx
    return cx


def make_channel(rng, E, T, nint, stride=0):
    """Random offset-binary samples (uniform [-8,7] re/im) for nint
    integrations of T samples, `stride` bytes apart (default E)."""
    st = stride or E
    vals = rng.integers(0, 256, size=(nint * T, st), dtype=np.uint8)
    return vals, st


def oracle_blocks(host, E, T, nint, ut):
    nb = orc.num_blocks(E)
    out = np.empty((nint, nb * 2048), dtype=np.int32)
    for i in range(nint):
        x = np.ascontiguousarray(host[i * T:(i + 1) * T, :E])
        out[i] = orc.correlate_blocks(x, T, 1, E, ut).reshape(-1)
    return out


def run_batch(cx, specs, ut=1, seed=7):
    rng = np.random.default_rng(seed)
    chans, hosts = [], []
    for (E, T, nint, stride) in specs:
        host, st = make_channel(rng, E, T, nint, stride)
        packed = torch.from_numpy(host.reshape(-1)).cuda()
        blocks = torch.full((nint * orc.num_blocks(E) * 2048,), -1, dtype=torch.int32,
                            device="cuda")
        chans.append((packed, blocks, E, T, nint, stride))
        hosts.append(host)
    b = cx.Batch(chans, ut)
    return b, chans, hosts


@pytest.mark.gpu
@pytest.mark.parametrize("ut", [0, 1])
def test_ragged_batch_small_tile(chimex, ut):
    # the costliest channel (E=128) spans one tile of 128 elements: the
    # one-SM tile for every channel
    specs = [(96, 77, 2, 128), (128, 300, 3, 0), (32, 33, 1, 48), (64, 1, 2, 0),
             (128, 95, 2, 256), (96, 64, 1, 0)]
    b, chans, hosts = run_batch(chimex, specs, ut)
    b.run(accumulate=False)
    b.check_device()
    for (E, T, nint, _), (packed, blocks, *_), host in zip(specs, chans, hosts):
        ref = oracle_blocks(host, E, T, nint, ut)
        np.testing.assert_array_equal(blocks.cpu().numpy().reshape(nint, -1), ref)
    b.run(accumulate=True)
    b.check_device()
    for (E, T, nint, _), (packed, blocks, *_), host in zip(specs, chans, hosts):
        ref = oracle_blocks(host, E, T, nint, ut)
        np.testing.assert_array_equal(blocks.cpu().numpy().reshape(nint, -1), 2 * ref)
    b.close()


@pytest.mark.gpu
def test_ragged_batch_pair_tile(chimex):
    # the costliest channel (E=512) spans 4 tiles of 128, an even count: the
    # SM-pair tile for every channel
    specs = [(512, 200, 2, 0), (96, 77, 1, 0), (288, 64, 3, 320), (640, 129, 1, 0)]
    b, chans, hosts = run_batch(chimex, specs, 1, seed=11)
    b.run()
    b.check_device()
    for (E, T, nint, _), (packed, blocks, *_), host in zip(specs, chans, hosts):
        ref = oracle_blocks(host, E, T, nint, 1)
        np.testing.assert_array_equal(blocks.cpu().numpy().reshape(nint, -1), ref)
    assert b.work_units > 0
    ops = sum(8.0 * E * (E + 1) / 2 * T * n for (E, T, n, _) in specs)
    assert b.ops == pytest.approx(ops)


@pytest.mark.gpu
def test_batch_split_integration(chimex):
    # an integration above 2^18 samples is cut into split units that meet by
    # TMA reduce-add in zeroed outputs
    specs = [(64, 300000, 1, 0), (32, 5, 1, 0)]
    b, chans, hosts = run_batch(chimex, specs, 1, seed=3)
    for accumulate, factor in ((False, 1), (True, 2)):
        b.run(accumulate=accumulate)
        b.check_device()
        for (E, T, nint, _), (packed, blocks, *_), host in zip(specs, chans, hosts):
            ref = oracle_blocks(host, E, T, nint, 1)
            np.testing.assert_array_equal(blocks.cpu().numpy().reshape(nint, -1), factor * ref)


@pytest.mark.gpu
def test_batch_of_few_long_channels_is_split(chimex):
    # two E=512 channels (three integrations) make only 9 SM-pair units for 74
    # clusters: the batch splits their samples (8 ranges by the makespan
    # estimate, 72 units), and the
    # ranges of each tile pair meet by TMA reduce-add, twice in a row and in
    # accumulate mode
    specs = [(512, 4096, 1, 0), (512, 2000, 2, 0)]
    b, chans, hosts = run_batch(chimex, specs, 1, seed=5)
    assert b.work_units > 9
    refs = [oracle_blocks(host, E, T, nint, 1)
            for (E, T, nint, _), host in zip(specs, hosts)]
    for accumulate, factor in ((False, 1), (False, 1), (True, 2)):
        b.run(accumulate=accumulate)
        b.check_device()
        for (E, T, nint, _), (packed, blocks, *_), ref in zip(specs, chans, refs):
            np.testing.assert_array_equal(blocks.cpu().numpy().reshape(nint, -1), factor * ref)


@pytest.mark.gpu
def test_batch_graph_replays_match_plain_plans(chimex):
    """64-channel ragged batch (E in {256..2048}, TA in [64, 1912], 4
    integrations) against per-integration plain launches, compared by an
    FNV-1a hash per channel."""
    cx = chimex
    rng = np.random.default_rng(42)
    Es = rng.choice([256, 512, 1024, 1536, 2048], size=64)
    TAs = rng.integers(64, 1913, size=64)
    chans = []
    for E, T in zip(Es, TAs):
        E, T = int(E), int(T)
        packed = torch.randint(0, 256, (4 * T * E,), dtype=torch.uint8, device="cuda")
        blocks = torch.empty(4 * orc.num_blocks(E) * 2048, dtype=torch.int32, device="cuda")
        chans.append((packed, blocks, E, T, 4))
    b = cx.Batch(chans)
    for _ in range(2):
        b.run()
    b.check_device()
    for (packed, blocks, E, T, nint) in chans:
        p = cx.Plan(E, 1, T, T)
        nbw = orc.num_blocks(E) * 2048
        for i in range(nint):
            ref = p.correlate(packed[i * T * E:(i + 1) * T * E])
            assert torch.equal(blocks[i * nbw:(i + 1) * nbw], ref), (E, T, i)
        p.close()


@pytest.mark.gpu
def test_config4_with_reference_generator_against_oracle(chimex):
    """The batched configuration as specified: 64 channels, E and time_accum
    drawn with seed 42, channel c's samples from the reference generator
    (random, seed 42 + c, no repeat), 4 integrations each, one batch launch.
    Every integration of every channel is compared word for word with the
    oracle (computed on all host cores)."""
    cx = chimex
    rng = np.random.default_rng(42)
    Es = [int(e) for e in rng.choice([256, 512, 1024, 1536, 2048], size=64)]
    TAs = [int(t) for t in rng.integers(64, 1913, size=64)]
    nint = 4
    chans, hosts = [], []
    for c, (E, T) in enumerate(zip(Es, TAs)):
        host = orc.generate(nint * T, 1, E, 4, 42 + c, no_repeat=1)
        hosts.append(host)
        chans.append((torch.from_numpy(host).cuda(),
                      torch.full((nint * orc.num_blocks(E) * 2048,), -1, dtype=torch.int32,
                                 device="cuda"), E, T, nint))
    b = cx.Batch(chans)
    b.run()
    b.check_device()
    for c, ((packed, blocks, E, T, n), host) in enumerate(zip(chans, hosts)):
        out = blocks.cpu().numpy().reshape(n, -1)
        for i in range(n):
            ref = orc.correlate_channel(host, n * T, 1, E, 0, 1, t0=i * T, t1=(i + 1) * T)
            np.testing.assert_array_equal(out[i], ref, err_msg="channel %d integration %d" % (c, i))
    b.close()


@pytest.mark.gpu
def test_autotune_choice_is_exact(chimex):
    cx = chimex
    E, T = 1024, 2048
    x = torch.randint(0, 256, (T * E,), dtype=torch.uint8, device="cuda")
    out = torch.empty(orc.num_blocks(E) * 2048, dtype=torch.int32, device="cuda")
    tile, split, ms = cx.autotune(E, T, x, out)
    assert tile in (1, 2) and split in (1, 2, 4) and ms > 0
    # a batch of this shape now uses the tuned tile (its own split)
    blocks = torch.full_like(out, -7)
    b = cx.Batch([(x, blocks, E, T, 1)])
    b.run()
    b.check_device()
    p = cx.Plan(E, 1, T, T)
    p.set_option(cx.OPT_ALGO, cx.ALGO_SIMT)
    ref = p.correlate(x)
    assert torch.equal(blocks, ref)
    # a plan of this shape created now takes the tuned tile too
    q = cx.Plan(E, 1, T, T)
    assert torch.equal(q.correlate(x), ref)
    q.check_device()


def test_batch_validation_without_device():
    import ctypes

    import chimex as cx
    h = ctypes.c_void_p()
    lib = cx.lib()
    assert lib.chx_batch_create(ctypes.byref(h), 0, None, 1, 0) == cx.E_INVALID
    d = (cx.ChannelDesc * 1)(cx.ChannelDesc(33, 16, 1, 0, 16, 16))
    assert lib.chx_batch_create(ctypes.byref(h), 1, d, 1, 0) == cx.E_INVALID
    d = (cx.ChannelDesc * 1)(cx.ChannelDesc(64, 16, 1, 72, 16, 16))  # stride not 16-aligned
    assert lib.chx_batch_create(ctypes.byref(h), 1, d, 1, 0) == cx.E_INVALID
    d = (cx.ChannelDesc * 1)(cx.ChannelDesc(64, 16, 0, 0, 16, 16))
    assert lib.chx_batch_create(ctypes.byref(h), 1, d, 1, 0) == cx.E_INVALID
    assert not h.value
    assert lib.chx_batch_run(None, None, 0) == cx.E_INVALID
    assert lib.chx_batch_destroy(None) == cx.OK
