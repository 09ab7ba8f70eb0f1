"""GPU parity of libchimex against the CPU oracle, through the C ABI.

Bit-exact integer comparisons: every output word must equal the oracle's.
Small and golden cases compare whole buffers.  At the full benchmark sizes one
channel per configuration is compared word for word with the oracle run on
all host cores, and every channel is checked by size-independent properties:
weighted checksums over every visibility (complex nonzero weights, four
draws), exact constant-input values and spot visibilities against O(T)
direct sums.
"""
import json
import os

import numpy as np
import pytest

import fullsize_checks as fc
import pyoracle as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KAT = json.load(open(os.path.join(GOLD, "kat.json")))["cases"]


@pytest.fixture(scope="module")
def chimex():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chimex as cx
    return cx


ALGOS = ["simt", "tc", "tc2"]  # tc: one-SM tile, tc2: SM-pair tile


def make_plan(cx, E, F, T, TA=256, ut=1, kb=0, algo="auto", tsplit=0, tile=0):
    p = cx.Plan(E, F, T, TA, ut, kb, 0)
    if tile:
        p.set_option(cx.OPT_TILE, tile)
    if algo == "simt":
        p.set_option(cx.OPT_ALGO, cx.ALGO_SIMT)
    elif algo in ("tc", "tc2"):
        if algo == "tc2":
            tile = 2
        elif not tile:
            tile = 1
        p.set_option(cx.OPT_TILE, tile)
        try:
            p.set_option(cx.OPT_ALGO, cx.ALGO_TC)
        except cx.ChimexError as e:
            if e.code == cx.E_UNSUPPORTED:
                pytest.skip("tensor-core path not available for this shape")
            raise
    if tsplit:
        p.set_option(cx.OPT_TSPLIT, tsplit)
    return p


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_blocks(cx, packed, E, F, T, ut=1, algo="auto", tsplit=0, tile=0):
    p = make_plan(cx, E, F, T, ut=ut, algo=algo, tsplit=tsplit, tile=tile)
    out = p.correlate(to_dev(packed))
    p.check_device()
    return out.cpu().numpy()


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("case", KAT, ids=[c["key"] for c in KAT])
def test_golden_cases(chimex, case, algo):
    T, F, E, ut = case["T"], case["F"], case["E"], case["ut"]
    packed = orc.generate(T, F, E, case["gen"], case["seed"], case["default_re"],
                          case["default_im"], case["initial_re"], case["initial_im"],
                          case["single_freq"], case["no_repeat"])
    blocks = gpu_blocks(chimex, packed, E, F, T, ut, algo)
    tri = orc.blocks_to_triangle(blocks, F, E)
    assert orc.fnv1a(tri) == case["tri_fnv"]
    if E <= 256:
        np.testing.assert_array_equal(blocks, orc.correlate_blocks(packed, T, F, E, ut))


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("E,F,T,ut", [
    (32, 1, 1, 1), (32, 1, 3, 0), (64, 2, 31, 1), (96, 3, 17, 1), (128, 1, 129, 0),
    (160, 2, 200, 1), (224, 1, 64, 1), (384, 1, 100, 1), (640, 2, 48, 0),
])
def test_edge_shapes(chimex, algo, E, F, T, ut):
    packed = orc.generate(T, F, E, 4, 1000 + E + T, no_repeat=1)
    blocks = gpu_blocks(chimex, packed, E, F, T, ut, algo)
    np.testing.assert_array_equal(blocks, orc.correlate_blocks(packed, T, F, E, ut))


@pytest.mark.parametrize("algo", ALGOS)
def test_extreme_values(chimex, algo):
    """All 256 byte values as elements; constant -8 is the int32 worst case."""
    T, F, E = 40, 1, 256
    packed = np.tile(np.arange(256, dtype=np.uint8), T)
    blocks = gpu_blocks(chimex, packed, E, F, T, 1, algo)
    np.testing.assert_array_equal(blocks, orc.correlate_blocks(packed, T, F, E, 1))
    T = 2048
    packed = np.zeros(T * 128, dtype=np.uint8)  # re = im = -8 everywhere
    blocks = gpu_blocks(chimex, packed, 128, 1, T, 1, algo)
    assert (blocks[0::2] == 128 * T).all() and (blocks[1::2] == 0).all()


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("tsplit", [1, 2, 3, 7])
def test_sample_splits_and_accumulate(chimex, algo, tsplit):
    T, F, E = 300, 2, 128
    packed = orc.generate(T, F, E, 4, 77, no_repeat=1)
    ref = orc.correlate_blocks(packed, T, F, E, 1)
    p = make_plan(chimex, E, F, T, algo=algo, tsplit=tsplit)
    d = to_dev(packed)
    out = p.correlate(d)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    p.correlate(d, out, accumulate=True)
    np.testing.assert_array_equal(out.cpu().numpy(), (ref.astype(np.int64) * 2).astype(np.int32))


@pytest.mark.parametrize("algo", ["tc", "tc2"])
@pytest.mark.parametrize("tsplit", [0, 2, 5, 16])
def test_split_units_meet_by_reduce_add(chimex, algo, tsplit):
    """The sample ranges of one tile pair run as separate units on different
    CTAs at the same time and add into the zeroed (or accumulating) output with
    TMA reduce-adds; repeated runs must equal the unsplit dp4a result exactly.
    tsplit 0 takes the automatic choice (this small shape is split)."""
    E, F, T = 512, 2, 4096
    packed = orc.generate(T, F, E, 4, 91, no_repeat=1)
    d = to_dev(packed)
    want = make_plan(chimex, E, F, T, algo="simt").correlate(d).cpu().numpy()
    p = make_plan(chimex, E, F, T, algo=algo, tsplit=tsplit)
    for _ in range(3):
        out = p.correlate(d)
        p.check_device()
        np.testing.assert_array_equal(out.cpu().numpy(), want)
    p.correlate(d, out, accumulate=True)
    p.check_device()
    np.testing.assert_array_equal(out.cpu().numpy(), (want.astype(np.int64) * 2).astype(np.int32))


def test_offset_accumulate_and_preseed(chimex):
    T, F, E = 96, 3, 96
    packed = orc.generate(T, F, E, 4, 5, no_repeat=1)
    for kb in (0, 1):
        for ut in (0, 1):
            p = chimex.Plan(E, F, T, 32, ut, kb, 0)
            d = to_dev(packed)
            sums = p.offset_accumulate(d)
            np.testing.assert_array_equal(sums.cpu().numpy().view(np.uint32),
                                          orc.offset_accumulate(packed, T, F, E))
            blocks = p.preseed(sums)
            ref = orc.preseed(orc.offset_accumulate(packed, T, F, E), T, F, E, kb, ut)
            np.testing.assert_array_equal(blocks.cpu().numpy(), ref)
            # accumulate=1 adds to the existing sums like the reference atomic_add
            p.offset_accumulate(d, sums, accumulate=True)
            np.testing.assert_array_equal(sums.cpu().numpy().view(np.uint32),
                                          2 * orc.offset_accumulate(packed, T, F, E))


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("kb,ut,F,TA", [(0, 1, 3, 256), (0, 0, 2, 288), (0, 1, 1, 8),
                                          (1, 1, 1, 1912), (1, 0, 1, 256)])
def test_reference_pipeline_compat(chimex, kb, ut, F, TA, algo):
    """accumulate -> preseed -> corr_compat reproduces the reference pipeline:
    the preseed values and the corr partials each match the oracle's
    restatement of the reference kernels, and their sum is exact."""
    E = 128
    T = TA * 2
    while T % 32:
        T += TA
    packed = orc.generate(T, F, E, 4, 9, no_repeat=1)
    p = make_plan(chimex, E, F, T, TA, ut, kb, algo)
    d = to_dev(packed)
    zero = torch.zeros(p.block_words, dtype=torch.int32, device="cuda")
    partial = p.corr_compat(d, zero).cpu().numpy()
    np.testing.assert_array_equal(partial, orc.corr_partials(packed, T, F, E, kb, ut))
    full = p.reference_pipeline(d).cpu().numpy()
    np.testing.assert_array_equal(full, orc.correlate_blocks(packed, T, F, E, ut))


@pytest.mark.parametrize("E,F,T,tsplit", [(1920, 2, 2048, 0), (1408, 3, 1000, 3), (384, 4, 777, 2),
                                          (1952, 1, 333, 0), (1888, 1, 500, 1)])
def test_odd_tile_counts(chimex, E, F, T, tsplit):
    """An odd number of 128-element tiles: the SM-pair kernel's last x pair
    and last y pair hold one tile each (the missing tile's cells are computed
    but never stored).  Every channel word for word against the oracle on
    every kernel, then accumulated once more on the SM pair (E=1952 is an
    even tile count with a partial last tile, E=1888 an odd one with a
    partial last tile)."""
    packed = orc.generate(T, F, E, 4, 5000 + E + T, no_repeat=1)
    ref = np.concatenate([orc.correlate_channel(packed, T, F, E, f, 1) for f in range(F)])
    for algo in ("tc2", "tc", "auto"):
        np.testing.assert_array_equal(
            gpu_blocks(chimex, packed, E, F, T, 1, algo, tsplit=tsplit), ref, err_msg=algo)
    p = make_plan(chimex, E, F, T, algo="tc2", tsplit=tsplit)
    d = to_dev(packed)
    out = p.correlate(d)
    p.correlate(d, out, accumulate=True)
    p.check_device()
    np.testing.assert_array_equal(out.cpu().numpy(), (ref.astype(np.int64) * 2).astype(np.int32))


@pytest.mark.parametrize("kb,ut", [(0, 1), (0, 0), (1, 1)])
def test_reference_pipeline_compat_odd_tiles(chimex, kb, ut):
    """The reference corr partials (offset-nibble value maps) on the SM-pair
    kernel with an odd tile count: E=384 (three tiles), F=1, TA=256."""
    E, F, TA = 384, 1, 256
    T = 2 * TA
    packed = orc.generate(T, F, E, 4, 19, no_repeat=1)
    p = make_plan(chimex, E, F, T, TA, ut, kb, "tc2")
    d = to_dev(packed)
    zero = torch.zeros(p.block_words, dtype=torch.int32, device="cuda")
    np.testing.assert_array_equal(p.corr_compat(d, zero).cpu().numpy(),
                                  orc.corr_partials(packed, T, F, E, kb, ut))
    np.testing.assert_array_equal(p.reference_pipeline(d).cpu().numpy(),
                                  orc.correlate_blocks(packed, T, F, E, ut))


@pytest.mark.parametrize("kb,F,T,TA", [(0, 1, 592, 296), (0, 1, 100, 20), (0, 1, 120, 12),
                                         (1, 2, 512, 256), (1, 1, 4608, 2304)])
def test_compat_rejects_outside_reference_domain(chimex, kb, F, T, TA):
    p = chimex.Plan(64, F, T, TA, 1, kb, 0)
    d = torch.zeros(p.input_bytes, dtype=torch.uint8, device="cuda")
    out = torch.zeros(p.block_words, dtype=torch.int32, device="cuda")
    with pytest.raises(chimex.ChimexError) as ei:
        p.corr_compat(d, out)
    assert ei.value.code in (chimex.E_INVALID, chimex.E_UNSUPPORTED)


def test_reorg_kernels(chimex):
    T, F, E = 32, 2, 96
    packed = orc.generate(T, F, E, 4, 8, no_repeat=1)
    p = chimex.Plan(E, F, T, 32, 1, 0, 0)
    blocks = p.correlate(to_dev(packed))
    ref_blocks = orc.correlate_blocks(packed, T, F, E, 1)
    np.testing.assert_array_equal(p.blocks_to_triangle(blocks).cpu().numpy(),
                                  orc.blocks_to_triangle(ref_blocks, F, E))
    np.testing.assert_array_equal(p.blocks_to_full(blocks).cpu().numpy(),
                                  orc.blocks_to_full(ref_blocks, F, E))


# ------------------------------------------------------------------ full sizes
# Configs 2 and 3 at their own sizes.  One channel of each is compared word for
# word (every cell of every block, diagonal-block lower halves included) with
# the oracle computed on all host cores; every channel is checked by four
# weighted checksums with complex nonzero weights and by spot visibilities.

_FULL = {}


def _config2():
    """E=2048, F=8, T=16384, reference generator (random, seed 42, no repeat)."""
    if "c2" not in _FULL:
        E, F, T = 2048, 8, 16384
        packed = orc.generate(T, F, E, 4, 42, no_repeat=1)
        f = 5
        _FULL["c2"] = (E, F, T, packed, f, orc.correlate_channel(packed, T, F, E, f, 1))
    return _FULL["c2"]


def _config3():
    """E=2048, F=16, time_accum=1912, T=1912*8; channels 0-7 constant -8 (the
    int32 worst case |Re| = 128 T), channels 8-15 random (seed 42, no repeat)."""
    if "c3" not in _FULL:
        E, F, T = 2048, 16, 1912 * 8
        const = orc.generate(T, 8, E, 1, 42, initial_re=-8, initial_im=-8)
        rnd = orc.generate(T, 8, E, 4, 42, no_repeat=1)
        packed = np.concatenate([const.reshape(T, 8, E), rnd.reshape(T, 8, E)], axis=1).ravel()
        f = 12
        _FULL["c3"] = (E, F, T, packed, f, orc.correlate_channel(packed, T, F, E, f, 1))
    return _FULL["c3"]


def _config3_single_channel():
    """The overflow workload with generate_frequency = 5: channel 5 random (seed 42, no
    repeat), every other channel the default value re = 7, im = -8
    (input_generator.c:84-96)."""
    if "c3q" not in _FULL:
        E, F, T, q = 2048, 16, 1912 * 8, 5
        packed = orc.generate(T, F, E, 4, 42, 7, -8, 0, 0, q, 1)
        _FULL["c3q"] = (E, F, T, packed, q, orc.correlate_channel(packed, T, F, E, q, 1))
    return _FULL["c3q"]


@pytest.mark.parametrize("algo", ALGOS)
def test_full_size_plain_config(chimex, algo):
    """The full-size plain workload: E=2048, F=8, T=16384, random no-repeat."""
    E, F, T, packed, f, ref = _config2()
    blocks = gpu_blocks(chimex, packed, E, F, T, 1, algo)
    np.testing.assert_array_equal(fc.channel_blocks(blocks, E, f), ref)
    rng = np.random.default_rng(1)
    for g in range(F):
        fc.weighted_checks(packed, blocks, T, F, E, g, rng)
        fc.spot_checks(packed, blocks, T, F, E, g, rng, 16)


def test_full_size_plain_config_nonstandard_convention(chimex):
    """The full-size plain workload with upper_triangle_convention = 0 on the
    SM-pair kernel: the same channel word for word (imaginary parts negated,
    cpu_corr_test.c:91-96)."""
    E, F, T, packed, f, ref = _config2()
    blocks = gpu_blocks(chimex, packed, E, F, T, 0, "tc2")
    want = ref.copy()
    want[1::2] = (0 - want[1::2].astype(np.int64)).astype(np.int32)
    np.testing.assert_array_equal(fc.channel_blocks(blocks, E, f), want)


@pytest.mark.parametrize("algo", ALGOS)
def test_full_size_overflow_edge_config(chimex, algo):
    """The long-integration overflow workload: constant -8 channels reach |Re| = 128 T exactly;
    the random channels are checked word for word (one) and by checksums."""
    E, F, T, packed, f, ref = _config3()
    blocks = gpu_blocks(chimex, packed, E, F, T, 1, algo)
    nbw = orc.num_blocks(E) * 2048
    head = blocks[: 8 * nbw]
    assert (head[0::2] == 128 * T).all() and (head[1::2] == 0).all()
    np.testing.assert_array_equal(fc.channel_blocks(blocks, E, f), ref)
    rng = np.random.default_rng(2)
    for g in range(8, F):
        fc.weighted_checks(packed, blocks, T, F, E, g, rng)
        fc.spot_checks(packed, blocks, T, F, E, g, rng, 8)


@pytest.mark.parametrize("algo", ALGOS)
def test_full_size_single_channel_generator(chimex, algo):
    """The overflow workload with generate_frequency: the fixed channels hold exactly
    T * |7 - 8i|^2 = 113 T (imaginary 0) in every cell, the generated channel
    equals the oracle word for word."""
    E, F, T, packed, q, ref = _config3_single_channel()
    blocks = gpu_blocks(chimex, packed, E, F, T, 1, algo)
    for g in range(F):
        ch = fc.channel_blocks(blocks, E, g)
        if g == q:
            np.testing.assert_array_equal(ch, ref)
        else:
            assert (ch[0::2] == 113 * T).all() and (ch[1::2] == 0).all(), g


@pytest.mark.parametrize("kb", [0, 1])
@pytest.mark.parametrize("ut", [0, 1])
def test_full_size_offset_sums_and_preseed(chimex, kb, ut):
    """The standalone offset_accumulator and all four preseed variants at
    the overflow workload's size (E=2048, F=16, T=15296), word for word against the
    oracle's restatement of offset_accumulator.cl:18-47 and
    preseed_multifreq*_UT.cl / preseed_multifreq*.cl."""
    E, F, T, packed, _, _ = _config3()
    p = chimex.Plan(E, F, T, 1912, ut, kb, 0)
    d = to_dev(packed)
    sums = p.offset_accumulate(d)
    ref_sums = _FULL.get("c3sums")
    if ref_sums is None:
        ref_sums = _FULL["c3sums"] = orc.offset_accumulate(packed, T, F, E)
    np.testing.assert_array_equal(sums.cpu().numpy().view(np.uint32), ref_sums)
    blocks = p.preseed(sums)
    np.testing.assert_array_equal(blocks.cpu().numpy(), orc.preseed(ref_sums, T, F, E, kb, ut))
    p.check_device()
    p.close()


@pytest.mark.parametrize("E,F,T", [(2048, 16, 4096), (1024, 16, 15296), (2048, 32, 2048),
                                   (2048, 4, 4000), (1536, 24, 1000)])
def test_tc_repeatable_against_simt(chimex, E, F, T):
    """Persistent tensor-core launches over many units, repeated: every run
    must equal the CUDA-core kernel bit for bit (catches pipeline races that a
    single run can miss).  The CUDA-core kernel is itself pinned to the oracle
    by the tests above."""
    gen = torch.Generator(device="cuda")
    gen.manual_seed(E + F + T)
    d = torch.randint(0, 256, (T * F * E,), dtype=torch.uint8, device="cuda", generator=gen)
    ref = make_plan(chimex, E, F, T, algo="simt").correlate(d)
    for algo in ("tc", "tc2"):
        p = make_plan(chimex, E, F, T, algo=algo)
        out = torch.empty_like(ref)
        for _ in range(4):
            p.correlate(d, out)
            p.check_device()
            assert torch.equal(out, ref), algo


def test_tensor_core_path_rejects_unaligned_buffers(chimex):
    """TMA needs 16-byte aligned input and block buffers: an unaligned pointer is
    refused with CHX_E_INVALID before anything is enqueued."""
    import ctypes
    cx = chimex
    E, F, T = 256, 1, 64
    p = make_plan(cx, E, F, T, algo="tc2")
    x = torch.zeros(p.input_bytes + 64, dtype=torch.uint8, device="cuda")
    y = torch.zeros(p.block_words + 16, dtype=torch.int32, device="cuda")
    lib = cx.lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h = p._h
    assert lib.chx_correlate(h, ctypes.c_void_p(x.data_ptr() + 4), ctypes.c_void_p(y.data_ptr()),
                             s, 0) == cx.E_INVALID
    assert lib.chx_correlate(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr() + 4),
                             s, 0) == cx.E_INVALID
    assert "aligned" in lib.chx_last_error().decode()
    assert lib.chx_correlate(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                             s, 0) == cx.OK
    p.check_device()
    # the CUDA-core path and the helper kernels refuse them too
    p.set_option(cx.OPT_ALGO, cx.ALGO_SIMT)
    assert lib.chx_correlate(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr() + 8),
                             s, 0) == cx.E_INVALID
    sums = torch.zeros(p.sum_words + 8, dtype=torch.int32, device="cuda")
    assert lib.chx_offset_accumulate(h, ctypes.c_void_p(x.data_ptr() + 4),
                                     ctypes.c_void_p(sums.data_ptr()), s, 0) == cx.E_INVALID
    assert lib.chx_preseed(h, ctypes.c_void_p(sums.data_ptr() + 4), ctypes.c_void_p(y.data_ptr()),
                           s) == cx.E_INVALID
    tri = torch.zeros(p.triangle_words + 8, dtype=torch.int32, device="cuda")
    assert lib.chx_blocks_to_triangle(h, ctypes.c_void_p(y.data_ptr()),
                                      ctypes.c_void_p(tri.data_ptr() + 8), s) == cx.E_INVALID


@pytest.mark.parametrize("algo", ["tc", "tc2"])
def test_large_element_count(chimex, algo):
    """E=8192 (256 blocks per row, 32,896 blocks, 270 MB of output per channel)
    on both tensor-core tiles, word for word against the oracle."""
    E, F, T = 8192, 1, 96
    packed = orc.generate(T, F, E, 4, 8192, no_repeat=1)
    blocks = gpu_blocks(chimex, packed, E, F, T, 1, algo)
    np.testing.assert_array_equal(blocks, orc.correlate_channel(packed, T, F, E, 0, 1))


@pytest.mark.parametrize("algo", ["tc", "tc2"])
def test_plan_above_the_unit_sample_limit(chimex, algo):
    """T above 262144 samples: every tile pair is cut into ranges that meet by
    TMA reduce-add, unsplit by the plan's own choice (tsplit 1) and split."""
    E, F, T = 256, 2, 262144 + 100
    packed = orc.generate(T, F, E, 4, 262, no_repeat=1)
    ref = np.concatenate([orc.correlate_channel(packed, T, F, E, f, 1) for f in range(F)])
    for tsplit in (1, 3):
        np.testing.assert_array_equal(gpu_blocks(chimex, packed, E, F, T, 1, algo, tsplit=tsplit),
                                      ref)
