"""CPU tests pinning the oracle (oracle/chx_oracle.c) to the reference.

The golden fixtures in tests/golden/ were produced by the reference's own CPU
code (tests/golden/make_golden.py); when oracle/_ref is present the same
comparisons also run live against it.
"""
import json
import os

import numpy as np
import pytest

import pyoracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLD, "kat.json")) as _fh:
    KAT = json.load(_fh)["cases"]
SMALL = np.load(os.path.join(GOLD, "small_tri.npz"))


def _gen(c):
    return orc.generate(c["T"], c["F"], c["E"], c["gen"], c["seed"], c["default_re"],
                        c["default_im"], c["initial_re"], c["initial_im"],
                        c["single_freq"], c["no_repeat"])


@pytest.mark.parametrize("case", KAT, ids=[c["key"] for c in KAT])
def test_generator_matches_golden(case):
    packed = _gen(case)
    if packed.size <= 1 << 20:
        assert orc.fnv1a_bytes(packed) == case["input_fnv"]
    if orc.ref_available():
        ref = orc.ref_generate(case["T"], case["F"], case["E"], case["gen"], case["seed"],
                               case["default_re"], case["default_im"], case["initial_re"],
                               case["initial_im"], case["single_freq"], case["no_repeat"])
        np.testing.assert_array_equal(packed, ref)


@pytest.mark.parametrize("case", KAT, ids=[c["key"] for c in KAT])
def test_triangle_matches_golden(case):
    T, F, E, ut = case["T"], case["F"], case["E"], case["ut"]
    packed = _gen(case)
    tri = orc.correlate_triangle(packed, T, F, E, ut)
    assert orc.fnv1a(tri) == case["tri_fnv"]
    assert tri[:8].tolist() == case["head"]
    if case["key"] in SMALL:
        np.testing.assert_array_equal(tri, SMALL[case["key"]])


@pytest.mark.parametrize("case", KAT, ids=[c["key"] for c in KAT])
def test_block_layout_reorgs_to_golden(case):
    T, F, E, ut = case["T"], case["F"], case["E"], case["ut"]
    if E > 256:
        pytest.skip("large case covered by the triangle test")
    packed = _gen(case)
    blocks = orc.correlate_blocks(packed, T, F, E, ut)
    tri = orc.blocks_to_triangle(blocks, F, E)
    assert orc.fnv1a(tri) == case["tri_fnv"]
    if orc.ref_available():
        np.testing.assert_array_equal(orc.ref_blocks_to_triangle(blocks, F, E), tri)


def test_reference_live_small_cases():
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    for (T, F, E, seed, ut) in [(24, 2, 64, 3, 1), (24, 2, 64, 3, 0), (5, 1, 32, 9, 1)]:
        packed = orc.generate(T, F, E, 4, seed, no_repeat=1)
        ours = orc.correlate_triangle(packed, T, F, E, ut)
        theirs = orc.ref_correlate_triangle(T, F, E, 4, seed, no_repeat=1, ut=ut)
        np.testing.assert_array_equal(ours, theirs)


def test_unpack_all_byte_values():
    """four_bit_macros.h:8-9 semantics: re = HI_NIBBLE - 8, im = LO_NIBBLE - 8."""
    T, F, E = 1, 1, 256
    packed = np.arange(256, dtype=np.uint8)
    blocks = orc.correlate_blocks(packed, T, F, E, 1)
    for b in range(256):
        re, im = (b >> 4) - 8, (b & 15) - 8
        off = orc.block_cell_offset(E, 0, b, b)
        assert blocks[off] == re * re + im * im and blocks[off + 1] == 0
    # a cross term pins the sign convention of Im (cpu_corr_test.c:189)
    y, x = 0x3A, 0xC5
    off = orc.block_cell_offset(E, 0, y, x)
    yr, yi, xr, xi = (y >> 4) - 8, (y & 15) - 8, (x >> 4) - 8, (x & 15) - 8
    assert blocks[off] == xr * yr + xi * yi
    assert blocks[off + 1] == xr * yi - xi * yr


def test_block_enumeration_matches_id_maps():
    """main_wrapper.c:529-540: for j (row) for i >= j (column)."""
    for E in (32, 64, 256, 2048):
        nb1 = E // 32
        idx = 0
        for by in range(nb1):
            for bx in range(by, nb1):
                assert orc.block_cell_offset(E, 0, by * 32, bx * 32) == idx * 2048
                idx += 1
        assert idx == orc.num_blocks(E)


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("ut", [0, 1])
def test_compat_pipeline_reconstructs_visibilities(variant, ut):
    """offsetAccumulate -> preseed -> corr (offset partials) == true visibilities."""
    T, F, E = 64, 3, 96
    packed = orc.generate(T, F, E, 4, 11, no_repeat=1)
    sums = orc.offset_accumulate(packed, T, F, E)
    blocks = orc.preseed(sums, T, F, E, variant, ut)
    orc.corr_partials(packed, T, F, E, variant, ut, out=blocks)
    np.testing.assert_array_equal(blocks, orc.correlate_blocks(packed, T, F, E, ut))


def test_compat_pipeline_worst_case_constant():
    """Constant -8 (offset 0) is the int32-magnitude worst case: |Re| = 128 T."""
    T, F, E = 1912, 1, 64
    packed = orc.generate(T, F, E, 1, 42, initial_re=-8, initial_im=-8)
    for variant in (0, 1):
        sums = orc.offset_accumulate(packed, T, F, E)
        blocks = orc.preseed(sums, T, F, E, variant, 1)
        orc.corr_partials(packed, T, F, E, variant, 1, out=blocks)
        assert blocks[0] == 128 * T and blocks[1] == 0
        np.testing.assert_array_equal(blocks, orc.correlate_blocks(packed, T, F, E, 1))


def test_offset_accumulate_values():
    T, F, E = 32, 2, 64
    packed = orc.generate(T, F, E, 4, 5, no_repeat=1)
    sums = orc.offset_accumulate(packed, T, F, E).reshape(F * E, 2)
    p = packed.reshape(T, F * E)
    np.testing.assert_array_equal(sums[:, 0], (p >> 4).sum(0))
    np.testing.assert_array_equal(sums[:, 1], (p & 15).sum(0))


def test_weighted_power_identity_and_spot_checks():
    T, F, E = 48, 2, 128
    packed = orc.generate(T, F, E, 4, 99, no_repeat=1)
    blocks = orc.correlate_blocks(packed, T, F, E, 1)
    rng = np.random.default_rng(0)
    for f in range(F):
        w = rng.integers(-3, 4, size=2 * E).astype(np.int32)
        assert orc.weighted_power(packed, T, F, E, f, w) == \
            orc.weighted_from_blocks(blocks, F, E, f, w)
        for _ in range(20):
            y = int(rng.integers(0, E))
            x = int(rng.integers(32 * (y // 32), E))
            off = orc.block_cell_offset(E, f, y, x)
            assert orc.visibility(packed, T, F, E, f, y, x) == \
                (blocks[off], blocks[off + 1])


def test_split_ranges_are_additive():
    """Integer sums are associative: any split of T gives the same result."""
    T, F, E = 40, 1, 64
    packed = orc.generate(T, F, E, 4, 3, no_repeat=1)
    whole = orc.correlate_blocks(packed, T, F, E, 1)
    part = orc.correlate_blocks(packed, T, F, E, 1, 0, 13)
    orc.correlate_blocks(packed, T, F, E, 1, 13, 40, out=part)
    np.testing.assert_array_equal(whole, part)


def test_full_matrix_view_is_hermitian():
    T, F, E = 16, 1, 64
    packed = orc.generate(T, F, E, 4, 21, no_repeat=1)
    full = orc.blocks_to_full(orc.correlate_blocks(packed, T, F, E, 1), F, E)
    m = full.reshape(E, E, 2)
    np.testing.assert_array_equal(m[:, :, 0], m[:, :, 0].T)
    np.testing.assert_array_equal(m[:, :, 1], -m[:, :, 1].T)


@pytest.mark.parametrize("E,F,T,ut,f", [(32, 1, 1, 1, 0), (96, 3, 37, 1, 2), (256, 2, 100, 0, 1),
                                         (160, 4, 64, 1, 3)])
def test_threaded_channel_oracle_equals_restatement(E, F, T, ut, f):
    """The threaded per-channel oracle used for word-for-word checks at full
    size gives exactly the single-threaded restatement's blocks, for whole
    sample ranges and sub-ranges, on one thread and on several."""
    packed = orc.generate(T, F, E, 4, 31 + E, no_repeat=1)
    nbw = orc.num_blocks(E) * 2048
    full = orc.correlate_blocks(packed, T, F, E, ut)[f * nbw:(f + 1) * nbw]
    for threads in (1, 3):
        np.testing.assert_array_equal(orc.correlate_channel(packed, T, F, E, f, ut,
                                                            threads=threads), full)
    t0, t1 = T // 3, T - T // 4
    sub = orc.correlate_blocks(packed, T, F, E, ut, t0=t0, t1=t1)[f * nbw:(f + 1) * nbw]
    np.testing.assert_array_equal(orc.correlate_channel(packed, T, F, E, f, ut, t0=t0, t1=t1), sub)


def test_weighted_checks_catch_single_cell_errors():
    """The full-size checks (four draws of complex nonzero weights) detect an
    error of one unit in the real part of any single visibility and in the
    imaginary part of any off-diagonal one, including imaginary-part errors
    that a real-valued weight product would miss.  (V[y][y] is real by
    definition and the identity weighs it by |w_y|^2, so its imaginary part
    is left to the word-for-word and spot checks.)"""
    import fullsize_checks as fc
    T, F, E = 24, 1, 64
    packed = orc.generate(T, F, E, 4, 8, no_repeat=1)
    good = orc.correlate_blocks(packed, T, F, E, 1)
    fc.weighted_checks(packed, good, T, F, E, 0, np.random.default_rng(0))
    rng = np.random.default_rng(1)
    for trial in range(40):
        y = int(rng.integers(0, E - 1))
        x = int(rng.integers(y if trial % 2 == 0 else y + 1, E))
        bad = good.copy()
        bad[orc.block_cell_offset(E, 0, y, x) + (trial % 2)] += 1
        with pytest.raises(AssertionError):
            fc.weighted_checks(packed, bad, T, F, E, 0, np.random.default_rng(trial))
