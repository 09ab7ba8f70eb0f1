"""Parity checks for outputs too large to compare against a full oracle run
in every test: weighted checksums over every upper-triangle visibility and
spot visibilities, both computed by the CPU oracle (oracle/chx_oracle.c).

The checksum identity is sum_t |sum_e w_e s_e(t)|^2 =
sum_y |w_y|^2 V[y][y] + 2 Re sum_{x>y} w_y conj(w_x) V[y][x].  Its weights
are complex with nonzero real and imaginary parts (magnitudes 1-3), so that
w_y conj(w_x) is complex for most pairs and an error in either the real or
the imaginary part of a visibility changes the sum; several independent
draws per channel make an error that cancels in one draw show in another.
"""
import numpy as np

import pyoracle as orc


def nonzero_weights(rng, E):
    """2E int32 weights (re, im interleaved), each in {-3..-1, 1..3}."""
    mag = rng.integers(1, 4, size=2 * E)
    sign = rng.choice(np.array([-1, 1]), size=2 * E)
    return (mag * sign).astype(np.int32)


def weighted_checks(packed, blocks, T, F, E, f, rng, draws=4):
    """`draws` independent weighted checksums of channel f."""
    for k in range(draws):
        w = nonzero_weights(rng, E)
        assert orc.weighted_power(packed, T, F, E, f, w) == \
            orc.weighted_from_blocks(blocks, F, E, f, w), "checksum %d of channel %d" % (k, f)


def spot_checks(packed, blocks, T, F, E, f, rng, n):
    """n visibilities of channel f against direct O(T) sums."""
    for _ in range(n):
        y = int(rng.integers(0, E))
        x = int(rng.integers(32 * (y // 32), E))
        off = orc.block_cell_offset(E, f, y, x)
        assert orc.visibility(packed, T, F, E, f, y, x) == \
            (blocks[off], blocks[off + 1]), (f, y, x)


def channel_blocks(blocks, E, f):
    """Channel f's NB*2048 words of a block buffer."""
    nbw = orc.num_blocks(E) * 2048
    return blocks[f * nbw:(f + 1) * nbw]
