"""Generate the golden fixtures in this directory from the reference's own CPU
code (cpu_corr_test.c, input_generator.c, gpu_data_reorg.c), compiled from the
reference sources into oracle/_ref/libchx_ref.so by oracle/Makefile.

Run from the repository root (needs the reference checkout, so only on the
development machine):

    make -C oracle && python tests/golden/make_golden.py

Outputs:
  kat.json         one record per case: generator/correlator arguments, the
                   FNV-1a hash of the generated input bytes, the FNV-1a hash of
                   the reference's upper-triangle output (int32 words as uint32),
                   and a few leading visibilities.
  small_tri.npz    full reference triangles for the small cases (E <= 64).
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libchx_ref.so")


def fnv1a_words(a):
    """64-bit FNV-1a over int32 words taken as uint32 (vectorised in chunks)."""
    h = 0xCBF29CE484222325
    for w in np.asarray(a).astype(np.uint32).ravel().tolist():
        h ^= w
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return "%016x" % h


def fnv1a_bytes(b):
    h = 0xCBF29CE484222325
    for w in bytes(b):
        h ^= w
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return "%016x" % h


# (T, F, E, gen, seed, dre, dim, ire, iim, single_freq, no_repeat, ut)
CASES = [
    # The small plain case: E=256 F=1 T=TA=256, seed 42, repeating random.
    (256, 1, 256, 4, 42, 0, 0, 0, 0, -1, 0, 1),
    (256, 1, 256, 4, 42, 0, 0, 0, 0, -1, 1, 1),
    (256, 1, 256, 1, 42, 0, 0, 0, 0, -1, 0, 1),
    (64, 1, 2048, 4, 42, 0, 0, 0, 0, -1, 1, 1),
    # multi-channel, every generator, both conventions
    (64, 8, 256, 4, 42, 0, 0, 0, 0, -1, 1, 1),
    (64, 8, 256, 4, 42, 0, 0, 0, 0, -1, 1, 0),
    (96, 4, 128, 1, 42, 0, 0, -8, -8, -1, 0, 1),
    (96, 4, 128, 1, 42, 0, 0, 7, 7, -1, 0, 1),
    (96, 4, 128, 1, 42, 0, 0, 7, -8, -1, 0, 0),
    (64, 4, 128, 2, 42, 0, 0, 0, 0, -1, 0, 1),
    (64, 4, 128, 3, 42, 0, 0, 0, 0, -1, 0, 1),
    (64, 4, 128, 2, 42, 0, 0, 3, -5, -1, 0, 0),
    # single-channel override (default (7, -8) in every other channel)
    (64, 4, 128, 4, 42, 7, -8, 0, 0, 2, 1, 1),
    (64, 4, 128, 4, 42, 7, -8, 0, 0, 4, 1, 1),  # == F: every channel default
    # small shapes kept whole in small_tri.npz
    (8, 1, 32, 4, 42, 0, 0, 0, 0, -1, 1, 1),
    (8, 1, 32, 4, 42, 0, 0, 0, 0, -1, 1, 0),
    (40, 2, 64, 4, 7, 0, 0, 0, 0, -1, 1, 1),
    (40, 2, 64, 4, 7, 0, 0, 0, 0, -1, 1, 0),
    (17, 3, 96, 4, 1234, 0, 0, 0, 0, -1, 1, 1),
    (1, 1, 32, 2, 42, 0, 0, -8, 7, -1, 0, 1),
]


def main():
    if not os.path.exists(REF_SO):
        sys.exit("missing %s: run `make -C oracle` with the reference present" % REF_SO)
    ref = ctypes.CDLL(REF_SO)
    vp = ctypes.c_void_p
    records = []
    small = {}
    for (T, F, E, gen, seed, dre, dim, ire, iim, sf, nr, ut) in CASES:
        packed = np.zeros(T * F * E, dtype=np.uint8)
        ref.generate_char_data_set(gen, seed, dre, dim, ire, iim, sf, T, F, E, nr,
                                   packed.ctypes.data_as(vp))
        tri = np.zeros(F * E * (E + 1), dtype=np.int32)
        fn = (ref.cpu_data_generate_and_correlate_upper_triangle_only if ut else
              ref.cpu_data_generate_and_correlate_upper_triangle_only_nonstandard_convention)
        err = fn(T, F, E, tri.ctypes.data_as(vp), gen, seed, dre, dim, ire, iim, sf, nr, 0)
        assert err == 0
        key = "T%d_F%d_E%d_g%d_s%d_d%d_%d_i%d_%d_q%d_p%d_u%d" % (
            T, F, E, gen, seed, dre, dim, ire, iim, sf, nr, ut)
        records.append(dict(
            key=key, T=T, F=F, E=E, gen=gen, seed=seed, default_re=dre,
            default_im=dim, initial_re=ire, initial_im=iim, single_freq=sf,
            no_repeat=nr, ut=ut,
            input_fnv=fnv1a_bytes(packed.tobytes()),
            tri_fnv=fnv1a_words(tri),
            head=tri[:8].tolist(),
        ))
        if E <= 64:
            small[key] = tri
        print(key, records[-1]["tri_fnv"], records[-1]["head"][:4])
    with open(os.path.join(HERE, "kat.json"), "w") as fh:
        json.dump(dict(
            source="reference CPU path (cpu_corr_test.c, input_generator.c) "
                   "built by oracle/Makefile",
            hash="64-bit FNV-1a; input over bytes, output over int32 words as uint32",
            cases=records), fh, indent=1)
    np.savez_compressed(os.path.join(HERE, "small_tri.npz"), **small)


if __name__ == "__main__":
    main()
