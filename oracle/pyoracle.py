"""ctypes binding of the CPU oracle (chx_oracle.c) and of the reference's own
CPU code (oracle/_ref/libchx_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, and there only as the checker.  The product
library never loads it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libchx_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libchx_ref.so")
REF_DRIVER = os.path.join(HERE, "_ref", "cpu_corr_ref")

_vp = ctypes.c_void_p
_lib = None
_ref = None


def build():
    """Compile the restatement (and the reference CPU code when present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        i, p = ctypes.c_int, _vp
        L.orc_generate.argtypes = [i] * 11 + [p]
        L.orc_num_blocks.restype = ctypes.c_int64
        L.orc_num_blocks.argtypes = [i]
        L.orc_correlate_blocks.argtypes = [p, i, i, i, i, i, p]
        L.orc_correlate_blocks_range.argtypes = [p, i, i, i, i, i, i, i, p]
        L.orc_correlate_triangle.argtypes = [p, i, i, i, i, p]
        L.orc_correlate_channel_mt.restype = i
        L.orc_correlate_channel_mt.argtypes = [p, i, i, i, i, i, i, i, i, p]
        L.orc_blocks_to_triangle.argtypes = [p, i, i, p]
        L.orc_blocks_to_full.argtypes = [p, i, i, p]
        L.orc_offset_accumulate.argtypes = [p, i, i, i, i, p]
        L.orc_preseed.argtypes = [p, i, i, i, i, i, p]
        L.orc_corr_partials.argtypes = [p, i, i, i, i, i, p]
        L.orc_fnv1a32.restype = ctypes.c_uint64
        L.orc_fnv1a32.argtypes = [p, ctypes.c_size_t]
        L.orc_weighted_power.restype = ctypes.c_int64
        L.orc_weighted_power.argtypes = [p, i, i, i, i, p]
        L.orc_weighted_from_blocks.restype = ctypes.c_int64
        L.orc_weighted_from_blocks.argtypes = [p, i, i, i, p]
        L.orc_visibility.argtypes = [p, i, i, i, i, i, i, p, p]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    """The reference's CPU routines compiled from its own sources."""
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
    return _ref


def _ptr(a):
    return a.ctypes.data_as(_vp)


def num_blocks(E):
    n = E // 32
    return n * (n + 1) // 2


def generate(T, F, E, gen=4, seed=42, default_re=0, default_im=0, initial_re=0,
             initial_im=0, single_freq=-1, no_repeat=0):
    out = np.zeros(T * F * E, dtype=np.uint8)
    lib().orc_generate(gen, seed, default_re, default_im, initial_re, initial_im,
                       single_freq, T, F, E, no_repeat, _ptr(out))
    return out


def ref_generate(T, F, E, gen=4, seed=42, default_re=0, default_im=0,
                 initial_re=0, initial_im=0, single_freq=-1, no_repeat=0):
    out = np.zeros(T * F * E, dtype=np.uint8)
    ref().generate_char_data_set(gen, seed, default_re, default_im, initial_re,
                                 initial_im, single_freq, T, F, E, no_repeat,
                                 _ptr(out))
    return out


def correlate_blocks(packed, T, F, E, ut=1, t0=0, t1=None, out=None):
    nb = num_blocks(E)
    acc = 1 if out is not None else 0
    if out is None:
        out = np.zeros(F * nb * 2048, dtype=np.int32)
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    lib().orc_correlate_blocks_range(_ptr(packed), T, F, E, t0,
                                     T if t1 is None else t1, ut, acc, _ptr(out))
    return out


def correlate_channel(packed, T, F, E, f, ut=1, t0=0, t1=None, threads=None):
    """Channel f's blocks int32[NB*2048] over samples [t0, t1), computed on
    `threads` host threads (default: every core); the same values as
    correlate_blocks for that channel."""
    out = np.empty(num_blocks(E) * 2048, dtype=np.int32)
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    n = threads or os.cpu_count() or 1
    rc = lib().orc_correlate_channel_mt(_ptr(packed), T, F, E, f, t0,
                                        T if t1 is None else t1, ut, n, _ptr(out))
    assert rc == 0, rc
    return out


def correlate_triangle(packed, T, F, E, ut=1):
    out = np.zeros(F * E * (E + 1), dtype=np.int32)
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    lib().orc_correlate_triangle(_ptr(packed), T, F, E, ut, _ptr(out))
    return out


def ref_correlate_triangle(T, F, E, gen=4, seed=42, default_re=0, default_im=0,
                           initial_re=0, initial_im=0, single_freq=-1,
                           no_repeat=0, ut=1):
    out = np.zeros(F * E * (E + 1), dtype=np.int32)
    fn = (ref().cpu_data_generate_and_correlate_upper_triangle_only if ut else
          ref().cpu_data_generate_and_correlate_upper_triangle_only_nonstandard_convention)
    err = fn(T, F, E, _ptr(out), gen, seed, default_re, default_im, initial_re,
             initial_im, single_freq, no_repeat, 0)
    assert err == 0
    return out


def ref_blocks_to_triangle(blocks, F, E):
    out = np.zeros(F * E * (E + 1), dtype=np.int32)
    blocks = np.ascontiguousarray(blocks, dtype=np.int32)
    ref().reorganize_GPU_to_upper_triangle(32, num_blocks(E), F, E, _ptr(blocks),
                                           _ptr(out))
    return out


def blocks_to_triangle(blocks, F, E):
    out = np.zeros(F * E * (E + 1), dtype=np.int32)
    blocks = np.ascontiguousarray(blocks, dtype=np.int32)
    lib().orc_blocks_to_triangle(_ptr(blocks), F, E, _ptr(out))
    return out


def blocks_to_full(blocks, F, E):
    out = np.zeros(F * E * E * 2, dtype=np.int32)
    blocks = np.ascontiguousarray(blocks, dtype=np.int32)
    lib().orc_blocks_to_full(_ptr(blocks), F, E, _ptr(out))
    return out


def offset_accumulate(packed, T, F, E, out=None):
    acc = 1 if out is not None else 0
    if out is None:
        out = np.zeros(F * E * 2, dtype=np.uint32)
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    lib().orc_offset_accumulate(_ptr(packed), T, F, E, acc, _ptr(out))
    return out


def preseed(sums, T, F, E, packed_variant=0, ut=1):
    out = np.zeros(F * num_blocks(E) * 2048, dtype=np.int32)
    sums = np.ascontiguousarray(sums, dtype=np.uint32)
    lib().orc_preseed(_ptr(sums), T, F, E, packed_variant, ut, _ptr(out))
    return out


def corr_partials(packed, T, F, E, packed_variant=0, ut=1, out=None):
    if out is None:
        out = np.zeros(F * num_blocks(E) * 2048, dtype=np.int32)
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    lib().orc_corr_partials(_ptr(packed), T, F, E, packed_variant, ut, _ptr(out))
    return out


def fnv1a(words):
    a = np.ascontiguousarray(words).view(np.int32).ravel()
    return "%016x" % lib().orc_fnv1a32(_ptr(a), a.size)


def fnv1a_bytes(b):
    h = 0xCBF29CE484222325
    b = np.ascontiguousarray(b, dtype=np.uint8).ravel()
    # Chunked pure-Python loop; only used on small inputs.
    for w in b.tolist():
        h ^= w
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return "%016x" % h


def weighted_power(packed, T, F, E, f, w):
    w = np.ascontiguousarray(w, dtype=np.int32)
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    return int(lib().orc_weighted_power(_ptr(packed), T, F, E, f, _ptr(w)))


def weighted_from_blocks(blocks, F, E, f, w):
    w = np.ascontiguousarray(w, dtype=np.int32)
    blocks = np.ascontiguousarray(blocks, dtype=np.int32)
    return int(lib().orc_weighted_from_blocks(_ptr(blocks), F, E, f, _ptr(w)))


def visibility(packed, T, F, E, f, y, x):
    re, im = ctypes.c_int32(), ctypes.c_int32()
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    lib().orc_visibility(_ptr(packed), T, F, E, f, y, x, ctypes.byref(re),
                         ctypes.byref(im))
    return re.value, im.value


def block_cell_offset(E, f, y, x):
    """int32 offset of (y, x)'s real part in the block layout (x >= 32*(y//32))."""
    nb1, nb = E // 32, num_blocks(E)
    by, bx = y // 32, x // 32
    b = by * nb1 - by * (by - 1) // 2 + (bx - by)
    return ((f * nb + b) * 32 + (y % 32)) * 64 + 2 * (x % 32)
