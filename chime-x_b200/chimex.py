"""Python host binding of libchimex (ctypes over the C ABI in include/chimex.h).

Mirrors the reference's correlator_test pipeline (main_wrapper.c) with the
same argument meaning: a Plan fixes E (num_elements), F (num_freq), T
(time_steps), time_accum, upper_triangle_convention and kernel_batch, like
the -D build options of main_wrapper.c:310.  Device buffers are torch CUDA
tensors (uint8 packed input [T][F][E], int32 block output [F][NB][32][32][2]);
torch only provides memory and streams, every computation runs in
libchimex's CUDA kernels.  There is no CPU fallback: importing this module
without a built libchimex.so raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchimex.so")

OK = 0
E_INVALID, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_TIMEOUT, E_NOT_READY, E_ADMISSION = \
    -1, -2, -3, -4, -5, -6, -7
KERNEL_CONFERENCE, KERNEL_PACKED = 0, 1
ALGO_AUTO, ALGO_SIMT, ALGO_TC = 0, 1, 2
OPT_ALGO, OPT_TSPLIT, OPT_TILE = 1, 2, 3

_ERRNAMES = {E_INVALID: "CHX_E_INVALID", E_UNSUPPORTED: "CHX_E_UNSUPPORTED",
             E_CUDA: "CHX_E_CUDA", E_NOMEM: "CHX_E_NOMEM", E_TIMEOUT: "CHX_E_TIMEOUT",
             E_NOT_READY: "CHX_E_NOT_READY", E_ADMISSION: "CHX_E_ADMISSION"}


class ChimexError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (_ERRNAMES.get(code, str(code)), msg))
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError("libchimex.so is not built (run python chime-x_b200/build.py)")

_lib = ctypes.CDLL(LIB_PATH)
_vp, _i, _i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


_sig("chx_version", ctypes.c_char_p, [])
_sig("chx_last_error", ctypes.c_char_p, [])
_sig("chx_plan_create", _i, [ctypes.POINTER(_vp), _i, _i, _i, _i, _i, _i, _i])
_sig("chx_plan_destroy", _i, [_vp])
_sig("chx_plan_set_option", _i, [_vp, _i, _i64])
for _n in ("chx_plan_block_words", "chx_plan_input_bytes", "chx_plan_sum_words",
           "chx_plan_triangle_words"):
    _sig(_n, _i64, [_vp])
_sig("chx_correlate", _i, [_vp, _vp, _vp, _vp, _i])
_sig("chx_offset_accumulate", _i, [_vp, _vp, _vp, _vp, _i])
_sig("chx_preseed", _i, [_vp, _vp, _vp, _vp])
_sig("chx_corr_compat", _i, [_vp, _vp, _vp, _vp])
_sig("chx_blocks_to_triangle", _i, [_vp, _vp, _vp, _vp])
_sig("chx_blocks_to_full", _i, [_vp, _vp, _vp, _vp])
_sig("chx_plan_check", _i, [_vp, _vp])
_sig("chx_correlate_noalloc", _i, [_vp, _vp, _i, _i, _i, _i, _i, _vp])

EXPORTED = [
    "chx_version", "chx_last_error", "chx_plan_create", "chx_plan_destroy",
    "chx_plan_set_option", "chx_plan_block_words", "chx_plan_input_bytes",
    "chx_plan_sum_words", "chx_plan_triangle_words", "chx_correlate",
    "chx_offset_accumulate", "chx_preseed", "chx_corr_compat", "chx_blocks_to_triangle",
    "chx_blocks_to_full", "chx_plan_check", "chx_correlate_noalloc",
]


def lib():
    return _lib


def version():
    return _lib.chx_version().decode()


def check(code):
    if code != OK:
        raise ChimexError(code, _lib.chx_last_error().decode())
    return code


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def num_blocks(E):
    n = E // 32
    return n * (n + 1) // 2


def correlate_noalloc(packed, blocks, E, F, T, upper_triangle_convention=1, accumulate=False,
                      stream=None):
    """chx_correlate_noalloc: the fused correlator without a plan and without
    any allocation (for loops that must not allocate); `blocks` must already
    hold F*NB*2048 int32."""
    check(_lib.chx_correlate_noalloc(_ptr(packed), _ptr(blocks), E, F, T,
                                     upper_triangle_convention, 1 if accumulate else 0,
                                     _stream(stream)))
    return blocks


class Plan:
    """One correlator configuration (the -D sizes of main_wrapper.c:310)."""

    def __init__(self, num_elements, num_freq, num_timesamples, time_accum=256,
                 upper_triangle_convention=1, kernel_batch=KERNEL_CONFERENCE, device=0):
        self.E, self.F, self.T = num_elements, num_freq, num_timesamples
        self.time_accum = time_accum
        self.ut = upper_triangle_convention
        self.kernel_batch = kernel_batch
        self.device = device
        h = ctypes.c_void_p()
        check(_lib.chx_plan_create(ctypes.byref(h), num_elements, num_freq, num_timesamples,
                                   time_accum, upper_triangle_convention, kernel_batch, device))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.chx_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # sizes
    @property
    def block_words(self):
        return _lib.chx_plan_block_words(self._h)

    @property
    def input_bytes(self):
        return _lib.chx_plan_input_bytes(self._h)

    @property
    def sum_words(self):
        return _lib.chx_plan_sum_words(self._h)

    @property
    def triangle_words(self):
        return _lib.chx_plan_triangle_words(self._h)

    def set_option(self, option, value):
        check(_lib.chx_plan_set_option(self._h, option, int(value)))
        return self

    def _dev(self):
        import torch
        return torch.device("cuda", self.device)

    def _check_input(self, packed):
        import torch
        if packed.dtype != torch.uint8 or not packed.is_cuda or not packed.is_contiguous():
            raise ValueError("packed must be a contiguous uint8 CUDA tensor")
        if packed.numel() != self.input_bytes:
            raise ValueError("packed has %d bytes, plan needs %d" % (packed.numel(), self.input_bytes))

    def _out(self, t, n, dtype):
        import torch
        if t is None:
            return torch.empty(n, dtype=dtype, device=self._dev())
        if t.dtype != dtype or not t.is_cuda or not t.is_contiguous() or t.numel() != n:
            raise ValueError("output tensor must be a contiguous %s CUDA tensor of %d" % (dtype, n))
        return t

    def correlate(self, packed, blocks=None, accumulate=False, stream=None):
        """Fused exact correlator into the block layout (chx_correlate)."""
        import torch
        self._check_input(packed)
        blocks = self._out(blocks, self.block_words, torch.int32)
        check(_lib.chx_correlate(self._h, _ptr(packed), _ptr(blocks), _stream(stream),
                                 1 if accumulate else 0))
        return blocks

    def offset_accumulate(self, packed, sums=None, accumulate=False, stream=None):
        import torch
        self._check_input(packed)
        sums = self._out(sums, self.sum_words, torch.int32)
        check(_lib.chx_offset_accumulate(self._h, _ptr(packed), _ptr(sums), _stream(stream),
                                         1 if accumulate else 0))
        return sums

    def preseed(self, sums, blocks=None, stream=None):
        import torch
        blocks = self._out(blocks, self.block_words, torch.int32)
        check(_lib.chx_preseed(self._h, _ptr(sums), _ptr(blocks), _stream(stream)))
        return blocks

    def corr_compat(self, packed, blocks, stream=None):
        import torch
        self._check_input(packed)
        blocks = self._out(blocks, self.block_words, torch.int32)
        check(_lib.chx_corr_compat(self._h, _ptr(packed), _ptr(blocks), _stream(stream)))
        return blocks

    def reference_pipeline(self, packed, stream=None):
        """offsetAccumulate -> preseed -> corr, as main_wrapper.c:693-777 runs it."""
        sums = self.offset_accumulate(packed, stream=stream)
        blocks = self.preseed(sums, stream=stream)
        return self.corr_compat(packed, blocks, stream=stream)

    def blocks_to_triangle(self, blocks, tri=None, stream=None):
        import torch
        tri = self._out(tri, self.triangle_words, torch.int32)
        check(_lib.chx_blocks_to_triangle(self._h, _ptr(blocks), _ptr(tri), _stream(stream)))
        return tri

    def blocks_to_full(self, blocks, full=None, stream=None):
        import torch
        full = self._out(full, self.F * self.E * self.E * 2, torch.int32)
        check(_lib.chx_blocks_to_full(self._h, _ptr(blocks), _ptr(full), _stream(stream)))
        return full

    def check_device(self, stream=None):
        check(_lib.chx_plan_check(self._h, _stream(stream)))
