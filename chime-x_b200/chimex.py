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
_sig("chx_noalloc_check", _i, [_vp])
_sig("chx_selftest_bounded_wait", _i, [_i, _i, ctypes.POINTER(_i)])


class ChannelDesc(ctypes.Structure):
    """chx_channel_desc: one channel of a batch."""
    _fields_ = [("num_elements", _i), ("num_timesamples", _i), ("num_integrations", _i),
                ("input_stride", _i64), ("d_packed", _vp), ("d_blocks", _vp)]


class StreamStats(ctypes.Structure):
    """chx_stream_stats."""
    _fields_ = [("frames", _i64), ("dumps", _i64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("resident_bytes", _i64)]


_sig("chx_batch_create", _i, [ctypes.POINTER(_vp), _i, ctypes.POINTER(ChannelDesc), _i, _i])
_sig("chx_batch_run", _i, [_vp, _vp, _i])
_sig("chx_batch_work_units", _i64, [_vp])
_sig("chx_batch_ops", ctypes.c_double, [_vp])
_sig("chx_batch_check", _i, [_vp, _vp])
_sig("chx_batch_destroy", _i, [_vp])
_sig("chx_autotune", _i, [_i, _i, _vp, _vp, _vp, ctypes.POINTER(_i), ctypes.POINTER(_i),
                          ctypes.POINTER(ctypes.c_double)])
_sig("chx_stream_create", _i, [ctypes.POINTER(_vp), _i, _i, _i, _i64, _i])
_sig("chx_stream_admit", _i, [_vp, _i, _i, ctypes.POINTER(_i)])
_sig("chx_stream_frame_slot", _i, [_vp, _i, ctypes.POINTER(_vp)])
_sig("chx_stream_submit", _i, [_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_vp),
                               ctypes.POINTER(_i64), _vp])
_sig("chx_stream_last_dump", _i, [_vp, _i, ctypes.POINTER(_vp), ctypes.POINTER(_i64)])
_sig("chx_stream_stats_get", _i, [_vp, ctypes.POINTER(StreamStats)])
_sig("chx_stream_reset_stats", _i, [_vp])
_sig("chx_stream_check", _i, [_vp])
_sig("chx_stream_sync", _i, [_vp])
_sig("chx_stream_destroy", _i, [_vp])

EXPORTED = [
    "chx_version", "chx_last_error", "chx_plan_create", "chx_plan_destroy",
    "chx_plan_set_option", "chx_plan_block_words", "chx_plan_input_bytes",
    "chx_plan_sum_words", "chx_plan_triangle_words", "chx_correlate",
    "chx_offset_accumulate", "chx_preseed", "chx_corr_compat", "chx_blocks_to_triangle",
    "chx_blocks_to_full", "chx_plan_check", "chx_correlate_noalloc", "chx_noalloc_check",
    "chx_selftest_bounded_wait",
    "chx_batch_create", "chx_batch_run", "chx_batch_work_units", "chx_batch_ops",
    "chx_batch_check", "chx_batch_destroy", "chx_autotune", "chx_stream_create",
    "chx_stream_admit", "chx_stream_frame_slot", "chx_stream_submit", "chx_stream_last_dump",
    "chx_stream_stats_get", "chx_stream_reset_stats", "chx_stream_check", "chx_stream_sync",
    "chx_stream_destroy",
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


class _DeviceArray:
    """A raw device allocation seen through __cuda_array_interface__."""

    def __init__(self, addr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (addr, False), "version": 3}


def device_view(addr, n, dtype="int32", device=0):
    """A torch tensor viewing n words at device address addr (no copy)."""
    import torch
    ts = {"int32": "<i4", "uint8": "|u1", "uint32": "<u4"}[dtype]
    return torch.as_tensor(_DeviceArray(addr, n, ts), device=torch.device("cuda", device))


def selftest_bounded_wait(mode=0, device=0):
    """Runs the bounded-wait self-test (chx_selftest_bounded_wait); returns
    (status code, elapsed ms).  CHX_E_TIMEOUT is the expected status."""
    ms = _i()
    code = _lib.chx_selftest_bounded_wait(device, mode, ctypes.byref(ms))
    return code, ms.value


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


def noalloc_check(stream=None):
    """chx_noalloc_check: raises ChimexError(E_TIMEOUT) when a bounded device
    wait of chx_correlate_noalloc gave up since the last check."""
    check(_lib.chx_noalloc_check(_stream(stream)))


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


def autotune(E, T, scratch_in, scratch_out, stream=None):
    """Times the tile variants and sample splits for channels of (E, T) on the
    current device (chx_autotune), on enough channels to fill the GPU (it
    allocates temporary buffers beyond the one channel of scratch given);
    returns (tile, split, ms) and caches the tile for later plans and
    batches, which choose their own split."""
    tile, split, ms = _i(), _i(), ctypes.c_double()
    check(_lib.chx_autotune(E, T, _ptr(scratch_in), _ptr(scratch_out), _stream(stream),
                            ctypes.byref(tile), ctypes.byref(split), ctypes.byref(ms)))
    return tile.value, split.value, ms.value


class Batch:
    """Many channels (own E, integration length and count) in one persistent
    launch captured in a CUDA graph (chx_batch_*).

    channels: list of (packed, blocks, E, T, n_integrations[, input_stride]),
    packed a uint8 CUDA tensor of n_integrations*T samples (stride bytes
    apart, default E), blocks an int32 CUDA tensor of n_integrations*NB*2048.
    The tensors must stay alive while the batch is used."""

    def __init__(self, channels, upper_triangle_convention=1, device=0):
        n = len(channels)
        arr = (ChannelDesc * n)()
        self._keep = []
        for k, ch in enumerate(channels):
            packed, blocks, E, T, nint = ch[:5]
            stride = ch[5] if len(ch) > 5 else 0
            if blocks.numel() < nint * num_blocks(E) * 2048:
                raise ValueError("channel %d: blocks too small" % k)
            if packed.numel() < ((nint * T - 1) * (stride or E) + E):
                raise ValueError("channel %d: packed too small" % k)
            arr[k] = ChannelDesc(E, T, nint, stride, packed.data_ptr(), blocks.data_ptr())
            self._keep.append((packed, blocks))
        self.device = device
        h = ctypes.c_void_p()
        check(_lib.chx_batch_create(ctypes.byref(h), n, arr, upper_triangle_convention, device))
        self._h = h

    def run(self, accumulate=False, stream=None):
        check(_lib.chx_batch_run(self._h, _stream(stream), 1 if accumulate else 0))

    @property
    def work_units(self):
        return _lib.chx_batch_work_units(self._h)

    @property
    def ops(self):
        return _lib.chx_batch_ops(self._h)

    def check_device(self, stream=None):
        check(_lib.chx_batch_check(self._h, _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            _lib.chx_batch_destroy(self._h)
            self._h = None
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Stream:
    """Streaming correlation (chx_stream_*): frames of frame_len samples per
    channel; each channel's integration of time_accum samples is correlated
    and dumped as soon as its last frame is submitted."""

    def __init__(self, max_channels, frame_len, upper_triangle_convention=1,
                 hbm_budget_bytes=0, device=0):
        h = ctypes.c_void_p()
        check(_lib.chx_stream_create(ctypes.byref(h), max_channels, frame_len,
                                     upper_triangle_convention, hbm_budget_bytes, device))
        self._h = h
        self.frame_len = frame_len
        self.device = device
        self.elements = []

    def admit(self, E, time_accum):
        cid = _i()
        check(_lib.chx_stream_admit(self._h, E, time_accum, ctypes.byref(cid)))
        self.elements.append(E)
        return cid.value

    def frame_slot(self, cid):
        p = ctypes.c_void_p()
        check(_lib.chx_stream_frame_slot(self._h, cid, ctypes.byref(p)))
        return p.value

    def submit(self, ids, frames=None, arrival_ns=None, stream=None):
        """ids: channel ids (or a prepared ctypes int array); frames: None
        (already in place) or a list of uint8 CUDA tensors / device addresses."""
        n = len(ids)
        ids_arr = ids if isinstance(ids, ctypes.Array) else (_i * n)(*ids)
        fr = None
        if frames is not None:
            fr = (_vp * n)(*[f if isinstance(f, int) else f.data_ptr() for f in frames])
        arr = None
        if arrival_ns is not None:
            arr = arrival_ns if isinstance(arrival_ns, ctypes.Array) else (_i64 * n)(*arrival_ns)
        check(_lib.chx_stream_submit(self._h, n, ids_arr, fr, arr, _stream(stream)))

    def last_dump(self, cid):
        """(device address or None, sequence number) of the last completed dump."""
        p, seq = ctypes.c_void_p(), _i64()
        check(_lib.chx_stream_last_dump(self._h, cid, ctypes.byref(p), ctypes.byref(seq)))
        return p.value, seq.value

    def last_dump_tensor(self, cid):
        """(int32 tensor view of the last completed dump, or None; sequence)."""
        addr, seq = self.last_dump(cid)
        if not addr:
            return None, seq
        return device_view(addr, num_blocks(self.elements[cid]) * 2048, "int32",
                           self.device), seq

    def stats(self):
        st = StreamStats()
        check(_lib.chx_stream_stats_get(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in StreamStats._fields_}

    def reset_stats(self):
        check(_lib.chx_stream_reset_stats(self._h))

    def sync(self):
        """Waits until every submitted launch is complete and published."""
        check(_lib.chx_stream_sync(self._h))

    def check_device(self):
        check(_lib.chx_stream_check(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.chx_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
