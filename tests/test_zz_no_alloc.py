"""The allocation-free entry point chx_correlate_noalloc.

It serves callers that may not allocate device memory once they are running:
a real-time correlator loop whose memory is all reserved at start-up, where
cudaMalloc/cudaFree could stall the device's streams or fail, or where another
runtime owns the allocator.  Its work tables live in a fixed array inside the
library instead of in a plan, written there by a small kernel on every call.
These tests call it through the C ABI and check it bit for bit against
chx_correlate, the plan-based entry point, and against the CPU oracle, on two
calls in a row (the second call reuses the array the first one left).  The
file is collected last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes

import numpy as np
import pytest

import pyoracle as orc

torch = pytest.importorskip("torch")


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_noalloc_rejects_sizes_beyond_its_tables():
    """F above 64, or more than 4096 work units, fails before any CUDA call."""
    import chimex
    lib = chimex.lib()
    fake = ctypes.c_void_p(256)
    rc = lib.chx_correlate_noalloc(fake, fake, 256, 65, 256, 1, 0, None)
    assert rc == chimex.E_UNSUPPORTED
    assert b"at most 64 channels" in lib.chx_last_error()
    rc = lib.chx_correlate_noalloc(fake, fake, 4096, 40, 256, 1, 0, None)  # 40 x 136 units
    assert rc == chimex.E_UNSUPPORTED
    assert b"work units" in lib.chx_last_error()
    rc = lib.chx_correlate_noalloc(fake, fake, 2048, 60, 3 * 262144, 1, 0, None)  # 60 x 36 x 3
    assert rc == chimex.E_UNSUPPORTED
    assert lib.chx_correlate_noalloc(None, fake, 256, 1, 256, 1, 0, None) == chimex.E_INVALID
    assert lib.chx_correlate_noalloc(fake, ctypes.c_void_p(260), 256, 1, 256, 1, 0,
                                     None) == chimex.E_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("E,F,T,ut", [(2048, 4, 2048, 1), (384, 3, 1000, 0)])
def test_noalloc_matches_plan_entry_point_twice(E, F, T, ut):
    _need_gpu()
    import chimex
    lib = chimex.lib()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(E * 7 + F + T)
    packed = torch.randint(0, 256, (T * F * E,), dtype=torch.uint8, device="cuda", generator=gen)
    plan = chimex.Plan(E, F, T, 256, ut, 0, 0)
    ref = plan.correlate(packed)
    for call in range(2):  # the second call reuses the tables left by the first
        out = torch.full_like(ref, -1)
        rc = lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, ut, 0, _stream())
        assert rc == chimex.OK, lib.chx_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), "call %d differs from chx_correlate" % call
    # accumulate = 1 adds onto the existing buffer, like chx_correlate
    rc = lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, ut, 1, _stream())
    assert rc == chimex.OK
    torch.cuda.synchronize()
    twice = (ref.cpu().numpy().astype(np.int64) * 2).astype(np.int32)
    assert np.array_equal(out.cpu().numpy(), twice)
    assert lib.chx_noalloc_check(_stream()) == chimex.OK, lib.chx_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("E,F,T,ut", [(256, 2, 300, 1), (640, 1, 200, 0), (128, 3, 250, 1)])
def test_noalloc_matches_oracle_twice(E, F, T, ut):
    """Seeded reference-generator input, both tile variants (E=256 and 640,
    an odd tile count: SM pair; E=128: one SM), compared word for word with
    the CPU oracle."""
    _need_gpu()
    import chimex
    lib = chimex.lib()
    host = orc.generate(T, F, E, 4, 42, no_repeat=1)
    ref = orc.correlate_blocks(host, T, F, E, ut)
    packed = torch.from_numpy(host).cuda()
    for call in range(2):
        out = torch.full((F * orc.num_blocks(E) * 2048,), -1, dtype=torch.int32, device="cuda")
        rc = lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, ut, 0, _stream())
        assert rc == chimex.OK, lib.chx_last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), ref, err_msg="call %d" % call)
    assert lib.chx_noalloc_check(_stream()) == chimex.OK


@pytest.mark.gpu
def test_noalloc_split_ranges_meet_by_reduce_add():
    """T just above the 262144-sample unit limit: every tile pair becomes two
    units whose results meet by TMA reduce-add in the output, which the call
    zeroes first unless it accumulates."""
    _need_gpu()
    import chimex
    lib = chimex.lib()
    E, F, T = 256, 1, 262144 + 4096
    gen = torch.Generator(device="cuda")
    gen.manual_seed(17)
    packed = torch.randint(0, 256, (T * F * E,), dtype=torch.uint8, device="cuda", generator=gen)
    plan = chimex.Plan(E, F, T, 256, 1, 0, 0)
    ref = plan.correlate(packed)
    out = torch.full_like(ref, 12345)
    for call in range(2):
        rc = lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, 1, 0, _stream())
        assert rc == chimex.OK, lib.chx_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), "call %d" % call
    rc = lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, 1, 1, _stream())
    assert rc == chimex.OK
    torch.cuda.synchronize()
    assert torch.equal(out, ref * 2)
    assert lib.chx_noalloc_check(_stream()) == chimex.OK


@pytest.mark.gpu
def test_noalloc_check_reports_a_recorded_timeout_once():
    """A bounded wait that gives up records a code in the entry point's error
    word (the self-test writes it the way a correlator CTA would); the check
    reports it once and clears it, and the next call is unaffected."""
    _need_gpu()
    import chimex
    lib = chimex.lib()
    assert lib.chx_noalloc_check(_stream()) == chimex.OK
    code, ms = chimex.selftest_bounded_wait(mode=2)
    assert code == chimex.E_TIMEOUT and ms < 500
    assert lib.chx_noalloc_check(_stream()) == chimex.E_TIMEOUT
    assert b"0x1000" in lib.chx_last_error()
    assert lib.chx_noalloc_check(_stream()) == chimex.OK
    E, F, T = 256, 1, 64
    host = orc.generate(T, F, E, 4, 3, no_repeat=1)
    out = torch.empty(orc.num_blocks(E) * 2048, dtype=torch.int32, device="cuda")
    packed = torch.from_numpy(host).cuda()
    assert lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, 1, 0, _stream()) == chimex.OK
    assert lib.chx_noalloc_check(_stream()) == chimex.OK
    np.testing.assert_array_equal(out.cpu().numpy(), orc.correlate_blocks(host, T, F, E, 1))


@pytest.mark.gpu
def test_noalloc_full_size_matches_plan_entry_point():
    """The full-size plain workload (E=2048, F=8, T=16384: 288 SM-pair units)
    through the allocation-free entry point, twice, against chx_correlate."""
    _need_gpu()
    import chimex
    lib = chimex.lib()
    E, F, T = 2048, 8, 16384
    gen = torch.Generator(device="cuda")
    gen.manual_seed(2048)
    packed = torch.randint(0, 256, (T * F * E,), dtype=torch.uint8, device="cuda", generator=gen)
    ref = chimex.Plan(E, F, T, 256, 1, 0, 0).correlate(packed)
    out = torch.full_like(ref, -1)
    for call in range(2):
        rc = lib.chx_correlate_noalloc(_vp(packed), _vp(out), E, F, T, 1, 0, _stream())
        assert rc == chimex.OK, lib.chx_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), "call %d" % call
    assert lib.chx_noalloc_check(_stream()) == chimex.OK
