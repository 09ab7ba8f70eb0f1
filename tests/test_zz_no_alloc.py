"""The allocation-free entry point chx_correlate_noalloc.

It serves callers that may not allocate device memory once they are running:
a real-time correlator loop whose memory is all reserved at start-up, where
cudaMalloc/cudaFree could stall the device's streams or fail, or where another
runtime owns the allocator.  Its work tables live in a fixed array inside the
library instead of in a plan.  These tests call it through the C ABI and check
it against chx_correlate, the plan-based entry point, bit for bit.  The file
is collected last so that a run stopping at the first failure has run every
other test before it.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")


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
    assert lib.chx_correlate_noalloc(None, fake, 256, 1, 256, 1, 0, None) == chimex.E_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("E,F,T,ut", [(2048, 4, 2048, 1), (384, 3, 1000, 0)])
def test_noalloc_matches_plan_entry_point_twice(E, F, T, ut):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chimex
    lib = chimex.lib()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(E * 7 + F + T)
    packed = torch.randint(0, 256, (T * F * E,), dtype=torch.uint8, device="cuda", generator=gen)
    plan = chimex.Plan(E, F, T, 256, ut, 0, 0)
    ref = plan.correlate(packed)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # the second call reuses the tables left by the first
        out = torch.full_like(ref, -1)
        rc = lib.chx_correlate_noalloc(ctypes.c_void_p(packed.data_ptr()),
                                       ctypes.c_void_p(out.data_ptr()), E, F, T, ut, 0, stream)
        assert rc == chimex.OK, lib.chx_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), "call %d differs from chx_correlate" % call
    # accumulate = 1 adds onto the existing buffer, like chx_correlate
    rc = lib.chx_correlate_noalloc(ctypes.c_void_p(packed.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), E, F, T, ut, 1, stream)
    assert rc == chimex.OK
    torch.cuda.synchronize()
    twice = (ref.cpu().numpy().astype(np.int64) * 2).astype(np.int32)
    assert np.array_equal(out.cpu().numpy(), twice)
