"""The bounded device-side waits that keep every tensor-core kernel from
hanging the GPU: a wait on a barrier that nothing completes must give up at
its time limit (or at once when the CTA's abort flag is raised), report it to
the host, and leave the context usable."""
import ctypes

import numpy as np
import pytest

import pyoracle as orc

torch = pytest.importorskip("torch")


def test_selftest_validates_arguments_without_device():
    import chimex as cx
    ms = ctypes.c_int()
    assert cx.lib().chx_selftest_bounded_wait(0, 7, ctypes.byref(ms)) == cx.E_INVALID


@pytest.mark.gpu
def test_wait_gives_up_at_the_limit_and_on_abort():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chimex as cx
    code, ms = cx.selftest_bounded_wait(mode=0)
    assert code == cx.E_TIMEOUT, cx.lib().chx_last_error()
    assert 1900 <= ms <= 4000, ms          # the 2 s limit
    code, ms = cx.selftest_bounded_wait(mode=1)
    assert code == cx.E_TIMEOUT
    assert ms < 500, ms                    # abort after ~10 ms, not the full limit
    # the context still works: a small correlation equals the oracle
    T, F, E = 64, 1, 256
    packed = orc.generate(T, F, E, 4, 5, no_repeat=1)
    p = cx.Plan(E, F, T, 64)
    out = p.correlate(torch.from_numpy(packed).cuda())
    p.check_device()
    np.testing.assert_array_equal(out.cpu().numpy(), orc.correlate_blocks(packed, T, F, E, 1))
