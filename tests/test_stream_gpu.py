"""Streaming correlation: frames submitted per channel, each completed
integration's dump must equal the oracle's blocks for exactly that
integration's samples; admission by HBM budget; latency statistics."""
import ctypes

import numpy as np
import pytest

import pyoracle as orc

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def chimex():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import chimex as cx
    return cx


def dump_of(s, c):
    t, seq = s.last_dump_tensor(c)
    return t.cpu().numpy(), seq


@pytest.mark.gpu
def test_stream_dumps_match_oracle(chimex):
    cx = chimex
    frame = 64
    s = cx.Stream(8, frame)
    layout = [(64, 128), (256, 192), (96, 64), (512, 256)]  # (E, time_accum)
    ids = [s.admit(E, ta) for E, ta in layout]
    rng = np.random.default_rng(5)
    history = {c: [] for c in ids}   # host frames per channel
    checked = 0
    for tick in range(12):
        # a varying subset of channels gets a frame each tick
        sub = [c for c in ids if (tick + c) % 3 != 0]
        frames, host = [], []
        for c in sub:
            E = layout[c][0]
            h = rng.integers(0, 256, size=(frame, E), dtype=np.uint8)
            frames.append(torch.from_numpy(h.reshape(-1)).cuda())
            host.append(h)
        s.submit(sub, frames)
        s.sync()
        for c, h in zip(sub, host):
            history[c].append(h)
            E, ta = layout[c]
            per = ta // frame
            if len(history[c]) % per == 0:
                seq = len(history[c]) // per - 1
                got, got_seq = dump_of(s, c)
                assert got_seq == seq
                x = np.concatenate(history[c][seq * per:(seq + 1) * per])
                ref = orc.correlate_blocks(x, ta, 1, E, 1).reshape(-1)
                np.testing.assert_array_equal(got, ref)
                checked += 1
    s.check_device()
    st = s.stats()
    assert st["dumps"] == checked and checked >= 8
    assert st["p99_ms"] >= st["p50_ms"] > 0
    s.close()


@pytest.mark.gpu
def test_stream_config5_shape_dumps_match_oracle(chimex):
    """The streaming workload's channel shape: E=2048 and E=1024 channels, time_accum 1024,
    frames of 256 samples, three integrations per channel with staggered
    starts (so completions of different channels fall on different ticks and
    on the same tick); every dump is compared word for word with the oracle
    for exactly its integration's frames."""
    cx = chimex
    frame, ta, nint = 256, 1024, 3
    layout = [2048, 1024, 2048, 1024, 2048]
    s = cx.Stream(len(layout), frame)
    ids = [s.admit(E, ta) for E in layout]
    per = ta // frame
    start = {c: (c * 3) % per for c in ids}   # first tick of channel c
    rng = np.random.default_rng(55)
    history = {c: [] for c in ids}
    checked = 0
    for tick in range(per * nint + per):
        sub = [c for c in ids if tick >= start[c] and len(history[c]) < per * nint]
        if not sub:
            continue
        host = [rng.integers(0, 256, size=(frame, layout[c]), dtype=np.uint8) for c in sub]
        s.submit(sub, [torch.from_numpy(h.reshape(-1)).cuda() for h in host])
        s.sync()
        for c, h in zip(sub, host):
            history[c].append(h)
            if len(history[c]) % per == 0:
                seq = len(history[c]) // per - 1
                got, got_seq = dump_of(s, c)
                assert got_seq == seq
                x = np.concatenate(history[c][seq * per:(seq + 1) * per]).reshape(-1)
                ref = orc.correlate_channel(x, ta, 1, layout[c], 0, 1)
                np.testing.assert_array_equal(got, ref, err_msg="channel %d dump %d" % (c, seq))
                checked += 1
    s.check_device()
    assert checked == len(layout) * nint
    assert s.stats()["dumps"] == checked
    s.close()


@pytest.mark.gpu
def test_stream_in_place_frames_reuse_ring(chimex):
    """Frames submitted in place (no copy) correlate what the ring holds: two
    integrations after a copied integration, the same ring half gives the
    same dump."""
    cx = chimex
    s = cx.Stream(2, 32)
    c = s.admit(128, 64)
    rng = np.random.default_rng(9)
    dumps = []
    for k in range(4):
        frames = [torch.from_numpy(rng.integers(0, 256, size=32 * 128, dtype=np.uint8)).cuda()
                  for _ in range(2)]
        for f in frames:
            s.submit([c], [f])
        s.sync()
        dumps.append(dump_of(s, c)[0])
    for k in range(2):
        for _ in range(2):
            s.submit([c], None)
        s.sync()
        got, seq = dump_of(s, c)
        assert seq == 4 + k
        np.testing.assert_array_equal(got, dumps[2 + k])
    s.close()


@pytest.mark.gpu
def test_stream_admission_by_budget(chimex):
    cx = chimex
    E, ta = 1024, 1024
    per = 2 * ta * E + 2 * orc.num_blocks(E) * 2048 * 4
    budget = 64 * 192 + 3 * per + per // 2   # channel table + 3.5 channels
    s = cx.Stream(64, 256, hbm_budget_bytes=budget)
    admitted = 0
    with pytest.raises(cx.ChimexError) as ei:
        for _ in range(10):
            s.admit(E, ta)
            admitted += 1
    assert ei.value.code == cx.E_ADMISSION
    assert admitted == 3
    assert s.stats()["resident_bytes"] <= budget
    s.close()


def test_stream_validation_without_device():
    import chimex as cx
    h = ctypes.c_void_p()
    lib = cx.lib()
    assert lib.chx_stream_create(ctypes.byref(h), 0, 256, 1, 0, 0) == cx.E_INVALID
    assert lib.chx_stream_create(ctypes.byref(h), 4, 100, 1, 0, 0) == cx.E_INVALID
    assert lib.chx_stream_create(ctypes.byref(h), 4, 256, 2, 0, 0) == cx.E_INVALID
    assert not h.value
    cid = ctypes.c_int()
    assert lib.chx_stream_admit(None, 256, 256, ctypes.byref(cid)) == cx.E_INVALID
    assert lib.chx_stream_submit(None, 0, None, None, None, None) == cx.E_INVALID
    assert lib.chx_stream_destroy(None) == cx.OK
