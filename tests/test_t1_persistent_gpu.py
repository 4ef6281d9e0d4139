"""Tier-1 encoding as one persistent launch (tuning knob t1Persistent): its warps take
context modelling, the largest-first order, MQ coding and truncation lengths from device
queues in turn. Its Tier-1 frames must equal the four-launch path's byte for byte: single
frames through the plain encoder (2K and 4K, every pass and with early termination), and
16 frames of all six DCI profiles plus two Y'CbCr PQ frames batched into shared launches by
the engine. Its bounded waits give up with a status bit instead of hanging."""
import numpy as np
import pytest

from libgail_b200 import autotune as AT
from libgail_b200 import plugin as P
from libgail_b200 import synth
from libgail_b200.engine import Engine


def _same(a: P.Tier1Frame, b: P.Tier1Frame):
    return (np.array_equal(a.info, b.info) and np.array_equal(a.pass_len, b.pass_len)
            and np.array_equal(a.pass_dist, b.pass_dist) and np.array_equal(a.data, b.data))


def _persistent(on: bool):
    for prof in (0, 1):
        AT.set_tuning(prof, {"t1Persistent": 1} if on else None)


@pytest.fixture(scope="module")
def dev():
    d = P.Plugin().device(0)
    yield d
    _persistent(False)
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("W,H,fk", [(1998, 1080, 0), (3996, 2160, 1)])
def test_plain_encoder_one_launch_equals_four(dev, W, H, fk):
    """Each mode has its own encoder, so that no table of the persistent launch holds the
    four-launch results beforehand."""
    frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=900 + fk + i)) for i in range(3)]
    lay = P.LayoutHolder(W, H, fk)
    four = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
    one = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
    try:
        for slope in (0.0, 800.0):  # every pass; early termination at a fixed threshold
            four.set_slope(slope)
            one.set_slope(slope)
            _persistent(False)
            want = [four.encode(f)[0] for f in frames]
            _persistent(True)
            for rep in range(2):  # the work area is cleared for every launch
                for f, w in zip(frames, want):
                    got = one.encode(f)[0]
                    assert _same(got, w), f"slope {slope}, pass {rep}: the persistent launch differs"
            if slope > 0:  # the threshold left passes out
                four.set_slope(0.0)
                _persistent(False)
                assert len(want[0].pass_len) < len(four.encode(frames[0])[0].pass_len)
    finally:
        _persistent(False)
        four.close()
        one.close()


@pytest.mark.gpu
def test_engine_batches_one_launch_equals_four(dev):
    """16 X'Y'Z' frames over the six DCI profiles and two Y'CbCr 4:2:2 PQ 4K frames, submitted
    interleaved to an engine batching up to 18 frames: every frame's Tier-1 frame equals its
    plain four-launch encode."""
    profiles = [(1998, 1080, 0, 3), (2048, 858, 0, 3), (2048, 1080, 0, 3), (3996, 2160, 1, 3), (4096, 1716, 1, 2),
                (4096, 2160, 1, 2)]
    cases = []
    for W, H, fk, nf in profiles:
        frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=300 + 7 * fk + W % 89 + i)) for i in range(nf)]
        cases.append(((W, H, fk), P.rgb48_format(W, H), P.color_passthrough(), frames))
    W, H = 3996, 2160
    cases.append(((W, H, 1), P.planar_format(W, H, bits=10, sx=1, sy=0), P.color("pq", "bt2020"),
                  [synth.yuv422p10(W, H, seed=330 + i) for i in range(2)]))
    _persistent(False)
    alone = []
    for (W, H, fk), fmt, col, frames in cases:
        enc = dev.encoder(P.LayoutHolder(W, H, fk), fmt, col)
        alone.append([enc.encode(f)[0] for f in frames])
        enc.close()
    _persistent(True)
    eng = Engine(0, 0, max_batch=18)
    try:
        layouts = [P.LayoutHolder(W, H, fk) for (W, H, fk), _, _, _ in cases]
        classes = [eng.add_encoder(lay, fmt, col)[0] for lay, (_, fmt, col, _) in zip(layouts, cases)]
        want = {}
        for fi in range(3):  # interleaved profiles
            for ci, (_, _, _, frames) in enumerate(cases):
                if fi < len(frames):
                    want[eng.submit(classes[ci], frames[fi])] = alone[ci][fi]
        for _ in range(len(want)):
            rid, t1, _, st = eng.wait(60000)
            assert rid >= 0, "timed out"
            assert st == 0
            assert _same(t1, want[rid]), f"request {rid} differs from its plain four-launch encode"
            eng.release(rid)
        s = eng.stats()
        assert s["frames"] == len(want) and s["batch_frames"] == len(want)
    finally:
        eng.close()
        _persistent(False)


@pytest.mark.gpu
def test_queue_wait_gives_up_and_the_device_stays_usable(dev):
    """The launch's failure detection without a fault: a wait on a flag that nothing sets,
    its limit lowered to 200 ms, returns with the queue-wait status bit after about that
    long, and a frame encoded afterwards equals one encoded before."""
    import ctypes as C

    import libgail_b200 as gb
    L = gb.lib()
    L.gb_t1_wait_selftest.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]
    W, H = 1998, 1080
    frame = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=404))
    enc = dev.encoder(P.LayoutHolder(W, H, 0), P.rgb48_format(W, H), P.color_passthrough())
    try:
        before = enc.encode(frame)[0]
        status, ms = C.c_uint32(), C.c_float()
        gb.check(L.gb_t1_wait_selftest(200, C.byref(status), C.byref(ms)))
        assert status.value == 16, f"status {status.value}"
        assert 190.0 <= ms.value <= 1200.0, f"the wait took {ms.value:.1f} ms"
        assert _same(enc.encode(frame)[0], before)
    finally:
        enc.close()
    with pytest.raises(gb.GailError):
        gb.check(L.gb_t1_wait_selftest(0, C.byref(status), None))
