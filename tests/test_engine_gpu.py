"""The batched, served encoder: every frame's Tier-1 frame must be the same whether it was
encoded alone through the plain per-frame path (the plugin's encoder_encode) or in a mix
of frames of all six DCI profiles batched into shared Tier-1 launches, its PCRD hull points
computed on the GPU must equal the host's, and the admission by HBM budget must let every
request finish."""
import numpy as np
import pytest

from libgail_b200 import plugin as P
from libgail_b200 import synth
from libgail_b200.engine import Engine


def _same(a: P.Tier1Frame, b: P.Tier1Frame):
    return (np.array_equal(a.info, b.info) and np.array_equal(a.pass_len, b.pass_len)
            and np.array_equal(a.pass_dist, b.pass_dist) and np.array_equal(a.data, b.data))


def _same_hull(eng, rid, layout, t1):
    """The PCRD hull points the engine computed on the GPU equal the host's (themselves
    pinned to the reference's buildHull) bit for bit."""
    from libgail_b200 import codestream as CS
    gp, gs = eng.hull(rid, len(t1.pass_len))
    hp, hs = CS.hull(layout, t1)
    return np.array_equal(gp, hp) and np.array_equal(gs.view(np.uint64), hs.view(np.uint64))


@pytest.fixture(scope="module")
def dev():
    d = P.Plugin().device(0)
    yield d
    d.close()


# the six DCI profiles (width, height, 4K layout flag) and frames of each in the mix: 16
# X'Y'Z' 12-bit frames in all, plus two Y'CbCr 4:2:2 PQ 4K frames for the colour path
PROFILES = [(1998, 1080, 0, 3), (2048, 858, 0, 3), (2048, 1080, 0, 3), (3996, 2160, 1, 3), (4096, 1716, 1, 2),
            (4096, 2160, 1, 2)]


def _cases():
    # (layout args, format, colour, frames)
    out = []
    for W, H, fk, nf in PROFILES:
        frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=100 * (1 + fk) + W % 97 + i)) for i in range(nf)]
        out.append(((W, H, fk), P.rgb48_format(W, H), P.color_passthrough(), frames))
    W, H = 3996, 2160
    frames = [synth.yuv422p10(W, H, seed=200 + i) for i in range(2)]
    out.append(((W, H, 1), P.planar_format(W, H, bits=10, sx=1, sy=0), P.color("pq", "bt2020"), frames))
    return out


@pytest.mark.gpu
def test_engine_mix_equals_alone(dev):
    cases = _cases()
    alone = []
    for (W, H, fk), fmt, col, frames in cases:
        enc = dev.encoder(P.LayoutHolder(W, H, fk), fmt, col)
        alone.append([enc.encode(f)[0] for f in frames])
        enc.close()
    eng = Engine(0, 0, max_batch=16)
    try:
        layouts = [P.LayoutHolder(W, H, fk) for (W, H, fk), _, _, _ in cases]
        classes = [eng.add_encoder(lay, fmt, col)[0] for lay, (_, fmt, col, _) in zip(layouts, cases)]
        want = {}
        order = [(ci, fi) for fi in range(3) for ci in range(len(cases)) if fi < len(cases[ci][3])]
        assert sum(len(c[3]) for c in cases[:6]) == 16
        lay_of = {}
        for ci, fi in order:  # interleaved profiles
            rid = eng.submit(classes[ci], cases[ci][3][fi])
            want[rid] = alone[ci][fi]
            lay_of[rid] = layouts[ci]
        got = 0
        while got < len(want):
            rid, t1, lat, st = eng.wait(60000)
            assert rid >= 0, "timed out"
            assert st == 0
            assert _same(t1, want[rid]), f"request {rid} differs from its plain encode"
            assert _same_hull(eng, rid, lay_of[rid], t1), f"request {rid}: GPU hull differs from the host's"
            eng.release(rid)
            got += 1
        s = eng.stats()
        assert s["frames"] == len(want)
        assert s["batch_frames"] == len(want)
    finally:
        eng.close()


@pytest.mark.gpu
def test_engine_admission_by_budget(dev):
    """A budget of two 2K frame slots: ten requests still all finish, in bounded slots."""
    W, H = 1998, 1080
    frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=300 + i)) for i in range(10)]
    lay = P.LayoutHolder(W, H, 0)
    enc = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
    ref = [enc.encode(f)[0] for f in frames[:2]]
    enc.close()
    probe = Engine(0, 0, 4)
    _, per_frame = probe.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
    probe.close()
    eng = Engine(0, 2 * per_frame + 1, max_batch=4)
    try:
        cid, _ = eng.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
        ids = [eng.submit(cid, f) for f in frames]
        seen = 0
        while seen < len(ids):
            rid, t1, _, st = eng.wait(60000)
            assert rid >= 0 and st == 0
            if rid < 2:
                assert _same(t1, ref[rid])
            eng.release(rid)
            seen += 1
        assert eng.stats()["slots"] <= 2
    finally:
        eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [True, False])
def test_engine_codestreams(dev, on_device):
    """Codestreams made by the engine (rate control and Tier-2 on the device, or on the host
    workers): each equals the host codec's on the frame's plain Tier-1 output, passes the DCI
    check, and (for one frame) equals the reference's rate control and codestream on the same
    Tier-1 frame; the Tier-1 frames and hull points handed out alongside are the plain ones."""
    from libgail_b200 import codestream as CS
    from oracle.oracle import Reference, have_reference, ref_codestream
    cases = [c for c in _cases() if c[0] in ((1998, 1080, 0), (3996, 2160, 1))]
    alone = []
    for (W, H, fk), fmt, col, frames in cases:
        enc = dev.encoder(P.LayoutHolder(W, H, fk), fmt, col)
        alone.append([enc.encode(f)[0] for f in frames[:2]])
        enc.close()
    eng = Engine(0, 0, max_batch=8)
    try:
        layouts = [P.LayoutHolder(W, H, fk) for (W, H, fk), _, _, _ in cases]
        classes = [eng.add_encoder(lay, fmt, col)[0] for lay, (_, fmt, col, _) in zip(layouts, cases)]
        eng.set_codestream(fps=24.0, label=CS.DEFAULT_LABEL, tag="b200", threads=3, on_device=on_device, tier1=True)
        want = {}
        for fi in range(2):
            for ci in range(len(cases)):
                rid = eng.submit(classes[ci], cases[ci][3][fi])
                want[rid] = (ci, fi)
        for _ in want:
            rid, t1, _, st = eng.wait(120000)
            assert rid >= 0 and st == 0
            cs, ok = eng.codestream(rid)
            ci, fi = want[rid]
            assert _same(t1, alone[ci][fi])
            assert _same_hull(eng, rid, layouts[ci], t1)
            host, _, _ = CS.rate_and_build(layouts[ci], alone[ci][fi], fps=24.0, label=CS.DEFAULT_LABEL, tag="b200")
            assert cs == host
            assert ok == 1 and CS.check_dci(cs)[0]
            if have_reference() and fi == 0:
                (W, H, fk) = cases[ci][0]
                ref_cs, _, _, _ = ref_codestream(Reference(), W, H, fk, alone[ci][fi], fps=24.0, tag=b"b200")
                assert cs == ref_cs
            eng.release(rid)
    finally:
        eng.close()


@pytest.mark.gpu
def test_engine_device_codestreams_keep_tier1_on_device(dev):
    """Device rate control without Tier-1 frames in host memory: the codestreams are the host
    codec's, wait() hands out empty Tier-1 views, and far fewer bytes come back than the
    Tier-1 frames hold."""
    from libgail_b200 import codestream as CS
    W, H = 3996, 2160
    frames = [synth.yuv422p10(W, H, seed=600 + i) for i in range(3)]
    lay = P.LayoutHolder(W, H, 1)
    fmt, col = P.planar_format(W, H, bits=10, sx=1, sy=0), P.color("pq", "bt2020")
    enc = dev.encoder(lay, fmt, col)
    alone = [enc.encode(f)[0] for f in frames]
    enc.close()
    eng = Engine(0, 0, max_batch=4)
    try:
        cid, _ = eng.add_encoder(lay, fmt, col)
        eng.set_codestream(label=CS.DEFAULT_LABEL, tag="b200", threads=2)
        ids = [eng.submit(cid, f) for f in frames]
        for _ in ids:
            rid, t1, _, st = eng.wait(60000)
            assert st == 0 and len(t1.info) == 0
            cs, ok = eng.codestream(rid)
            assert ok == 1
            assert cs == CS.rate_and_build(lay, alone[ids.index(rid)], tag="b200")[0]
            eng.release(rid)
        h2d, d2h = eng.transfer_bytes()
        tier1_bytes = sum(len(t.data) + 17 * len(t.pass_len) + 20 * len(t.info) for t in alone)
        assert h2d == sum(f.nbytes for f in frames)
        assert d2h < tier1_bytes / 3
    finally:
        eng.close()


@pytest.mark.gpu
def test_slot_pipeline_codestreams(dev):
    """The plain path with slots gives each frame the same codestream as the engine."""
    from libgail_b200 import codestream as CS
    from libgail_b200.slots import SlotPipeline
    W, H = 1998, 1080
    frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=400 + i)) for i in range(5)]
    lay = P.LayoutHolder(W, H, 0)
    sp = SlotPipeline(dev, lay, P.rgb48_format(W, H), P.color_passthrough(), slots=2, tag="b200")
    try:
        res, _ = sp.run(frames)
    finally:
        sp.close()
    eng = Engine(0, 0, max_batch=4)
    try:
        cid, _ = eng.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
        eng.set_codestream(label=CS.DEFAULT_LABEL, tag="b200", threads=2)
        ids = [eng.submit(cid, f) for f in frames]
        got = {}
        for _ in ids:
            rid, _, _, st = eng.wait(60000)
            assert st == 0
            got[rid] = eng.codestream(rid)
            eng.release(rid)
    finally:
        eng.close()
    for i, rid in enumerate(ids):
        assert res[i][0] == got[rid][0] and res[i][1] and got[rid][1] == 1


@pytest.mark.gpu
def test_engine_mixed_encode_decode(dev):
    """Encode and decode requests of several profiles in one engine: every decode gives the
    picture the plugin's decoder gives alone, every encode its plain Tier-1 output."""
    from libgail_b200 import codestream as CS
    jobs = []  # (kind, class index, payload, expected)
    profiles = [(1998, 1080, 0), (3996, 2160, 1)]
    eng = Engine(0, 0, max_batch=8)
    try:
        enc_cls, dec_cls = {}, {}
        for W, H, fk in profiles:
            lay = P.LayoutHolder(W, H, fk)
            frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=500 + i + W)) for i in range(3)]
            enc = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
            t1s = [enc.encode(f)[0] for f in frames]
            enc.close()
            streams = [CS.rate_and_build(lay, t, 24.0)[0] for t in t1s]
            dec = dev.decoder(lay)
            pics = [dec.decode(cs, CS.parse(cs)[1].view(P.CBLK_CODE_DTYPE))[0] for cs in streams]
            dec.close()
            enc_cls[(W, H)] = eng.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())[0]
            dec_cls[(W, H)] = eng.add_decoder(lay)[0]
            for i in range(3):
                jobs.append(("enc", (W, H), frames[i], t1s[i]))
                jobs.append(("dec", (W, H), streams[i], pics[i]))
        want = {}
        for kind, key, payload, expect in jobs:  # interleaved kinds and profiles
            rid = eng.submit(enc_cls[key], payload) if kind == "enc" else eng.submit_decode(dec_cls[key], payload)
            want[rid] = (kind, expect)
        for _ in want:
            rid, t1, _, st = eng.wait(120000)
            assert rid >= 0 and st == 0
            kind, expect = want[rid]
            if kind == "enc":
                assert _same(t1, expect)
            else:
                assert np.array_equal(eng.picture(rid), expect)
            eng.release(rid)
    finally:
        eng.close()


@pytest.mark.gpu
def test_engine_early_termination(dev):
    """Early termination as libgail's pipeline drives it: each frame's threshold is the last
    frame's lambda x factor. Every codestream equals the one the plain encoder and the host
    codec give for the same frame at the threshold it was coded with (every pass when it was
    coded again) and is DCI-valid; at 0.25 the thresholds leave passes out; a factor that puts
    the threshold above the frame's own lambda makes the engine code it again with every pass."""
    from libgail_b200 import codestream as CS
    W, H = 1998, 1080
    frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=700 + i)) for i in range(4)]
    lay = P.LayoutHolder(W, H, 0)
    fmt, col = P.rgb48_format(W, H), P.color_passthrough()
    enc = dev.encoder(lay, fmt, col)
    eng = Engine(0, 0, max_batch=4)
    try:
        cid, _ = eng.add_encoder(lay, fmt, col)
        eng.set_codestream(label=CS.DEFAULT_LABEL, tag="b200", threads=2)
        for factor in (0.25, 1e9):
            eng.set_slope_factor(factor)
            active = recoded_n = 0
            for f in frames:  # one at a time: each threshold comes from the frame before
                rid = eng.submit(cid, f)
                got, _, _, st = eng.wait(60000)
                assert got == rid and st == 0
                cs, ok = eng.codestream(rid)
                thr, recoded = eng.frame_info(rid)
                eng.release(rid)
                assert ok == 1
                enc.set_slope(0.0 if recoded else thr)
                t1 = enc.encode(f)[0]
                assert cs == CS.rate_and_build(lay, t1, tag="b200")[0]
                if thr > 0 and not recoded:
                    active += 1
                    enc.set_slope(0.0)
                    assert len(t1.pass_len) < len(enc.encode(f)[0].pass_len)  # passes left out
                recoded_n += recoded
            if factor == 0.25:
                assert active >= 2
            else:
                assert recoded_n == len(frames)  # the first threshold comes from the 0.25 run
    finally:
        eng.close()
        enc.close()


@pytest.mark.gpu
def test_engine_reserve_makes_slots_up_front(dev):
    """Slots reserved before serving are the ones frames use (no slot is made while the
    burst runs), and a reservation stops at the HBM budget."""
    W, H = 1998, 1080
    lay = P.LayoutHolder(W, H, 0)
    frame = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=808))
    eng = Engine(0, 0, max_batch=4)
    try:
        cid, frame_bytes = eng.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
        assert eng.reserve(cid, 5) == 5
        assert eng.stats()["slots"] == 5
        assert eng.reserve(cid, 3) == 5  # it has five already
        ids = [eng.submit(cid, frame) for _ in range(5)]
        for _ in ids:
            rid, _, _, st = eng.wait(60000, copy=False)
            assert rid >= 0 and st == 0
            eng.release(rid)
        assert eng.stats()["slots"] == 5
    finally:
        eng.close()
    eng = Engine(0, 2 * frame_bytes + 1, max_batch=4)
    try:
        cid, _ = eng.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
        assert eng.reserve(cid, 5) == 2
    finally:
        eng.close()
