"""Tuning changes launch shapes and work order, never results: Tier-1 frames and decoded
pictures are bit-identical under extreme tunings."""
import numpy as np
import pytest

from libgail_b200 import autotune as AT
from libgail_b200 import codestream as CS
from libgail_b200 import plugin as P
from libgail_b200 import synth


@pytest.mark.gpu
def test_tuning_does_not_change_results():
    W, H = 1998, 1080
    dev = P.Plugin().device(0)
    lay = P.LayoutHolder(W, H, 0)
    frame = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=77))
    try:
        enc = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
        ref = enc.encode(frame)[0]
        cs = CS.rate_and_build(lay, ref, 24.0)[0]
        blocks = CS.parse(cs)[1].view(P.CBLK_CODE_DTYPE)
        dec = dev.decoder(lay)
        pic = dec.decode(cs, blocks)[0]
        for t in ({"soloDecisions": 256, "cmCtasPerSm": 1, "mqCtasPerSm": 1, "decCtasPerSm": 1},
                  {"soloDecisions": 1 << 30, "cmCtasPerSm": 64, "mqCtasPerSm": 64, "decCtasPerSm": 64}):
            AT.set_tuning(0, t)
            got = enc.encode(frame)[0]
            assert np.array_equal(got.info, ref.info) and np.array_equal(got.data, ref.data)
            assert np.array_equal(got.pass_len, ref.pass_len) and np.array_equal(got.pass_dist, ref.pass_dist)
            assert np.array_equal(dec.decode(cs, blocks)[0], pic)
        dec.close()
        enc.close()
    finally:
        AT.set_tuning(0, None)
        dev.close()


@pytest.mark.gpu
@pytest.mark.parametrize("W,H,fk,planar", [(1998, 1080, 0, False), (3996, 2160, 1, True), (2001, 1077, 0, False)])
def test_tile_shapes_give_the_same_coefficients(W, H, fk, planar):
    """Every front-end tile shape (64 x 64, 128 x 64, 64 x 128 at level 1 and at the later
    levels) gives the same X'Y'Z' codes, wavelet planes, quantised words and Tier-1 frame."""
    prof = 1 if fk else 0
    dev = P.Plugin().device(0)
    lay = P.LayoutHolder(W, H, fk)
    if planar:
        fmt, col = P.planar_format(W, H, bits=10, sx=1, sy=0), P.color("pq", "bt2020")
        frame = synth.yuv422p10(W, H, seed=91)
    else:
        fmt, col = P.rgb48_format(W, H), P.color_passthrough()
        frame = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=91))
    try:
        enc = dev.encoder(lay, fmt, col)
        ref, _, rtaps = enc.encode(frame, debug=True)
        for t1, tn in ((1, 0), (2, 0), (0, 1), (0, 2), (1, 2), (2, 1)):
            AT.set_tuning(prof, {"dwtTile1": t1, "dwtTileN": tn})
            got, _, taps = enc.encode(frame, debug=True)
            for k in ("xyz12", "coeffs"):
                assert np.array_equal(taps[k], rtaps[k]), f"tiles {t1}/{tn}: {k} differ"
            assert np.array_equal(taps["wavelet"].view(np.uint32), rtaps["wavelet"].view(np.uint32)), \
                f"tiles {t1}/{tn}: wavelet planes differ"
            assert np.array_equal(got.info, ref.info) and np.array_equal(got.data, ref.data)
            assert np.array_equal(got.pass_len, ref.pass_len) and np.array_equal(got.pass_dist, ref.pass_dist)
        enc.close()
    finally:
        AT.set_tuning(prof, None)
        dev.close()
