"""The managed colour routes on the GPU against the reference CPU encoder, as the reference's
own GPU colour test compares its backends (tests/test_main.cpp:965-1060, testGpuColor):
an HDR PQ BT.2020 source through the shoulder and BT.2390 tone maps on each norm with gamut
compression, HLG, the tone-map-free settings, and application 3D LUTs (in memory and by
.cube path), each encoded through the plugin table with the debug taps and compared with
the reference CpuSlot's taps (FrameDebug::xyz12 / coeffs) on the same frame:

  * every route without a power function on the way (shoulder tone maps, gamut
    compression, the 3D LUTs, the tone-map-free settings): X'Y'Z' codes and quantised
    code-block words identical;
  * the BT.2390 routes, which take each value to PQ and back (four chained powers, two of
    them to the 78.8th power or its inverse): X'Y'Z' codes at most one apart on at most 1 in
    10^4 pixels. The GPU's powers are correctly rounded; the host C library's powf is not
    (glibc 2.39 differs from the correctly rounded power on 0.07-0.12 % of arguments), and
    the 78.8th power turns one such difference into a code now and then. A code one off
    moves the quantised words of the wavelet coefficients it feeds, so those are counted
    and reported, not held to 1 in 10^5. The reference's own GPU backend is allowed 2 % of
    codes one off on these routes.

The counts found are reported in the failure message; the engine's batched front end is
checked to give the plain path's Tier-1 frame on two of the routes."""
import numpy as np
import pytest

from libgail_b200 import plugin as P
from oracle.oracle import RefEncoder, Reference, have_reference, ref_color

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")]

W, H = 1998, 1080


def hdr_frame(w, h, seed):
    """Interleaved 16-bit R'G'B' over the whole PQ range: saturated random colours (gamut
    and per-channel tone stages), a grey ramp with small channel offsets (the knee and the
    curve's top), smooth colour gradients, and a near-black band."""
    rng = np.random.default_rng(seed)
    a = h // 4
    f = np.empty((h, w, 3), np.uint16)
    f[:a] = rng.integers(0, 65536, (a, w, 3))
    ramp = np.linspace(0, 65535, w)
    f[a:2 * a] = np.clip(ramp[None, :, None] + rng.normal(0, 1500, (a, w, 3)), 0, 65535)
    yy, xx = np.mgrid[0:a, 0:w]
    f[2 * a:3 * a] = np.stack([xx * 65535 // (w - 1), yy * 65535 // (a - 1), (xx + yy) * 40000 // (w + a)], -1)
    f[3 * a:] = rng.integers(0, 12000, (h - 3 * a, w, 3))
    return f


def _sin_lut(n):
    return np.array([0.5 + 0.4 * np.sin(i * 0.7 + c) for i in range(n ** 3) for c in range(3)], np.float32)


def _identity_lut(n):
    return np.array([v / (n - 1) for b in range(n) for g in range(n) for r in range(n) for v in (r, g, b)],
                    np.float32)


HDR = dict(transfer="pq", primaries="bt2020", hdr_peak=4000.0, gamut="p3d65")
MODES = {
    "pq-shoulder-channel": dict(HDR, tone_map="shoulder", tone_norm="channel"),
    "pq-shoulder-maxrgb": dict(HDR, tone_map="shoulder", tone_norm="maxrgb"),
    "pq-shoulder-luminance": dict(HDR, tone_map="shoulder", tone_norm="luminance"),
    "pq-bt2390-channel": dict(HDR, tone_map="bt2390", tone_norm="channel"),
    "pq-bt2390-maxrgb-dcip3": dict(HDR, tone_map="bt2390", tone_norm="maxrgb", gamut="dcip3", hdr_peak=1000.0),
    "pq-bt2390-luminance-nogamut": dict(HDR, tone_map="bt2390", tone_norm="luminance", gamut="none"),
    "hlg-shoulder-channel": dict(transfer="hlg", primaries="bt2020", tone_map="shoulder", gamut="p3d65"),
    "bt1886-gamut-only": dict(transfer="bt1886", primaries="bt709", gamut="dcip3", gamut_threshold=0.5),
    "pq-signal": dict(transfer="pq", primaries="bt2020"),
    "lut3d-5-sin": dict(transfer="bt1886", primaries="bt709", lut="sin5"),
    "lut3d-17-identity": dict(transfer="bt1886", primaries="bt709", lut="id17"),
    "lut3d-cube-path": dict(transfer="bt1886", primaries="bt709", lut="cube9"),
}


def _colours(mode, tmp_path):
    kw = dict(MODES[mode])
    lut = kw.pop("lut", None)
    lut_kw = {}
    if lut == "sin5":
        lut_kw = dict(lut=_sin_lut(5), lut_size=5)
    elif lut == "id17":
        lut_kw = dict(lut=_identity_lut(17), lut_size=17)
    elif lut == "cube9":
        data = _sin_lut(9).reshape(-1, 3)
        path = tmp_path / "nine.cube"
        path.write_text("# a 9^3 LUT\nTITLE \"nine\"\nLUT_3D_SIZE 9\n" +
                        "".join(f"{r:.6f} {g:.6f} {b:.6f}\n" for r, g, b in data))
        lut_kw = dict(lut_path=str(path))
    mine = P.color_managed(**kw, **{k: v for k, v in lut_kw.items()})
    rkw = dict(transfer=P.TRANSFER[kw.pop("transfer")], primaries=P.PRIMARIES[kw.pop("primaries")],
               tone_map=P.TONE_MAP[kw.pop("tone_map", "signal")],
               tone_norm=P.TONE_NORM[kw.pop("tone_norm", "channel")], gamut=P.GAMUT[kw.pop("gamut", "none")])
    if "lut_path" in lut_kw:
        rkw["lut_path"] = lut_kw["lut_path"].encode()
    elif lut_kw:
        rkw.update(lut=lut_kw["lut"], lut_size=lut_kw["lut_size"])
    rkw.update(kw)
    return mine, ref_color(**rkw)


@pytest.fixture(scope="module")
def dev():
    d = P.Plugin().device(0)
    yield d
    d.close()


@pytest.fixture(scope="module")
def frame():
    return hdr_frame(W, H, 77)


@pytest.mark.parametrize("mode", list(MODES))
def test_color_route_against_reference(dev, frame, mode, tmp_path):
    mine, theirs = _colours(mode, tmp_path)
    route, _, _ = P.color_route(mine)
    lay = P.LayoutHolder(W, H, 0)
    enc = dev.encoder(lay, P.rgb48_format(W, H), mine)
    try:
        _, _, taps = enc.encode(frame, debug=True)
    finally:
        enc.close()
    renc = RefEncoder(Reference(), W, H, 0, color=theirs, threads=0)
    try:
        rt1 = renc.encode(frame, debug=True)
    finally:
        renc.close()
    d = np.abs(taps["xyz12"].astype(np.int32) - rt1.xyz12.astype(np.int32))
    ncodes = int(np.count_nonzero(d))
    q, rq = taps["coeffs"], rt1.coeffs
    nq = int(np.count_nonzero(q != rq))
    msg = f"route {route}: {ncodes} of {d.size} X'Y'Z' codes differ (max {d.max()}), {nq} of {q.size} quantised words"
    print(mode, msg)
    if "bt2390" in mode:
        assert d.max() <= 1, msg
        assert ncodes <= d.size * 1e-4, msg
    else:
        assert ncodes == 0 and nq == 0, msg
    if mode.startswith("lut"):
        assert route == 2
    elif mode == "pq-signal":
        assert route == 0
    else:
        assert route == 1


def test_engine_route_equals_plain(dev, frame, tmp_path):
    """The engine's front end takes the same route constants and LUT as the plain encoder."""
    from libgail_b200.engine import Engine
    lay = P.LayoutHolder(W, H, 0)
    for mode in ("pq-bt2390-channel", "lut3d-5-sin"):
        mine, _ = _colours(mode, tmp_path)
        enc = dev.encoder(lay, P.rgb48_format(W, H), mine)
        want = enc.encode(frame)[0]
        enc.close()
        eng = Engine(0, 0, max_batch=4)
        try:
            cid, _ = eng.add_encoder(lay, P.rgb48_format(W, H), mine)
            rid = eng.submit(cid, frame)
            got_id, t1, _, st = eng.wait(60000)
            assert got_id == rid and st == 0
            assert (np.array_equal(t1.info, want.info) and np.array_equal(t1.pass_len, want.pass_len)
                    and np.array_equal(t1.data, want.data)), f"{mode}: engine differs from the plain encoder"
            eng.release(rid)
        finally:
            eng.close()
