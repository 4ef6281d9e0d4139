"""Frame encoding through the plugin table (encoder_create / encoder_encode with the debug
taps, as the reference's testGpu does, tests/test_main.cpp:468-562) against the reference
CPU encoder itself (oracle/_ref: the CpuSlot built from the reference sources):

  * X'Y'Z' codes and quantised code-block words against the CpuSlot's own debug taps
    (FrameDebug::xyz12 / coeffs, src/core/cpu_backend.cpp:61-96);
  * wavelet planes against the reference fdwt97_2d on the reference colour planes (the
    CpuSlot has no wavelet tap);
  * Tier-1 of every code-block against the CpuSlot's Tier1Frame: nbps, pass count, every
    truncation length and distortion, the codeword bytes.

All bit-identical (the specification allows 1 in 10^5 quantised words off by one; the count
found is 0 and the tests require 0)."""
import numpy as np
import pytest

from libgail_b200 import plugin as P
from libgail_b200 import synth
from oracle.oracle import Planar, RefEncoder, Reference, have_reference

pytestmark = pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")


@pytest.fixture(scope="module")
def dev():
    d = P.Plugin().device(0)
    yield d
    d.close()


@pytest.fixture(scope="module")
def ref():
    return Reference()


def _ref_block(rt1, i):
    nbps, np_, off, ln, pb = (int(x) for x in rt1.info[i])
    return nbps, np_, bytes(rt1.data[off:off + ln]), rt1.pass_len[pb:pb + np_], rt1.pass_dist[pb:pb + np_]


def _compare_tier1(t1, rt1):
    """(blocks whose results differ, blocks whose pass count differs)."""
    n = rt1.info.shape[0]
    assert t1.info.shape[0] == n
    bad, stops = [], []
    for i in range(n):
        nbps, np_, data, pl, pd = t1.block(i)
        rn, rnp, rdata, rpl, rpd = _ref_block(rt1, i)
        if np_ != rnp:
            stops.append(i)
        elif np_ and (nbps != rn or data != rdata or not np.array_equal(pl, rpl) or not np.array_equal(pd, rpd)):
            bad.append(i)
    return bad, stops


def _frame_parity(dev, ref, width, height, fourk, fmt, col, frame, transfer, primaries, planar=None):
    lay = P.LayoutHolder(width, height, fourk)
    enc = dev.encoder(lay, fmt, col)
    try:
        t1, tm, taps = enc.encode(frame, debug=True)
    finally:
        enc.close()
    renc = RefEncoder(ref, width, height, fourk, transfer, primaries, planar=planar, threads=0)
    try:
        rt1 = renc.encode(frame, debug=True)
    finally:
        renc.close()
    assert np.array_equal(taps["xyz12"], rt1.xyz12), \
        f"{np.count_nonzero(taps['xyz12'] != rt1.xyz12)} X'Y'Z' codes differ from the reference CpuSlot"
    rgb = ref.planar_to_rgb48(planar, frame) if planar is not None else frame
    planes, _ = ref.color_frame(rgb, transfer, primaries)
    levels = 6 if fourk else 5
    wav = np.stack([ref.fdwt(planes[c], levels) for c in range(3)])
    got = taps["wavelet"].reshape(3, height, width)
    diff = np.count_nonzero(got.view(np.uint32) != wav.view(np.uint32))
    assert diff == 0, f"{diff} wavelet coefficients differ (max |d| {np.abs(got - wav).max()})"
    q = taps["coeffs"].reshape(-1, 1024)
    rq = rt1.coeffs.reshape(-1, 1024)
    nq = np.count_nonzero(q != rq)
    assert nq == 0, f"{nq} of {q.size} quantised words differ from the reference CpuSlot"
    bad, stops = _compare_tier1(t1, rt1)
    assert not bad and not stops, f"{len(bad) + len(stops)} of {rt1.info.shape[0]} code-blocks differ, " \
                                  f"first {(bad + stops)[:8]}"
    return t1, tm


@pytest.mark.gpu
def test_2k_xyz_frame_bit_exact(dev, ref):
    W, H = 1998, 1080
    rgb = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=11))
    t1, tm = _frame_parity(dev, ref, W, H, 0, P.rgb48_format(W, H), P.color_passthrough(), rgb, 5, 4)
    assert tm.symbols > 0 and t1.data.size > 0


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,fourk", [(333, 200, 1), (100, 77, 0), (2048, 858, 0), (4096, 1716, 1), (64, 64, 0),
                                        (65, 67, 1)])
def test_ragged_sizes_bit_exact(dev, ref, w, h, fourk):
    rgb = synth.xyz12_to_rgb48(synth.xyz12_planes(w, h, seed=5))
    _frame_parity(dev, ref, w, h, fourk, P.rgb48_format(w, h), P.color_passthrough(), rgb, 5, 4)


@pytest.mark.gpu
def test_largest_container_and_extreme_pictures(dev, ref):
    """The largest DCI container (4096 x 2160) with seeded content; then pictures at the
    ends of the code range: black (every X'Y'Z' code 0: after the DC shift only the lowest
    band codes anything), white (every code 4095) and a one-pixel checkerboard of both
    (every high band at its largest magnitudes)."""
    W, H = 4096, 2160
    rgb = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=17))
    _frame_parity(dev, ref, W, H, 1, P.rgb48_format(W, H), P.color_passthrough(), rgb, 5, 4)
    W, H = 1998, 1080
    yy, xx = np.mgrid[0:H, 0:W]
    for planes in (np.zeros((3, H, W), np.uint16), np.full((3, H, W), 4095, np.uint16),
                   np.broadcast_to((((yy + xx) & 1) * 4095).astype(np.uint16), (3, H, W)).copy()):
        _frame_parity(dev, ref, W, H, 0, P.rgb48_format(W, H), P.color_passthrough(), synth.xyz12_to_rgb48(planes),
                      5, 4)


@pytest.mark.gpu
def test_4k_yuv422_pq_frame_bit_exact(dev, ref):
    W, H = 3996, 2160
    frame = synth.yuv422p10(W, H, seed=21)
    fmt = P.planar_format(W, H, bits=10, sx=1, sy=0, kr=0.2627, kb=0.0593)
    pl = Planar(width=W, height=H, active_w=W, active_h=H, ox=0, oy=0, sx=1, sy=0, rgb=0, bits=10, full_range=0,
                chroma=0, kr=0.2627, kb=0.0593)
    _frame_parity(dev, ref, W, H, 1, fmt, P.color("pq", "bt2020"), frame, 2, 1, pl)


@pytest.mark.gpu
def test_planar_variants_bit_exact(dev, ref):
    """Letterboxed 4:2:0 8-bit BT.709 with centred chroma, full-range 4:4:4 12-bit, planar
    G'B'R' 10-bit and 16-bit, letterboxed 4:2:2 8-bit, and 4:2:0 12-bit with an odd active
    picture and left-sited chroma (the reference's GAIL_PIX_* planar formats, gail.h:125-141)."""
    for (aw, ah, bits, sx, sy, chroma, full, rgbf, kr, kb) in [(180, 101, 8, 1, 1, 1, 0, 0, 0.2126, 0.0722),
                                                               (200, 120, 12, 0, 0, 2, 1, 0, 0.299, 0.114),
                                                               (200, 120, 10, 0, 0, 0, 0, 1, 0.2627, 0.0593),
                                                               (200, 120, 16, 0, 0, 0, 1, 1, 0.2627, 0.0593),
                                                               (198, 108, 8, 1, 0, 0, 0, 0, 0.2126, 0.0722),
                                                               (199, 119, 12, 1, 1, 0, 0, 0, 0.2627, 0.0593)]:
        W, H = 200, 120
        rng = np.random.default_rng(bits + rgbf)
        cw, ch = (aw + sx) >> sx, (ah + sy) >> sy
        dt = np.uint8 if bits == 8 else np.uint16
        src = rng.integers(0, 1 << bits, aw * ah + 2 * cw * ch).astype(dt)
        fmt = P.planar_format(W, H, bits=bits, sx=sx, sy=sy, kr=kr, kb=kb, chroma=chroma, full_range=bool(full),
                              active=(aw, ah), rgb=bool(rgbf))
        pl = Planar(width=W, height=H, active_w=aw, active_h=ah, ox=(W - aw) // 2, oy=(H - ah) // 2, sx=sx, sy=sy,
                    rgb=rgbf, bits=bits, full_range=full, chroma=chroma, kr=kr, kb=kb)
        _frame_parity(dev, ref, W, H, 0, fmt, P.color("bt1886", "bt709"), src, 0, 0, pl)


@pytest.mark.gpu
def test_early_termination_frame(dev, ref):
    """Early termination with a fixed threshold against the reference CpuSlot at the same
    threshold: at least 99 % of the blocks make the reference's stop decision (the device
    log2f may differ from glibc's in the last place), and every block that does is
    bit-exact."""
    W, H = 1998, 1080
    rgb = synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=3))
    lay = P.LayoutHolder(W, H, 0)
    enc = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
    enc.set_slope(800.0)
    try:
        t1, _, _ = enc.encode(rgb, debug=True)
    finally:
        enc.close()
    renc = RefEncoder(ref, W, H, 0, 5, 4, threads=0)
    try:
        rt1 = renc.encode(rgb, slope=800.0)
    finally:
        renc.close()
    info = rt1.info
    stopped = np.count_nonzero((info[:, 1] > 0) & (info[:, 1] < 3 * info[:, 0] - 2))
    assert stopped > 100, "threshold too low to exercise the rule"
    bad, stops = _compare_tier1(t1, rt1)
    assert not bad, f"{len(bad)} blocks with the reference's stop decision differ"
    assert len(stops) <= 0.01 * info.shape[0], f"{len(stops)} stop decisions differ"
