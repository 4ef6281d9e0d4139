"""Frame encoding through the plugin table (encoder_create / encoder_encode with the debug
taps, as the reference's testGpu does, tests/test_main.cpp:468-562) against the oracle:
X'Y'Z' codes, the wavelet planes and the quantised code-block words must be bit-identical
to the CPU path's, and Tier-1 bit-exact (bytes, truncation lengths, distortions) on every
code-block."""
import numpy as np
import pytest

from libgail_b200 import plugin as P
from libgail_b200 import synth
from oracle.oracle import Oracle, Planar


@pytest.fixture(scope="module")
def dev():
    d = P.Plugin().device(0)
    yield d
    d.close()


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def _check_tier1(o, t1, coeffs, bands, cblks, slope=0.0, dscale=None):
    geom = np.array([[k.w, k.h, bands[k.band].orient, 64] for k in cblks], np.int32)
    info, plen, pdist, words = o.t1_encode_many(coeffs.reshape(-1, 1024), geom, slope, dscale)
    n = len(cblks)
    assert t1.info.shape[0] == n
    bad, stops = [], []
    for i in range(n):
        nbps, np_, data, pl, pd = t1.block(i)
        if np_ != int(info[i, 1]):
            stops.append(i)
            continue
        if np_ and (nbps != int(info[i, 0]) or data != words[i] or not np.array_equal(pl, plen[i, :np_])
                    or not np.array_equal(pd, pdist[i, :np_])):
            bad.append(i)
    return bad + stops if slope == 0.0 else bad, info, stops


def _frame_parity(dev, o, width, height, fourk, fmt, col, frame, rgb48, transfer, primaries):
    lay = P.LayoutHolder(width, height, fourk)
    enc = dev.encoder(lay, fmt, col)
    try:
        t1, tm, taps = enc.encode(frame, debug=True)
    finally:
        enc.close()
    planes, xyz = o.color_frame(rgb48, transfer, primaries)
    assert np.array_equal(taps["xyz12"], xyz.ravel()), "X'Y'Z' codes differ"
    levels = 6 if fourk else 5
    wav = np.stack([o.fdwt(planes[c], levels) for c in range(3)])
    got = taps["wavelet"].reshape(3, height, width)
    diff = np.count_nonzero(got.view(np.uint32) != wav.view(np.uint32))
    assert diff == 0, f"{diff} wavelet coefficients differ (max |d| {np.abs(got - wav).max()})"
    bands, cblks = o.layout(width, height, fourk)
    q = o.quantize_frame(wav, bands, cblks)
    assert np.array_equal(taps["coeffs"].reshape(-1, 1024), q), "quantised words differ"
    bad, info, _ = _check_tier1(o, t1, q, bands, cblks)
    assert not bad, f"{len(bad)} of {len(cblks)} code-blocks differ, first {bad[:8]}"
    return t1, tm


@pytest.mark.gpu
def test_2k_xyz_frame_bit_exact(dev, oracle):
    W, H = 1998, 1080
    planes = synth.xyz12_planes(W, H, seed=11)
    rgb = synth.xyz12_to_rgb48(planes)
    t1, tm = _frame_parity(dev, oracle, W, H, 0, P.rgb48_format(W, H), P.color_passthrough(), rgb, rgb, 5, 4)
    assert tm.symbols > 0 and t1.data.size > 0


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,fourk", [(333, 200, 1), (100, 77, 0), (2048, 858, 0)])
def test_ragged_sizes_bit_exact(dev, oracle, w, h, fourk):
    planes = synth.xyz12_planes(w, h, seed=5)
    rgb = synth.xyz12_to_rgb48(planes)
    _frame_parity(dev, oracle, w, h, fourk, P.rgb48_format(w, h), P.color_passthrough(), rgb, rgb, 5, 4)


@pytest.mark.gpu
def test_4k_yuv422_pq_frame_bit_exact(dev, oracle):
    W, H = 3996, 2160
    frame = synth.yuv422p10(W, H, seed=21)
    fmt = P.planar_format(W, H, bits=10, sx=1, sy=0, kr=0.2627, kb=0.0593)
    pl = Planar(width=W, height=H, active_w=W, active_h=H, ox=0, oy=0, sx=1, sy=0, rgb=0, bits=10, full_range=0,
                chroma=0, kr=0.2627, kb=0.0593)
    rgb = oracle.planar_to_rgb48(pl, frame)
    _frame_parity(dev, oracle, W, H, 1, fmt, P.color("pq", "bt2020"), frame, rgb, 2, 1)


@pytest.mark.gpu
def test_planar_variants_bit_exact(dev, oracle):
    """Letterboxed 4:2:0 8-bit BT.709 with centred chroma, and full-range 4:4:4 12-bit."""
    for (aw, ah, bits, sx, sy, chroma, full, kr, kb) in [(180, 101, 8, 1, 1, 1, 0, 0.2126, 0.0722),
                                                         (200, 120, 12, 0, 0, 2, 1, 0.299, 0.114)]:
        W, H = 200, 120
        rng = np.random.default_rng(bits)
        cw, ch = (aw + sx) >> sx, (ah + sy) >> sy
        dt = np.uint8 if bits == 8 else np.uint16
        src = rng.integers(0, 1 << bits, aw * ah + 2 * cw * ch).astype(dt)
        fmt = P.planar_format(W, H, bits=bits, sx=sx, sy=sy, kr=kr, kb=kb, chroma=chroma, full_range=bool(full),
                              active=(aw, ah))
        pl = Planar(width=W, height=H, active_w=aw, active_h=ah, ox=(W - aw) // 2, oy=(H - ah) // 2, sx=sx, sy=sy,
                    rgb=0, bits=bits, full_range=full, chroma=chroma, kr=kr, kb=kb)
        rgb = oracle.planar_to_rgb48(pl, src)
        _frame_parity(dev, oracle, W, H, 0, fmt, P.color("bt1886", "bt709"), src, rgb, 0, 0)


@pytest.mark.gpu
def test_early_termination_frame(dev, oracle):
    """Early termination with a fixed threshold: at least 99% of the blocks make the CPU's
    stop decision, and every block that does is bit-exact."""
    W, H = 1998, 1080
    planes = synth.xyz12_planes(W, H, seed=3)
    rgb = synth.xyz12_to_rgb48(planes)
    lay = P.LayoutHolder(W, H, 0)
    enc = dev.encoder(lay, P.rgb48_format(W, H), P.color_passthrough())
    enc.set_slope(800.0)
    try:
        t1, _, taps = enc.encode(rgb, debug=True)
    finally:
        enc.close()
    bands, cblks = oracle.layout(W, H, 0)
    q = taps["coeffs"].reshape(-1, 1024)
    dscale = np.array([np.float32(np.float64(bands[k.band].delta) ** 2 * bands[k.band].weight) for k in cblks],
                      np.float32)
    bad, info, stops = _check_tier1(oracle, t1, q, bands, cblks, 800.0, dscale)
    stopped = np.count_nonzero((info[:, 1] > 0) & (info[:, 1] < 3 * info[:, 0] - 2))
    assert stopped > 100, "threshold too low to exercise the rule"
    assert not bad, f"{len(bad)} blocks with the CPU's stop decision differ"
    assert len(stops) <= 0.01 * len(cblks), f"{len(stops)} stop decisions differ"
