"""Decoding through the plugin table against the reference CPU decoder: codestreams made by
the reference CPU encoder (rate-controlled to the DCI budget, DCI-checked), parsed by the
reference's packet parser; the dequantised coefficients must be bit-identical to the CPU
decoder's and the picture within one code value of it (as the reference's testGpuDecode,
tests/test_main.cpp:2420-2499), at full and half size."""
import numpy as np
import pytest

from libgail_b200 import plugin as P
from libgail_b200 import synth
from oracle.oracle import Reference, RefEncoder, have_reference, ref_check, ref_codestream, ref_decode, ref_parse

pytestmark = pytest.mark.skipif(not have_reference(), reason="reference build not present")


@pytest.fixture(scope="module")
def dev():
    d = P.Plugin().device(0)
    yield d
    d.close()


def _codestream(W, H, fourk, seed):
    ref = Reference()
    planes = synth.xyz12_planes(W, H, seed=seed)
    enc = RefEncoder(ref, W, H, fourk)
    t1 = enc.encode(synth.xyz12_to_rgb48(planes))
    enc.close()
    cs, _, _, _ = ref_codestream(ref, W, H, fourk, t1, mbps=250.0)
    if (W, H) in ((1998, 1080), (2048, 858), (2048, 1080), (3996, 2160), (4096, 1716), (4096, 2160)):
        ok, msg = ref_check(ref, cs)  # the checker knows the DCI containers only
        assert ok, msg
    return ref, cs


@pytest.mark.gpu
@pytest.mark.parametrize("W,H,fourk,reduce,high", [(1998, 1080, 0, 0, False), (1998, 1080, 0, 1, False),
                                                   (1998, 1080, 0, 2, True), (3996, 2160, 1, 0, False),
                                                   (3996, 2160, 1, 1, False), (3996, 2160, 1, 2, False),
                                                   (333, 200, 1, 0, True), (64, 64, 0, 0, False),
                                                   (65, 67, 1, 1, False)])
def test_decode_matches_cpu(dev, W, H, fourk, reduce, high):
    """Full, half and quarter size; `high`: the codes in the high 12 bits of each word (the
    reference decoder's xyz12le output)."""
    ref, cs = _codestream(W, H, fourk, seed=7 + W)
    blocks, w, h, lv = ref_parse(ref, cs, reduce)
    lay = P.LayoutHolder(W, H, fourk)
    dec = dev.decoder(lay, reduce=reduce, high_bits=high)
    try:
        pic, tm, wl = dec.decode(cs, blocks.view(P.CBLK_CODE_DTYPE), wavelet=True)
    finally:
        dec.close()
    want, wref, _ = ref_decode(ref, cs, W, H, reduce, high_bits=high, wavelet=True)
    if high:  # the low four bits are zero on both sides; compare the codes
        assert not np.any(pic & 15) and not np.any(want & 15)
        pic, want = pic >> 4, want >> 4
    # coefficients of the decoded resolutions: bit-identical
    wl = wl.reshape(3, H, W)
    mask = np.zeros((H, W), bool)
    bands, _ = Reference().layout(W, H, fourk)
    for b in bands:
        if b.res <= lv - reduce:
            mask[b.py0:b.py0 + b.h, b.px0:b.px0 + b.w] = True
    diff = np.count_nonzero((wl.view(np.uint32) != wref.view(np.uint32)) & mask[None])
    assert diff == 0, f"{diff} dequantised coefficients differ"
    d = np.abs(pic.astype(np.int32) - want.astype(np.int32))
    assert d.max() <= 1, f"picture differs by up to {d.max()} codes"
    assert np.count_nonzero(d) <= 0.02 * d.size


@pytest.mark.gpu
def test_decode_damaged_input_stays_in_bounds(dev):
    """Blocks pointing past the codestream decode as zero; junk bytes decode to
    something without error."""
    W, H = 333, 200
    ref, cs = _codestream(W, H, 1, seed=1)
    blocks, _, _, _ = ref_parse(ref, cs, 0)
    b = blocks.copy()
    b["offset"][::3] = len(cs) + 100
    b["len"][1::5] = 0xFFFFFF
    lay = P.LayoutHolder(W, H, 1)
    dec = dev.decoder(lay)
    try:
        junk = bytes(np.random.default_rng(0).integers(0, 256, len(cs), dtype=np.uint8))
        pic, _, _ = dec.decode(junk, b.view(P.CBLK_CODE_DTYPE))
        pic2, _, _ = dec.decode(cs, blocks.view(P.CBLK_CODE_DTYPE))
    finally:
        dec.close()
    want, _, _ = ref_decode(ref, cs, W, H, 0)
    assert np.abs(pic2.astype(np.int32) - want.astype(np.int32)).max() <= 1


@pytest.mark.gpu
def test_decode_extreme_pictures(dev):
    """Codestreams of black, white and one-pixel checkerboard pictures (the checkerboard
    fills every high band at its largest magnitudes, truncated hard by the rate control):
    coefficients bit-identical to the reference CPU decoder's, picture within one code."""
    W, H, fk = 1998, 1080, 0
    ref = Reference()
    yy, xx = np.mgrid[0:H, 0:W]
    lay = P.LayoutHolder(W, H, fk)
    dec = dev.decoder(lay)
    try:
        for planes in (np.zeros((3, H, W), np.uint16), np.full((3, H, W), 4095, np.uint16),
                       np.broadcast_to((((yy + xx) & 1) * 4095).astype(np.uint16), (3, H, W)).copy()):
            enc = RefEncoder(ref, W, H, fk)
            t1 = enc.encode(synth.xyz12_to_rgb48(planes))
            enc.close()
            cs, _, _, _ = ref_codestream(ref, W, H, fk, t1, mbps=250.0)
            blocks, _, _, _ = ref_parse(ref, cs, 0)
            pic, _, wl = dec.decode(cs, blocks.view(P.CBLK_CODE_DTYPE), wavelet=True)
            want, wref, _ = ref_decode(ref, cs, W, H, 0, wavelet=True)
            assert np.array_equal(wl.reshape(3, H, W).view(np.uint32), wref.view(np.uint32))
            assert np.abs(pic.astype(np.int32) - want.astype(np.int32)).max() <= 1
    finally:
        dec.close()
