"""The CPU oracle (oracle/gail_oracle.c, the C restatement) pinned to the reference.

Two anchors:
  * the committed golden fixtures made by the reference itself (tests/golden/make_golden.py):
    the reference tests' random code-block suites (testT1Truncation seed 42, testT1PassLimit
    seed 9, tests/test_main.cpp:340-393, :652-676) with the reference coder's outputs, and
    small frames through the reference encoder's front end (planarToRgb48, the CpuSlot's
    X'Y'Z' and quantised-word taps, fdwt97_2d);
  * the reference CPU path compiled from its sources (oracle/_ref/libgailref.so), where it
    is present: odd-size forward / inverse 9/7, every colour route the encoder takes on
    random pixels and all 4096 pass-through codes, planar variants, the frame quantiser and
    the block decoder at every truncation point.
The GPU parity tests compare the CUDA path with the reference directly; these tests make
the restatement a checked stand-in wherever the reference build is absent."""
import os
import zlib

import numpy as np
import pytest

from oracle.oracle import Oracle, Planar, Reference, have_reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not have_reference(), reason="reference build not present")


@pytest.fixture(scope="module")
def o():
    return Oracle()


@pytest.fixture(scope="module")
def ref():
    return Reference()


@pytest.fixture(scope="module")
def fe():
    return np.load(os.path.join(ROOT, "tests", "golden", "front_end.npz"))


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


# ---- Tier-1 against the golden suites -------------------------------------------------

def test_t1_encode_matches_golden_suites(o, golden_t1):
    """Every block of both suites with their pass limits: nbps, passes, truncation lengths,
    distortions and codeword bytes as the reference coded them."""
    g = golden_t1
    info, plen, pdist, words = o.t1_encode_many(g["coeffs"], g["meta"])
    ofs = g["s0_data_ofs"]
    assert np.array_equal(info[:, 1].astype(np.int32), g["s0_passes"])
    for i in range(len(g["meta"])):
        np_ = int(g["s0_passes"][i])
        if np_:
            assert int(info[i, 0]) == int(g["s0_nbps"][i]), f"block {i}: nbps"
        assert words[i] == bytes(g["s0_data"][ofs[i]:ofs[i + 1]]), f"block {i}: codeword"
        assert np.array_equal(plen[i, :np_], g["s0_pass_len"][i, :np_]), f"block {i}: pass lengths"
        assert np.array_equal(pdist[i, :np_], g["s0_pass_dist"][i, :np_]), f"block {i}: distortions"


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_t1_early_termination_matches_golden(o, golden_t1, variant):
    """Early termination at three thresholds with per-block distortion scales: the same
    stop decisions and, by CRC-32, the same codewords. The stop rule calls log2f, which
    glibc evaluates the same way in both builds, so every block must agree."""
    g = golden_t1
    meta = g["meta"].copy()
    meta[:, 3] = 64
    info, plen, pdist, words = o.t1_encode_many(g["coeffs"], meta, float(g["slopes"][variant]), g["dscale"])
    assert np.array_equal(info[:, 1].astype(np.int32), g[f"s{variant}_passes"])
    crc = np.array([zlib.crc32(w) for w in words], np.uint32)
    assert np.array_equal(crc, g[f"s{variant}_crc"])
    for i in range(len(meta)):
        np_ = int(info[i, 1])
        assert np.array_equal(plen[i, :np_], g[f"s{variant}_pass_len"][i, :np_])
        assert np.array_equal(pdist[i, :np_], g[f"s{variant}_pass_dist"][i, :np_])


@needs_ref
def test_t1_decode_every_truncation_point_matches_reference(o, ref, golden_t1):
    """The block decoder on the golden codewords cut at every truncation point (the
    reference's testT1Truncation decodes each prefix): the restatement's words equal the
    reference decoder's."""
    g = golden_t1
    ofs = g["s0_data_ofs"]
    points = 0
    for i in range(0, len(g["meta"]), 5):
        w, h, orient, _ = (int(x) for x in g["meta"][i])
        nbps, np_ = int(g["s0_nbps"][i]), int(g["s0_passes"][i])
        data = bytes(g["s0_data"][ofs[i]:ofs[i + 1]])
        for k in range(np_):
            n = int(g["s0_pass_len"][i, k])
            want = ref.t1_decode(data[:n], w, h, orient, nbps, k + 1)
            got = o.t1_decode(data[:n], w, h, orient, nbps, k + 1)
            assert np.array_equal(got, want), f"block {i} pass {k}"
            points += 1
    assert points > 2000


# ---- front end against the golden frames ----------------------------------------------

def _planar_from(geom, krkb):
    w, h, aw, ah, bits, sx, sy, chroma, full, rgb = (int(x) for x in geom)
    return Planar(width=w, height=h, active_w=aw, active_h=ah, ox=(w - aw) // 2, oy=(h - ah) // 2, sx=sx, sy=sy,
                  rgb=rgb, bits=bits, full_range=full, chroma=chroma, kr=float(krkb[0]), kb=float(krkb[1]))


@pytest.mark.parametrize("name", ["yuv420p8_letterbox", "yuv444p12_full", "gbrp10"])
def test_planar_variants_match_golden(o, fe, name):
    pl = _planar_from(fe[f"{name}_geom"], fe[f"{name}_krkb"])
    assert np.array_equal(o.planar_to_rgb48(pl, fe[f"{name}_input"]), fe[f"{name}_rgb48"])


@pytest.mark.parametrize("name", ["xyz2k", "pq4k"])
def test_front_end_matches_golden(o, fe, name):
    """X'Y'Z' codes, wavelet planes and quantised words of the reference encoder, bit for
    bit, for a pass-through 2K-profile frame and a 4:2:2 PQ 4K-profile frame."""
    w, h, fourk, transfer, primaries = (int(x) for x in fe[f"{name}_geom"])
    frame = fe[f"{name}_input"]
    if name == "pq4k":
        pl = Planar(width=w, height=h, active_w=w, active_h=h, ox=0, oy=0, sx=1, sy=0, rgb=0, bits=10, full_range=0,
                    chroma=0, kr=0.2627, kb=0.0593)
        rgb = o.planar_to_rgb48(pl, frame)
        assert np.array_equal(rgb, fe[f"{name}_rgb48"])
    else:
        rgb = frame
    planes, xyz = o.color_frame(rgb, transfer, primaries)
    assert np.array_equal(xyz, fe[f"{name}_xyz12"]), "X'Y'Z' codes"
    wav = np.stack([o.fdwt(planes[c], 6 if fourk else 5) for c in range(3)])
    assert np.array_equal(_bits(wav), _bits(fe[f"{name}_wavelet"])), "wavelet planes"
    bands, cblks = o.layout(w, h, fourk)
    assert np.array_equal(o.quantize_frame(wav, bands, cblks), fe[f"{name}_coeffs"]), "quantised words"


# ---- front end against the reference build --------------------------------------------

@needs_ref
@pytest.mark.parametrize("w,h,levels", [(333, 200, 6), (100, 77, 5), (17, 3, 5), (1, 9, 5), (64, 64, 6),
                                        (1998, 1080, 5)])
def test_dwt_odd_sizes_match_reference(o, ref, w, h, levels):
    rng = np.random.default_rng(w * 1000 + h)
    plane = rng.uniform(-2048, 2048, (h, w)).astype(np.float32)
    f_o, f_r = o.fdwt(plane, levels), ref.fdwt(plane, levels)
    assert np.array_equal(_bits(f_o), _bits(f_r)), "forward 9/7"
    for skip in (0, 1):
        assert np.array_equal(_bits(o.idwt(f_r, levels, skip)), _bits(ref.idwt(f_r, levels, skip))), \
            f"inverse 9/7, {skip} levels skipped"


ROUTES = [("gamma26", "xyz", 5, 4), ("pq", "bt2020", 2, 1), ("bt1886", "bt709", 0, 0), ("srgb", "p3d65", 1, 2),
          ("linear", "dcip3", 4, 3), ("hlg", "bt2020", 3, 1), ("pq", "p3d65", 2, 2)]


@needs_ref
@pytest.mark.parametrize("tname,pname,transfer,primaries", ROUTES)
def test_color_per_pixel_matches_reference(o, ref, tname, pname, transfer, primaries):
    """Random 16-bit R'G'B' pixels plus the full range of each channel: the float planes
    (after the DC shift and ICT) and the 12-bit X'Y'Z' codes of every pixel."""
    rng = np.random.default_rng(transfer * 10 + primaries)
    rgb = rng.integers(0, 65536, (256, 257, 3)).astype(np.uint16)
    rgb[0, :, :] = np.linspace(0, 65535, 257).astype(np.uint16)[:, None]
    p_o, x_o = o.color_frame(rgb, transfer, primaries)
    p_r, x_r = ref.color_frame(rgb, transfer, primaries)
    assert np.array_equal(x_o, x_r), f"{np.count_nonzero(x_o != x_r)} X'Y'Z' codes differ"
    assert np.array_equal(_bits(p_o), _bits(p_r)), "colour planes differ"


@needs_ref
def test_pass_through_all_codes_match_reference(o, ref):
    """Every 12-bit X'Y'Z' code through the public API's 16-bit fill comes back as itself
    (the reference's testXyzPassThrough, tests/test_main.cpp:886-901), in both builds."""
    v = np.arange(4096, dtype=np.uint32)
    rgb = np.repeat(((v * 65535 + 2047) // 4095).astype(np.uint16)[:, None], 3, 1).reshape(64, 64, 3)
    _, x_o = o.color_frame(rgb, 5, 4)
    _, x_r = ref.color_frame(rgb, 5, 4)
    assert np.array_equal(x_r[..., 0].ravel(), v)
    assert np.array_equal(x_o, x_r)


@needs_ref
def test_planar_variants_match_reference(o, ref):
    rng = np.random.default_rng(3)
    cases = [(3996, 64, 3996, 64, 10, 1, 0, 0, 0, 0, 0.2627, 0.0593),   # 4:2:2 PQ rows at 4K width
             (333, 201, 301, 181, 8, 1, 1, 1, 0, 0, 0.2126, 0.0722),   # odd 4:2:0 letterbox, centred chroma
             (200, 120, 200, 120, 12, 0, 0, 2, 1, 0, 0.299, 0.114),    # 4:4:4 full range
             (128, 65, 127, 63, 10, 1, 1, 2, 0, 0, 0.2627, 0.0593),    # 4:2:0 top-left chroma, odd active
             (96, 50, 96, 50, 16, 0, 0, 0, 1, 1, 0.2627, 0.0593)]      # planar G'B'R' 16-bit
    for (w, h, aw, ah, bits, sx, sy, chroma, full, rgbf, kr, kb) in cases:
        pl = Planar(width=w, height=h, active_w=aw, active_h=ah, ox=(w - aw) // 2, oy=(h - ah) // 2, sx=sx, sy=sy,
                    rgb=rgbf, bits=bits, full_range=full, chroma=chroma, kr=kr, kb=kb)
        cw, ch = (aw + sx) >> sx, (ah + sy) >> sy
        dt = np.uint8 if bits == 8 else np.uint16
        src = rng.integers(0, 1 << bits, aw * ah + 2 * cw * ch).astype(dt)
        assert np.array_equal(o.planar_to_rgb48(pl, src), ref.planar_to_rgb48(pl, src)), (w, h, bits, sx, sy)


@needs_ref
@pytest.mark.parametrize("w,h,fourk", [(333, 200, 1), (100, 77, 0), (1998, 1080, 0)])
def test_quantiser_matches_reference(o, ref, w, h, fourk):
    """The frame quantiser on wavelet planes of a generator frame, scaled so that every
    band reaches its magnitude clamp somewhere."""
    from libgail_b200 import synth
    planes, _ = ref.color_frame(synth.xyz12_to_rgb48(synth.xyz12_planes(w, h, seed=4)), 5, 4)
    wav = np.stack([ref.fdwt(planes[c], 6 if fourk else 5) for c in range(3)])
    wav[:, ::7, ::5] *= np.float32(300.0)
    bands, cblks = o.layout(w, h, fourk)
    assert np.array_equal(o.quantize_frame(wav, bands, cblks), ref.quantize_frame(wav, w, h, fourk))


@needs_ref
def test_front_end_golden_is_the_reference(ref, fe):
    """The committed front-end fixtures are what the reference build gives today."""
    w, h, fourk, transfer, primaries = (int(x) for x in fe["xyz2k_geom"])
    planes, xyz = ref.color_frame(fe["xyz2k_input"], transfer, primaries)
    assert np.array_equal(xyz, fe["xyz2k_xyz12"])
    wav = np.stack([ref.fdwt(planes[c], 5) for c in range(3)])
    assert np.array_equal(_bits(wav), _bits(fe["xyz2k_wavelet"]))
