"""The host codec against the reference's own (built from its sources into oracle/_ref):
rate control and codestream bytes, the codestream with given passes, the empty codestream,
the DCI checker's verdicts on good and damaged codestreams, and the packet parser's
per-block code. Tier-1 frames come from the reference CPU encoder on seeded frames, so
these run without a GPU."""
import ctypes as C

import numpy as np
import pytest

from libgail_b200 import codestream as CS
from libgail_b200 import plugin as P
from libgail_b200 import synth
from oracle.oracle import (RefEncoder, Reference, _p, _ref_bind, have_reference, ref_check, ref_codestream,
                           ref_hull, ref_parse)

pytestmark = pytest.mark.skipif(not have_reference(), reason="reference CPU build (oracle/_ref) not present")

LABEL = "GAIL 1.1.0"  # the reference build's COM label
PROFILES = [(1998, 1080, 0), (2048, 858, 0), (4096, 1716, 1)]


@pytest.fixture(scope="module")
def ref():
    r = Reference()
    _ref_bind(r.lib)
    return r


@pytest.fixture(scope="module")
def frames(ref):
    out = {}
    for W, H, fk in PROFILES:
        enc = RefEncoder(ref, W, H, fk)
        out[(W, H, fk)] = enc.encode(synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=7 + W)))
        enc.close()
    return out


def _ref_build(ref, W, H, fk, t1, passes, tag=b""):
    info = np.ascontiguousarray(t1.info, np.uint32)
    pl = np.ascontiguousarray(t1.pass_len, np.uint32)
    pd = np.ascontiguousarray(t1.pass_dist, np.int32)
    data = np.ascontiguousarray(t1.data, np.uint8)
    p = np.ascontiguousarray(passes, np.uint8)
    cs = np.zeros(64 << 20, np.uint8)
    n = ref.lib.ref_build(W, H, fk, C.c_double(1.0), _p(info), info.shape[0], _p(pl), _p(pd), pl.size, _p(data),
                          data.size, _p(p), tag, _p(cs), cs.size)
    assert n >= 0, ref.error()
    return bytes(cs[:n])


@pytest.mark.parametrize("prof", PROFILES)
@pytest.mark.parametrize("mbps,fps", [(230.0, 24.0), (90.0, 24.0), (230.0, 48.0), (230.0, 25.0)])
def test_rate_and_build_matches_reference(ref, frames, prof, mbps, fps):
    """Rate control and codestream against the reference's allocateRate + buildCodestream, at
    the DCI rate and a low one, and at 48 and 25 frames/s (the per-frame budget follows the
    frame rate, dciLimits, rate_control.cpp:11-26)."""
    W, H, fk = prof
    t1 = frames[prof]
    lay = P.LayoutHolder(W, H, fk)
    want, wpasses, wlam, _ = ref_codestream(ref, W, H, fk, t1, fps=fps, mbps=mbps, tag=b"cuda13.0")
    got, passes, lam = CS.rate_and_build(lay, t1, fps=fps, max_mbps=mbps, label=LABEL, tag="cuda13.0")
    assert np.array_equal(passes, wpasses)
    assert lam == wlam
    assert got == want
    ok, msg = CS.check_dci(got, fps)
    assert ok, msg
    assert msg == LABEL + " cuda13.0"


@pytest.mark.parametrize("prof", PROFILES)
def test_hull_matches_reference(ref, frames, prof):
    """The host PCRD hull points equal the reference's buildHull bit for bit (the pass
    counts, and the slopes as IEEE bit patterns)."""
    W, H, fk = prof
    t1 = frames[prof]
    passes, slope = CS.hull(P.LayoutHolder(W, H, fk), t1)
    wp, ws = ref_hull(ref, W, H, fk, t1)
    assert np.array_equal(passes, wp)
    assert np.array_equal(slope.view(np.uint64), ws.view(np.uint64))
    assert (passes > 0).sum() > len(t1.info)  # blocks with several points


@pytest.mark.parametrize("prof", PROFILES)
def test_rate_and_build_with_given_hull(ref, frames, prof):
    """Rate control fed the hull points (as the engine feeds it those computed on the GPU)
    gives the same codestream as computing them; a malformed hull is refused."""
    W, H, fk = prof
    t1 = frames[prof]
    lay = P.LayoutHolder(W, H, fk)
    hp, hs = CS.hull(lay, t1)
    for mbps in (230.0, 90.0):
        want = CS.rate_and_build(lay, t1, max_mbps=mbps, tag="cuda13.0")
        got = CS.rate_and_build(lay, t1, max_mbps=mbps, tag="cuda13.0", hull_points=(hp, hs))
        assert got[0] == want[0] and np.array_equal(got[1], want[1]) and got[2] == want[2]
    b = int(np.argmax(t1.info[:, 1] >= 2))  # a block with two or more passes
    base = int(t1.info[b, 4])
    bad = hp.copy()
    bad[base], bad[base + 1] = 2, 1  # pass counts not increasing
    with pytest.raises(P.GailError):
        CS.rate_and_build(lay, t1, hull_points=(bad, hs))
    bad = hp.copy()
    bad[base] = t1.info[b, 1] + 1  # beyond the block's passes
    with pytest.raises(P.GailError):
        CS.rate_and_build(lay, t1, hull_points=(bad, hs))


@pytest.mark.parametrize("prof", PROFILES)
def test_build_with_given_passes_matches_reference(ref, frames, prof):
    W, H, fk = prof
    t1 = frames[prof]
    lay = P.LayoutHolder(W, H, fk)
    full = t1.info[:, 1].astype(np.uint8)
    rng = np.random.default_rng(W)
    subset = (rng.random(full.size) * (full.astype(np.float64) + 1)).astype(np.uint8)  # 0..numPasses
    subset[rng.random(full.size) < 0.2] = 0
    for passes, tag in [(full, ""), (subset, "vulk"), (np.zeros_like(full), "cuda99.99")]:
        assert CS.build(lay, t1, passes, LABEL, tag) == _ref_build(ref, W, H, fk, t1, passes, tag.encode())


@pytest.mark.parametrize("prof,want", [((1998, 1080, 0), 376), ((2048, 858, 0), 334), ((3996, 2160, 1), 890),
                                       ((4096, 1716, 1), 752)])
def test_empty_codestream(ref, prof, want):
    W, H, fk = prof
    assert CS.empty_bytes(P.LayoutHolder(W, H, fk), LABEL) == want == ref.lib.ref_empty_codestream_bytes(W, H, fk)


def test_dci_limits(ref):
    for fps in (24.0, 25.0, 48.0, 60.0):
        t, c = C.c_uint64(), C.c_uint64()
        ref.lib.ref_dci_limits(fps, 230.0, 200.0, C.byref(t), C.byref(c))
        assert CS.dci_limits(fps) == (t.value, c.value)
    assert CS.dci_limits(0.0) == (0, 0)


def _damaged(cs: bytes):
    """Codestreams that break one DCI rule each (and two that stay valid)."""
    b = bytearray(cs)
    out = {"good": bytes(b)}
    out["truncated"] = bytes(b[:-100])
    out["no_eoc"] = bytes(b[:-2])
    out["after_eoc"] = bytes(b) + b"\x00"
    r = bytearray(b)
    r[7] ^= 1  # Rsiz
    out["rsiz"] = bytes(r)
    cod = b.find(b"\xff\x52")
    r = bytearray(b)
    r[cod + 5] = 0  # progression LRCP
    out["progression"] = bytes(r)
    r = bytearray(b)
    r[cod + 12] = 0x40  # code-block style with a mode switch (vertically causal)
    out["style"] = bytes(r)
    r = bytearray(b)
    r[cod + 13] = 1  # the 5/3 wavelet
    out["wavelet"] = bytes(r)
    tlm = b.find(b"\xff\x55")
    r = bytearray(b)
    r[tlm + 10] ^= 1  # a TLM length
    out["tlm"] = bytes(r)
    sot = b.find(b"\xff\x90")
    r = bytearray(b)
    r[sot + 10] = 9  # TPsot out of order
    out["tp_order"] = bytes(r)
    r = bytearray(b)
    r[sot + 16:sot + 18] = b"\xff\x91"  # a marker code inside packet data
    out["false_marker"] = bytes(r)
    r = bytearray(b)
    r[2:4] = b"\xff\x52"  # SIZ missing
    out["no_siz"] = bytes(r)
    r = bytearray(b)
    r[5] ^= 2  # Lsiz
    out["lsiz"] = bytes(r)
    r = bytearray(b)
    r[42] = 7  # Ssiz of component 0: 8-bit
    out["ssiz"] = bytes(r)
    r = bytearray(b)
    r[44] = 2  # YRsiz of component 0: subsampled
    out["subsampled"] = bytes(r)
    qcd = b.find(b"\xff\x5c")
    r = bytearray(b)
    r[qcd + 4] ^= 0x20  # guard bits
    out["guard"] = bytes(r)
    r = bytearray(b)
    r[cod + 14] = 0x66  # precincts of the lowest resolution
    out["precinct"] = bytes(r)
    r = bytearray(b)
    r[sot + 11] ^= 1  # TNsot
    out["tnsot"] = bytes(r)
    r = bytearray(b)
    r[sot + 6] = 0xFF  # Psot past the data
    out["psot"] = bytes(r)
    r = bytearray(b)
    r[cod + 1] = 0x60  # COD becomes a marker DCI does not allow (PPM)
    out["ppm"] = bytes(r)
    poc = b.find(b"\xff\x5f", 0, sot)  # in the main header (4K only)
    if poc > 0:
        r = bytearray(b)
        r[poc + 7] = 5  # POC: resolutions 0-4 first
        out["poc"] = bytes(r)
        out["no_poc"] = bytes(b[:poc]) + bytes(b[poc + 18:])
    last = b.rfind(b"\xff\x90")
    out["missing_tile_part"] = bytes(b[:last]) + b"\xff\xd9"
    return out


@pytest.mark.parametrize("prof", PROFILES)
def test_checker_agrees_with_reference(ref, frames, prof):
    W, H, fk = prof
    cs, _, _, _ = ref_codestream(ref, W, H, fk, frames[prof], fps=24.0)
    for name, d in _damaged(cs).items():
        for fps in (24.0, 60.0, 200.0):
            want, _ = ref_check(ref, d, fps)
            got, msg = CS.check_dci(d, fps)
            assert got == want, f"{name} at {fps} fps: ours {got} ({msg}), reference {want}"
    assert CS.check_dci(cs)[0]
    assert not CS.check_dci(cs, 400.0)[0]  # far over the byte cap at 400 fps


@pytest.mark.parametrize("prof", PROFILES)
def test_checker_agrees_with_reference_under_header_damage(ref, frames, prof):
    """Seeded random damage to the main header, the tile-part headers and the bytes around
    them (one to three bytes each): the verdict equals the reference checker's in every case,
    at the frame rate and at the rate where the frame sits exactly on the 250 Mbit/s cap."""
    W, H, fk = prof
    cs, _, _, _ = ref_codestream(ref, W, H, fk, frames[prof], fps=24.0)
    b = np.frombuffer(cs, np.uint8)
    sots = [i for i in range(len(b) - 1) if b[i] == 0xFF and b[i + 1] == 0x90][:6]
    hot = list(range(0, cs.find(b"\xff\x90") + 14)) + [s + k for s in sots for k in range(16)] + \
        list(range(len(b) - 4, len(b)))
    rng = np.random.default_rng(W + H)
    exact = 250e6 / 8.0 / len(cs)  # frame rate whose cap is this frame's size
    disagree = []
    for t in range(300):
        d = bytearray(cs)
        for _ in range(int(rng.integers(1, 4))):
            d[hot[int(rng.integers(0, len(hot)))]] = int(rng.integers(0, 256))
        for fps in (24.0, exact):
            want, _ = ref_check(ref, bytes(d), fps)
            got, msg = CS.check_dci(bytes(d), fps)
            if got != want:
                disagree.append((t, fps, msg))
    assert not disagree, disagree[:5]


@pytest.mark.parametrize("prof", PROFILES)
def test_parse_matches_reference(ref, frames, prof):
    W, H, fk = prof
    for mbps in (230.0, 60.0):
        cs, _, _, _ = ref_codestream(ref, W, H, fk, frames[prof], fps=24.0, mbps=mbps)
        lay, blocks = CS.parse(cs)
        want, w, h, levels = ref_parse(ref, cs)
        assert (lay.width, lay.height, lay.abi.levels) == (w, h, levels) == (W, H, 6 if fk else 5)
        for f in ("offset", "len", "passes", "nbps"):
            assert np.array_equal(blocks[f], want[f]), f
        ours = P.LayoutHolder(W, H, fk)
        for a, b in zip(lay.bands, ours.bands):
            assert (a.eps, a.mu, a.Mb, a.delta, a.cblkBase) == (b.eps, b.mu, b.Mb, b.delta, b.cblkBase)


def test_parse_rejects_damage(ref, frames):
    W, H, fk = PROFILES[0]
    cs, _, _, _ = ref_codestream(ref, W, H, fk, frames[PROFILES[0]], fps=24.0)
    for cut in (10, 100, len(cs) // 2):
        with pytest.raises(Exception):
            CS.parse(cs[:cut])
    rng = np.random.default_rng(3)
    for _ in range(40):  # damaged anywhere: an error or a result, never a crash
        b = bytearray(cs)
        for i in rng.integers(0, len(b), 4):
            b[i] = int(rng.integers(0, 256))
        try:
            CS.parse(bytes(b))
        except Exception:
            pass
