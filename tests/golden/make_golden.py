"""Generates the committed golden fixtures from the reference itself.

Run in a tree where oracle/_ref/libgailref.so was built from the reference sources
(oracle/Makefile). Writes tests/golden/*.npz:

  t1_suite.npz   the reference tests' own random code-block suites (testT1Truncation,
                 std::mt19937 seed 42, 400 blocks; testT1PassLimit, seed 9, 300 blocks
                 with their pass limits), with the reference coder's output for each:
                 nbps, passes, pass lengths, pass distortions and codeword bytes (CRC-32 of each codeword for
                 the variants); plus
                 the same blocks coded with early termination at three thresholds.
  front_end.npz  small frames through the reference encoder front end: the inputs, the
                 planar-to-R'G'B' conversion (planarToRgb48), the reference CpuSlot's own
                 debug taps (X'Y'Z' codes, quantised code-block words) and the wavelet
                 planes of the reference fdwt97_2d on the reference colour planes, for an
                 X'Y'Z' pass-through frame (2K profile), a 4:2:2 10-bit PQ BT.2020 frame
                 (4K profile), and the planar variants 4:2:0 8-bit letterboxed with centred
                 chroma, 4:4:4 12-bit full range and planar G'B'R'.
"""
import os
import sys

import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.oracle import Planar, RefEncoder, Reference  # noqa: E402


def t1_suite(ref: Reference) -> dict:
    out = {}
    c0, m0 = ref.suite(0, 400)
    c1, m1 = ref.suite(1, 300)
    coeffs = np.concatenate([c0, c1])
    meta = np.concatenate([m0, m1])
    # early termination variants: thresholds and per-block distortion scales
    rng = np.random.default_rng(7)
    slopes = np.array([0.0, 0.5, 5.0, 50.0], np.float32)
    dscale = rng.uniform(0.05, 2.0, len(coeffs)).astype(np.float32)
    for si, s in enumerate(slopes):
        nb, npass, plen, pdist, data, dofs = [], [], [], [], [], [0]
        for i in range(len(coeffs)):
            w, h, o, lim = (int(x) for x in meta[i])
            r = ref.t1_encode(coeffs[i], w, h, o, lim if s == 0 else 64, float(s), float(dscale[i]))
            nb.append(r.nbps)
            npass.append(r.num_passes)
            pl = np.zeros(64, np.uint32)
            pd = np.zeros(64, np.int32)
            pl[: r.num_passes] = r.pass_len
            pd[: r.num_passes] = r.pass_dist
            plen.append(pl)
            pdist.append(pd)
            data.append(np.frombuffer(r.data, np.uint8))
            dofs.append(dofs[-1] + len(r.data))
        out[f"s{si}_nbps"] = np.array(nb, np.int32)
        out[f"s{si}_passes"] = np.array(npass, np.int32)
        out[f"s{si}_pass_len"] = np.array(plen)
        out[f"s{si}_pass_dist"] = np.array(pdist)
        if si == 0:
            out["s0_data"] = np.concatenate(data)
            out["s0_data_ofs"] = np.array(dofs, np.int64)
        # every variant keeps a CRC-32 of each codeword
        out[f"s{si}_crc"] = np.array([zlib.crc32(d.tobytes()) for d in data], np.uint32)
    out["coeffs"] = coeffs
    out["meta"] = meta
    out["slopes"] = slopes
    out["dscale"] = dscale
    return out


# colour settings (the reference's Transfer / Primaries numbering)
PASS_THROUGH = (5, 4)   # gamma 2.6, XYZ
PQ_BT2020 = (2, 1)
BT1886_BT709 = (0, 0)

# planar variants: (name, width, height, active w, active h, bits, sx, sy, chroma, full range, rgb, kr, kb)
PLANAR_VARIANTS = [
    ("yuv420p8_letterbox", 100, 60, 90, 51, 8, 1, 1, 1, 0, 0, 0.2126, 0.0722),
    ("yuv444p12_full", 64, 40, 64, 40, 12, 0, 0, 2, 1, 0, 0.299, 0.114),
    ("gbrp10", 48, 32, 48, 32, 10, 0, 0, 0, 0, 1, 0.2627, 0.0593),
]


def planar_of(w, h, aw, ah, bits, sx, sy, chroma, full, rgb, kr, kb):
    return Planar(width=w, height=h, active_w=aw, active_h=ah, ox=(w - aw) // 2, oy=(h - ah) // 2, sx=sx, sy=sy,
                  rgb=rgb, bits=bits, full_range=full, chroma=chroma, kr=kr, kb=kb)


def _frame_taps(ref, out, name, frame, w, h, fourk, colour, planar=None):
    """The reference encoder's front end on one frame, stored under name_*."""
    levels = 6 if fourk else 5
    enc = RefEncoder(ref, w, h, fourk, colour[0], colour[1], planar=planar, threads=1)
    t = enc.encode(frame, debug=True)
    enc.close()
    rgb = ref.planar_to_rgb48(planar, frame) if planar is not None else frame
    planes, xyz = ref.color_frame(rgb, colour[0], colour[1])
    assert np.array_equal(xyz.ravel(), t.xyz12), "reference colour and CpuSlot taps disagree"
    wav = np.stack([ref.fdwt(planes[c], levels) for c in range(3)])
    q = ref.quantize_frame(wav, w, h, fourk)
    assert np.array_equal(q.ravel(), t.coeffs), "reference quantiser and CpuSlot taps disagree"
    out[f"{name}_input"] = np.ascontiguousarray(frame)
    if planar is not None:  # an R'G'B' 16-bit input is its own rgb48
        out[f"{name}_rgb48"] = rgb
    out[f"{name}_xyz12"] = t.xyz12.reshape(h, w, 3)
    out[f"{name}_wavelet"] = wav
    out[f"{name}_coeffs"] = t.coeffs.reshape(-1, 1024)
    out[f"{name}_geom"] = np.array([w, h, fourk, colour[0], colour[1]], np.int32)


def front_end(ref: Reference) -> dict:
    from libgail_b200 import synth
    out = {}
    w, h = 144, 80
    _frame_taps(ref, out, "xyz2k", synth.xyz12_to_rgb48(synth.xyz12_planes(w, h, seed=31)), w, h, 0, PASS_THROUGH)
    w, h = 128, 72
    pl = planar_of(w, h, w, h, 10, 1, 0, 0, 0, 0, 0.2627, 0.0593)
    _frame_taps(ref, out, "pq4k", synth.yuv422p10(w, h, seed=32), w, h, 1, PQ_BT2020, pl)
    rng = np.random.default_rng(33)
    for (name, w, h, aw, ah, bits, sx, sy, chroma, full, rgb, kr, kb) in PLANAR_VARIANTS:
        pl = planar_of(w, h, aw, ah, bits, sx, sy, chroma, full, rgb, kr, kb)
        cw, ch = (aw + sx) >> sx, (ah + sy) >> sy
        dt = np.uint8 if bits == 8 else np.uint16
        src = rng.integers(0, 1 << bits, aw * ah + 2 * cw * ch).astype(dt)
        out[f"{name}_input"] = src
        out[f"{name}_rgb48"] = ref.planar_to_rgb48(pl, src)
        out[f"{name}_geom"] = np.array([w, h, aw, ah, bits, sx, sy, chroma, full, rgb], np.int32)
        out[f"{name}_krkb"] = np.array([kr, kb], np.float64)
    return out


def main():
    ref = Reference()
    np.savez_compressed(os.path.join(HERE, "t1_suite.npz"), **t1_suite(ref))
    print("wrote t1_suite.npz")
    np.savez_compressed(os.path.join(HERE, "front_end.npz"), **front_end(ref))
    print("wrote front_end.npz")


if __name__ == "__main__":
    main()
