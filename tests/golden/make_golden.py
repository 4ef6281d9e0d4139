"""Generates the committed golden fixtures from the reference itself.

Run in a tree where oracle/_ref/libgailref.so was built from the reference sources
(oracle/Makefile). Writes tests/golden/*.npz:

  t1_suite.npz   the reference tests' own random code-block suites (testT1Truncation,
                 std::mt19937 seed 42, 400 blocks; testT1PassLimit, seed 9, 300 blocks
                 with their pass limits), with the reference coder's output for each:
                 nbps, passes, pass lengths, pass distortions and codeword bytes (CRC-32 of each codeword for
                 the variants); plus
                 the same blocks coded with early termination at three thresholds.
"""
import os
import sys

import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.oracle import Reference  # noqa: E402


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


def main():
    ref = Reference()
    np.savez_compressed(os.path.join(HERE, "t1_suite.npz"), **t1_suite(ref))
    print("wrote t1_suite.npz")


if __name__ == "__main__":
    main()
