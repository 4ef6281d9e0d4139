"""Tier-1 encoder kernels against the reference coder's own outputs (golden fixtures made
by the reference build, tests/golden/make_golden.py): every block of the reference tests'
random suites (seed 42 and seed 9 with pass limits) must come out bit-exact: nbps, pass
count, every truncation length, every pass distortion and the codeword bytes."""
import zlib

import numpy as np
import pytest

import libgail_b200 as gb


def _run(golden, variant):
    coeffs, meta = golden["coeffs"], golden["meta"].copy()
    slope = float(golden["slopes"][variant])
    if variant != 0:
        meta[:, 3] = 64  # early-termination variants code without a pass limit
    info, plen, pdist, words = gb.t1_encode_blocks(coeffs, meta, slope, golden["dscale"] if variant else None)
    return info, plen, pdist, words


@pytest.mark.gpu
def test_t1_suites_bit_exact(golden_t1):
    g = golden_t1
    info, plen, pdist, words = _run(g, 0)
    n = len(g["meta"])
    assert np.array_equal(info[:, 0], np.where(g["s0_passes"] > 0, g["s0_nbps"], info[:, 0]))
    assert np.array_equal(info[:, 1].astype(np.int32), g["s0_passes"])
    ofs = g["s0_data_ofs"]
    bad = []
    points = 0
    for i in range(n):
        np_ = int(g["s0_passes"][i])
        points += np_
        want = bytes(g["s0_data"][ofs[i]:ofs[i + 1]])
        if (words[i] != want or not np.array_equal(plen[i, :np_], g["s0_pass_len"][i, :np_])
                or not np.array_equal(pdist[i, :np_], g["s0_pass_dist"][i, :np_])):
            bad.append(i)
    assert not bad, f"{len(bad)} of {n} blocks differ, first {bad[:10]}"
    assert points > 15000


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [1, 2, 3])
def test_t1_early_termination_agreement(golden_t1, variant):
    """With early termination the stop rule uses float log2 and the GPU's log2f may round
    differently from the host's in the last place; blocks whose stop decision agrees must
    be bit-exact, and at least 99% of blocks must agree."""
    g = golden_t1
    info, plen, pdist, words = _run(g, variant)
    n = len(g["meta"])
    agree = exact = 0
    for i in range(n):
        np_ = int(g[f"s{variant}_passes"][i])
        if int(info[i, 1]) != np_:
            continue
        agree += 1
        if (zlib.crc32(words[i]) == int(g[f"s{variant}_crc"][i])
                and np.array_equal(plen[i, :np_], g[f"s{variant}_pass_len"][i, :np_])
                and np.array_equal(pdist[i, :np_], g[f"s{variant}_pass_dist"][i, :np_])):
            exact += 1
    assert exact == agree, f"{agree - exact} blocks with the same stop point differ"
    assert agree >= 0.99 * n, f"stop decisions agree on only {agree} of {n} blocks"
