"""gb_t1_encode_blocks_noalloc, the Tier-1 entry point that allocates nothing (for callers
that may not allocate device memory, e.g. a real-time frame thread or a process with a
fixed device-memory budget), against gb_t1_encode_blocks, which allocates per call: the
same blocks must give the same results, bit for bit, on two calls in a row (the second
call reuses the static array the first one left its data in). This file is collected last
so that a failure here comes after every other test has run."""
import ctypes as C

import numpy as np
import pytest

import libgail_b200 as gb

MAX_BLOCKS = 64


SENTINEL = 0xA5


def _call(fn, coeffs, geom, slope=0.0, dscale=None, stride=65536, rows=None):
    n = len(geom)
    info = np.zeros((n, 4), np.uint32)
    plen = np.zeros((n, 64), np.uint32)
    pdist = np.zeros((n, 64), np.int32)
    data = np.full((n, stride), SENTINEL, np.uint8)
    c = np.ascontiguousarray(coeffs, np.uint32)
    g = np.ascontiguousarray(geom, np.int32)
    ds = None if dscale is None else np.ascontiguousarray(dscale, np.float32)
    st = fn(c.ctypes.data, g.ctypes.data, n, C.c_float(slope), None if ds is None else ds.ctypes.data, info.ctypes.data,
            plen.ctypes.data, pdist.ctypes.data, data.ctypes.data, stride)
    if rows is not None:
        rows.append(data)
    return st, info, plen, pdist, [bytes(data[i, : info[i, 3]]) for i in range(n)]


def _lib():
    L = gb.lib()
    for name in ("gb_t1_encode_blocks_noalloc", "gb_t1_encode_blocks"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    return L


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(golden_t1):
    L = _lib()
    coeffs, meta = golden_t1["coeffs"], golden_t1["meta"]
    slope = float(golden_t1["slopes"][2])
    dscale = golden_t1["dscale"]
    # two calls in a row with different blocks and settings: the second one runs over what
    # the first left in the shared array
    for k, (lo, sl) in enumerate([(0, 0.0), (MAX_BLOCKS, slope)]):
        sel = slice(lo, lo + MAX_BLOCKS)
        geom = meta[sel].copy()
        if sl:
            geom[:, 3] = 64
        ds = dscale[sel] if sl else None
        st_a, *want = _call(L.gb_t1_encode_blocks, coeffs[sel], geom, sl, ds)
        st_b, *got = _call(L.gb_t1_encode_blocks_noalloc, coeffs[sel], geom, sl, ds)
        assert st_a == 0, gb.lib().gb_last_error()
        assert st_b == 0, gb.lib().gb_last_error()
        info_a, len_a, dist_a, words_a = want
        info_b, len_b, dist_b, words_b = got
        assert np.array_equal(info_a, info_b), f"call {k + 1}: block results differ"
        assert words_a == words_b, f"call {k + 1}: codewords differ"
        # a block's pass tables are defined up to its pass count (the rest of each
        # 64-entry row is whatever the device memory held)
        for i in range(len(geom)):
            np_ = int(info_a[i, 1])
            assert np.array_equal(len_a[i, :np_], len_b[i, :np_]), f"call {k + 1}: block {i} pass lengths differ"
            assert np.array_equal(dist_a[i, :np_], dist_b[i, :np_]), f"call {k + 1}: block {i} distortions differ"


@pytest.mark.gpu
def test_noalloc_refuses_more_than_its_maximum(golden_t1):
    L = _lib()
    coeffs, meta = golden_t1["coeffs"][: MAX_BLOCKS + 1], golden_t1["meta"][: MAX_BLOCKS + 1]
    st, *_ = _call(L.gb_t1_encode_blocks_noalloc, coeffs, meta)
    assert st == 4  # GAIL_CUDA_MISUSE
    assert b"at most 64" in gb.lib().gb_last_error()


@pytest.mark.gpu
def test_noalloc_writes_only_each_codeword(golden_t1):
    """Rows narrower than the array's per-block region (8 KB here, where the region is
    about 56 KB): each codeword lands in its row exactly, and the bytes after it keep the
    caller's contents, as gb_t1_encode_blocks leaves them."""
    L = _lib()
    coeffs, meta = golden_t1["coeffs"], golden_t1["meta"]
    sel = slice(2 * MAX_BLOCKS, 3 * MAX_BLOCKS)
    geom = meta[sel].copy()
    longest = 0
    for fn in (L.gb_t1_encode_blocks, L.gb_t1_encode_blocks_noalloc):
        rows = []
        st, info, _, _, words = _call(fn, coeffs[sel], geom, stride=8192, rows=rows)
        assert st == 0, gb.lib().gb_last_error()
        data = rows[0]
        for i in range(len(geom)):
            n = int(info[i, 3])
            longest = max(longest, n)
            assert np.all(data[i, n:] == SENTINEL), f"block {i}: bytes after the codeword were overwritten"
        if fn is L.gb_t1_encode_blocks:
            want = words
        else:
            assert words == want, "codewords differ from the allocating entry point"
    assert 0 < longest <= 8192
