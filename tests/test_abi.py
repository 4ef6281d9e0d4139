"""The C-ABI boundary, without a GPU: the library loads, exports every entry point the
headers declare, and its plugin table is the one libgail accepts (ABI 1, table size,
layout hash of the structure sizes); the host-side layout and colour tables equal the
reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import libgail_b200 as gb
from libgail_b200 import plugin as P
from oracle.oracle import Oracle, Reference, have_reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in ("gail_b200.h", "gail_cuda_plugin_abi.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names.update(re.findall(r"GB_API\s+[\w\s\*]+?\b(gb_\w+)\s*\(", text))
        if "gail_cuda_plugin_get" in text:
            names.add("gail_cuda_plugin_get")
    return names


def test_library_exports_declared_symbols():
    lib = gb.lib()
    names = _declared_symbols()
    assert {"gail_cuda_plugin_get", "gb_t1_encode_blocks", "gb_last_error", "gb_make_layout"} <= names
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"


def test_plugin_table_header():
    t = P.table()
    assert t.abi == 1
    assert t.size == C.sizeof(P.PluginTable)
    assert t.name == b"gail_cuda13"
    assert t.archs == b"100a"
    assert t.toolkit.startswith(b"12.9")
    assert t.layout == gb.lib().gb_plugin_layout_hash()


@pytest.mark.skipif(not have_reference(), reason="reference build not present")
def test_plugin_layout_matches_reference():
    ref = Reference()
    sizes = ref.plugin_sizes()
    mine = [C.sizeof(x) for x in (P.Subband, P.CblkInfo, P.CblkCode, P.FrameFormat, P.FrameTimings, P.DeviceDesc,
                                  P.Layout, P.EncodeSettings, P.Tier1, P.Debug, P.DecodeTimings, P.PluginTable)]
    assert mine == sizes
    L = gb.lib()
    L.gb_plugin_layout_hash.restype = C.c_uint64
    assert L.gb_plugin_layout_hash() == ref.plugin_layout_hash()
    assert P.table().layout == ref.plugin_layout_hash()
    assert P.table().size == sizes[-1]


@pytest.mark.skipif(not have_reference(), reason="reference build not present")
@pytest.mark.parametrize("w,h,fourk", [(1998, 1080, 0), (2048, 858, 0), (2048, 1080, 0), (3996, 2160, 1),
                                       (4096, 1716, 1), (4096, 2160, 1), (100, 77, 0), (333, 200, 1)])
def test_layout_matches_reference(w, h, fourk):
    mine = P.make_layout(w, h, fourk, 1.0)
    rb, _ = Reference().layout(w, h, fourk, 1.0)
    assert len(mine) == len(rb)
    for a, b in zip(mine, rb):
        assert (a.comp, a.res, a.level, a.orient, a.px0, a.py0, a.w, a.h, a.ncbx, a.ncby, a.cblkBase, a.eps, a.mu,
                a.Mb) == (b.comp, b.res, b.level, b.orient, b.px0, b.py0, b.w, b.h, b.ncbx, b.ncby, b.cblk_base,
                          b.eps, b.mu, b.mb)
        assert np.float32(a.delta) == np.float32(b.delta) and a.weight == b.weight


def _tables(col):
    eotf = np.zeros(65536, np.float32)
    m = np.zeros(9, np.float32)
    thr = np.zeros(4096, np.float32)
    gb.lib().gb_color_tables.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    gb.check(gb.lib().gb_color_tables(C.byref(col), eotf.ctypes.data, m.ctypes.data, thr.ctypes.data))
    return eotf, m, thr


@pytest.mark.skipif(not have_reference(), reason="reference build not present")
@pytest.mark.parametrize("transfer,primaries", [("gamma26", "xyz"), ("pq", "bt2020"), ("bt1886", "bt709"),
                                                ("srgb", "p3d65"), ("linear", "dcip3")])
def test_color_tables_match_reference(transfer, primaries):
    col = P.color(transfer, primaries)
    eotf, m, thr = _tables(col)
    ref_eotf, params = Reference().color_tables(P.TRANSFER[transfer], P.PRIMARIES[primaries], 48.0)
    assert np.array_equal(eotf.view(np.uint32), ref_eotf.view(np.uint32))
    assert np.array_equal(m.reshape(3, 3), params[[0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(3, 3))


def test_dci_thresholds_are_exact():
    """Each threshold is the first float whose 12-bit code (the oracle's powf arithmetic)
    reaches k: the code at it is >= k and at the float just below it is < k."""
    _, _, thr = _tables(P.color_passthrough())
    o = Oracle()
    assert thr[0] == 0.0
    bits = thr.view(np.uint32)
    for k in range(1, 4096):
        assert o.dci_code(float(thr[k])) >= k
        below = np.array([bits[k] - 1], np.uint32).view(np.float32)[0]
        assert o.dci_code(float(below)) < k
    assert np.all(np.diff(thr) > 0)


def test_dci_code_is_monotone_on_a_dense_sweep():
    """The thresholds assume the encoding never decreases in n: check it on 2^20 evenly
    spaced floats of [0, 1] and on every float near each threshold."""
    o = Oracle()
    L = o.lib
    xs = np.linspace(0, 1, 1 << 14, dtype=np.float32)
    codes = np.array([L.or_dci_code(C.c_float(x)) for x in xs])
    assert np.all(np.diff(codes) >= 0)


def test_unsupported_color_routes_are_refused():
    col = P.color("pq", "bt2020")
    col.toneMap = 1
    with pytest.raises(gb.GailError):
        _tables(col)
