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


# colour settings across the managed route's branches: tone map x norm x target gamut,
# the shoulder's knee clamp and its no-shoulder case, BT.2390 with a source peak at or below
# the cinema peak (no tone map), HLG, pass-through (tone settings ignored), LUTs
ROUTE_CASES = [
    dict(tone_map="shoulder", tone_norm="channel", gamut="p3d65", hdr_peak=4000.0),
    dict(tone_map="shoulder", tone_norm="maxrgb", gamut="p3d65", hdr_peak=4000.0),
    dict(tone_map="shoulder", tone_norm="luminance", gamut="p3d65", hdr_peak=4000.0),
    dict(tone_map="bt2390", tone_norm="channel", gamut="p3d65", hdr_peak=4000.0),
    dict(tone_map="bt2390", tone_norm="maxrgb", gamut="dcip3", hdr_peak=1000.0, cinema_peak=48.0),
    dict(tone_map="bt2390", tone_norm="luminance", gamut="none", hdr_peak=40.0),
    dict(tone_map="shoulder", knee=0.001, hdr_peak=600.0, gamut_threshold=1.5),
    dict(tone_map="shoulder", knee=2.0, hdr_peak=100.0, cinema_ref_white=10.0, gamut="dcip3", gamut_threshold=-1.0),
    dict(transfer="hlg", tone_map="shoulder", tone_norm="maxrgb", gamut="p3d65"),
    dict(transfer="hlg", tone_map="none"),
    dict(tone_map="signal", gamut="p3d65"),
    dict(transfer="bt1886", primaries="bt709", gamut="dcip3", gamut_threshold=0.5),
    dict(transfer="gamma26", primaries="xyz", tone_map="shoulder", gamut="p3d65"),
    dict(transfer="srgb", primaries="bt709", lut_size=5, lut="sin"),
]


def _lut_of(case):
    if case.get("lut") == "sin":
        n = case["lut_size"]
        return np.array([0.5 + 0.4 * np.sin(i * 0.7 + c) for i in range(n ** 3) for c in range(3)], np.float32)
    return None


def _route_case(case):
    kw = dict(case)
    lut = _lut_of(kw)
    kw["lut"] = lut
    mine = P.color_managed(**kw)
    from oracle.oracle import ref_color
    rkw = dict(transfer=P.TRANSFER[kw.pop("transfer", "pq")], primaries=P.PRIMARIES[kw.pop("primaries", "bt2020")],
               tone_map=P.TONE_MAP[kw.pop("tone_map", "signal")], tone_norm=P.TONE_NORM[kw.pop("tone_norm", "channel")],
               gamut=P.GAMUT[kw.pop("gamut", "none")])
    rkw.update(lut=kw.pop("lut"), lut_size=kw.pop("lut_size", 0))
    rkw.update(kw)
    return mine, ref_color(**rkw)


@pytest.mark.skipif(not have_reference(), reason="reference build not present")
@pytest.mark.parametrize("case", ROUTE_CASES, ids=lambda c: "-".join(str(v) for k, v in c.items() if k != "lut"))
def test_color_route_constants_match_reference(case):
    """The managed route's constants, bit for bit in the positions of the reference's
    parameter block (ColorConverter::params), and the route chosen."""
    mine, theirs = _route_case(case)
    route, params, n = P.color_route(mine)
    ref_params, ref_n = Reference().color_params(theirs)
    assert n == ref_n
    assert np.array_equal(params.view(np.uint32), ref_params.view(np.uint32)), \
        [(i, params[i], ref_params[i]) for i in range(48) if params.view(np.uint32)[i] != ref_params.view(np.uint32)[i]]
    want = 2 if ref_n > 1 else 1 if (ref_params[12] != 0 or ref_params[18] != 0) else 0
    assert route == want


CUBE_GOOD = """# comment
TITLE "test"
LUT_3D_SIZE 2
DOMAIN_MIN 0 0 0
DOMAIN_MAX 1 1 1

0 0 0
1 0 0
0 1 0
1 1 0
  0 0 1
1 0 1 trailing words
0 1 1
1 1 1
"""


@pytest.mark.skipif(not have_reference(), reason="reference build not present")
@pytest.mark.parametrize("name,text", [
    ("good", CUBE_GOOD),
    ("one_d", "LUT_1D_SIZE 4\n0 0 0\n"),
    ("count", "LUT_3D_SIZE 2\n0 0 0\n1 1 1\n"),
    ("domain", CUBE_GOOD.replace("DOMAIN_MAX 1 1 1", "DOMAIN_MAX 1 2 1")),
    ("size1", "LUT_3D_SIZE 1\n0 0 0\n"),
    ("crlf", CUBE_GOOD.replace("\n", "\r\n")),
])
def test_cube_reader_matches_reference(tmp_path, name, text):
    """A .cube LUT given by path: read as the reference's readCubeLut reads it (the same
    nodes, or an error where it gives one)."""
    path = tmp_path / f"{name}.cube"
    path.write_bytes(text.encode())
    try:
        rn, rdata = Reference().read_cube(str(path))
    except RuntimeError:
        rn = None
    col = P.color_managed(transfer="srgb", primaries="bt709", lut_path=str(path))
    if rn is None:
        with pytest.raises(gb.GailError):
            P.color_route(col)
        return
    route, params, n = P.color_route(col)
    assert (route, n) == (2, rn)


def test_lut_data_must_match_its_size():
    lut = np.zeros(5 ** 3 * 3 - 1, np.float32)
    with pytest.raises(gb.GailError):
        P.color_route(P.color_managed(lut=lut, lut_size=5))
