"""The host codec from Python: rate control and codestream assembly over a Tier-1 frame,
the DCI check, and the reading of a codestream for the decoder (gb_* codestream entry
points of include/gail_b200.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import check, lib
from .plugin import CblkCode, CblkInfo, LayoutHolder, Subband, Tier1, Tier1Frame

# the COM label of the reference encoder's release build ("GAIL " + its version)
DEFAULT_LABEL = "GAIL 1.1.0"


def _bind():
    L = lib()
    if getattr(L, "_codestream_bound", False):
        return L
    u64p = C.POINTER(C.c_uint64)
    L.gb_dci_limits.argtypes = [C.c_double, C.c_double, C.c_double, u64p, u64p]
    L.gb_empty_codestream_bytes.argtypes = [C.c_void_p, C.c_char_p, u64p]
    L.gb_build_codestream.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_char_p, C.c_void_p,
                                      C.c_uint64, u64p]
    L.gb_rate_and_build.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_char_p,
                                    C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, u64p, C.POINTER(C.c_double)]
    L.gb_rate_and_build_hull.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                         C.c_double, C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, u64p,
                                         C.POINTER(C.c_double)]
    L.gb_device_rate_and_build.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                           C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, u64p,
                                           C.POINTER(C.c_double)]
    L.gb_tier1_hull.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.gb_check_dci.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_char_p, C.c_uint64, C.POINTER(C.c_int)]
    L.gb_parse_codestream.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                      C.c_uint64, u64p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L._codestream_bound = True
    return L


class Tier1Arrays:
    """A GailCudaTier1 view over a Tier1Frame's arrays (kept alive with it)."""

    def __init__(self, t: Tier1Frame):
        self.info = np.ascontiguousarray(t.info, np.uint32)
        self.pass_len = np.ascontiguousarray(t.pass_len, np.uint32)
        self.pass_dist = np.ascontiguousarray(t.pass_dist, np.int32)
        self.data = np.ascontiguousarray(t.data, np.uint8)
        self.abi = Tier1(info=self.info.ctypes.data_as(C.POINTER(CblkInfo)),
                         passLen=self.pass_len.ctypes.data_as(C.POINTER(C.c_uint32)),
                         passDist=self.pass_dist.ctypes.data_as(C.POINTER(C.c_int32)),
                         data=self.data.ctypes.data_as(C.POINTER(C.c_uint8)), numInfo=len(self.info),
                         numPasses=len(self.pass_len), numData=len(self.data))


class _View:
    def __init__(self, t: Tier1):
        self.abi = t


def _t1(t):
    """Tier1Arrays as given; a plugin's Tier1 view used in place; else its arrays wrapped."""
    if isinstance(t, (Tier1Arrays, _View)):
        return t
    if isinstance(t, Tier1):
        return _View(t)
    return Tier1Arrays(t)


def dci_limits(fps: float, max_mbps: float = 230.0, comp_mbps: float = 200.0):
    tot, comp = C.c_uint64(), C.c_uint64()
    check(_bind().gb_dci_limits(fps, max_mbps, comp_mbps, C.byref(tot), C.byref(comp)))
    return tot.value, comp.value


def empty_bytes(layout: LayoutHolder, label: str = DEFAULT_LABEL) -> int:
    n = C.c_uint64()
    check(_bind().gb_empty_codestream_bytes(C.byref(layout.abi), label.encode(), C.byref(n)))
    return n.value


def build(layout: LayoutHolder, t1, passes, label: str = DEFAULT_LABEL, tag: str = "") -> bytes:
    L, t = _bind(), _t1(t1)
    p = np.ascontiguousarray(passes, np.uint8)
    n = C.c_uint64()
    check(L.gb_build_codestream(C.byref(layout.abi), C.byref(t.abi), p.ctypes.data, label.encode(), tag.encode(), None,
                                0, C.byref(n)))
    out = np.empty(n.value, np.uint8)
    check(L.gb_build_codestream(C.byref(layout.abi), C.byref(t.abi), p.ctypes.data, label.encode(), tag.encode(),
                                out.ctypes.data, out.size, C.byref(n)))
    return out.tobytes()


def rate_and_build(layout: LayoutHolder, t1, fps: float = 24.0, max_mbps: float = 230.0, comp_mbps: float = 200.0,
                   label: str = DEFAULT_LABEL, tag: str = "", hull_points=None):
    """(codestream bytes, passes per block, lambda). hull_points: (passes, slope) arrays as
    hull() gives them (e.g. computed on the GPU by the engine), taken instead of computing
    the hull."""
    L, t = _bind(), _t1(t1)
    passes = np.zeros(layout.abi.numCblks, np.uint8)
    cap = 1 << 22
    out = np.empty(cap, np.uint8)
    n, lam = C.c_uint64(), C.c_double()
    hp = hs = None
    if hull_points is not None:
        hp = np.ascontiguousarray(hull_points[0], np.uint8)
        hs = np.ascontiguousarray(hull_points[1], np.float64)
        if hp.size < t.abi.numPasses or hs.size < t.abi.numPasses:
            raise ValueError("hull arrays shorter than the Tier-1 frame's passes")
    check(L.gb_rate_and_build_hull(C.byref(layout.abi), C.byref(t.abi), None if hp is None else hp.ctypes.data,
                                   None if hs is None else hs.ctypes.data, fps, max_mbps, comp_mbps, label.encode(),
                                   tag.encode(), passes.ctypes.data, out.ctypes.data, cap, C.byref(n), C.byref(lam)))
    return out[: n.value].tobytes(), passes, lam.value


def device_rate_and_build(layout: LayoutHolder, t1, fps: float = 24.0, max_mbps: float = 230.0,
                          comp_mbps: float = 200.0, label: str = DEFAULT_LABEL, tag: str = "", device: int = 0):
    """rate_and_build on a GPU (hull, slope histogram, size measurements and packets
    computed there): (codestream bytes, passes per block, lambda), the same as rate_and_build."""
    L, t = _bind(), _t1(t1)
    passes = np.zeros(layout.abi.numCblks, np.uint8)
    cap = 1 << 22
    out = np.empty(cap, np.uint8)
    n, lam = C.c_uint64(), C.c_double()
    check(L.gb_device_rate_and_build(device, C.byref(layout.abi), C.byref(t.abi), fps, max_mbps, comp_mbps,
                                     label.encode(), tag.encode(), passes.ctypes.data, out.ctypes.data, cap,
                                     C.byref(n), C.byref(lam)))
    return out[: n.value].tobytes(), passes, lam.value


def hull(layout: LayoutHolder, t1):
    """Every block's PCRD hull points on the host: (passes uint8, slope float64) per pass slot
    of the Tier-1 frame; block i's points from its passBase on, ending at its pass count or
    the first 0 in passes."""
    L, t = _bind(), _t1(t1)
    n = t.abi.numPasses
    p, s = np.zeros(max(n, 1), np.uint8), np.zeros(max(n, 1), np.float64)
    check(L.gb_tier1_hull(C.byref(layout.abi), C.byref(t.abi), p.ctypes.data, s.ctypes.data))
    return p[:n], s[:n]


def check_dci(cs: bytes, fps: float = 24.0):
    """(compliant, COM text or the first error)."""
    d = np.frombuffer(cs, np.uint8)
    msg = C.create_string_buffer(512)
    ok = C.c_int()
    check(_bind().gb_check_dci(d.ctypes.data, d.size, fps, msg, 512, C.byref(ok)))
    return bool(ok.value), msg.value.decode(errors="replace")


def parse(cs: bytes):
    """(LayoutHolder with the signalled steps, structured CblkCode array)."""
    L = _bind()
    d = np.frombuffer(cs, np.uint8)
    nb, nblk, w, h, prof = C.c_int(), C.c_uint64(), C.c_int(), C.c_int(), C.c_int()
    # room for the largest DCI layout (4096 x 2160: 57 bands, 26,292 code-blocks): one call
    bands = (Subband * 64)()
    blocks = np.zeros(60000, dtype=np.dtype([("offset", "<u4"), ("len", "<u4"), ("passes", "u1"), ("nbps", "u1"),
                                             ("_pad", "u1", 2)]))
    assert blocks.itemsize == C.sizeof(CblkCode)
    check(L.gb_parse_codestream(d.ctypes.data, d.size, bands, 64, C.byref(nb), blocks.ctypes.data, blocks.size,
                                C.byref(nblk), C.byref(w), C.byref(h), C.byref(prof)))
    lay = LayoutHolder(w.value, h.value, prof.value, bands=list(bands)[: nb.value])
    return lay, blocks[: nblk.value]
