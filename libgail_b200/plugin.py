"""The GAIL CUDA plugin table from Python: the ctypes mirror of gail_cuda_plugin_abi.h.

`Plugin` wraps the table gail_cuda_plugin_get(1) returns, exactly as libgail's CudaHost
drives it (Josephur/libgail src/cuda/cuda_host.cpp:152-255): devices, encoder slots
(encoder_bytes / create / input / set_slope / encode) and decoder slots. Results come
back as numpy arrays copied out of the plugin's views (which stay valid only until the
next call on the same object).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import GailError, check, lib


class Subband(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("comp", "res", "level", "orient", "px0", "py0", "w", "h", "ncbx", "ncby",
                                         "cblkBase", "eps", "mu", "Mb")] + [("delta", C.c_float), ("weight", C.c_double)]


class CblkInfo(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("nbps", "numPasses", "dataOffset", "dataLen", "passBase")]


class CblkCode(C.Structure):
    _fields_ = [("offset", C.c_uint32), ("len", C.c_uint32), ("passes", C.c_uint8), ("nbps", C.c_uint8)]


class FrameFormat(C.Structure):
    _fields_ = [("kind", C.c_int32), ("chroma", C.c_int32), ("width", C.c_int32), ("height", C.c_int32),
                ("activeW", C.c_int32), ("activeH", C.c_int32), ("ox", C.c_int32), ("oy", C.c_int32),
                ("sx", C.c_int32), ("sy", C.c_int32), ("rgb", C.c_uint8), ("bits", C.c_int32),
                ("fullRange", C.c_uint8), ("kr", C.c_double), ("kb", C.c_double)]


class FrameTimings(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("upload", "color", "dwt", "quant", "t1", "t1cm", "t1mq", "download", "gpu",
                                          "total", "symbols", "codedBytes")]


class DeviceDesc(C.Structure):
    _fields_ = [("index", C.c_int32), ("smMajor", C.c_int32), ("smMinor", C.c_int32), ("memoryBytes", C.c_uint64),
                ("name", C.c_char * 256), ("uuid", C.c_char * 48), ("pciBusId", C.c_char * 32)]


class Layout(C.Structure):
    _fields_ = [("profile", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("levels", C.c_int32),
                ("guardBits", C.c_int32), ("numBands", C.c_int32), ("numCblks", C.c_int32),
                ("baseStep", C.c_double), ("bands", C.POINTER(Subband))]


class Color(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("transfer", "primaries", "toneMap", "toneNorm", "gamut", "lut3dSize")] + \
        [(n, C.c_double) for n in ("sdrWhite", "hdrPeak", "cinemaPeak", "hdrRefWhite", "cinemaRefWhite", "knee",
                                   "gamutThreshold")] + \
        [("lut3d", C.c_char_p), ("lut3dData", C.POINTER(C.c_float)), ("lut3dCount", C.c_uint64)]


class EncodeSettings(C.Structure):
    _fields_ = [("profile", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("baseStep", C.c_double),
                ("slopeFactor", C.c_double), ("bitsPerSymbol", C.c_double), ("input", FrameFormat), ("color", Color)]


class DecodeSettings(C.Structure):
    _fields_ = [("reduce", C.c_int32), ("highBits", C.c_int32)]


class Memory(C.Structure):
    _fields_ = [("total", C.c_uint64), ("available", C.c_uint64), ("budgeted", C.c_int32)]


class Tier1(C.Structure):
    _fields_ = [("info", C.POINTER(CblkInfo)), ("passLen", C.POINTER(C.c_uint32)), ("passDist", C.POINTER(C.c_int32)),
                ("data", C.POINTER(C.c_uint8)), ("numInfo", C.c_uint64), ("numPasses", C.c_uint64),
                ("numData", C.c_uint64)]


class Debug(C.Structure):
    _fields_ = [("full", C.c_int32), ("xyz12", C.POINTER(C.c_uint16)), ("coeffs", C.POINTER(C.c_uint32)),
                ("wavelet", C.POINTER(C.c_float)), ("numXyz12", C.c_uint64), ("numCoeffs", C.c_uint64),
                ("numWavelet", C.c_uint64)]


class DecodeTimings(C.Structure):
    _fields_ = [("t1", C.c_double), ("dwt", C.c_double), ("color", C.c_double), ("total", C.c_double),
                ("wantWavelet", C.c_int32), ("wavelet", C.POINTER(C.c_float) * 3), ("numWavelet", C.c_uint64)]


LogFn = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_char_p)
_vp = C.c_void_p


class PluginTable(C.Structure):
    _fields_ = [
        ("abi", C.c_uint32), ("size", C.c_uint32), ("layout", C.c_uint64), ("name", C.c_char_p),
        ("toolkit", C.c_char_p), ("archs", C.c_char_p),
        ("last_error", C.CFUNCTYPE(C.c_char_p)),
        ("device_count", C.CFUNCTYPE(C.c_int)),
        ("device_desc", C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(DeviceDesc))),
        ("device_usable", C.CFUNCTYPE(C.c_int, C.c_int)),
        ("device_create", C.CFUNCTYPE(C.c_int, C.c_int, LogFn, _vp, C.POINTER(_vp))),
        ("device_destroy", C.CFUNCTYPE(None, _vp)),
        ("device_name", C.CFUNCTYPE(C.c_char_p, _vp)),
        ("device_memory", C.CFUNCTYPE(C.c_int, _vp, C.POINTER(Memory))),
        ("encoder_bytes", C.CFUNCTYPE(C.c_uint64, _vp, C.POINTER(Layout), C.POINTER(EncodeSettings))),
        ("encoder_create", C.CFUNCTYPE(C.c_int, _vp, C.POINTER(Layout), C.POINTER(EncodeSettings), C.POINTER(_vp))),
        ("encoder_destroy", C.CFUNCTYPE(None, _vp)),
        ("encoder_input", C.CFUNCTYPE(_vp, _vp)),
        ("encoder_set_slope", C.CFUNCTYPE(None, _vp, C.c_double)),
        ("encoder_encode", C.CFUNCTYPE(C.c_int, _vp, _vp, C.POINTER(Tier1), C.POINTER(FrameTimings), C.POINTER(Debug))),
        ("decoder_bytes", C.CFUNCTYPE(C.c_uint64, _vp, C.POINTER(Layout), C.POINTER(DecodeSettings))),
        ("decoder_create", C.CFUNCTYPE(C.c_int, _vp, C.POINTER(Layout), C.POINTER(DecodeSettings), C.POINTER(_vp))),
        ("decoder_destroy", C.CFUNCTYPE(None, _vp)),
        ("decoder_decode", C.CFUNCTYPE(C.c_int, _vp, C.POINTER(Layout), _vp, C.c_size_t, C.POINTER(CblkCode),
                                       C.c_size_t, _vp, C.c_ssize_t, C.POINTER(DecodeTimings))),
    ]


def table(path: str | None = None) -> PluginTable:
    """This library's plugin table, or that of another build of the plugin ABI at `path`."""
    L = lib() if path is None else C.CDLL(path)
    L.gail_cuda_plugin_get.restype = C.POINTER(PluginTable)
    L.gail_cuda_plugin_get.argtypes = [C.c_uint32]
    p = L.gail_cuda_plugin_get(1)
    if not p:
        raise RuntimeError("plugin refused ABI 1")
    return p.contents


# transfer / primaries codes of GailCudaColor
TRANSFER = {"bt1886": 0, "srgb": 1, "pq": 2, "hlg": 3, "linear": 4, "gamma26": 5}
PRIMARIES = {"bt709": 0, "bt2020": 1, "p3d65": 2, "dcip3": 3, "xyz": 4}


def color_passthrough() -> Color:
    """X'Y'Z' input: gamma 2.6 with identity primaries (gail_api.cpp:608-610)."""
    return color(transfer="gamma26", primaries="xyz")


def color(transfer="bt1886", primaries="bt709", sdr_white=48.0) -> Color:
    """The managed route with the preset defaults (gail_color_preset, gail_api.cpp:497-524)."""
    return Color(transfer=TRANSFER[transfer], primaries=PRIMARIES[primaries], toneMap=0, toneNorm=0, gamut=2,
                 lut3dSize=0, sdrWhite=sdr_white, hdrPeak=1000.0, cinemaPeak=48.0, hdrRefWhite=203.0,
                 cinemaRefWhite=16.0, knee=0.25, gamutThreshold=0.8, lut3d=b"", lut3dData=None, lut3dCount=0)


TONE_MAP = {"signal": 0, "shoulder": 1, "bt2390": 2, "none": 3}
TONE_NORM = {"channel": 0, "maxrgb": 1, "luminance": 2}
GAMUT = {"p3d65": 0, "dcip3": 1, "none": 2}


def color_managed(transfer="pq", primaries="bt2020", tone_map="signal", tone_norm="channel", gamut="none",
                  sdr_white=48.0, hdr_peak=1000.0, cinema_peak=48.0, hdr_ref_white=203.0, cinema_ref_white=16.0,
                  knee=0.25, gamut_threshold=0.8, lut=None, lut_size=0, lut_path="") -> Color:
    """Every colour setting of ColorParams (core/color.h:84-100): tone map and its norm,
    target gamut, or a 3D LUT (float32 lut_size^3 * 3, red fastest, or a .cube path) that
    replaces them. The LUT array is kept alive by the returned structure."""
    c = Color(transfer=TRANSFER[transfer], primaries=PRIMARIES[primaries], toneMap=TONE_MAP[tone_map],
              toneNorm=TONE_NORM[tone_norm], gamut=GAMUT[gamut], lut3dSize=lut_size, sdrWhite=sdr_white,
              hdrPeak=hdr_peak, cinemaPeak=cinema_peak, hdrRefWhite=hdr_ref_white, cinemaRefWhite=cinema_ref_white,
              knee=knee, gamutThreshold=gamut_threshold, lut3d=lut_path.encode(), lut3dData=None, lut3dCount=0)
    if lut is not None:
        arr = np.ascontiguousarray(lut, dtype=np.float32)
        c._lut = arr
        c.lut3dData = arr.ctypes.data_as(C.POINTER(C.c_float))
        c.lut3dCount = arr.size
    return c


def color_route(col: Color):
    """(route, the reference-layout 48-float parameter block, LUT nodes per axis) the
    library derives from a colour setting: route 0 direct, 1 tone map / gamut, 2 3D LUT."""
    L = lib()
    L.gb_color_route.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    params = np.zeros(48, np.float32)
    route, n = C.c_int32(), C.c_int32()
    check(L.gb_color_route(C.byref(col), params.ctypes.data, C.byref(route), C.byref(n)))
    return route.value, params, n.value


def rgb48_format(width, height) -> FrameFormat:
    return FrameFormat(kind=0, chroma=0, width=width, height=height, activeW=0, activeH=0, ox=0, oy=0, sx=1, sy=1,
                       rgb=0, bits=8, fullRange=0, kr=0.2627, kb=0.0593)


def planar_format(width, height, bits=10, sx=1, sy=0, kr=0.2627, kb=0.0593, chroma=0, full_range=False,
                  active=None, rgb=False) -> FrameFormat:
    aw, ah = active or (width, height)
    return FrameFormat(kind=1, chroma=chroma, width=width, height=height, activeW=aw, activeH=ah,
                       ox=(width - aw) // 2, oy=(height - ah) // 2, sx=sx, sy=sy, rgb=int(rgb), bits=bits,
                       fullRange=int(full_range), kr=kr, kb=kb)


class LayoutHolder:
    """A frame layout (bands with steps) kept alive for the calls that point into it."""

    def __init__(self, width, height, fourk, base_step=1.0, bands=None):
        self.width, self.height, self.fourk = width, height, bool(fourk)
        if bands is None:
            bands = make_layout(width, height, fourk, base_step)
        self.bands = (Subband * len(bands))(*bands)
        n_cblks = sum(b.ncbx * b.ncby for b in bands)
        self.abi = Layout(profile=int(fourk), width=width, height=height, levels=6 if fourk else 5,
                          guardBits=2 if fourk else 1, numBands=len(bands), numCblks=n_cblks, baseStep=base_step,
                          bands=C.cast(self.bands, C.POINTER(Subband)))

    @property
    def num_cblks(self):
        return self.abi.numCblks


def make_layout(width, height, fourk, base_step=1.0):
    """The DCI layout (makeLayout, core/layout.h:87) computed by the library."""
    L = lib()
    L.gb_make_layout.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]
    bands = (Subband * 200)()
    nb, nc = C.c_int(), C.c_int()
    st = L.gb_make_layout(width, height, int(fourk), C.c_double(base_step), bands, 200, C.byref(nb), C.byref(nc))
    if st != 0:
        raise GailError(st, L.gb_last_error().decode())
    return list(bands[: nb.value])


class Plugin:
    def __init__(self, path: str | None = None):
        self.t = table(path)

    def err(self):
        return self.t.last_error().decode(errors="replace")

    def check(self, st):
        if st != 0:
            raise GailError(st, self.err())

    def device_count(self):
        return self.t.device_count()

    def device(self, index=0) -> "Device":
        return Device(self, index)


class Device:
    def __init__(self, plugin: Plugin, index: int):
        self.p = plugin
        h = C.c_void_p()
        self._log = LogFn(lambda u, lvl, m: None)
        self.p.check(self.p.t.device_create(index, self._log, None, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.p.t.device_destroy(self.h)
            self.h = None

    def name(self):
        return self.p.t.device_name(self.h).decode()

    def memory(self):
        m = Memory()
        self.p.check(self.p.t.device_memory(self.h, C.byref(m)))
        return m

    def encoder(self, layout: LayoutHolder, fmt: FrameFormat, col: Color) -> "Encoder":
        return Encoder(self, layout, fmt, col)

    def decoder(self, layout: LayoutHolder, reduce=0, high_bits=False) -> "Decoder":
        return Decoder(self, layout, reduce, high_bits)


class Tier1Frame:
    """A copy of one encode's Tier-1 output (the reference's Tier1Frame)."""

    def __init__(self, t: Tier1):
        n, npass, nd = t.numInfo, t.numPasses, t.numData
        self.info = np.ctypeslib.as_array(C.cast(t.info, C.POINTER(C.c_uint32)), (n * 5,)).reshape(n, 5).copy() \
            if n else np.zeros((0, 5), np.uint32)
        self.pass_len = np.ctypeslib.as_array(t.passLen, (npass,)).copy() if npass else np.zeros(0, np.uint32)
        self.pass_dist = np.ctypeslib.as_array(t.passDist, (npass,)).copy() if npass else np.zeros(0, np.int32)
        self.data = np.ctypeslib.as_array(t.data, (nd,)).copy() if nd else np.zeros(0, np.uint8)

    def block(self, i):
        nbps, np_, off, ln, pb = (int(x) for x in self.info[i])
        return nbps, np_, bytes(self.data[off:off + ln]), self.pass_len[pb:pb + np_], self.pass_dist[pb:pb + np_]


class Encoder:
    def __init__(self, dev: Device, layout: LayoutHolder, fmt: FrameFormat, col: Color):
        self.d, self.layout = dev, layout
        self.settings = EncodeSettings(profile=layout.abi.profile, width=layout.width, height=layout.height,
                                       baseStep=layout.abi.baseStep, slopeFactor=0.0, bitsPerSymbol=0.5, input=fmt,
                                       color=col)
        t = dev.p.t
        self.bytes = t.encoder_bytes(dev.h, C.byref(layout.abi), C.byref(self.settings))
        h = C.c_void_p()
        dev.p.check(t.encoder_create(dev.h, C.byref(layout.abi), C.byref(self.settings), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.d.p.t.encoder_destroy(self.h)
            self.h = None

    def input_buffer(self):
        return self.d.p.t.encoder_input(self.h)

    def set_slope(self, thr: float):
        self.d.p.t.encoder_set_slope(self.h, C.c_double(thr))

    def encode_view(self, frame_ptr):
        """encoder_encode of the frame at host address frame_ptr (the input buffer, or any
        host memory of the input format). Returns (the plugin's Tier1 view, valid until the
        next call on this encoder, and the timings), without copying the output."""
        out, tm = Tier1(), FrameTimings()
        self.d.p.check(self.d.p.t.encoder_encode(self.h, C.c_void_p(frame_ptr), C.byref(out), C.byref(tm), None))
        return out, tm

    def encode(self, frame: np.ndarray, debug: bool = False, full: bool = True):
        """frame: the input bytes (RGB48 interleaved or planar). Returns (Tier1Frame,
        timings, taps) where taps = dict(xyz12, coeffs, wavelet) when debug."""
        f = np.ascontiguousarray(frame)
        out = Tier1()
        tm = FrameTimings()
        dbg = Debug(full=int(full)) if debug else None
        st = self.d.p.t.encoder_encode(self.h, f.ctypes.data_as(C.c_void_p), C.byref(out), C.byref(tm),
                                       C.byref(dbg) if dbg is not None else None)
        self.d.p.check(st)
        t1 = Tier1Frame(out)
        taps = None
        if dbg is not None:
            taps = {"xyz12": np.ctypeslib.as_array(dbg.xyz12, (dbg.numXyz12,)).copy()}
            if full:
                taps["coeffs"] = np.ctypeslib.as_array(dbg.coeffs, (dbg.numCoeffs,)).copy()
                taps["wavelet"] = np.ctypeslib.as_array(dbg.wavelet, (dbg.numWavelet,)).copy()
        return t1, tm, taps


class Decoder:
    def __init__(self, dev: Device, layout: LayoutHolder, reduce=0, high_bits=False):
        self.d, self.layout = dev, layout
        self.settings = DecodeSettings(reduce=reduce, highBits=int(high_bits))
        h = C.c_void_p()
        dev.p.check(dev.p.t.decoder_create(dev.h, C.byref(layout.abi), C.byref(self.settings), C.byref(h)))
        self.h = h
        w, hh = layout.width, layout.height
        for _ in range(reduce):
            w, hh = (w + 1) // 2, (hh + 1) // 2
        self.out_w, self.out_h = w, hh

    def close(self):
        if self.h:
            self.d.p.t.decoder_destroy(self.h)
            self.h = None

    def decode(self, codestream: bytes, blocks: np.ndarray, frame_layout: LayoutHolder = None, wavelet=False,
               out: np.ndarray = None):
        """blocks: structured CblkCode array (one per code-block); out: an (H, W, 3) uint16
        picture to write into (a new one when None). Returns (picture, timings, wavelet
        planes or None)."""
        lay = frame_layout or self.layout
        data = np.frombuffer(codestream, np.uint8)
        if out is None:
            out = np.zeros((self.out_h, self.out_w, 3), np.uint16)
        elif out.shape != (self.out_h, self.out_w, 3) or out.dtype != np.uint16 or not out.flags.c_contiguous:
            raise ValueError("picture buffer of the wrong shape or type")
        tm = DecodeTimings(wantWavelet=int(wavelet))
        b = np.ascontiguousarray(blocks)
        st = self.d.p.t.decoder_decode(self.h, C.byref(lay.abi), data.ctypes.data_as(C.c_void_p), data.size,
                                       b.ctypes.data_as(C.POINTER(CblkCode)), len(b), out.ctypes.data_as(C.c_void_p),
                                       self.out_w * 6, C.byref(tm))
        self.d.p.check(st)
        wl = None
        if wavelet:
            n = tm.numWavelet
            wl = np.stack([np.ctypeslib.as_array(tm.wavelet[c], (n,)).copy() for c in range(3)])
        return out, tm, wl


CBLK_CODE_DTYPE = np.dtype({"names": ["offset", "len", "passes", "nbps"],
                            "formats": [np.uint32, np.uint32, np.uint8, np.uint8],
                            "offsets": [0, 4, 8, 9], "itemsize": 12})
