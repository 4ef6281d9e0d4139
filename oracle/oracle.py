"""ctypes bindings for the CPU oracle: TEST INFRASTRUCTURE ONLY.

`Oracle` wraps liboracle.so, the plain-C restatement of the reference hot path
(oracle/gail_oracle.c). `Reference` wraps _ref/libgailref.so, the reference's own CPU
sources compiled by oracle/Makefile (present where the reference tree was available at
build time; the built file travels with the repository tree).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module;
the product (libgail_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgailref.so")

MAX_PASSES = 64


class T1Result(C.Structure):
    _fields_ = [("nbps", C.c_int32), ("num_passes", C.c_int32), ("data_len", C.c_uint32),
                ("num_symbols", C.c_uint32), ("pass_len", C.c_uint32 * 64), ("pass_dist", C.c_int32 * 64)]


class OrBand(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("comp", "res", "level", "orient", "px0", "py0", "w", "h", "ncbx", "ncby",
                                         "cblk_base", "eps", "mu", "mb")] + [("delta", C.c_float), ("weight", C.c_double)]


class OrCblk(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("band", "x0", "y0", "w", "h")]


class RefColor(C.Structure):
    """Every colour setting of the reference (ColorParams, core/color.h:84-100)."""
    _fields_ = [(n, C.c_int32) for n in ("transfer", "primaries", "toneMap", "toneNorm", "gamut", "lutSize")] + \
        [(n, C.c_double) for n in ("sdrWhite", "hdrPeak", "cinemaPeak", "hdrRefWhite", "cinemaRefWhite", "knee",
                                   "gamutThreshold")] + \
        [("lutData", C.POINTER(C.c_float)), ("lutCount", C.c_uint64), ("lutPath", C.c_char_p)]


def ref_color(transfer=0, primaries=0, tone_map=0, tone_norm=0, gamut=2, sdr_white=48.0, hdr_peak=1000.0,
              cinema_peak=48.0, hdr_ref_white=203.0, cinema_ref_white=16.0, knee=0.25, gamut_threshold=0.8,
              lut=None, lut_size=0, lut_path=b"") -> RefColor:
    """A RefColor with the reference's defaults; `lut` (float32, lut_size^3 * 3) is kept
    alive by the returned structure."""
    c = RefColor(transfer=transfer, primaries=primaries, toneMap=tone_map, toneNorm=tone_norm, gamut=gamut,
                 lutSize=lut_size, sdrWhite=sdr_white, hdrPeak=hdr_peak, cinemaPeak=cinema_peak,
                 hdrRefWhite=hdr_ref_white, cinemaRefWhite=cinema_ref_white, knee=knee,
                 gamutThreshold=gamut_threshold, lutData=None, lutCount=0, lutPath=lut_path)
    if lut is not None:
        arr = np.ascontiguousarray(lut, dtype=np.float32)
        c._lut = arr
        c.lutData = arr.ctypes.data_as(C.POINTER(C.c_float))
        c.lutCount = arr.size
    return c


class Planar(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("width", "height", "active_w", "active_h", "ox", "oy", "sx", "sy", "rgb",
                                         "bits", "full_range", "chroma")] + [("kr", C.c_double), ("kb", C.c_double)]


def _p(a, t=C.c_void_p):
    return a.ctypes.data_as(t)


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and the reference library when GAIL_REFERENCE_SRC names the
    reference source tree)."""
    import subprocess
    src = os.environ.get("GAIL_REFERENCE_SRC", "")
    subprocess.run(["make", "-s", "-C", HERE, "all" if ref else "liboracle.so", f"REF={src}"], check=True)


class T1Block:
    """The result of coding one block: the fields of the reference's T1Result."""

    def __init__(self, r: T1Result, data: bytes):
        self.nbps = r.nbps
        self.num_passes = r.num_passes
        self.data = data
        self.pass_len = list(r.pass_len[: r.num_passes])
        self.pass_dist = list(r.pass_dist[: r.num_passes])
        self.num_symbols = r.num_symbols

    def key(self):
        return (self.nbps, self.num_passes, self.data, tuple(self.pass_len), tuple(self.pass_dist))


class _Common:
    lib: C.CDLL

    def _t1(self, fn, coeffs, w, h, orient, max_passes=64, slope=0.0, dist_scale=1.0) -> T1Block:
        c = np.ascontiguousarray(coeffs, dtype=np.uint32).reshape(-1)
        assert c.size == 1024
        buf = np.zeros(4096 * 24 + 64, np.uint8)
        r = T1Result()
        rc = fn(_p(c), w, h, orient, max_passes, C.c_float(slope), C.c_float(dist_scale), _p(buf), buf.size, C.byref(r))
        if rc != 0:
            raise RuntimeError(f"Tier-1 encode failed ({rc})")
        return T1Block(r, bytes(buf[: r.data_len]))


class Oracle(_Common):
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        L = self.lib = C.CDLL(path)
        L.or_t1_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p,
                                   C.c_size_t, C.c_void_p]
        L.or_quantize.restype = C.c_uint32
        L.or_quantize.argtypes = [C.c_float, C.c_float, C.c_uint32]
        L.or_fdwt97_2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_idwt97_2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.or_synthesis_norm.restype = C.c_double
        L.or_synthesis_norm.argtypes = [C.c_int, C.c_int]
        L.or_geometry_counts.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.or_make_layout.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.or_color_init.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
        L.or_color_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_planar_to_rgb48.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_t1_decode.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.or_ict_inverse_pack.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]
        L.or_t1_encode_many.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        L.or_quantize_frame.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.or_dci_code.argtypes = [C.c_float]
        L.or_dci_code.restype = C.c_int

    def t1_encode(self, coeffs, w, h, orient, max_passes=64, slope=0.0, dist_scale=1.0) -> T1Block:
        return self._t1(self.lib.or_t1_encode, coeffs, w, h, orient, max_passes, slope, dist_scale)

    def quantize(self, v, inv_delta, max_mag):
        return self.lib.or_quantize(C.c_float(v), C.c_float(inv_delta), max_mag)

    def t1_encode_many(self, coeffs, geom4, slope=0.0, dist_scale=None, stride=65536):
        """or_t1_encode over n blocks: (info4, pass_len, pass_dist, codewords)."""
        c = np.ascontiguousarray(coeffs, np.uint32).reshape(-1, 1024)
        g = np.ascontiguousarray(geom4, np.int32).reshape(-1, 4)
        n = c.shape[0]
        ds = None if dist_scale is None else np.ascontiguousarray(dist_scale, np.float32)
        info = np.zeros((n, 4), np.uint32)
        plen = np.zeros((n, 64), np.uint32)
        pdist = np.zeros((n, 64), np.int32)
        data = np.zeros((n, stride), np.uint8)
        rc = self.lib.or_t1_encode_many(_p(c), _p(g), n, C.c_float(slope), None if ds is None else _p(ds), _p(info),
                                        _p(plen), _p(pdist), _p(data), stride)
        if rc != 0:
            raise RuntimeError(f"oracle Tier-1 failed ({rc})")
        return info, plen, pdist, [bytes(data[i, : info[i, 3]]) for i in range(n)]

    def quantize_frame(self, planes: np.ndarray, bands, cblks) -> np.ndarray:
        p = np.ascontiguousarray(planes, np.float32)
        _, h, w = p.shape
        b = (OrBand * len(bands))(*bands)
        k = (OrCblk * len(cblks))(*cblks)
        out = np.zeros((len(cblks), 1024), np.uint32)
        self.lib.or_quantize_frame(_p(p), w, h, b, k, len(cblks), _p(out))
        return out

    def dci_code(self, n: float) -> int:
        return self.lib.or_dci_code(C.c_float(n))

    def fdwt(self, plane: np.ndarray, levels: int) -> np.ndarray:
        p = np.ascontiguousarray(plane, dtype=np.float32).copy()
        h, w = p.shape
        self.lib.or_fdwt97_2d(_p(p), w, w, h, levels)
        return p

    def idwt(self, plane: np.ndarray, levels: int, skip: int = 0) -> np.ndarray:
        p = np.ascontiguousarray(plane, dtype=np.float32).copy()
        h, w = p.shape
        self.lib.or_idwt97_2d(_p(p), w, w, h, levels, skip)
        return p

    def layout(self, width, height, fourk, base_step=1.0):
        nb, nc = C.c_int(), C.c_int()
        self.lib.or_geometry_counts(width, height, 6 if fourk else 5, C.byref(nb), C.byref(nc))
        bands = (OrBand * nb.value)()
        cblks = (OrCblk * nc.value)()
        if self.lib.or_make_layout(width, height, int(fourk), C.c_double(base_step), bands, cblks) != 0:
            raise RuntimeError("layout: step size out of range")
        return list(bands), list(cblks)

    def color_frame(self, rgb48: np.ndarray, transfer: int, primaries: int, sdr_white: float = 48.0):
        """Interleaved R'G'B' 16-bit (H, W, 3) -> (planes (3, H, W) float32, xyz12 (H, W, 3))."""
        buf = C.create_string_buffer(65536 * 4 + 9 * 4 + 64)
        self.lib.or_color_init(buf, transfer, primaries, C.c_double(sdr_white))
        rgb = np.ascontiguousarray(rgb48, dtype=np.uint16)
        h, w = rgb.shape[:2]
        planes = np.zeros((3, h, w), np.float32)
        xyz = np.zeros((h, w, 3), np.uint16)
        self.lib.or_color_frame(buf, _p(rgb), h * w, _p(planes[0]), _p(planes[1]), _p(planes[2]), _p(xyz))
        return planes, xyz

    def planar_to_rgb48(self, fmt: Planar, src: np.ndarray) -> np.ndarray:
        out = np.zeros((fmt.height, fmt.width, 3), np.uint16)
        s = np.ascontiguousarray(src)
        self.lib.or_planar_to_rgb48(C.byref(fmt), _p(s), _p(out))
        return out

    def t1_decode(self, data: bytes, w, h, orient, nbps, passes, length=None) -> np.ndarray:
        out = np.zeros(1024, np.uint32)
        d = np.frombuffer(bytes(data) + b"\0", np.uint8)
        n = len(data) if length is None else length
        self.lib.or_t1_decode(_p(d), n, w, h, orient, nbps, passes, _p(out))
        return out


class Reference(_Common):
    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_t1_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p,
                                    C.c_size_t, C.c_void_p]
        L.ref_quantize.restype = C.c_uint32
        L.ref_quantize.argtypes = [C.c_float, C.c_float, C.c_uint32]
        L.ref_t1_decode.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.ref_quantize_frame.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
        L.ref_fdwt97_2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.ref_idwt97_2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_layout_counts.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.ref_make_layout.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.ref_synthesis_norm.restype = C.c_double
        L.ref_synthesis_norm.argtypes = [C.c_int, C.c_int]
        L.ref_color_frame.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        L.ref_color_tables.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.ref_planar_to_rgb48.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_suite_blocks.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.ref_plugin_layout_hash.restype = C.c_uint64
        L.ref_plugin_sizes.argtypes = [C.c_void_p]
        L.ref_usable_cpus.restype = C.c_int
        L.ref_color_params.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_color_frame_full.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p]
        L.ref_read_cube.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64]

    def error(self) -> str:
        return self.lib.ref_last_error().decode()

    def t1_encode(self, coeffs, w, h, orient, max_passes=64, slope=0.0, dist_scale=1.0) -> T1Block:
        return self._t1(self.lib.ref_t1_encode, coeffs, w, h, orient, max_passes, slope, dist_scale)

    def quantize(self, v, inv_delta, max_mag):
        return self.lib.ref_quantize(C.c_float(v), C.c_float(inv_delta), max_mag)

    def quantize_frame(self, planes: np.ndarray, width, height, fourk, base_step=1.0) -> np.ndarray:
        """The reference quantiser (quantizeFrame) on three Mallat planes: (numCblks, 1024) words."""
        p = np.ascontiguousarray(planes, np.float32).reshape(3, height, width)
        nb, nc = C.c_int(), C.c_int()
        if self.lib.ref_layout_counts(width, height, int(fourk), C.byref(nb), C.byref(nc)) != 0:
            raise RuntimeError(self.error())
        out = np.zeros((nc.value, 1024), np.uint32)
        if self.lib.ref_quantize_frame(width, height, int(fourk), C.c_double(base_step), _p(p[0]), _p(p[1]), _p(p[2]),
                                       _p(out)) != 0:
            raise RuntimeError(self.error())
        return out

    def t1_decode(self, data: bytes, w, h, orient, nbps, passes, length=None) -> np.ndarray:
        out = np.zeros(1024, np.uint32)
        d = np.frombuffer(bytes(data) + b"\0", np.uint8)
        n = len(data) if length is None else length
        self.lib.ref_t1_decode(_p(d), n, w, h, orient, nbps, passes, _p(out))
        return out

    def fdwt(self, plane: np.ndarray, levels: int) -> np.ndarray:
        p = np.ascontiguousarray(plane, dtype=np.float32).copy()
        h, w = p.shape
        self.lib.ref_fdwt97_2d(_p(p), w, h, levels)
        return p

    def idwt(self, plane: np.ndarray, levels: int, skip: int = 0) -> np.ndarray:
        p = np.ascontiguousarray(plane, dtype=np.float32).copy()
        h, w = p.shape
        self.lib.ref_idwt97_2d(_p(p), w, h, levels, skip)
        return p

    def layout(self, width, height, fourk, base_step=1.0):
        nb, nc = C.c_int(), C.c_int()
        if self.lib.ref_layout_counts(width, height, int(fourk), C.byref(nb), C.byref(nc)) != 0:
            raise RuntimeError(self.error())
        bands = (OrBand * nb.value)()
        cblks = np.zeros((nc.value, 5), np.int32)
        if self.lib.ref_make_layout(width, height, int(fourk), C.c_double(base_step), bands, _p(cblks)) != 0:
            raise RuntimeError(self.error())
        return list(bands), cblks

    def color_frame(self, rgb48: np.ndarray, transfer: int, primaries: int, sdr_white: float = 48.0):
        rgb = np.ascontiguousarray(rgb48, dtype=np.uint16)
        h, w = rgb.shape[:2]
        planes = np.zeros((3, h, w), np.float32)
        xyz = np.zeros((h, w, 3), np.uint16)
        self.lib.ref_color_frame(transfer, primaries, C.c_double(sdr_white), _p(rgb), h * w, _p(planes[0]),
                                 _p(planes[1]), _p(planes[2]), _p(xyz))
        return planes, xyz

    def color_tables(self, transfer: int, primaries: int, sdr_white: float = 48.0):
        eotf = np.zeros(65536, np.float32)
        params = np.zeros(48, np.float32)
        self.lib.ref_color_tables(transfer, primaries, C.c_double(sdr_white), _p(eotf), _p(params))
        return eotf, params

    def planar_to_rgb48(self, fmt: Planar, src: np.ndarray) -> np.ndarray:
        out = np.zeros((fmt.height, fmt.width, 3), np.uint16)
        s = np.ascontiguousarray(src)
        self.lib.ref_planar_to_rgb48(C.byref(fmt), _p(s), _p(out))
        return out

    def color_params(self, color: RefColor):
        """ColorConverter's parameter block (48 floats) and its 3D LUT size."""
        params = np.zeros(48, np.float32)
        n = C.c_int()
        if self.lib.ref_color_params(C.byref(color), _p(params), C.byref(n)) != 0:
            raise RuntimeError(self.error())
        return params, n.value

    def color_frame_full(self, rgb48: np.ndarray, color: RefColor):
        """convertFrame under any colour setting: ICT planes and X'Y'Z' codes."""
        rgb = np.ascontiguousarray(rgb48, dtype=np.uint16)
        h, w = rgb.shape[:2]
        planes = np.zeros((3, h, w), np.float32)
        xyz = np.zeros((h, w, 3), np.uint16)
        if self.lib.ref_color_frame_full(C.byref(color), _p(rgb), h * w, _p(planes[0]), _p(planes[1]),
                                         _p(planes[2]), _p(xyz)) != 0:
            raise RuntimeError(self.error())
        return planes, xyz

    def read_cube(self, path: str):
        """readCubeLut: (n, n^3 * 3 floats); raises RuntimeError with the reference's message."""
        n = C.c_int()
        out = np.zeros(256 ** 3 * 3 // 64, np.float32)
        if self.lib.ref_read_cube(path.encode(), C.byref(n), _p(out), out.size) != 0:
            raise RuntimeError(self.error())
        return n.value, out[: n.value ** 3 * 3].copy()

    def suite(self, which: int, ntrials: int):
        coeffs = np.zeros((ntrials, 1024), np.uint32)
        meta = np.zeros((ntrials, 4), np.int32)
        if self.lib.ref_suite_blocks(which, ntrials, _p(coeffs), _p(meta)) != 0:
            raise ValueError("unknown suite")
        return coeffs, meta

    def plugin_layout_hash(self) -> int:
        return self.lib.ref_plugin_layout_hash()

    def plugin_sizes(self):
        out = np.zeros(12, np.uint64)
        self.lib.ref_plugin_sizes(_p(out))
        return [int(x) for x in out]


def have_reference() -> bool:
    return os.path.exists(REF_SO)


class RefEncOut(C.Structure):
    _fields_ = [("info", C.POINTER(C.c_uint32)), ("passLen", C.POINTER(C.c_uint32)), ("passDist", C.POINTER(C.c_int32)),
                ("data", C.POINTER(C.c_uint8)), ("numInfo", C.c_uint64), ("numPasses", C.c_uint64),
                ("numData", C.c_uint64), ("xyz12", C.POINTER(C.c_uint16)), ("coeffs", C.POINTER(C.c_uint32)),
                ("ms", C.c_double)]


class RefTier1:
    """A copy of the reference CPU encoder's Tier1Frame."""

    def __init__(self, o: RefEncOut):
        n, npass, nd = o.numInfo, o.numPasses, o.numData
        self.info = np.ctypeslib.as_array(o.info, (n * 5,)).reshape(n, 5).copy()
        self.pass_len = np.ctypeslib.as_array(o.passLen, (npass,)).copy() if npass else np.zeros(0, np.uint32)
        self.pass_dist = np.ctypeslib.as_array(o.passDist, (npass,)).copy() if npass else np.zeros(0, np.int32)
        self.data = np.ctypeslib.as_array(o.data, (nd,)).copy() if nd else np.zeros(0, np.uint8)
        self.ms = o.ms


def _ref_bind(L):
    L.ref_encoder_create.restype = C.c_void_p
    L.ref_encoder_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                     C.c_int]
    L.ref_encoder_encode.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.POINTER(RefEncOut)]
    L.ref_encoder_destroy.argtypes = [C.c_void_p]
    L.ref_encoder_create_color.restype = C.c_void_p
    L.ref_encoder_create_color.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
    L.ref_rate_and_build.restype = C.c_longlong
    L.ref_rate_and_build.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_uint64, C.c_void_p,
                                     C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_double, C.c_double,
                                     C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]
    L.ref_build.restype = C.c_longlong
    L.ref_build.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                            C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64]
    L.ref_hull.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                           C.c_uint64, C.c_void_p, C.c_void_p]
    L.ref_check_dci.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_char_p, C.c_uint64]
    L.ref_parse.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_int),
                            C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ref_decode.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong, C.c_void_p,
                             C.POINTER(C.c_double)]
    L.ref_empty_codestream_bytes.restype = C.c_longlong
    L.ref_empty_codestream_bytes.argtypes = [C.c_int, C.c_int, C.c_int]
    L.ref_dci_limits.argtypes = [C.c_double, C.c_double, C.c_double, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]


CBLK_CODE = np.dtype({"names": ["offset", "len", "passes", "nbps"], "formats": [np.uint32, np.uint32, np.uint8, np.uint8],
                      "offsets": [0, 4, 8, 9], "itemsize": 12})


class RefEncoder:
    """The reference CPU encoder (CpuSlot through createCpuDevice) on one frame format."""

    def __init__(self, ref: "Reference", width, height, fourk, transfer=5, primaries=4, sdr_white=48.0,
                 planar: Planar = None, threads=0, base_step=1.0, color: RefColor = None):
        self.ref = ref
        _ref_bind(ref.lib)
        pl = C.byref(planar) if planar is not None else None
        if color is not None:  # every colour setting (tone map, gamut, 3D LUT)
            self._color = color
            self.h = ref.lib.ref_encoder_create_color(width, height, int(fourk), C.c_double(base_step),
                                                      C.byref(color), pl, threads)
        else:
            self.h = ref.lib.ref_encoder_create(width, height, int(fourk), C.c_double(base_step), transfer,
                                                primaries, C.c_double(sdr_white), pl, threads)
        if not self.h:
            raise RuntimeError(ref.error())
        self.width, self.height, self.fourk = width, height, fourk

    def encode(self, frame: np.ndarray, slope=0.0, debug=False) -> RefTier1:
        o = RefEncOut()
        f = np.ascontiguousarray(frame)
        if self.ref.lib.ref_encoder_encode(self.h, _p(f), C.c_double(slope), int(debug), C.byref(o)) != 0:
            raise RuntimeError(self.ref.error())
        t = RefTier1(o)
        if debug:
            t.xyz12 = np.ctypeslib.as_array(o.xyz12, (self.width * self.height * 3,)).copy()
            t.coeffs = np.ctypeslib.as_array(o.coeffs, (t.info.shape[0] * 1024,)).copy()
        return t

    def close(self):
        if self.h:
            self.ref.lib.ref_encoder_destroy(self.h)
            self.h = None


def ref_codestream(ref: "Reference", width, height, fourk, t1, fps=24.0, mbps=230.0, tag=b"", base_step=1.0):
    """allocateRate + buildCodestream on a Tier-1 frame (info (n, 5), pass arrays, data)."""
    _ref_bind(ref.lib)
    info = np.ascontiguousarray(t1.info, np.uint32)
    n = info.shape[0]
    pl = np.ascontiguousarray(t1.pass_len, np.uint32)
    pd = np.ascontiguousarray(t1.pass_dist, np.int32)
    data = np.ascontiguousarray(t1.data, np.uint8)
    passes = np.zeros(n, np.uint8)
    cs = np.zeros(4 << 20, np.uint8)
    lam, ms = C.c_double(), C.c_double()
    size = ref.lib.ref_rate_and_build(width, height, int(fourk), C.c_double(base_step), _p(info), n, _p(pl), _p(pd),
                                      pl.size, _p(data), data.size, C.c_double(fps), C.c_double(mbps), tag, _p(passes),
                                      _p(cs), cs.size, C.byref(lam), C.byref(ms))
    if size < 0:
        raise RuntimeError(ref.error())
    return bytes(cs[:size]), passes, lam.value, ms.value


def ref_hull(ref: "Reference", width, height, fourk, t1, base_step=1.0):
    """The reference's PCRD hull points (buildHull) per pass slot of the Tier-1 frame:
    (passes uint8, slope float64), a block's points from its passBase on, then zeros."""
    _ref_bind(ref.lib)
    info = np.ascontiguousarray(t1.info, np.uint32)
    pl = np.ascontiguousarray(t1.pass_len, np.uint32)
    pd = np.ascontiguousarray(t1.pass_dist, np.int32)
    passes = np.zeros(max(pl.size, 1), np.uint8)
    slope = np.zeros(max(pl.size, 1), np.float64)
    if ref.lib.ref_hull(width, height, int(fourk), C.c_double(base_step), _p(info), info.shape[0], _p(pl), _p(pd),
                        pl.size, _p(passes), _p(slope)) != 0:
        raise RuntimeError(ref.error())
    return passes[: pl.size], slope[: pl.size]


def ref_parse(ref: "Reference", cs: bytes, reduce=0):
    _ref_bind(ref.lib)
    d = np.frombuffer(cs, np.uint8)
    blocks = np.zeros(40000, CBLK_CODE)
    nb, w, h, lv = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    if ref.lib.ref_parse(_p(d), d.size, reduce, _p(blocks), len(blocks), C.byref(nb), C.byref(w), C.byref(h),
                         C.byref(lv)) != 0:
        raise RuntimeError(ref.error())
    return blocks[: nb.value].copy(), w.value, h.value, lv.value


def ref_decode(ref: "Reference", cs: bytes, width, height, reduce=0, high_bits=False, threads=0, wavelet=False):
    _ref_bind(ref.lib)
    d = np.frombuffer(cs, np.uint8)
    ow, oh = width, height
    for _ in range(reduce):
        ow, oh = (ow + 1) // 2, (oh + 1) // 2
    out = np.zeros((oh, ow, 3), np.uint16)
    wl = np.zeros((3, height, width), np.float32) if wavelet else None
    ms = C.c_double()
    if ref.lib.ref_decode(_p(d), d.size, reduce, int(high_bits), threads, _p(out), ow * 6,
                          _p(wl) if wavelet else None, C.byref(ms)) != 0:
        raise RuntimeError(ref.error())
    return out, wl, ms.value


def ref_check(ref: "Reference", cs: bytes, fps=24.0):
    _ref_bind(ref.lib)
    d = np.frombuffer(cs, np.uint8)
    msg = C.create_string_buffer(512)
    ok = ref.lib.ref_check_dci(_p(d), d.size, C.c_double(fps), msg, 512)
    return bool(ok), msg.value.decode(errors="replace")
