"""The batched, served encoder from Python (gb_engine_* in include/gail_b200.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import GailError, check, lib
from .plugin import Color, DecodeSettings, EncodeSettings, FrameFormat, LayoutHolder, Tier1, Tier1Frame


def _bind():
    L = lib()
    if getattr(L, "_engine_bound", False):
        return L
    L.gb_engine_create.argtypes = [C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_void_p)]
    L.gb_engine_destroy.argtypes = [C.c_void_p]
    L.gb_engine_destroy.restype = None
    L.gb_engine_add_encoder.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint64)]
    L.gb_engine_reserve.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
    L.gb_engine_submit.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int64)]
    L.gb_engine_wait.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(Tier1), C.POINTER(C.c_double),
                                 C.POINTER(C.c_int)]
    L.gb_engine_release.argtypes = [C.c_void_p, C.c_int64]
    L.gb_engine_stats.argtypes = [C.c_void_p, C.c_void_p]
    L.gb_engine_stage_timing.argtypes = [C.c_void_p, C.c_int]
    L.gb_engine_decode_times.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.gb_engine_open_loop.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
    L.gb_engine_stage_times.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.gb_engine_set_codestream.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_char_p, C.c_char_p,
                                           C.c_int, C.c_int, C.c_int]
    L.gb_engine_set_slope_factor.argtypes = [C.c_void_p, C.c_double]
    L.gb_engine_frame_info.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.gb_engine_counters.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.gb_engine_codestream.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.POINTER(C.c_uint8)),
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
    L.gb_engine_set_policy.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
    L.gb_engine_add_decoder.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint64)]
    L.gb_engine_submit_decode.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_int64)]
    L.gb_engine_picture.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.POINTER(C.c_uint16)), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int)]
    L.gb_engine_hull.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.POINTER(C.c_uint8)),
                                 C.POINTER(C.POINTER(C.c_double))]
    L._engine_bound = True
    return L


class Engine:
    def __init__(self, device: int = 0, hbm_budget: int = 0, max_batch: int = 16):
        L = _bind()
        h = C.c_void_p()
        check(L.gb_engine_create(device, hbm_budget, max_batch, C.byref(h)))
        self.h = h
        self._keep = {}   # frames the engine still reads, by request id
        self._classes = []

    def close(self):
        if self.h:
            lib().gb_engine_destroy(self.h)
            self.h = None
            self._keep.clear()

    def add_encoder(self, layout: LayoutHolder, fmt: FrameFormat, col: Color):
        s = EncodeSettings(profile=layout.abi.profile, width=layout.width, height=layout.height,
                           baseStep=layout.abi.baseStep, slopeFactor=0.0, bitsPerSymbol=0.5, input=fmt, color=col)
        cid, nbytes = C.c_int(), C.c_uint64()
        check(lib().gb_engine_add_encoder(self.h, C.byref(layout.abi), C.byref(s), C.byref(cid), C.byref(nbytes)))
        self._classes.append((layout, s))
        return cid.value, nbytes.value

    def reserve(self, cls: int, slots: int) -> int:
        """Makes frame slots for class cls now, until it has `slots` (or the HBM budget is
        spent): serving capacity set up before the first request. Returns how many it has."""
        have = C.c_int()
        check(lib().gb_engine_reserve(self.h, cls, slots, C.byref(have)))
        return have.value

    def submit(self, cls: int, frame, slope: float = 0.0) -> int:
        """frame: a numpy array (host) or a torch CUDA tensor (device)."""
        on_device = hasattr(frame, "is_cuda") and frame.is_cuda
        ptr = frame.data_ptr() if on_device or hasattr(frame, "data_ptr") else frame.ctypes.data
        rid = C.c_int64()
        check(lib().gb_engine_submit(self.h, cls, C.c_void_p(ptr), int(on_device), C.c_double(slope), C.byref(rid)))
        self._keep[rid.value] = frame
        return rid.value

    def wait(self, timeout_ms: int = 60000, copy: bool = True):
        """(id, Tier1Frame or None, latency ms, status); id -1 on timeout."""
        rid, lat, st = C.c_int64(), C.c_double(), C.c_int()
        t = Tier1()
        check(lib().gb_engine_wait(self.h, timeout_ms, C.byref(rid), C.byref(t), C.byref(lat), C.byref(st)))
        if rid.value < 0:
            return -1, None, 0.0, 0
        return rid.value, (Tier1Frame(t) if copy else t), lat.value, st.value

    def set_policy(self, max_batch: int = 16, min_batch_pct: int = 25, max_wait_ms: float = 2.0):
        """Batch policy (the autotuner's engine knobs)."""
        check(lib().gb_engine_set_policy(self.h, max_batch, min_batch_pct, max_wait_ms))

    def set_codestream(self, fps: float = 24.0, max_mbps: float = 230.0, comp_mbps: float = 200.0,
                       label: str = "GAIL 1.1.0", tag: str = "", threads: int = 4, check_dci: bool = True,
                       on_device: bool = True, tier1: bool = False):
        """Every frame from now on also gets its DCI codestream, driven by `threads` host
        workers: rate control and Tier-2 on the device (on_device) or on the host workers;
        tier1: the Tier-1 frames (and hull points) also handed out in host memory."""
        flags = (0 if on_device else 1) | (2 if tier1 else 0)
        check(lib().gb_engine_set_codestream(self.h, fps, max_mbps, comp_mbps, label.encode(), tag.encode(), threads,
                                             int(check_dci), flags))

    def set_slope_factor(self, factor: float):
        """Tier-1 early termination at threshold = last frame's lambda x factor, with the
        frame coded again with every pass when its own lambda comes out lower (libgail's
        pipeline; its gail.h encoder uses 0.25). Needs codestreams on; 0 turns it off."""
        check(lib().gb_engine_set_slope_factor(self.h, factor))

    def frame_info(self, rid: int):
        """(the early-termination threshold a finished encode was first coded with, whether
        it was coded again with every pass)."""
        t, rc = C.c_double(), C.c_int()
        check(lib().gb_engine_frame_info(self.h, rid, C.byref(t), C.byref(rc)))
        return t.value, bool(rc.value)

    def counters(self):
        """For the engine's encodes so far: (host-to-device bytes, device-to-host bytes,
        kernels launched)."""
        a, b, k = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().gb_engine_counters(self.h, C.byref(a), C.byref(b), C.byref(k)))
        return a.value, b.value, k.value

    def transfer_bytes(self):
        """(host-to-device, device-to-host) bytes the engine's encodes copied so far."""
        return self.counters()[:2]

    def codestream(self, rid: int, copy: bool = True):
        """(codestream bytes, or (pointer, size) without copy; DCI verdict 1/0, -1 unchecked)."""
        p, n, ok = C.POINTER(C.c_uint8)(), C.c_uint64(), C.c_int()
        check(lib().gb_engine_codestream(self.h, rid, C.byref(p), C.byref(n), C.byref(ok)))
        if not copy:
            return (p, n.value), ok.value
        return (C.string_at(p, n.value) if n.value else b""), ok.value

    def add_decoder(self, layout: LayoutHolder, reduce: int = 0, high_bits: bool = False):
        """A decode class; returns its id and the device bytes one decode in flight takes."""
        ds = DecodeSettings(reduce=reduce, highBits=int(high_bits))
        cid, nbytes = C.c_int(), C.c_uint64()
        check(lib().gb_engine_add_decoder(self.h, C.byref(layout.abi), C.byref(ds), C.byref(cid), C.byref(nbytes)))
        self._classes.append((layout, ds))
        return cid.value, nbytes.value

    def submit_decode(self, cls: int, codestream: bytes) -> int:
        rid = C.c_int64()
        check(lib().gb_engine_submit_decode(self.h, cls, codestream, len(codestream), C.byref(rid)))
        return rid.value

    def picture(self, rid: int, copy: bool = True):
        """A finished decode's picture, (height, width, 3) uint16."""
        p, w, h = C.POINTER(C.c_uint16)(), C.c_int(), C.c_int()
        check(lib().gb_engine_picture(self.h, rid, C.byref(p), C.byref(w), C.byref(h)))
        a = np.ctypeslib.as_array(p, (h.value, w.value, 3))
        return a.copy() if copy else a

    def hull(self, rid: int, num_passes: int, copy: bool = True):
        """A finished encode's PCRD hull points computed on the GPU: (passes uint8, slope
        float64), num_passes entries each (its Tier-1 frame's pass count), in the layout of
        codestream.hull()."""
        p, s = C.POINTER(C.c_uint8)(), C.POINTER(C.c_double)()
        check(lib().gb_engine_hull(self.h, rid, C.byref(p), C.byref(s)))
        if num_passes == 0:
            return np.zeros(0, np.uint8), np.zeros(0, np.float64)
        a, b = np.ctypeslib.as_array(p, (num_passes,)), np.ctypeslib.as_array(s, (num_passes,))
        return (a.copy(), b.copy()) if copy else (a, b)

    def release(self, rid: int):
        check(lib().gb_engine_release(self.h, rid))
        self._keep.pop(rid, None)

    def open_loop(self, requests, arrivals):
        """An open-loop load driven by the library's own threads: requests[i] = (class id,
        kind, item) with kind "encode" (item: a numpy array or a torch tensor, host or
        device) or "decode" (item: codestream bytes), submitted arrivals[i] seconds after the
        start. Returns (latency ms per request, status per request, seconds to the last
        finish)."""
        n = len(requests)
        cls = np.array([r[0] for r in requests], np.int32)
        kind = np.array([0 if r[1] == "encode" else 1 for r in requests], np.int32)
        items = (C.c_void_p * max(1, n))()
        sizes = np.zeros(max(1, n), np.uint64)
        ondev = np.zeros(max(1, n), np.int32)
        keep = []
        for i, (_, k, it) in enumerate(requests):
            if k == "encode":
                on_device = hasattr(it, "is_cuda") and it.is_cuda
                items[i] = it.data_ptr() if hasattr(it, "data_ptr") else it.ctypes.data
                ondev[i] = int(on_device)
            else:
                b = C.create_string_buffer(bytes(it), len(it))
                keep.append(b)
                items[i] = C.cast(b, C.c_void_p).value
                sizes[i] = len(it)
            keep.append(it)
        arr = np.ascontiguousarray(arrivals, np.float64)
        lat = np.zeros(max(1, n), np.float64)
        st = np.zeros(max(1, n), np.int32)
        el = C.c_double()
        check(lib().gb_engine_open_loop(self.h, n, cls.ctypes.data, kind.ctypes.data, items, sizes.ctypes.data,
                                        ondev.ctypes.data, arr.ctypes.data, lat.ctypes.data, st.ctypes.data,
                                        C.byref(el)))
        return lat[:n], st[:n], el.value

    def decode_times(self, reset: bool = False):
        """For the decode requests since the last reset: host ms waiting for a decoder slot,
        parsing and in the slot; decodes; decoder slots made after their class was added."""
        ms = np.zeros(3, np.float64)
        n = np.zeros(2, np.uint64)
        check(lib().gb_engine_decode_times(self.h, int(bool(reset)), ms.ctypes.data, n.ctypes.data))
        return {"wait_ms": float(ms[0]), "parse_ms": float(ms[1]), "run_ms": float(ms[2]), "decodes": int(n[0]),
                "slots_made_later": int(n[1])}

    def stage_timing(self, on: bool):
        """Per-stage timing of the served path (CUDA events; a little overhead) on or off."""
        check(lib().gb_engine_stage_timing(self.h, int(bool(on))))

    def stage_times(self, reset: bool = False):
        """Totals since the last reset: ms by stage (front, cm, order, mq, pack, rc) and the
        counts they cover (front_frames, batches, batch_frames, rc_frames)."""
        ms = np.zeros(6, np.float64)
        n = np.zeros(4, np.uint64)
        check(lib().gb_engine_stage_times(self.h, int(bool(reset)), ms.ctypes.data, n.ctypes.data))
        return (dict(zip(["front", "cm", "order", "mq", "pack", "rc"], (float(x) for x in ms))),
                dict(zip(["front_frames", "batches", "batch_frames", "rc_frames"], (int(x) for x in n))))

    def stats(self):
        out = np.zeros(5, np.uint64)
        check(lib().gb_engine_stats(self.h, out.ctypes.data))
        return dict(zip(["frames", "batches", "batch_frames", "slots", "slot_bytes"], (int(x) for x in out)))
