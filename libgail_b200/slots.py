"""The plain per-frame path as libgail drives a CUDA plugin: slot threads, each with its
own encoder object (src/core/pipeline.cpp:166-249). Frames are taken in order; a slot
copies its frame into its encoder's pinned input buffer, encodes it through the plugin
table's encoder_encode (upload, device stages, download of the Tier-1 frame), then makes
the DCI codestream (rate control, Tier-2) and checks it, all on its own thread. Different
encoders run concurrently; one encoder is never called from two threads at once."""
from __future__ import annotations

import ctypes as C
import threading
import time

from . import codestream as CS
from . import plugin as P


class SlotPipeline:
    def __init__(self, dev: P.Device, layout: P.LayoutHolder, fmt, col, slots: int = 3, fps: float = 24.0,
                 max_mbps: float = 230.0, label: str = CS.DEFAULT_LABEL, tag: str = "", check: bool = True):
        self.layout, self.fps, self.max_mbps, self.label, self.tag, self.check = layout, fps, max_mbps, label, tag, check
        self.encoders = [dev.encoder(layout, fmt, col) for _ in range(slots)]

    def close(self):
        for e in self.encoders:
            e.close()
        self.encoders = []

    def run(self, frames, arrivals=None):
        """Encodes frames (host arrays) in order; arrivals: seconds after the start at which
        each frame may start (None: all at once). Returns per frame (codestream bytes, DCI
        verdict (None unchecked), latency in ms from its arrival to its codestream), and the
        wall time of the whole run in seconds."""
        n = len(frames)
        results = [None] * n
        nxt = [0]
        lock = threading.Lock()
        errors = []
        t0 = time.perf_counter()

        def slot(enc):
            buf = enc.input_buffer()
            try:
                while True:
                    with lock:
                        i = nxt[0]
                        nxt[0] += 1
                    if i >= n:
                        return
                    due = arrivals[i] if arrivals is not None else 0.0
                    while time.perf_counter() - t0 < due:
                        time.sleep(0.0002)
                    f = frames[i]
                    C.memmove(buf, f.ctypes.data, f.nbytes)
                    view, _ = enc.encode_view(buf)
                    cs, _, _ = CS.rate_and_build(self.layout, view, self.fps, self.max_mbps, label=self.label,
                                                 tag=self.tag)
                    ok = CS.check_dci(cs, self.fps)[0] if self.check else None
                    results[i] = (cs, ok, (time.perf_counter() - t0 - due) * 1e3)
            except Exception as ex:  # reported after the others finish
                errors.append(ex)

        threads = [threading.Thread(target=slot, args=(e,)) for e in self.encoders]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        return results, time.perf_counter() - t0
