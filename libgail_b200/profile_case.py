"""Small, fixed encode cases for profiler captures.

  python -m libgail_b200.profile_case --path plain --frames 2 [--persistent]
  python -m libgail_b200.profile_case --path served --frames 8 --batch 8 [--size 2k] [--repeat 3] [--codestreams]
  python -m libgail_b200.profile_case --path decode --frames 2

Encodes seeded synthetic frames that are already in device memory, through the plain
per-frame encoder or the batched engine, and prints the stage times of the plain path, or
decodes the frames' DCI codestreams (made and parsed by the host codec) through the
plugin's decoder; --persistent runs Tier-1 encoding as one persistent launch (the
t1Persistent tuning knob) instead of four:
4K (3996x2160 Y'CbCr 4:2:2 10-bit, BT.2020 PQ, as the benchmark uses) or 2K (1998x1080
X'Y'Z' 12-bit, whose small frame slots keep a batched case to a few GB of device memory).
Exits non-zero on any encoder error, so that a profiler run after it sees the same
launches of a program that ended cleanly.
"""
from __future__ import annotations

import argparse
import ctypes as C

import numpy as np

W4K, H4K = 3996, 2160


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--path", choices=["plain", "served", "decode"], default="plain")
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--size", choices=["4k", "2k"], default="4k")
    ap.add_argument("--repeat", type=int, default=1, help="served: passes over the frames (the first warms up)")
    ap.add_argument("--codestreams", action="store_true",
                    help="served: DCI codestreams too (rate control and Tier-2 on the device)")
    ap.add_argument("--persistent", action="store_true", help="Tier-1 encoding as one persistent launch")
    args = ap.parse_args()

    import torch

    import libgail_b200 as gb
    from libgail_b200 import plugin as P
    from libgail_b200 import synth
    from libgail_b200.engine import Engine

    if args.size == "4k":
        frames = synth.many(synth.yuv422p10, args.frames, W4K, H4K, seed=1000)
        lay = P.LayoutHolder(W4K, H4K, 1)
        fmt = P.planar_format(W4K, H4K, bits=10, sx=1, sy=0)
        col = P.color("pq", "bt2020")
    else:
        W, H = 1998, 1080
        frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=1000 + i)) for i in range(args.frames)]
        lay = P.LayoutHolder(W, H, 0)
        fmt = P.rgb48_format(W, H)
        col = P.color_passthrough()
    dframes = [torch.from_numpy(f.view(np.int16)).to("cuda:0") for f in frames]
    torch.cuda.synchronize()
    if args.persistent:
        from libgail_b200 import autotune as AT
        AT.set_tuning(1 if args.size == "4k" else 0, {"t1Persistent": 1})
    dev = P.Plugin().device(0)
    try:
        if args.path == "plain":
            L = gb.lib()
            L.gb_encoder_enqueue_device.argtypes = [C.c_void_p, C.c_void_p]
            L.gb_encoder_finish.argtypes = [C.c_void_p]
            L.gb_encoder_stage_timing.argtypes = [C.c_void_p, C.c_int]
            L.gb_encoder_stage_times.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            enc = dev.encoder(lay, fmt, col)
            gb.check(L.gb_encoder_stage_timing(enc.h, 1))
            for f in dframes:
                gb.check(L.gb_encoder_enqueue_device(enc.h, C.c_void_p(f.data_ptr())))
            gb.check(L.gb_encoder_finish(enc.h))
            ms = np.zeros(5)
            n = C.c_int()
            gb.check(L.gb_encoder_stage_times(enc.h, ms.ctypes.data, C.byref(n)))
            print("ms per frame (front, cm, order, mq, pack):", np.round(ms / max(n.value, 1), 4).tolist())
            enc.close()
        elif args.path == "decode":
            from libgail_b200 import codestream as CS
            enc = dev.encoder(lay, fmt, col)
            streams = []
            for f in frames:
                view, _ = enc.encode_view(f.ctypes.data)
                streams.append(CS.rate_and_build(lay, view, 24.0)[0])
            enc.close()
            dec = dev.decoder(lay)
            pic = np.zeros((dec.out_h, dec.out_w, 3), np.uint16)
            for cs in streams:
                _, tm, _ = dec.decode(cs, CS.parse(cs)[1].view(P.CBLK_CODE_DTYPE), out=pic)
                print(f"decode ms: t1 {tm.t1:.3f} dwt {tm.dwt:.3f} colour+download {tm.color:.3f} ({len(cs)} bytes)")
            dec.close()
        else:
            import time
            eng = Engine(0, 0, max_batch=args.batch)
            cid, _ = eng.add_encoder(lay, fmt, col)
            eng.reserve(cid, len(dframes))  # a slot for every frame of the burst, made before it
            if args.codestreams:
                from libgail_b200 import codestream as CS
                eng.set_codestream(label=CS.DEFAULT_LABEL, tag="b200", threads=8)
            for rep in range(args.repeat):
                t0 = time.perf_counter()
                ids = [eng.submit(cid, f) for f in dframes]
                lat = []
                for _ in ids:
                    rid, _, ms, st = eng.wait(120000, copy=False)
                    if rid < 0 or st != 0:
                        raise SystemExit(f"engine frame failed (id {rid}, status {st})")
                    if args.codestreams and eng.codestream(rid, copy=False)[1] != 1:
                        raise SystemExit(f"codestream of request {rid} failed the DCI check")
                    lat.append(ms)
                    eng.release(rid)
                dt = time.perf_counter() - t0
                what = "DCI codestreams" if args.codestreams else "Tier-1 frames to host memory"
                print(f"engine pass {rep}: {len(ids) / dt:.1f} frames/s ({what}), mean latency {np.mean(lat):.1f} ms")
            print("engine:", eng.stats())
            eng.close()
    finally:
        dev.close()


if __name__ == "__main__":
    main()
