"""The project's autotuner: per frame profile (2K, 4K) on this GPU, the launch knobs whose
best value depends on the workload and the device -- the front end's tile shape at level 1
and at the later levels (64 x 64, 128 x 64, 64 x 128), the MQ solo threshold, the grid caps
of context modelling, MQ coding and Tier-1 decoding, Tier-1 as one persistent launch or
four, the decoder's heavy-block threshold -- and the engine's batch policy, chosen by
timing candidates on seeded synthetic frames. Every candidate gives bit-identical output
(the knobs change launch shapes and work order, never the arithmetic), so only speed is
compared. The result is a JSON file keyed by the GPU's name; apply() loads it into the
library (gb_set_tuning) and returns the engine policy for Engine.set_policy().

  python -m libgail_b200.autotune --out libgail_b200/tuning_b200.json [--quick]
  python -m libgail_b200.autotune --tiles     # the front-end tile-shape grid alone
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import check, lib

DEFAULTS = {"soloDecisions": 16384, "cmCtasPerSm": 16, "mqCtasPerSm": 16, "decCtasPerSm": 32, "t1Persistent": 0,
            "decHeavyPct": 150, "dwtTile1": 0, "dwtTileN": 0}
POLICY_DEFAULT = {"maxBatch": 16, "minBatchPct": 25, "maxWaitMs": 2.0}
PROFILES = {"2k": 0, "4k": 1}


class GbTuning(C.Structure):
    _fields_ = [("soloDecisions", C.c_uint32), ("cmCtasPerSm", C.c_int32), ("mqCtasPerSm", C.c_int32),
                ("decCtasPerSm", C.c_int32), ("t1Persistent", C.c_int32), ("decHeavyPct", C.c_int32),
                ("dwtTile1", C.c_int32), ("dwtTileN", C.c_int32)]


def _bind():
    L = lib()
    if not getattr(L, "_tuning_bound", False):
        L.gb_set_tuning.argtypes = [C.c_int, C.c_void_p]
        L.gb_get_tuning.argtypes = [C.c_int, C.c_void_p]
        L._tuning_bound = True
    return L


def set_tuning(profile: int, t: dict | None):
    """Stores a profile's knobs in the library (None restores the defaults; a knob left out
    takes its default)."""
    L = _bind()
    if t is None:
        check(L.gb_set_tuning(profile, None))
    else:
        v = GbTuning(**{k: int(t.get(k, DEFAULTS[k])) for k in DEFAULTS})
        check(L.gb_set_tuning(profile, C.byref(v)))


def get_tuning(profile: int) -> dict:
    v = GbTuning()
    check(_bind().gb_get_tuning(profile, C.byref(v)))
    return {k: int(getattr(v, k)) for k in DEFAULTS}


def coordinate_search(start: dict, space: dict, measure, rounds: int = 1, log=None):
    """Minimises measure(config) one knob at a time over its candidates (keeping the others),
    `rounds` sweeps over the knobs. Returns (best config, its cost, every (config, cost))."""
    best = dict(start)
    best_cost = measure(best)
    seen = [(dict(best), best_cost)]
    for _ in range(rounds):
        for knob, values in space.items():
            for v in values:
                if v == best[knob]:
                    continue
                cand = dict(best, **{knob: v})
                cost = measure(cand)
                seen.append((dict(cand), cost))
                if log:
                    log(f"  {knob}={v}: {cost:.4f}")
                if cost < best_cost:
                    best, best_cost = cand, cost
    return best, best_cost, seen


def apply(path: str, device_name: str | None = None) -> dict:
    """Loads a tuning file into the library; returns its engine policy. A file made on a
    different GPU is not applied (the defaults stay) and the default policy is returned."""
    with open(path) as f:
        d = json.load(f)
    if device_name is not None and d.get("device") != device_name:
        return dict(POLICY_DEFAULT)
    for name, prof in PROFILES.items():
        if name in d.get("profiles", {}):
            set_tuning(prof, d["profiles"][name])
    return dict(POLICY_DEFAULT, **d.get("policy", {}))


# ---------------------------------------------------------------------------- measuring
def _workload(name: str, nframes: int):
    from . import plugin as P
    from . import synth
    if name == "4k":
        W, H = 3996, 2160
        frames = synth.many(synth.yuv422p10, nframes, W, H, seed=4242)
        return P.LayoutHolder(W, H, 1), P.planar_format(W, H, bits=10, sx=1, sy=0), P.color("pq", "bt2020"), frames
    W, H = 1998, 1080
    frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=4242 + i)) for i in range(nframes)]
    return P.LayoutHolder(W, H, 0), P.rgb48_format(W, H), P.color_passthrough(), frames


def _stage_timer(L, enc, dframes, prof: int, n: int):
    """stage_ms(cfg, stages): the plain encoder's device time per frame of the given stages
    (0 front end, 1 context modelling, 2 ordering, 3 MQ, 4 packing; CUDA events) over n
    device-resident frames, with the profile's knobs set to cfg first."""
    def stage_ms(cfg, stages):
        set_tuning(prof, cfg)
        for f in dframes[:2]:
            check(L.gb_encoder_enqueue_device(enc.h, C.c_void_p(f.data_ptr())))
        check(L.gb_encoder_finish(enc.h))
        ms5, cnt = np.zeros(5), C.c_int()
        check(L.gb_encoder_stage_timing(enc.h, 1))
        check(L.gb_encoder_stage_times(enc.h, ms5.ctypes.data, C.byref(cnt)))
        for f in dframes[:n]:
            check(L.gb_encoder_enqueue_device(enc.h, C.c_void_p(f.data_ptr())))
        check(L.gb_encoder_stage_times(enc.h, ms5.ctypes.data, C.byref(cnt)))
        check(L.gb_encoder_stage_timing(enc.h, 0))
        return float(sum(ms5[k] for k in stages)) / max(cnt.value, 1)
    return stage_ms


def _bind_encoder_timing(L):
    L.gb_encoder_enqueue_device.argtypes = [C.c_void_p, C.c_void_p]
    L.gb_encoder_finish.argtypes = [C.c_void_p]
    L.gb_encoder_stage_timing.argtypes = [C.c_void_p, C.c_int]
    L.gb_encoder_stage_times.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]


def _best_of(measure, runs: int):
    """The fastest of `runs` measurements (noise on a shared host only ever adds time)."""
    return lambda cfg: min(measure(cfg) for _ in range(runs))


def tune(quick: bool = False, log=print, runs: int = 2) -> dict:
    import torch

    import libgail_b200 as gb
    from . import codestream as CS
    from . import plugin as P
    from .engine import Engine

    L = gb.lib()
    _bind_encoder_timing(L)
    dev = P.Plugin().device(0)
    out = {"device": torch.cuda.get_device_name(0), "sms": torch.cuda.get_device_properties(0).multi_processor_count,
           "profiles": {}, "policy": {}, "measured": {}}
    try:
        for name, prof in PROFILES.items():
            n = 4 if name == "4k" else 8
            if quick:
                n //= 2
            lay, fmt, col, frames = _workload(name, 3 * n)
            dframes = [torch.from_numpy(f.view(np.int16)).to("cuda:0") for f in frames]
            torch.cuda.synchronize()
            enc = dev.encoder(lay, fmt, col)
            stage_ms = _stage_timer(L, enc, dframes, prof, n)  # plain one-frame launches

            def tier1_ms(cfg):  # context modelling + MQ
                return stage_ms(cfg, (1, 3))

            def front_ms(cfg):  # colour + wavelet + quantisation
                return stage_ms(cfg, (0,))

            eng = Engine(0, 0, max_batch=POLICY_DEFAULT["maxBatch"])
            cid, _ = eng.add_encoder(lay, fmt, col)
            eng.reserve(cid, len(dframes))  # a slot per frame of a burst before the first one

            def served_ms(cfg):  # wall time per frame of a burst through the engine, Tier-1 only
                set_tuning(prof, cfg)
                ids = [eng.submit(cid, f) for f in dframes[:n]]  # warm
                for _ in ids:
                    eng.release(eng.wait(120000, copy=False)[0])
                t0 = time.perf_counter()
                ids = [eng.submit(cid, f) for f in dframes]
                for _ in ids:
                    eng.release(eng.wait(120000, copy=False)[0])
                return (time.perf_counter() - t0) * 1e3 / len(dframes)

            cfg = dict(DEFAULTS)
            log(f"[{name}] front-end tile shapes (front-end ms per frame)")
            tiles = {"dwtTile1": [1, 2], "dwtTileN": [1, 2]}
            cfg, _, seen0 = coordinate_search(cfg, tiles, _best_of(front_ms, runs), log=log)
            log(f"[{name}] MQ solo threshold (Tier-1 ms per frame)")
            solo = {"soloDecisions": [4096, 8192, 32768, 1 << 30]}
            cfg, _, seen1 = coordinate_search(cfg, solo, _best_of(tier1_ms, runs), log=log)
            log(f"[{name}] grid caps (served ms per frame)")
            caps = {"cmCtasPerSm": [8, 12, 24], "mqCtasPerSm": [8, 12, 24], "t1Persistent": [1]}
            cfg, _, seen2 = coordinate_search(cfg, caps, _best_of(served_ms, runs), log=log)
            # the decoder's cap on this profile's own codestreams
            streams = []
            for f in frames[:2]:
                view, _ = enc.encode_view(f.ctypes.data)
                streams.append(CS.rate_and_build(lay, view, 24.0)[0])
            # as decode requests to the engine, several in flight: the cap that serves most
            dcls, _ = eng.add_decoder(lay)

            def decode_ms(c):  # wall time per decode of a burst through the engine
                set_tuning(prof, c)
                for rep in range(2):  # the first burst warms up (and makes the decoder slots)
                    t0 = time.perf_counter()
                    ids = [eng.submit_decode(dcls, s) for s in streams * 4]
                    for _ in ids:
                        eng.release(eng.wait(120000, copy=False)[0])
                return (time.perf_counter() - t0) * 1e3 / len(ids)

            log(f"[{name}] decoder grid cap (served decode ms per frame)")
            cfg, _, seen3 = coordinate_search(cfg, {"decCtasPerSm": [16, 24, 48, 64]}, _best_of(decode_ms, runs),
                                             log=log)
            # the heavy-block threshold by one frame's Tier-1 decode on its own (the latency of
            # decoder_decode: the longest codewords' serial chains set it)
            blocks = [CS.parse(s)[1].view(P.CBLK_CODE_DTYPE) for s in streams]
            dec = dev.decoder(lay)
            pic = np.zeros((lay.height, lay.width, 3), np.uint16)

            def decode_t1_ms(c):
                set_tuning(prof, c)
                t = []
                for s, b in zip(streams, blocks):
                    dec.decode(s, b, out=pic)
                    t.append(dec.decode(s, b, out=pic)[1].t1)
                return float(np.mean(t))

            log(f"[{name}] decoder heavy-block threshold (Tier-1 decode ms of one frame)")
            cfg, _, seen5 = coordinate_search(cfg, {"decHeavyPct": [0, 150, 400, 800]}, _best_of(decode_t1_ms, runs),
                                             log=log)
            seen3 = seen3 + seen5
            dec.close()
            if name == "4k":
                log("[4k] engine batch policy (served ms per frame)")
                pol = dict(POLICY_DEFAULT)

                def policy_ms(p):
                    eng.set_policy(p["maxBatch"], p["minBatchPct"], p["maxWaitMs"])
                    return served_ms(cfg)

                space = {"maxBatch": [8, 32], "minBatchPct": [10, 50]}
                pol, _, seen4 = coordinate_search(pol, space, _best_of(policy_ms, runs), log=log)
                out["policy"] = pol
                out["measured"]["policy"] = [[c, round(v, 4)] for c, v in seen4]
            eng.close()
            enc.close()
            out["profiles"][name] = cfg
            out["measured"][name] = [[c, round(v, 4)] for c, v in seen0 + seen1 + seen2 + seen3]
            set_tuning(prof, None)
    finally:
        dev.close()
    return out


def tile_sweep(runs: int = 3, nframes: int = 8, log=print) -> dict:
    """The front end's device time per frame (colour, every 9/7 level and quantisation; ms,
    best of `runs`) for every pair of tile shapes, level 1 x the later levels (0 = 64 x 64,
    1 = 128 x 64, 2 = 64 x 128), on the 4K and 2K workloads: the whole grid the autotuner's
    coordinate search walks part of."""
    import torch

    import libgail_b200 as gb
    from . import plugin as P

    L = gb.lib()
    _bind_encoder_timing(L)
    dev = P.Plugin().device(0)
    out = {"device": torch.cuda.get_device_name(0)}
    try:
        for name in ("4k", "2k"):
            prof = PROFILES[name]
            lay, fmt, col, frames = _workload(name, nframes)
            dframes = [torch.from_numpy(f.view(np.int16)).to("cuda:0") for f in frames]
            torch.cuda.synchronize()
            enc = dev.encoder(lay, fmt, col)
            try:
                stage_ms = _stage_timer(L, enc, dframes, prof, nframes)
                table = {}
                for t1 in range(3):
                    for tn in range(3):
                        cfg = dict(DEFAULTS, dwtTile1=t1, dwtTileN=tn)
                        table[f"{t1},{tn}"] = round(min(stage_ms(cfg, (0,)) for _ in range(runs)), 4)
                        log(f"[{name}] dwtTile1={t1} dwtTileN={tn}: {table[f'{t1},{tn}']:.4f} ms")
            finally:
                enc.close()
                set_tuning(prof, None)
            out[name] = table
    finally:
        dev.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="tuning.json")
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--tiles", action="store_true",
                    help="only time every pair of front-end tile shapes and print the table")
    args = ap.parse_args()
    if args.tiles:
        print(json.dumps(tile_sweep()))
        return
    res = tune(quick=args.quick)
    with open(args.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({"device": res["device"], "profiles": res["profiles"], "policy": res["policy"]}))


if __name__ == "__main__":
    main()
