"""Serving a mix of encode and decode requests as they arrive, over all six DCI profiles.

  python -m libgail_b200.serve_mix [--requests 20000] [--loads 50,100,150,200,250,300,350,400]
                                   [--budget-gb 150] [--workers 14] [--seed 11] [--out FILE]

Requests arrive as a Poisson process at each offered load in turn: 70 % encodes and 30 %
decodes; per request a profile, 50 % 4K flat (3996x2160), 30 % 2K flat (1998x1080) and 20 %
spread evenly over the other four (2048x858, 2048x1080, 4096x1716, 4096x2160). Encodes take
seeded X'Y'Z' 12-bit frames of their profile (in pinned host memory) to DCI codestreams (PCRD to 230 Mbit/s at 24
fps, every codestream checked); decodes take codestreams this engine made of the same
frames back to pictures. One engine serves them all, admitting frames against an HBM budget
of its measured per-frame footprints. Per load it prints one JSON line: the achieved rate
and the p50 / p99 latency (arrival to result) by kind and by profile. With the defaults a
run takes about 18 minutes on one B200 (20,000 requests per load); --requests and --loads
make shorter ones.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

# (width, height, 4K layout, share of the requests)
PROFILES = [(3996, 2160, 1, 0.50), (1998, 1080, 0, 0.30), (2048, 858, 0, 0.05), (2048, 1080, 0, 0.05),
            (4096, 1716, 1, 0.05), (4096, 2160, 1, 0.05)]
ENCODE_SHARE = 0.7
FRAMES_PER_PROFILE = 4
WARM_BURST = 8  # requests of each class at once before the timed loads
RESERVE = 16    # frame slots reserved per encode class before serving


def arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Seconds after the start at which each of n Poisson requests arrives."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def draw(n: int, seed: int):
    """Per request: encode (True) or decode, its profile index and a frame pick."""
    rng = np.random.default_rng(seed)
    kinds = rng.random(n) < ENCODE_SHARE
    shares = np.array([p[3] for p in PROFILES])
    prof = rng.choice(len(PROFILES), size=n, p=shares / shares.sum())
    picks = rng.integers(0, FRAMES_PER_PROFILE, n)
    return kinds, prof, picks


def percentiles(v) -> dict:
    if not v:
        return {"requests": 0}
    return {"requests": len(v), "p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99))}


def serve(requests: int, loads, budget_gb: float, workers: int, seed: int, log=print):
    import torch

    from . import autotune as AT
    from . import codestream as CS
    from . import plugin as P
    from . import synth
    from .engine import Engine

    dev = P.Plugin().device(0)
    policy = AT.apply(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json"),
                      torch.cuda.get_device_name(0))
    eng = Engine(0, int(budget_gb * (1 << 30)), max_batch=policy["maxBatch"])
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    try:
        frames, enc_cls, dec_cls = [], [], []
        for i, (W, H, fk, _) in enumerate(PROFILES):
            lay = P.LayoutHolder(W, H, fk)
            # frames in pinned host memory, as a server receiving them would keep them (an
            # upload from pageable memory is staged by the driver on the engine's thread)
            frames.append([torch.from_numpy(synth.xyz12_to_rgb48(synth.xyz12_planes(W, H, seed=seed * 1000 + 10 * i + k))
                                            .view(np.int16)).pin_memory() for k in range(FRAMES_PER_PROFILE)])
            enc_cls.append(eng.add_encoder(lay, P.rgb48_format(W, H), P.color_passthrough())[0])
            eng.reserve(enc_cls[-1], RESERVE)  # serving capacity set up before the requests
            dec_cls.append(eng.add_decoder(lay)[0])
        eng.set_codestream(label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
        # the codestreams to decode, made by this engine; this also makes every class's slots
        streams = [[None] * FRAMES_PER_PROFILE for _ in PROFILES]
        ids = {eng.submit(enc_cls[p], frames[p][k]): (p, k) for p in range(len(PROFILES))
               for k in range(FRAMES_PER_PROFILE)}
        for _ in range(len(ids)):
            rid, _, _, st = eng.wait(120000, copy=False)
            if rid < 0 or st != 0:
                raise RuntimeError(f"warm-up encode failed (id {rid}, status {st})")
            cs, ok = eng.codestream(rid)
            if ok != 1:
                raise RuntimeError("a warm-up codestream failed the DCI check")
            p, k = ids[rid]
            streams[p][k] = cs
            eng.release(rid)
        # a burst of every class at once before the timed loads
        warm = [eng.submit(enc_cls[p], frames[p][k % FRAMES_PER_PROFILE]) for p in range(len(PROFILES))
                for k in range(WARM_BURST)]
        warm += [eng.submit_decode(dec_cls[p], streams[p][k % FRAMES_PER_PROFILE]) for p in range(len(PROFILES))
                 for k in range(WARM_BURST)]
        for _ in warm:
            rid, _, _, st = eng.wait(120000, copy=False)
            if rid < 0 or st != 0:
                raise RuntimeError(f"warm-up request failed (id {rid}, status {st})")
            eng.release(rid)

        kinds, prof, picks = draw(requests, seed)
        reqs = [(enc_cls[int(p)], "encode", frames[int(p)][int(k)]) if kd else
                (dec_cls[int(p)], "decode", streams[int(p)][int(k)]) for kd, p, k in zip(kinds, prof, picks)]
        rows = []
        for load in loads:
            # submitted and collected by the library's own threads at the arrival times
            # (open loop: a request arrives whether or not earlier ones have finished)
            lat, st, elapsed = eng.open_loop(reqs, arrivals(requests, load, seed + int(load)))
            bad = np.flatnonzero(st != 0)
            if bad.size:
                raise RuntimeError(f"{bad.size} requests failed at {load} requests/s, first {int(bad[0])}")
            kind = np.where(kinds, "encode", "decode")
            row = {"offered_per_s": load, "achieved_per_s": requests / elapsed, "requests": requests}
            for kd in ("encode", "decode"):
                row[kd] = percentiles(list(lat[kind == kd]))
            row["by_profile"] = {f"{W}x{H} {kd}": percentiles(list(lat[(kind == kd) & (prof == p)]))
                                 for p, (W, H, _, _) in enumerate(PROFILES) for kd in ("encode", "decode")}
            log(json.dumps(row))
            rows.append(row)
        return {"mix": "70 % encode / 30 % decode; 50 % 4K flat, 30 % 2K flat, 20 % over the other four "
                       "profiles; X'Y'Z' 12-bit frames, DCI codestreams at 230 Mbit/s",
                "budget_gb": budget_gb, "stats": eng.stats(), "loads": rows}
    finally:
        eng.close()
        dev.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--loads", default="50,100,150,200,250,300,350,400")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--workers", type=int, default=14)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    loads = [float(x) for x in args.loads.split(",") if x]
    res = serve(args.requests, loads, args.budget_gb, args.workers, args.seed)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
