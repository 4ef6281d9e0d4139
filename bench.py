#!/usr/bin/env python
"""Benchmark: 4K DCI JPEG 2000 encode on one B200 (and N replicas under torchrun).

Workload (the 4K configuration): 48 preloaded 3996x2160 frames of 10-bit Y'CbCr 4:2:2
BT.2020 PQ from the seeded generator (libgail_b200/synth.py), colour-converted on the GPU
to 12-bit X'Y'Z', 9/7 wavelet with 6 levels, 32x32 code-blocks, Tier-1 with every coding
pass (bit-exact with the CPU reference). One step = encoding all 48 frames; the 48 frames
(1.66 GB) are larger than L2, so no flush is needed between steps.

  value   DCI codestreams/s of the served path: the batched engine (continuous batching of
          Tier-1 over every frame in flight) on frames resident in HBM, rate control and
          Tier-2 on the device driven by host workers, every codestream DCI-checked. The K
          steps run as one job (all K x 48 requests submitted at once, the time to the last
          codestream). The work spans the engine's streams and threads, so the timed region
          is bracketed by a barrier and a device synchronisation on both sides; max over ranks.
  e2e     the same with the frames in pinned host memory: uploads and codestreams inside.
  served_* / plain_*  codestreams/s and p50 / p99 latency of both paths at one Poisson load
          (80 % of the plain rate, 480 requests each), and the served p99 at 90 % of its own
          end-to-end rate (480 requests).
          plain: the drop-in per-frame path as libgail drives the plugin (four slot threads,
          the frames in flight of the reference's own benchmark, each encoder_encode from
          host memory, then the host codec's rate control, Tier-2 and the DCI check).
  stages  the served path's stage split, live (the same job once more with the engine's
          CUDA-event stage timing on): ms per frame, algorithmic bytes and HBM fraction.
  roofline  the dominant kernel of the served run, t1CmKernel: integer-issue bound, so its
          roofline is the SM issue rate.
  decode  48 4K + 48 2K X'Y'Z' codestreams at 250 Mbit/s decoded at full and half size,
          one at a time (decoder_decode) and as engine decode requests.
  encode_decode_2k  the 2K configuration one frame at a time, encode and decode.
  six_profiles  16 frames over the six DCI profiles: Tier-1 as one persistent launch in
          the served engine against the plain per-frame path.
  mixed   Poisson encode and decode requests of 4K and 2K at four loads.

--impl reference times the reference's own CPU path (the CpuSlot encoder, then its rate
control, codestream writer and DCI checker, built from the reference sources into
oracle/_ref) on the same frames with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W4K, H4K, FRAMES = 3996, 2160, 48
FPS = 24.0  # DCI frame rate of the byte budgets
METRIC = "4K encode fps & p99 frame latency, served vs plain, 1 B200, Tier-1 bit-exact"
WORKLOAD = ("4K 3996x2160 Y'CbCr 4:2:2 10-bit BT.2020 PQ -> 12-bit X'Y'Z', 9/7 6 levels, 32x32 code-blocks, "
            "Tier-1 all passes, PCRD to the 230 Mbit/s DCI budget at 24 fps, every codestream DCI-checked, "
            "48 preloaded frames")


ET_FACTOR = 0.25  # the Tier-1 early-termination factor gail.h's encoder forces
DECODE_FRAMES = 48  # codestreams per profile of the decode configuration
# Per 4K frame of this workload, one batched t1CmKernel launch (context modelling of the
# frames' 25,986 code-blocks each) executes this many warp instructions and moves this many
# DRAM bytes: ncu counters smsp__inst_executed.sum and dram__bytes_read.sum +
# dram__bytes_write.sum of this build, divided by the frames in the launch. The achieved
# issue rate in the roofline divides them by the launch time measured in the run.
CM_WARP_INSTR_PER_FRAME = 685.89e6
CM_DRAM_BYTES_PER_FRAME = 220.35e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=None,
                    help="most frames per Tier-1 launch (served path; default: the tuning file's, else 16)")
    ap.add_argument("--tuning", default=os.path.join(ROOT, "libgail_b200", "tuning_b200.json"),
                    help="autotuner file applied when it was made on this GPU ('' for the defaults)")
    ap.add_argument("--slots", type=int, default=4,
                    help="slot threads (frames in flight) of the plain path, as libgail's gail-bench runs it (--slots 4)")
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


def gen_frames(count, seed=1000):
    from libgail_b200 import synth
    return synth.many(synth.yuv422p10, count, W4K, H4K, seed=seed)


def cpu_baseline(frames, sample=2):
    """The reference CPU encoder (or, without its build, the oracle port) on a bounded sample."""
    from oracle.oracle import Planar, Reference, RefEncoder, have_reference
    pl = Planar(width=W4K, height=H4K, active_w=W4K, active_h=H4K, ox=0, oy=0, sx=1, sy=0, rgb=0, bits=10,
                full_range=0, chroma=0, kr=0.2627, kb=0.0593)
    if have_reference():
        ref = Reference()
        cores = ref.lib.ref_usable_cpus()
        from oracle.oracle import ref_codestream
        enc = RefEncoder(ref, W4K, H4K, 1, transfer=2, primaries=1, planar=pl, threads=0)
        enc.encode(frames[0])  # warm-up
        t0 = time.perf_counter()
        for i in range(sample):
            t1 = enc.encode(frames[1 + i % (len(frames) - 1)])
            ref_codestream(ref, W4K, H4K, 1, t1, fps=FPS, tag=b"cpu")
        dt = time.perf_counter() - t0
        enc.close()
        from oracle.oracle import ref_decode
        cs, _, _, _ = ref_codestream(ref, W4K, H4K, 1, t1, fps=FPS, tag=b"cpu")
        ref_decode(ref, cs, W4K, H4K)  # warm-up
        t0 = time.perf_counter()
        for _ in range(sample):
            ref_decode(ref, cs, W4K, H4K)
        ddt = time.perf_counter() - t0
        return {"value": sample / dt, "unit": "frames/s", "cores": cores, "kind": "reference",
                "sample": f"{sample} 4K frames (after 1 warm-up) through the reference CpuSlot encoder, all "
                          f"passes, then its rate control and codestream writer",
                "decode": {"value": sample / ddt, "unit": "frames/s",
                           "sample": f"{sample} decodes of one 4K codestream through the reference CPU decoder"}}
    from oracle.oracle import Oracle
    o = Oracle()
    t0 = time.perf_counter()
    rgb = o.planar_to_rgb48(pl, frames[0])
    planes, _ = o.color_frame(rgb, 2, 1)
    wav = np.stack([o.fdwt(planes[c], 6) for c in range(3)])
    bands, cblks = o.layout(W4K, H4K, 1)
    q = o.quantize_frame(wav, bands, cblks)
    geom = np.array([[k.w, k.h, bands[k.band].orient, 64] for k in cblks], np.int32)
    o.t1_encode_many(q, geom)
    dt = time.perf_counter() - t0
    return {"value": 1 / dt, "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": "1 4K frame through the single-threaded C oracle"}


def run_reference(args):
    from libgail_b200.replicas import rank_info
    rank, local, world = rank_info()
    if rank != 0:
        return
    from oracle.oracle import Planar, Reference, RefEncoder, have_reference, ref_check, ref_codestream
    if not have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) not present"}))
        return
    frames = gen_frames(min(args.frames, args.steps + args.warmup + 1))
    ref = Reference()
    cores = ref.lib.ref_usable_cpus()
    pl = Planar(width=W4K, height=H4K, active_w=W4K, active_h=H4K, ox=0, oy=0, sx=1, sy=0, rgb=0, bits=10,
                full_range=0, chroma=0, kr=0.2627, kb=0.0593)
    enc = RefEncoder(ref, W4K, H4K, 1, transfer=2, primaries=1, planar=pl, threads=0)

    def step(f):
        t1 = enc.encode(f)
        cs, _, _, _ = ref_codestream(ref, W4K, H4K, 1, t1, fps=FPS, tag=b"cpu")
        return ref_check(ref, cs, FPS)[0]

    for i in range(args.warmup):
        step(frames[i % len(frames)])
    lat, valid = [], 0
    t0 = time.perf_counter()
    for i in range(args.steps):
        t = time.perf_counter()
        valid += step(frames[(args.warmup + i) % len(frames)])
        lat.append((time.perf_counter() - t) * 1e3)
    dt = time.perf_counter() - t0
    enc.close()
    fps = args.steps / dt
    out = {"impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32 (integer Tier-1), f32 (colour, wavelet)",
           "data": "synthetic (seeded generator)",
           "config": {"workload": WORKLOAD, "step": "one frame (bounded sample of the 48-frame workload)",
                      "path": "reference CpuSlot (colour, wavelet, quantisation, Tier-1), then its rate control, "
                              "codestream writer and DCI checker, all host threads"},
           "dci": {"frames": args.steps, "valid": int(valid)},
           "latency_ms": {"p50": statistics.median(lat), "p99": float(np.percentile(lat, 99))},
           "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": cores, "kind": "reference",
                            "sample": f"{args.steps} 4K frames after {args.warmup} warm-up"},
           "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def poisson_arrivals(n, rate, seed=7):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def _pct(a, q):
    return float(np.percentile(a, q)) if len(a) else None


def served_latency(eng, cid, frames, rate, n, seed=7):
    """p50 / p99 latency (ms, submit to codestream) of n requests at Poisson rate `rate`,
    submitted and collected by the engine's own threads (gb_engine_open_loop), and the
    rate achieved."""
    lat, st, el = eng.open_loop([(cid, "encode", frames[i % len(frames)]) for i in range(n)],
                                poisson_arrivals(n, rate, seed=seed))
    if np.any(st != 0):
        raise RuntimeError(f"{int(np.count_nonzero(st))} engine frames failed")
    return {"offered_fps": rate, "achieved_fps": n / el, "requests": n, "p50_ms": _pct(lat, 50),
            "p99_ms": _pct(lat, 99)}


def drain(eng, ids, keep=None):
    for _ in ids:
        rid, _, _, st = eng.wait(120000, copy=False)
        if rid < 0 or st != 0:
            raise RuntimeError(f"engine request failed (id {rid}, status {st})")
        if keep is not None:
            keep(rid)
        eng.release(rid)


def run_ours(args):
    import torch

    from libgail_b200.replicas import Replicas, rank_info
    rank, local, world = rank_info()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", timeout_s=120, device=f"cuda:{local}")
    import libgail_b200 as gb  # noqa: F401  (loads the CUDA library: no fallback exists)
    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    from libgail_b200.engine import Engine
    from libgail_b200.slots import SlotPipeline

    cuda = f"cuda:{local}"
    reduce_max = rep.max

    def barrier():
        torch.cuda.synchronize()
        rep.barrier()
        torch.cuda.synchronize()

    frames = gen_frames(args.frames, seed=rep.frame_seed(1000))
    nbytes = frames[0].nbytes
    pinned = [torch.from_numpy(f.view(np.int16)).pin_memory() for f in frames]
    dframes = [p.to(cuda) for p in pinned]
    torch.cuda.synchronize()
    # the autotuner's choices for this GPU (launch knobs per profile, batch policy)
    from libgail_b200 import autotune as AT
    policy = dict(AT.POLICY_DEFAULT)
    tuned = False
    if args.tuning and os.path.exists(args.tuning):
        policy = AT.apply(args.tuning, device_name=torch.cuda.get_device_name(local))
        tuned = json.load(open(args.tuning)).get("device") == torch.cuda.get_device_name(local)
    if args.batch is not None:
        policy["maxBatch"] = args.batch
    args.batch = policy["maxBatch"]
    plugin = P.Plugin()
    dev = plugin.device(local)
    lay = P.LayoutHolder(W4K, H4K, 1)
    fmt = P.planar_format(W4K, H4K, bits=10, sx=1, sy=0)
    col = P.color("pq", "bt2020")
    ncblk = lay.abi.numCblks
    budget, _ = CS.dci_limits(FPS)
    # host workers for the codestreams: the CPUs this process may use, shared by the ranks on
    # this node, less two for the engine's own threads
    usable = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 8)
    per_node = int(os.environ.get("LOCAL_WORLD_SIZE", world))
    workers = max(2, min(16, usable // max(1, per_node) - 2))
    sms = torch.cuda.get_device_properties(local).multi_processor_count

    # ---- served: the batched engine, rate control and Tier-2 on the device -------------
    # a budget of 48 frame slots: deep enough to keep two Tier-1 batches and the front ends
    # busy; all of them reserved up front (serving capacity set up before the first request),
    # none made inside the timed region
    probe = Engine(local, 0, max_batch=args.batch)
    _, frame_bytes = probe.add_encoder(lay, fmt, col)
    probe.close()
    eng = Engine(local, 48 * frame_bytes + 1, max_batch=args.batch)
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    cid, frame_bytes = eng.add_encoder(lay, fmt, col)
    eng.reserve(cid, 48)
    eng.set_codestream(fps=FPS, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
    served_cs, kept_cs = [], []

    def served_step(src, keep=False, repeat=1):
        """Returns the host-to-device and device-to-host bytes the engine copied and the
        kernels it launched."""
        b0 = eng.counters()
        ids = [eng.submit(cid, f) for _ in range(repeat) for f in src]

        def k(rid):
            if keep:
                (p, n), ok = eng.codestream(rid, copy=False)
                served_cs.append((n, ok))
                if len(kept_cs) < len(src):
                    kept_cs.append(C.string_at(p, n))
        drain(eng, ids, k)
        b1 = eng.counters()
        return tuple(y - x for x, y in zip(b0, b1))

    served_step(dframes, repeat=args.warmup)
    barrier()
    clocks = Clocks(local)
    clocks.start()
    # the K steps as one continuous job: every step's frames submitted at once, so that the
    # pipeline drains once at the end rather than after each step
    t0 = time.perf_counter()
    launches = served_step(dframes, keep=True, repeat=args.steps)[2]
    torch.cuda.synchronize()
    served_s = reduce_max(time.perf_counter() - t0)
    clk = clocks.stop()
    value = args.steps * len(dframes) * world / served_s
    st_eng = eng.stats()

    # served end to end: frames in pinned host memory, uploads and codestreams inside
    served_step(pinned)
    barrier()
    t0 = time.perf_counter()
    h2d_e2e, d2h, _ = (x / args.steps for x in served_step(pinned, repeat=args.steps))
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0)
    e2e_fps = args.steps * len(pinned) * world / e2e_s

    # the served path's stage split, live: the same job once more with the engine's stage
    # timing on (CUDA events around each frame's front-end graph and each Tier-1 batch's
    # stages; host wall time of each frame's rate-control round trips)
    eng.stage_timing(True)
    eng.stage_times(reset=True)
    t0 = time.perf_counter()
    served_step(dframes, repeat=2)
    split_s = time.perf_counter() - t0
    stage_ms, stage_n = eng.stage_times(reset=True)
    eng.stage_timing(False)
    split_fps = 2 * len(dframes) / split_s

    # ---- plain: slot threads, each encoder_encode + rate control + codestream + check ----
    slots = SlotPipeline(dev, lay, fmt, col, slots=args.slots, fps=FPS, tag="b200")
    slots.run(frames[: min(len(frames), 2 * args.slots)])  # warm-up
    barrier()
    plain_res, plain_s = [], 0.0
    for _ in range(args.steps):
        r, dt = slots.run(frames)
        plain_res += r
        plain_s += dt
    plain_fps = len(plain_res) * world / reduce_max(plain_s)
    # latency at a Poisson load both paths carry: 80 % of the plain rate
    rate = 0.8 * plain_fps / world
    # 480 requests: the 99th percentile is the fifth-largest latency, not one stray request
    nlat = 10 * len(frames)
    arr = poisson_arrivals(nlat, rate)
    plain_lat_res, _ = slots.run([frames[i % len(frames)] for i in range(nlat)], arrivals=arr)
    slots.close()
    plain_lat = [r[2] for r in plain_lat_res]
    lat_equal = served_latency(eng, cid, pinned, rate, nlat)
    # served latency near its own capacity: 90 % of the served end-to-end rate
    lat_90 = served_latency(eng, cid, pinned, 0.9 * e2e_fps / world, 10 * len(pinned), seed=9)
    eng.close()

    # decisions and codeword bytes per frame, from the plugin's own timings
    enc = dev.encoder(lay, fmt, col)
    inbuf = enc.input_buffer()
    decisions, coded = [], []
    for f in frames[: min(4, len(frames))]:
        C.memmove(inbuf, f.ctypes.data, nbytes)
        view, tm = enc.encode_view(inbuf)
        decisions.append(tm.symbols)
        coded.append(view.numData)
    enc.close()

    # ---- served with Tier-1 early termination, as libgail's gail.h encoder runs it --------
    # (slope factor 0.25, src/api/gail_api.cpp:607: each frame's threshold is the lambda of
    # the frame finished last x 0.25; a frame whose own lambda comes out lower is coded again
    # with every pass). Not the headline: its Tier-1 leaves passes out.
    eng = Engine(local, 48 * frame_bytes + 1, max_batch=args.batch)
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    cid_et, _ = eng.add_encoder(lay, fmt, col)
    eng.reserve(cid_et, 48)
    eng.set_codestream(fps=FPS, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
    eng.set_slope_factor(ET_FACTOR)
    et_res = []

    def et_keep(rid):
        (p, n), ok = eng.codestream(rid, copy=False)
        et_res.append((n, ok, eng.frame_info(rid)[1]))

    drain(eng, [eng.submit(cid_et, f) for _ in range(args.warmup) for f in dframes])
    barrier()
    t0 = time.perf_counter()
    drain(eng, [eng.submit(cid_et, f) for _ in range(args.steps) for f in dframes], et_keep)
    torch.cuda.synchronize()
    et_fps = args.steps * len(dframes) * world / reduce_max(time.perf_counter() - t0)
    eng.close()

    mixed = run_mixed(args, local, dev, lay, fmt, col, pinned, kept_cs, frame_bytes, workers, policy)
    cfg2 = run_decode_cfg(local, dev, workers, args.batch, policy)
    cfg0 = run_2k_frame(dev)
    cfg3 = run_six_profiles(local, dev, workers)

    out = None
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        npix = W4K * H4K
        dec, cod = float(np.mean(decisions)), float(np.mean(coded))
        nf = max(1, stage_n["batch_frames"])
        per = {"front": stage_ms["front"] / max(1, stage_n["front_frames"]), "cm": stage_ms["cm"] / nf,
               "order": stage_ms["order"] / nf, "mq": stage_ms["mq"] / nf, "pack": stage_ms["pack"] / nf,
               "rc": stage_ms["rc"] / max(1, stage_n["rc_frames"])}
        # algorithmic bytes per frame: the front end at 60 B per pixel (colour 16, the 9/7
        # levels 32, the quantised words 12); context modelling reads the coefficient words
        # and writes a byte per decision; MQ coding reads the decisions and writes the
        # codewords; packing moves the codewords and the per-block and per-pass tables
        alg = {"front": npix * 60, "cm": ncblk * 4096 + dec, "mq": dec + cod, "pack": 2 * cod + ncblk * 40}
        names = {"front": "front end (colour + 9/7 + quantisation; one CUDA graph per frame)",
                 "cm": "Tier-1 context modelling (t1CmKernel, batched)", "order": "Tier-1 ordering (t1OrderKernel)",
                 "mq": "Tier-1 MQ coding + truncation lengths (t1MqKernel, t1TruncKernel)",
                 "pack": "packing + PCRD hull points (tileSum, scan, hull, copy)",
                 "rc": "rate control + Tier-2 on the device (host wall time of the round trips, per frame)"}
        stages = []
        for k, nm in names.items():
            ms = per[k]
            row = {"stage": nm, "ms_per_frame": round(ms, 4)}
            if k in alg and ms > 0:
                ach = alg[k] / (ms * 1e-3) / 1e9
                row.update({"algorithmic_bytes": int(alg[k]), "achieved_gbs": ach, "hbm_frac": ach / hbm})
            stages.append(row)
        # the dominant kernel of the served run: context modelling, integer-issue bound; its
        # roofline is the SM issue rate (4 warp instructions per SM per cycle at the SM clock
        # sampled during the timed region)
        sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        issue_peak = sms * 4 * sm_mhz * 1e6
        batch_frames = stage_n["batch_frames"] / max(1, stage_n["batches"])
        cm_launch_ms = stage_ms["cm"] / max(1, stage_n["batches"])
        instr = CM_WARP_INSTR_PER_FRAME * batch_frames
        achieved = instr / (cm_launch_ms * 1e-3)
        roofline = {"bound": "issue", "kernel": "t1CmKernel (Tier-1 context modelling, batched launch)",
                    "achieved": achieved / 1e12, "peak": issue_peak / 1e12, "unit": "T warp-instr/s",
                    "frac": achieved / issue_peak, "traffic": CM_DRAM_BYTES_PER_FRAME * batch_frames,
                    "traffic_unit": "DRAM bytes per launch",
                    "algorithmic_bytes_per_launch": alg["cm"] * batch_frames,
                    "launch_ms": cm_launch_ms, "frames_per_launch": batch_frames,
                    "warp_instr_per_launch": instr,
                    "sources": "launch_ms: CUDA events on the batch stream in this run; warp instructions and "
                               "DRAM bytes per frame: ncu (smsp__inst_executed.sum, dram__bytes_read.sum + "
                               "dram__bytes_write.sum) on one batched launch of this build; peak: SMs x 4 issue "
                               "slots x the median SM clock sampled in this run",
                    "note": "elapsed on its stream while the other batch's MQ coding and the next front ends "
                            "run beside it; HBM is not the bound (traffic / launch_ms is far below the peak)"}
        front = stages[0]
        tier1 = {"code_blocks": ncblk, "decisions_per_frame": dec, "codeword_bytes_per_frame": cod,
                 "mq_decisions_per_s_served": dec / (per["mq"] * 1e-3) if per["mq"] else None,
                 "code_blocks_per_s_per_sm_served": ncblk * value / sms,
                 "cm_issue_frac_served": roofline["frac"]}
        pct = _pct
        dci = {"fps": FPS, "budget_bytes": budget,
               "served": {"frames": len(served_cs), "valid": sum(1 for _, ok in served_cs if ok == 1),
                          "max_bytes": max(n for n, _ in served_cs)},
               "plain": {"frames": len(plain_res), "valid": sum(1 for r in plain_res if r[1]),
                         "max_bytes": max(len(r[0]) for r in plain_res)}}
        out = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": served_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32 (integer Tier-1), f32 (colour, wavelet)",
            "data": f"synthetic (seeded generator, {len(dframes)} frames)",
            "served_fps": value, "plain_fps": plain_fps,
            "served_p50_ms": lat_equal["p50_ms"], "served_p99_ms": lat_equal["p99_ms"],
            "plain_p50_ms": pct(plain_lat, 50), "plain_p99_ms": pct(plain_lat, 99), "latency_offered_fps": rate,
            "served_p99_ms_at_90pct": lat_90["p99_ms"], "served_offered_fps_at_90pct": lat_90["offered_fps"],
            "config": {"workload": WORKLOAD, "frames_per_step": len(dframes), "path": "served (batched engine)",
                       "max_batch": args.batch, "codestream_workers": workers, "parallelism": f"replicas x{world}",
                       "tuning": {"file": os.path.relpath(args.tuning, ROOT) if tuned else None,
                                  "profiles": {"2k": AT.get_tuning(0), "4k": AT.get_tuning(1)}, "policy": policy},
                       "l2": f"inputs larger than L2 ({len(dframes)} frames, {len(dframes) * nbytes / 1e9:.2f} GB)"},
            "served": {"fps": value, "latency_equal_load": lat_equal, "latency_90pct_capacity": lat_90,
                       "batches": st_eng["batches"],
                       "frames_per_batch": st_eng["batch_frames"] / max(1, st_eng["batches"]),
                       "slots": st_eng["slots"], "frame_bytes": frame_bytes,
                       "stage_split_fps": split_fps},
            "early_termination": {
                "slope_factor": ET_FACTOR, "fps": et_fps, "frames": len(et_res),
                "coded_again": sum(1 for r in et_res if r[2]),
                "dci_valid": sum(1 for r in et_res if r[1] == 1), "max_bytes": max(r[0] for r in et_res),
                "path": "served engine as the headline, with gail.h's Tier-1 early termination (threshold = last "
                        "lambda x 0.25, frame coded again with every pass when its lambda comes out lower)",
                "reference_published": "171.1 frames/s on an RTX 3090 (CUDA backend, early termination 0.25, "
                                       "4 frames in flight, docs/BENCHMARKS.md:16)"},
            "plain": {"fps": plain_fps, "slots": args.slots,
                      "latency_ms": {"p50": pct(plain_lat, 50), "p99": pct(plain_lat, 99)}, "offered_fps": rate},
            "dci": dci,
            "mixed": mixed,
            "decode": cfg2,
            "encode_decode_2k": cfg0,
            "six_profiles": cfg3,
            "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": int(h2d_e2e),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "served engine, frames in pinned host memory; rate control and Tier-2 on the device, "
                            "codestreams (and a few numbers per size measurement) back to host memory"},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "stages": stages,
            "front_end_hbm": {"achieved_gbs": front.get("achieved_gbs"), "peak": hbm,
                              "frac": front.get("hbm_frac"),
                              "peak_source": "measured" if peaks else "fallback"},
            "tier1": tier1,
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline(frames)
            except Exception as e:  # a missing baseline must not hide the measurement
                out["cpu_baseline"] = {"unavailable": str(e)}
    dev.close()
    rep.close()
    if out is not None:
        print(json.dumps(out))


def _xyz_frames(w, h, count, seed):
    from libgail_b200 import synth
    return synth.many(lambda ww, hh, sd, i: synth.xyz12_to_rgb48(synth.xyz12_planes(ww, hh, sd, i)), count, w, h,
                      seed=seed)


def run_decode_cfg(local, dev, workers, batch, policy, count=DECODE_FRAMES):
    """Decode of `count` 4K and `count` 2K X'Y'Z' codestreams at 250 Mbit/s, at full size
    and at half size (reduce 1): one at a time through decoder_decode (host parse, device
    Tier-1 decode, dequantisation, inverse 9/7 and ICT, picture to host memory) and as
    engine decode requests with several in flight. The codestreams come from this
    library's encoder, whose codestream bytes equal the reference CPU encoder's on the same
    frames (the parity tests check that byte for byte)."""
    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    from libgail_b200.engine import Engine
    out = {"frames_per_profile": count, "mbps": 250.0,
           "source": "X'Y'Z' 12-bit generator frames encoded by this library at 250 Mbit/s (codestreams "
                     "byte-identical to the reference CPU encoder's)",
           "reference_published": "reduce 1: 301.4 (4K) / 566.6 (2K) frames/s on an RTX 3090 "
                                  "(docs/BENCHMARKS.md:117-118)"}
    for name, (w, h, fk) in (("4k", (W4K, H4K, 1)), ("2k", (1998, 1080, 0))):
        lay = P.LayoutHolder(w, h, fk)
        frames = _xyz_frames(w, h, count, 3000 + fk)
        eng = Engine(local, 0, max_batch=batch)
        eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
        cid, _ = eng.add_encoder(lay, P.rgb48_format(w, h), P.color_passthrough())
        eng.set_codestream(fps=FPS, max_mbps=250.0, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
        streams = []
        drain(eng, [eng.submit(cid, f) for f in frames], lambda rid: streams.append(eng.codestream(rid)[0]))
        eng.close()
        del frames
        parsed = [CS.parse(c)[1].view(P.CBLK_CODE_DTYPE) for c in streams]
        row = {"max_bytes": max(len(c) for c in streams)}
        for reduce in (0, 1):
            dec = dev.decoder(lay, reduce=reduce)
            pic = np.zeros((dec.out_h, dec.out_w, 3), np.uint16)
            for i in range(3):
                dec.decode(streams[i], parsed[i], out=pic)
            t0 = time.perf_counter()
            for c in streams:  # the host parse is part of each decode, as in decoder_decode's callers
                _, blocks = CS.parse(c)
                dec.decode(c, blocks.view(P.CBLK_CODE_DTYPE), out=pic)
            plain = len(streams) / (time.perf_counter() - t0)
            dec.close()
            eng = Engine(local, 0, max_batch=batch)
            dcls, _ = eng.add_decoder(lay, reduce=reduce)
            drain(eng, [eng.submit_decode(dcls, c) for c in streams])  # makes the decoder slots
            eng.decode_times(reset=True)
            t0 = time.perf_counter()
            drain(eng, [eng.submit_decode(dcls, c) for _ in range(2) for c in streams])
            served = 2 * len(streams) / (time.perf_counter() - t0)
            dt = eng.decode_times()
            eng.close()
            nd = max(1, dt["decodes"])
            row[f"reduce{reduce}"] = {"plain_fps": plain, "served_fps": served,
                                      "served_host_ms_per_decode": {k: dt[k] / nd for k in ("wait_ms", "parse_ms",
                                                                                             "run_ms")},
                                      "served_slots_made_later": dt["slots_made_later"]}
        out[name] = row
    return out


def run_2k_frame(dev, count=24):
    """The 2K configuration one frame at a time through the drop-in, as libgail's pipeline
    drives it: encoder_encode of a 1998x1080 X'Y'Z' frame, its codestream by the host codec
    (rate control and Tier-2, 230 Mbit/s at 24 fps), then the parse and decoder_decode of that
    codestream back to 12-bit X'Y'Z'."""
    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    w, h = 1998, 1080
    lay = P.LayoutHolder(w, h, 0)
    frames = _xyz_frames(w, h, count, 4000)
    enc = dev.encoder(lay, P.rgb48_format(w, h), P.color_passthrough())
    dec = dev.decoder(lay)
    buf = enc.input_buffer()
    pic = np.zeros((h, w, 3), np.uint16)

    def one(f):
        C.memmove(buf, f.ctypes.data, f.nbytes)
        view, _ = enc.encode_view(buf)
        cs, _, _ = CS.rate_and_build(lay, view, FPS, 230.0, tag="b200")
        t = time.perf_counter()
        _, blocks = CS.parse(cs)
        dec.decode(cs, blocks.view(P.CBLK_CODE_DTYPE), out=pic)
        return cs, time.perf_counter() - t

    for f in frames[:3]:
        one(f)
    enc_s = dec_s = 0.0
    ok = 0
    for f in frames:
        t = time.perf_counter()
        cs, ds = one(f)
        enc_s += time.perf_counter() - t - ds
        dec_s += ds
        ok += CS.check_dci(cs, FPS)[0]
    enc.close()
    dec.close()
    return {"frames": count, "encode_fps": count / enc_s, "decode_fps": count / dec_s,
            "encode_decode_fps": count / (enc_s + dec_s), "dci_valid": ok,
            "path": "encoder_encode + host rate control and Tier-2, then parse + decoder_decode, one frame at a time"}


SIX_PROFILES = [(1998, 1080, 0), (2048, 858, 0), (2048, 1080, 0), (3996, 2160, 1), (4096, 1716, 1), (4096, 2160, 1)]


def run_six_profiles(local, dev, workers, count=16, repeat=4):
    """16 X'Y'Z' frames over the six DCI profiles (uneven edge code-blocks): the served
    engine with Tier-1 as one persistent launch from a device work queue over every frame in
    flight (each frame's front end one CUDA graph; rate control and Tier-2 on the device),
    against the plain per-frame path (encoder_encode, then the host codec's rate control and
    Tier-2), both to DCI codestreams."""
    from libgail_b200 import autotune as AT
    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    from libgail_b200.engine import Engine
    from libgail_b200 import synth
    import torch
    profs = [SIX_PROFILES[i % 6] for i in range(count)]
    frames = [synth.xyz12_to_rgb48(synth.xyz12_planes(w, h, seed=5000 + i)) for i, (w, h, _) in enumerate(profs)]
    pinned = [torch.from_numpy(f.view(np.int16)).pin_memory() for f in frames]  # the served path's uploads
    lays = {p: P.LayoutHolder(*p) for p in SIX_PROFILES}
    saved = {k: AT.get_tuning(k) for k in (0, 1)}
    out = {"frames": count, "profiles": [f"{w}x{h}" for w, h, _ in SIX_PROFILES]}
    try:
        for k in (0, 1):
            AT.set_tuning(k, dict(saved[k], t1Persistent=1))
        eng = Engine(local, 0, max_batch=count)
        eng.set_policy(count, 100, 5.0)
        cls = {p: eng.add_encoder(lays[p], P.rgb48_format(p[0], p[1]), P.color_passthrough())[0] for p in SIX_PROFILES}
        for p in SIX_PROFILES:  # a slot for every frame of the burst, reserved up front
            eng.reserve(cls[p], repeat * profs.count(p))
        eng.set_codestream(fps=FPS, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
        # a warm-up burst as large as the timed one
        drain(eng, [eng.submit(cls[p], f) for _ in range(repeat) for p, f in zip(profs, pinned)])
        t0 = time.perf_counter()
        drain(eng, [eng.submit(cls[p], f) for _ in range(repeat) for p, f in zip(profs, pinned)])
        out["served_persistent_fps"] = repeat * count / (time.perf_counter() - t0)
        st = eng.stats()
        out["frames_per_tier1_launch"] = st["batch_frames"] / max(1, st["batches"])
        eng.close()
    finally:
        for k in (0, 1):
            AT.set_tuning(k, saved[k])
    encs = {p: dev.encoder(lays[p], P.rgb48_format(p[0], p[1]), P.color_passthrough()) for p in SIX_PROFILES}

    def plain_pass():
        for p, f in zip(profs, frames):
            e = encs[p]
            buf = e.input_buffer()
            C.memmove(buf, f.ctypes.data, f.nbytes)
            view, _ = e.encode_view(buf)
            CS.rate_and_build(lays[p], view, FPS, 230.0, tag="b200")

    plain_pass()
    t0 = time.perf_counter()
    for _ in range(repeat):
        plain_pass()
    out["plain_fps"] = repeat * count / (time.perf_counter() - t0)
    for e in encs.values():
        e.close()
    return out


def run_mixed(args, local, dev, lay4k, fmt4k, col4k, frames4k, streams4k, frame_bytes, workers, policy, n=480,
              loads=(100.0, 200.0, 300.0, 400.0), seed=11):
    """Serving a mix as it arrives: Poisson requests, 70 % encode / 30 % decode, 60 % 4K
    (the benchmark's Y'CbCr frames and their codestreams) / 40 % 2K X'Y'Z', one engine with
    codestreams on; per offered load the achieved rate and p50/p99 latency by kind."""
    import torch

    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    from libgail_b200 import synth
    from libgail_b200.engine import Engine
    W2, H2 = 1998, 1080
    lay2k = P.LayoutHolder(W2, H2, 0)
    fmt2k, col2k = P.rgb48_format(W2, H2), P.color_passthrough()
    frames2k = [torch.from_numpy(synth.xyz12_to_rgb48(synth.xyz12_planes(W2, H2, seed=seed + i)).view(np.int16))
                .pin_memory() for i in range(8)]
    eng = Engine(local, 64 * frame_bytes, max_batch=args.batch)
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    try:
        e4, _ = eng.add_encoder(lay4k, fmt4k, col4k)
        e2, _ = eng.add_encoder(lay2k, fmt2k, col2k)
        eng.reserve(e4, 32)
        eng.reserve(e2, 24)
        d4, _ = eng.add_decoder(lay4k)
        d2, _ = eng.add_decoder(lay2k)
        eng.set_codestream(fps=FPS, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
        # 2K codestreams to decode, made by this engine; and a warm-up of every class
        ids = [eng.submit(e2, f) for f in frames2k]
        streams2k = []
        for _ in ids:
            rid, _, _, st = eng.wait(120000, copy=False)
            streams2k.append(eng.codestream(rid)[0])
            eng.release(rid)
        # a burst of every class at once: the engine makes the frame and decoder slots the
        # timed loads will use
        warm = [eng.submit(e4, frames4k[i % len(frames4k)]) for i in range(32)]
        warm += [eng.submit(e2, frames2k[i % len(frames2k)]) for i in range(24)]
        warm += [eng.submit_decode(d4, streams4k[i % len(streams4k)]) for i in range(12)]
        warm += [eng.submit_decode(d2, streams2k[i % len(streams2k)]) for i in range(12)]
        for _ in warm:
            rid, _, _, _ = eng.wait(120000, copy=False)
            eng.release(rid)
        rng = np.random.default_rng(seed)
        kinds = rng.random(n) < 0.7           # encode
        big = rng.random(n) < 0.6             # 4K
        picks = rng.integers(0, 1 << 30, n)
        reqs = []
        for i in range(n):
            if kinds[i]:
                reqs.append((e4, "encode", frames4k[picks[i] % len(frames4k)]) if big[i] else
                            (e2, "encode", frames2k[picks[i] % len(frames2k)]))
            else:
                reqs.append((d4, "decode", streams4k[picks[i] % len(streams4k)]) if big[i] else
                            (d2, "decode", streams2k[picks[i] % len(streams2k)]))
        out = []
        for load in loads:
            lat, st, elapsed = eng.open_loop(reqs, poisson_arrivals(n, load, seed=seed + int(load)))
            if np.any(st != 0):
                raise RuntimeError("mixed requests failed")
            row = {"offered_fps": load, "achieved_fps": n / elapsed}
            for k, sel in (("encode", kinds), ("decode", ~kinds)):
                v = lat[sel]
                row[k] = {"requests": int(v.size), "p50_ms": float(np.percentile(v, 50)),
                          "p99_ms": float(np.percentile(v, 99))}
            out.append(row)
        return {"requests_per_load": n, "mix": "70 % encode / 30 % decode; 60 % 4K Y'CbCr PQ / 40 % 2K X'Y'Z'",
                "loads": out}
    finally:
        eng.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
