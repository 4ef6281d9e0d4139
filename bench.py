#!/usr/bin/env python
"""Benchmark: 4K DCI JPEG 2000 encode on one B200 (and N replicas under torchrun).

Workload (the 4K configuration): 48 preloaded 3996x2160 frames of 10-bit Y'CbCr 4:2:2
BT.2020 PQ from the seeded generator (libgail_b200/synth.py), colour-converted on the GPU
to 12-bit X'Y'Z', 9/7 wavelet with 6 levels, 32x32 code-blocks, Tier-1 with every coding
pass (bit-exact with the CPU reference). One step = encoding all 48 frames; the 48 frames
(1.66 GB) are larger than L2, so no flush is needed between steps.

  value   DCI codestreams/s of the served path: the batched engine (continuous batching of
          Tier-1 over every frame in flight) on frames resident in HBM, Tier-1 frames written
          to mapped host memory, each frame's rate control, Tier-2 and DCI check on the
          engine's host workers. The K steps run as one job (all K x 48 requests submitted
          at once, the time to the last codestream). The work spans the engine's streams and
          threads, so the timed region is bracketed by a barrier and a device
          synchronisation on both sides; max over ranks.
  plain   the drop-in per-frame path beside it, as libgail drives the plugin: slot threads,
          each encoder_encode from host memory then rate control, Tier-2 and the DCI check;
          codestreams/s and p50/p99 latency at a Poisson load of 80 % of that rate (served
          latency at the same load); and, frames resident in HBM, the device stages alone
          with the per-stage split (CUDA events on the encoder's stream).
  e2e     codestreams/s of the served path with the frames in pinned host memory: each
          frame's upload and its Tier-1 output in host memory are inside the timed region.
  dci     every codestream of the timed runs checked: how many passed, the largest.
  decode  the served codestreams of one step decoded through decoder_decode (host
          codestream in, 12-bit picture out) one after another, with the stage split.
  stages  per stage of the plain path: live ms per frame, algorithmic bytes, GB/s and the
          fraction of the measured HBM bandwidth; roofline is the dominant stage.

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


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch on one 4K
# frame, and Tier-1 issue figures, from the ncu captures summarised in the files below
# (encode kernels; decodeKernel's in the second)
NCU_SOURCE = "profiles/kernels_4k_encode_frame.md"
NCU_DECODE_SOURCE = "profiles/kernels_4k_decode_frame.md"
ET_FACTOR = 0.25  # the Tier-1 early-termination factor gail.h's encoder forces
NCU_TRAFFIC = {"t1CmKernel": 214.29e6, "t1MqKernel": 182.01e6}
NCU_TIER1 = {"cm_issue_active_pct": 71.1, "cm_warps_per_sm": 23.1, "mq_issue_active_pct": 27.1, "mq_warps_per_sm": 4.6,
             "decode_issue_active_pct": 72.5, "decode_warps_per_sm": 26.0}


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
    ap.add_argument("--slots", type=int, default=3, help="slot threads of the plain path")
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


def run_ours(args):
    import torch

    from libgail_b200.replicas import Replicas, rank_info
    rank, local, world = rank_info()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", timeout_s=120, device=f"cuda:{local}")
    import libgail_b200 as gb
    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    from libgail_b200.engine import Engine
    from libgail_b200.slots import SlotPipeline

    L = gb.lib()
    L.gb_encoder_stream.restype = C.c_void_p
    L.gb_encoder_stream.argtypes = [C.c_void_p]
    L.gb_encoder_enqueue_device.argtypes = [C.c_void_p, C.c_void_p]
    L.gb_encoder_finish.argtypes = [C.c_void_p]
    L.gb_encoder_stage_timing.argtypes = [C.c_void_p, C.c_int]
    L.gb_encoder_stage_times.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
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
    workers = max(2, min(16, (os.cpu_count() or 8) - 2))

    # ---- device stages of the plain path, frames resident in HBM: the per-stage split ---
    enc = dev.encoder(lay, fmt, col)
    h = enc.h
    stream = torch.cuda.ExternalStream(L.gb_encoder_stream(h), device=cuda)

    def plain_step():
        for f in dframes:
            gb.check(L.gb_encoder_enqueue_device(h, C.c_void_p(f.data_ptr())))

    for _ in range(args.warmup):
        plain_step()
    gb.check(L.gb_encoder_finish(h))
    ms5 = np.zeros(5)
    cnt = C.c_int()
    gb.check(L.gb_encoder_stage_timing(h, 1))
    gb.check(L.gb_encoder_stage_times(h, ms5.ctypes.data, C.byref(cnt)))  # reset
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plain_step()
    e1.record(stream)
    gb.check(L.gb_encoder_finish(h))
    torch.cuda.synchronize()
    plain_dev_ms = reduce_max(e0.elapsed_time(e1))
    gb.check(L.gb_encoder_stage_times(h, ms5.ctypes.data, C.byref(cnt)))
    gb.check(L.gb_encoder_stage_timing(h, 0))
    stage = ms5 / max(cnt.value, 1)  # ms per frame: front, cm, order, mq, pack
    plain_dev_fps = args.steps * len(dframes) * world / (plain_dev_ms / 1e3)
    # decisions and codeword bytes per frame, from the plugin's own timings
    inbuf = enc.input_buffer()
    decisions, coded, passes = [], [], []
    for f in frames[: min(4, len(frames))]:
        C.memmove(inbuf, f.ctypes.data, nbytes)
        view, tm = enc.encode_view(inbuf)
        decisions.append(tm.symbols)
        coded.append(view.numData)
        passes.append(view.numPasses)
    enc.close()

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
    nlat = min(2 * len(frames), 96)
    arr = poisson_arrivals(nlat, rate)
    lat_frames = [frames[i % len(frames)] for i in range(nlat)]
    plain_lat_res, _ = slots.run(lat_frames, arrivals=arr)
    slots.close()
    plain_lat = [r[2] for r in plain_lat_res]

    # ---- served: the batched engine; rate control and Tier-2 on the device, driven by
    # host workers (the Tier-1 frames stay in device memory, only codestreams come back)
    # a budget of 48 frame slots: deep enough to keep two Tier-1 batches and the front ends
    # busy; every slot is made during the warm-up, none inside the timed region
    probe = Engine(local, 0, max_batch=args.batch)
    _, frame_bytes = probe.add_encoder(lay, fmt, col)
    probe.close()
    eng = Engine(local, 48 * frame_bytes + 1, max_batch=args.batch)
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    cid, frame_bytes = eng.add_encoder(lay, fmt, col)
    eng.set_codestream(fps=FPS, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
    served_cs = []

    kept_cs = []  # codestreams of one step, for the decode run

    def served_step(src, keep=False, repeat=1):
        """Returns the host-to-device and device-to-host bytes the engine copied and the
        kernels it launched."""
        b0 = eng.counters()
        ids = [eng.submit(cid, f) for _ in range(repeat) for f in src]
        for _ in ids:
            rid, t, _, st = eng.wait(120000, copy=False)
            if rid < 0 or st != 0:
                raise RuntimeError(f"engine frame failed (id {rid}, status {st})")
            (p, n), ok = eng.codestream(rid, copy=False)
            if keep:
                served_cs.append((n, ok))
                if len(kept_cs) < len(src):
                    kept_cs.append(C.string_at(p, n))
            eng.release(rid)
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

    # served end to end: frames in pinned host memory, uploads and Tier-1 output inside
    served_step(pinned)
    barrier()
    t0 = time.perf_counter()
    h2d_e2e, d2h, _ = (x / args.steps for x in served_step(pinned, repeat=args.steps))
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0)
    e2e_fps = args.steps * len(pinned) * world / e2e_s

    # served latency at the same Poisson load
    served_lat = []
    import threading

    def collect():
        for _ in range(nlat):
            rid, _, lat_ms, st = eng.wait(120000, copy=False)
            served_lat.append(lat_ms)
            eng.release(rid)

    th = threading.Thread(target=collect)
    th.start()
    t0 = time.perf_counter()
    for i in range(nlat):
        while time.perf_counter() - t0 < arr[i]:
            pass
        eng.submit(cid, pinned[i % len(pinned)])
    th.join()
    eng.close()

    # ---- served with Tier-1 early termination, as libgail's gail.h encoder runs it --------
    # (slope factor 0.25, src/api/gail_api.cpp:607: each frame's threshold is the lambda of
    # the frame finished last x 0.25; a frame whose own lambda comes out lower is coded again
    # with every pass). Not the headline: its Tier-1 leaves passes out.
    eng = Engine(local, 48 * frame_bytes + 1, max_batch=args.batch)
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    cid_et, _ = eng.add_encoder(lay, fmt, col)
    eng.set_codestream(fps=FPS, label=CS.DEFAULT_LABEL, tag="b200", threads=workers)
    eng.set_slope_factor(ET_FACTOR)

    def et_step(src, repeat=1):
        ids = [eng.submit(cid_et, f) for _ in range(repeat) for f in src]
        res = []
        for _ in ids:
            rid, _, _, st = eng.wait(120000, copy=False)
            if rid < 0 or st != 0:
                raise RuntimeError(f"engine frame failed (id {rid}, status {st})")
            (p, n), ok = eng.codestream(rid, copy=False)
            res.append((n, ok, eng.frame_info(rid)[1]))
            eng.release(rid)
        return res

    et_step(dframes, repeat=args.warmup)
    barrier()
    t0 = time.perf_counter()
    et_res = et_step(dframes, repeat=args.steps)
    torch.cuda.synchronize()
    et_s = reduce_max(time.perf_counter() - t0)
    et_fps = args.steps * len(dframes) * world / et_s
    eng.close()

    # ---- decode: the served codestreams back to 12-bit pictures -------------------------
    # the host parses each codestream (gb_parse_codestream), decoder_decode does Tier-1
    # decode, dequantisation, the inverse 9/7 and ICT on the device and returns the picture
    parse_ms = []
    parsed = []
    for c in kept_cs:
        t = time.perf_counter()
        parsed.append(CS.parse(c)[1].view(P.CBLK_CODE_DTYPE))
        parse_ms.append((time.perf_counter() - t) * 1e3)
    dec = dev.decoder(lay, reduce=0)
    pic = np.zeros((H4K, W4K, 3), np.uint16)
    for i in range(min(3, len(kept_cs))):
        dec.decode(kept_cs[i], parsed[i], out=pic)
    dstage = np.zeros(3)
    t0 = time.perf_counter()
    for c, b in zip(kept_cs, parsed):
        _, tm, _ = dec.decode(c, b, out=pic)
        dstage += (tm.t1, tm.dwt, tm.color)
    dec_s = reduce_max(time.perf_counter() - t0)
    dec.close()
    decode_fps = len(kept_cs) * world / dec_s

    # the same codestreams as decode requests to the served engine: its host workers parse
    # them and decode them on decoder slots, each on its own stream, several in flight (the
    # pictures come back to host memory as above)
    eng = Engine(local, 0, max_batch=args.batch)
    dcls, _ = eng.add_decoder(lay)

    def dec_burst():
        ids = [eng.submit_decode(dcls, c) for c in kept_cs]
        for _ in ids:
            rid, _, _, st = eng.wait(120000, copy=False)
            if rid < 0 or st != 0:
                raise RuntimeError(f"engine decode failed (id {rid}, status {st})")
            eng.release(rid)

    dec_burst()  # makes the decoder slots
    barrier()
    t0 = time.perf_counter()
    for _ in range(2):
        dec_burst()
    dec_srv_s = reduce_max(time.perf_counter() - t0)
    eng.close()
    decode_served_fps = 2 * len(kept_cs) * world / dec_srv_s

    mixed = run_mixed(args, local, dev, lay, fmt, col, pinned, kept_cs, frame_bytes, workers, policy)

    out = None
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        npix = W4K * H4K
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        dec, cod, npas = float(np.mean(decisions)), float(np.mean(coded)), float(np.mean(passes))
        # algorithmic bytes per frame (one launch of each stage): the front end at 60 B per
        # pixel (colour 16, the 9/7 levels 32, the quantised words 12); context modelling
        # reads the coefficient words and writes one byte per decision; MQ coding reads the
        # decisions and writes the codewords; packing reads and writes the codewords and
        # the per-block and per-pass tables
        alg = [npix * 60, ncblk * 4096 + dec, ncblk * 16, dec + cod, 2 * cod + ncblk * 40 + npas * 16]
        names = ["front end (colour + 9/7 + quantisation)", "Tier-1 context modelling", "Tier-1 ordering",
                 "Tier-1 MQ coding", "Tier-1 packing"]
        stages = []
        for i, nm in enumerate(names):
            ms = float(stage[i])
            ach = alg[i] / (ms * 1e-3) / 1e9 if ms > 0 else None
            stages.append({"stage": nm, "ms_per_frame": round(ms, 4), "algorithmic_bytes": int(alg[i]),
                           "achieved_gbs": ach, "frac": ach / hbm if ach else None})
        # the dominant stage of the plain step: its roofline, with the DRAM traffic of one
        # launch from the committed ncu capture of the same workload
        k = int(np.argmax(stage))
        traffic = {1: NCU_TRAFFIC.get("t1CmKernel"), 3: NCU_TRAFFIC.get("t1MqKernel")}.get(k)
        roofline = {"bound": "hbm", "kernel": names[k], "achieved": stages[k]["achieved_gbs"], "peak": hbm,
                    "unit": "GB/s", "frac": stages[k]["frac"], "traffic": traffic,
                    "peak_source": "measured" if peaks else "fallback",
                    "traffic_source": NCU_SOURCE if traffic else None,
                    "note": "Tier-1 is integer-issue and latency bound (a serial MQ chain per code-block): "
                            "bytes move far below HBM speed; see tier1 for its own measures"}
        tier1 = {"code_blocks": ncblk, "decisions_per_frame": dec, "codeword_bytes_per_frame": cod,
                 "mq_decisions_per_s": dec / (stage[3] * 1e-3),
                 "code_blocks_per_s_per_sm_plain": ncblk / ((stage[1] + stage[3]) * 1e-3) / sms,
                 "code_blocks_per_s_per_sm_served": ncblk * value / sms,
                 "ncu": dict(NCU_TIER1, sources=[NCU_SOURCE, NCU_DECODE_SOURCE])}
        pct = lambda a, q: float(np.percentile(a, q))  # noqa: E731
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
            "config": {"workload": WORKLOAD, "frames_per_step": len(dframes), "path": "served (batched engine)",
                       "max_batch": args.batch, "codestream_workers": workers, "parallelism": f"replicas x{world}",
                       "tuning": {"file": os.path.relpath(args.tuning, ROOT) if tuned else None,
                                  "profiles": {"2k": AT.get_tuning(0), "4k": AT.get_tuning(1)}, "policy": policy},
                       "l2": f"inputs larger than L2 ({len(dframes)} frames, {len(dframes) * nbytes / 1e9:.2f} GB)"},
            "served": {"fps": value, "latency_ms": {"p50": pct(served_lat, 50), "p99": pct(served_lat, 99)},
                       "offered_fps": rate, "batches": st_eng["batches"],
                       "frames_per_batch": st_eng["batch_frames"] / max(1, st_eng["batches"]),
                       "slots": st_eng["slots"], "frame_bytes": frame_bytes},
            "early_termination": {
                "slope_factor": ET_FACTOR, "fps": et_fps, "frames": len(et_res),
                "coded_again": sum(1 for r in et_res if r[2]),
                "dci_valid": sum(1 for r in et_res if r[1] == 1), "max_bytes": max(r[0] for r in et_res),
                "path": "served engine as the headline, with gail.h's Tier-1 early termination (threshold = last "
                        "lambda x 0.25, frame coded again with every pass when its lambda comes out lower)",
                "reference_published": "171.1 frames/s on an RTX 3090 (CUDA backend, early termination 0.25, "
                                       "4 frames in flight, docs/BENCHMARKS.md:16)"},
            "plain": {"fps": plain_fps, "slots": args.slots,
                      "latency_ms": {"p50": pct(plain_lat, 50), "p99": pct(plain_lat, 99)}, "offered_fps": rate,
                      "device_resident_fps_tier1_only": plain_dev_fps,
                      "stage_ms_per_frame": dict(zip(["front", "t1_cm", "t1_order", "t1_mq", "pack"],
                                                     [round(x, 4) for x in stage]))},
            "dci": dci,
            "mixed": mixed,
            "decode": {"fps": decode_fps, "unit": "frames/s", "frames": len(kept_cs),
                       "path": "decoder_decode per frame: codestream from host memory, 12-bit picture to host memory",
                       "parse_ms_per_frame": float(np.mean(parse_ms)),
                       "served_fps": decode_served_fps,
                       "served_path": "engine decode requests: host workers parse, decoder slots on their own streams, "
                                      "several in flight, pictures to host memory",
                       "reference_published": "121.4 frames/s on an RTX 3090 (CUDA backend, 250 Mbit/s, 3 in flight, "
                                              "docs/BENCHMARKS.md:113)",
                       "stage_ms_per_frame": dict(zip(["t1_decode_dequant", "inverse_dwt", "ict_pack"],
                                                      [round(x / max(1, len(kept_cs)), 4) for x in dstage]))},
            "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": int(h2d_e2e),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "served engine, frames in pinned host memory; rate control and Tier-2 on the device, "
                            "codestreams (and a few numbers per size measurement) back to host memory"},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "stages": stages,
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


def run_mixed(args, local, dev, lay4k, fmt4k, col4k, frames4k, streams4k, frame_bytes, workers, policy, n=240,
              loads=(100.0, 200.0, 300.0), seed=11):
    """Serving a mix as it arrives: Poisson requests, 70 % encode / 30 % decode, 60 % 4K
    (the benchmark's Y'CbCr frames and their codestreams) / 40 % 2K X'Y'Z', one engine with
    codestreams on; per offered load the achieved rate and p50/p99 latency by kind."""
    import threading

    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P
    from libgail_b200 import synth
    from libgail_b200.engine import Engine
    W2, H2 = 1998, 1080
    lay2k = P.LayoutHolder(W2, H2, 0)
    fmt2k, col2k = P.rgb48_format(W2, H2), P.color_passthrough()
    frames2k = [synth.xyz12_to_rgb48(synth.xyz12_planes(W2, H2, seed=seed + i)) for i in range(8)]
    eng = Engine(local, 64 * frame_bytes, max_batch=args.batch)
    eng.set_policy(policy["maxBatch"], policy["minBatchPct"], policy["maxWaitMs"])
    try:
        e4, _ = eng.add_encoder(lay4k, fmt4k, col4k)
        e2, _ = eng.add_encoder(lay2k, fmt2k, col2k)
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
        out = []
        for load in loads:
            arr = poisson_arrivals(n, load, seed=seed + int(load))
            lat = {}
            kind_of = {}
            done = threading.Event()

            def collect():
                for _ in range(n):
                    rid, _, ms, st = eng.wait(120000, copy=False)
                    if rid < 0 or st != 0:
                        raise RuntimeError(f"mixed request failed (id {rid}, status {st})")
                    lat[rid] = ms
                    eng.release(rid)
                done.set()

            th = threading.Thread(target=collect)
            th.start()
            t0 = time.perf_counter()
            for i in range(n):
                while time.perf_counter() - t0 < arr[i]:
                    pass
                if kinds[i]:
                    rid = eng.submit(e4, frames4k[picks[i] % len(frames4k)]) if big[i] else \
                        eng.submit(e2, frames2k[picks[i] % len(frames2k)])
                    kind_of[rid] = "encode"
                else:
                    rid = eng.submit_decode(d4, streams4k[picks[i] % len(streams4k)]) if big[i] else \
                        eng.submit_decode(d2, streams2k[picks[i] % len(streams2k)])
                    kind_of[rid] = "decode"
            th.join()
            elapsed = time.perf_counter() - t0
            if len(lat) != n:
                raise RuntimeError("mixed serving lost requests")
            row = {"offered_fps": load, "achieved_fps": n / elapsed}
            for k in ("encode", "decode"):
                v = [lat[r] for r in lat if kind_of.get(r) == k]
                row[k] = {"requests": len(v), "p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99))}
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
