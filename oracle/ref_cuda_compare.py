"""Same-GPU comparison with the reference's own CUDA plugin: TEST INFRASTRUCTURE ONLY (the
product never imports or loads anything here).

The reference plugin is _ref/refcuda/libgail_cuda13.so (`make REF=<tree> refcuda`: the
reference's src/cuda and src/core compiled for sm_100 with the options of its own CUDA
recipe). On one B200 this runs, for that plugin and for libgail_b200/libgail_cuda13.so:

  A. the plugin table one frame at a time: encoder_encode on the 4K Y'CbCr 4:2:2 10-bit PQ
     BT.2020 frames of the headline workload (3996x2160) and on 2K X'Y'Z' 12-bit frames
     (1998x1080), with each plugin's own per-stage GPU timings, and decoder_decode of the
     same codestreams; the Tier-1 outputs and decoded pictures of the two are compared;
  B. the reference library's own pipeline (_ref/libgail.so through gail.h: send / receive,
     4 frames in flight, the DCI check on every frame, early termination from the second
     frame on), once with each plugin next to it: frames per second over a stream of 48
     distinct frames looped, as the reference's gail-bench measures its headline.

    python oracle/ref_cuda_compare.py [--frames 48] [--loops 2] [--out FILE]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_PLUGIN = os.path.join(HERE, "_ref", "refcuda", "libgail_cuda13.so")
OUR_PLUGIN = os.path.join(ROOT, "libgail_b200", "libgail_cuda13.so")
BACKEND_CUDA = 1
GAIL_PIX_XYZ12, GAIL_PIX_YUV422P10 = 1, 7
GAIL_MATRIX_BT2020, GAIL_PRESET_HDR_PQ_BT2020 = 1, 2
W4, H4, W2, H2 = 3996, 2160, 1998, 1080


def _frames(profile: str, n: int, seed: int):
    sys.path.insert(0, ROOT)
    from libgail_b200 import synth
    if profile == "4k":
        return [synth.yuv422p10(W4, H4, seed=seed + i) for i in range(n)]
    return [synth.xyz12_to_rgb48(synth.xyz12_planes(W2, H2, seed=seed + i)) for i in range(n)]


# ---------------------------------------------------------------- A: the plugin table
def plugin_table(nframes: int) -> dict:
    sys.path.insert(0, ROOT)
    from libgail_b200 import codestream as CS
    from libgail_b200 import plugin as P

    out = {}
    plugins = {"reference": P.Plugin(REF_PLUGIN), "b200": P.Plugin(OUR_PLUGIN)}
    for prof in ("4k", "2k"):
        frames = _frames(prof, nframes + 2, 900 if prof == "4k" else 950)
        if prof == "4k":
            lay = P.LayoutHolder(W4, H4, 1)
            fmt, col = P.planar_format(W4, H4, bits=10, sx=1, sy=0), P.color("pq", "bt2020")
        else:
            lay = P.LayoutHolder(W2, H2, 0)
            fmt, col = P.rgb48_format(W2, H2), P.color_passthrough()
        res, t1s, pics = {}, {}, {}
        streams = None
        for name, plug in plugins.items():
            dev = plug.device(0)
            enc = dev.encoder(lay, fmt, col)
            for f in frames[:2]:
                enc.encode(f)
            keys = ("color", "dwt", "t1cm", "t1mq", "t1", "download", "gpu", "total")
            acc = {k: 0.0 for k in keys}
            t1s[name] = []
            t0 = time.perf_counter()
            for f in frames[2:]:
                t1, tm, _ = enc.encode(f)
                t1s[name].append(t1)
                for k in keys:
                    acc[k] += getattr(tm, k)
            wall = (time.perf_counter() - t0) / nframes
            res[name] = {"encode_ms": {k: v / nframes for k, v in acc.items()}, "encode_wall_ms": wall * 1e3,
                         "device": dev.name()}
            if streams is None:  # this plugin's own codestreams, decoded by both
                streams = []
                for t1 in t1s[name][:4]:
                    streams.append(CS.rate_and_build(lay, t1, 24.0)[0])
            enc.close()
            dec = dev.decoder(lay)
            pic = np.zeros((lay.height, lay.width, 3), np.uint16)
            blocks = [CS.parse(s)[1].view(P.CBLK_CODE_DTYPE) for s in streams]
            for s, b in zip(streams[:1], blocks):
                dec.decode(s, b, out=pic)
            acc = {"t1": 0.0, "dwt": 0.0, "color": 0.0, "total": 0.0}
            pics[name] = []
            t0 = time.perf_counter()
            for s, b in zip(streams, blocks):
                p, tm, _ = dec.decode(s, b)
                pics[name].append(p)
                for k in acc:
                    acc[k] += getattr(tm, k)
            res[name]["decode_ms"] = {k: v / len(streams) for k, v in acc.items()}
            res[name]["decode_wall_ms"] = (time.perf_counter() - t0) / len(streams) * 1e3
            dec.close()
            dev.close()
        same = 0
        for a, b in zip(t1s["reference"], t1s["b200"]):
            same += int(np.array_equal(a.info, b.info) and np.array_equal(a.pass_len, b.pass_len)
                        and np.array_equal(a.data, b.data))
        res["tier1_frames_identical"] = f"{same} of {nframes}"
        res["decoded_max_code_difference"] = int(max(np.abs(a.astype(np.int32) - b.astype(np.int32)).max()
                                                     for a, b in zip(pics["reference"], pics["b200"])))
        out[prof] = res
        print(prof, json.dumps(res), flush=True)
    return out


# ------------------------------------------------------ B: the reference library's pipeline
def _install(plugin: str) -> str:
    d = tempfile.mkdtemp(prefix="gailref")
    for f in ("libgail.so", "libgail_api_probe.so"):
        shutil.copy(os.path.join(HERE, "_ref", f), os.path.join(d, f))
    os.symlink(plugin, os.path.join(d, "libgail_cuda13.so"))
    return d


def _child(install: str, profile: str, nframes: int, loops: int, result: str) -> None:
    L = C.CDLL(os.path.join(install, "libgail_api_probe.so"))
    L.probe_last_error.restype = C.c_char_p
    L.probe_version.restype = C.c_char_p
    L.probe_encode_timed.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                     C.c_char_p, C.c_size_t, C.POINTER(C.c_double)]
    if profile == "4k":
        frames = _frames(profile, nframes, 900)
        cw = (W4 + 1) // 2
        planes = [(f[: W4 * H4], f[W4 * H4: W4 * H4 + cw * H4], f[W4 * H4 + cw * H4:]) for f in frames]
        args = (1, 0, GAIL_PIX_YUV422P10, GAIL_MATRIX_BT2020, GAIL_PRESET_HDR_PQ_BT2020)
    else:  # interleaved 16-bit words holding the 12-bit X'Y'Z' codes
        sys.path.insert(0, ROOT)
        from libgail_b200 import synth
        planes = [(np.ascontiguousarray(synth.xyz12_planes(W2, H2, seed=950 + i).transpose(1, 2, 0)), None, None)
                  for i in range(nframes)]
        args = (0, 0, GAIL_PIX_XYZ12, 0, -1)
    count = nframes * loops
    ptrs = (C.c_void_p * (3 * count))()
    for i in range(count):
        for k in range(3):
            p = planes[i % nframes][k]
            ptrs[3 * i + k] = None if p is None else p.ctypes.data
    cap = 2 << 20
    cs = np.zeros((count, cap), np.uint8)
    sizes = np.zeros(count, np.uint64)
    ok = np.zeros(count, np.int32)
    devs = C.create_string_buffer(512)
    out = {"version": L.probe_version().decode()}
    for rep in range(2):  # the first stream warms up (GPU programs, pinned buffers)
        sec = C.c_double()
        st = L.probe_encode_timed(BACKEND_CUDA, *args, 24.0, 230.0, 4, ptrs, count, cs.ctypes.data, cap,
                                  sizes.ctypes.data, ok.ctypes.data, devs, 512, C.byref(sec))
        if st != 0:
            out["error"] = L.probe_last_error().decode()
            break
        out[f"fps_run{rep}"] = count / sec.value
    out["devices"] = devs.value.decode()
    out["all_compliant"] = bool(np.all(ok == 1))
    out["mean_bytes"] = float(sizes.mean())
    with open(result, "w") as f:
        json.dump(out, f)


def pipeline(nframes: int, loops: int) -> dict:
    out = {}
    for prof in ("4k", "2k"):
        for name, plugin in (("reference", REF_PLUGIN), ("b200", OUR_PLUGIN)):
            d = _install(plugin)
            res = os.path.join(d, "result.json")
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", d, prof, str(nframes),
                                str(loops), res], capture_output=True, text=True, timeout=1200)
            if r.returncode != 0:
                out[f"{prof}_{name}"] = {"error": r.stderr[-2000:]}
            else:
                out[f"{prof}_{name}"] = json.load(open(res))
            print(prof, name, json.dumps(out[f"{prof}_{name}"]), flush=True)
            shutil.rmtree(d, ignore_errors=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=48)
    ap.add_argument("--loops", type=int, default=2)
    ap.add_argument("--out", default=None)
    ap.add_argument("--child", nargs=5, default=None)
    a = ap.parse_args()
    if a.child:
        _child(a.child[0], a.child[1], int(a.child[2]), int(a.child[3]), a.child[4])
        return
    for f in (REF_PLUGIN, OUR_PLUGIN, os.path.join(HERE, "_ref", "libgail.so")):
        if not os.path.exists(f):
            raise SystemExit(f"{f} is missing (make REF=<reference tree> ref refcuda; libgail_b200/build.py)")
    res = {"pipeline": pipeline(a.frames, a.loops), "plugin_table": plugin_table(8)}
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
