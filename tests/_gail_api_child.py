"""Child process of tests/test_reference_loader.py: the reference's public gail.h API over
the reference library (oracle/_ref/libgail.so, built from the reference sources with its
CUDA plugin loader and no plugin of its own), with this repository's libgail_cuda13.so
placed next to it, so that libgail loads it exactly as it loads its own CUDA plugin.

    python tests/_gail_api_child.py <directory with libgail.so, libgail_api_probe.so and
                                     libgail_cuda13.so> <job .npz> <result .npz>

Runs in its own process so that libgail's CUDA host (a process-wide singleton) and the
device flags it sets are its own."""
import ctypes as C
import json
import os
import sys

import numpy as np

BACKEND = {"auto": 0, "cuda": 1, "vulkan": 2, "cpu": 3}


def bind(path):
    L = C.CDLL(os.path.join(path, "libgail_api_probe.so"))
    L.probe_last_error.restype = C.c_char_p
    L.probe_version.restype = C.c_char_p
    L.probe_list_devices.argtypes = [C.c_int, C.c_char_p, C.c_size_t]
    L.probe_encode_one.restype = C.c_longlong
    L.probe_encode_one.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_int),
                                   C.c_char_p, C.c_size_t]
    L.probe_encode.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                               C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p,
                               C.c_size_t]
    L.probe_decode.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_longlong, C.c_char_p,
                               C.c_size_t]
    return L


def planes_of(job, inputs, name):
    return [np.ascontiguousarray(inputs[f"{name}_p{k}"]) if f"{name}_p{k}" in inputs.files else None
            for k in range(3)]


def main(path, job_file, out_file):
    L = bind(path)
    inputs = np.load(job_file)
    jobs = json.loads(str(inputs["jobs"]))
    out = {"version": L.probe_version().decode()}
    buf = C.create_string_buffer(4096)
    L.probe_list_devices(1, buf, 4096)
    out["cuda_devices"] = buf.value.decode()
    cap = 4 << 20
    for j in jobs:
        name, kind = j["name"], j["kind"]
        devs = C.create_string_buffer(512)
        if kind == "encode_one":
            p = planes_of(j, inputs, j["frame"])
            cs = np.zeros(cap, np.uint8)
            ok = C.c_int()
            n = L.probe_encode_one(BACKEND[j["backend"]], j["profile"], 0, j["format"], j.get("matrix", 0),
                                   j.get("preset", -1), 24.0, 230.0, *[None if a is None else a.ctypes.data for a in p],
                                   cs.ctypes.data, cap, C.byref(ok), devs, 512)
            if n < 0:
                out[f"{name}_error"] = L.probe_last_error().decode()
                continue
            out[f"{name}_cs"] = cs[:n].copy()
            out[f"{name}_compliant"] = ok.value
        elif kind == "encode_seq":
            frames = [planes_of(j, inputs, f) for f in j["frames"]]
            count = len(frames)
            ptrs = (C.c_void_p * (3 * count))()
            for i, p in enumerate(frames):
                for k in range(3):
                    ptrs[3 * i + k] = None if p[k] is None else p[k].ctypes.data
            cs = np.zeros((count, cap), np.uint8)
            sizes = np.zeros(count, np.uint64)
            ok = np.zeros(count, np.int32)
            st = L.probe_encode(BACKEND[j["backend"]], j["profile"], 0, j["format"], j.get("matrix", 0),
                                j.get("preset", -1), 24.0, 230.0, 1, ptrs, count, cs.ctypes.data, cap,
                                sizes.ctypes.data, ok.ctypes.data, devs, 512)
            if st != 0:
                out[f"{name}_error"] = L.probe_last_error().decode()
                continue
            for i in range(count):
                out[f"{name}_cs{i}"] = cs[i, : int(sizes[i])].copy()
            out[f"{name}_compliant"] = ok
        elif kind == "decode":
            cs = np.ascontiguousarray(inputs[j["codestream"]])
            w, h = j["width"], j["height"]
            for _ in range(j["reduce"]):
                w, h = (w + 1) // 2, (h + 1) // 2
            pic = np.zeros((h, w, 3), np.uint16)
            st = L.probe_decode(BACKEND[j["backend"]], cs.ctypes.data, cs.size, j["reduce"], pic.ctypes.data, w * 6,
                                devs, 512)
            if st != 0:
                out[f"{name}_error"] = L.probe_last_error().decode()
                continue
            out[f"{name}_picture"] = pic
        out[f"{name}_devices"] = devs.value.decode()
    np.savez(out_file, **{k: (np.array(v) if not isinstance(v, np.ndarray) else v) for k, v in out.items()})


if __name__ == "__main__":
    main(*sys.argv[1:4])
