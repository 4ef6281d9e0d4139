"""The drop-in, proven through the reference's own loader and public API.

The reference library (oracle/_ref/libgail.so: src/api, src/core and the CUDA plugin
loader src/cuda/cuda_host.cpp, built from the reference sources by oracle/Makefile, with no
CUDA plugin of its own) is placed in a directory next to this repository's
libgail_cuda13.so. There, as in an installed libgail:

  * CudaHost::load (src/cuda/cuda_host.cpp:386-421) finds the plugin next to the library,
    calls gail_cuda_plugin_get(1) and accepts its ABI, table size and layout hash; the
    library reports it loaded (gail_version_string, the part after ';');
  * on a GPU, CudaHost lists the B200 for it (archs "100a" run on sm 100) and
    gail_encoder_encode on GAIL_BACKEND_CUDA (PluginEncoderSlot::encode under runPipeline,
    cuda_host.cpp:158-175, src/core/pipeline.cpp:42-291) gives DCI-valid 2K X'Y'Z' and 4K
    Y'CbCr 4:2:2 PQ codestreams equal to GAIL_BACKEND_CPU's once the COM segment (which
    names the device) is taken out, as the reference's own test compares them
    (withoutComment, tests/test_main.cpp:1488); a sequence through send / receive, where
    the pipeline's early termination (slope factor 0.25) applies from the second frame on,
    does the same;
  * gail_decoder_decode on the CUDA backend gives pictures within one code of the CPU
    decoder's, at full and at half size.
Each check runs in a child process (tests/_gail_api_child.py) with only the reference
library and this plugin loaded."""
import json
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from libgail_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
PLUGIN = os.path.join(ROOT, "libgail_b200", "libgail_cuda13.so")
HAVE = all(os.path.exists(os.path.join(REF_DIR, f)) for f in ("libgail.so", "libgail_api_probe.so"))
pytestmark = pytest.mark.skipif(not HAVE or not os.path.exists(PLUGIN),
                                reason="reference library build (oracle/_ref/libgail.so) or the plugin not present")

GAIL_PIX_XYZ12, GAIL_PIX_YUV422P10 = 1, 7
GAIL_MATRIX_BT2020, GAIL_PRESET_HDR_PQ_BT2020 = 1, 2


@pytest.fixture(scope="module")
def install(tmp_path_factory):
    """A directory laid out as an installed libgail: the library, and the plugin beside it
    (a symbolic link to this repository's build, so the process maps that very file)."""
    d = tmp_path_factory.mktemp("libgail")
    for f in ("libgail.so", "libgail_api_probe.so"):
        shutil.copy(os.path.join(REF_DIR, f), d / f)
    os.symlink(PLUGIN, d / "libgail_cuda13.so")
    return str(d)


def _run(install, jobs, arrays, timeout=600):
    job = os.path.join(install, "job.npz")
    res = os.path.join(install, "result.npz")
    np.savez(job, jobs=np.array(json.dumps(jobs)), **arrays)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "_gail_api_child.py"), install, job, res],
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-4000:]
    out = np.load(res)
    errors = {k: str(out[k]) for k in out.files if k.endswith("_error")}
    assert not errors, errors
    return out


def without_comment(cs: bytes) -> bytes:
    """The codestream with the main header's COM segment taken out."""
    at = 2
    while at + 4 <= len(cs) and cs[at] == 0xFF and cs[at + 1] != 0x90:
        seg = 2 + (cs[at + 2] << 8 | cs[at + 3])
        if cs[at + 1] == 0x64:
            return cs[:at] + cs[at + seg:]
        at += seg
    return cs


def _xyz12(w, h, seed):
    """Interleaved 16-bit words with the 12-bit X'Y'Z' codes in the low bits."""
    return np.ascontiguousarray(synth.xyz12_planes(w, h, seed=seed).transpose(1, 2, 0))


def _yuv422(w, h, seed):
    f = synth.yuv422p10(w, h, seed=seed)
    cw = (w + 1) // 2
    return f[: w * h].copy(), f[w * h: w * h + cw * h].copy(), f[w * h + cw * h:].copy()


def test_reference_loader_accepts_the_plugin(install):
    """No GPU needed: loading is dlopen and the table checks."""
    out = _run(install, [], {})
    version = str(out["version"])
    assert version.startswith("1.1.0"), version
    assert "gail_cuda13" in version.split(";")[-1], f"libgail did not load the plugin: {version}"


@pytest.mark.gpu
def test_gail_api_cuda_backend_equals_cpu_backend(install):
    W2, H2, W4, H4 = 1998, 1080, 3996, 2160
    arrays = {"x2k_p0": _xyz12(W2, H2, 61)}
    y, cb, cr = _yuv422(W4, H4, 62)
    arrays.update({"y4k_p0": y, "y4k_p1": cb, "y4k_p2": cr})
    for i in range(3):
        arrays[f"s{i}_p0"] = _xyz12(W2, H2, 70 + i)
    jobs = []
    for be in ("cuda", "cpu"):
        jobs.append({"name": f"x2k_{be}", "kind": "encode_one", "backend": be, "profile": 0, "format": GAIL_PIX_XYZ12,
                     "frame": "x2k"})
        jobs.append({"name": f"y4k_{be}", "kind": "encode_one", "backend": be, "profile": 1,
                     "format": GAIL_PIX_YUV422P10, "matrix": GAIL_MATRIX_BT2020, "preset": GAIL_PRESET_HDR_PQ_BT2020,
                     "frame": "y4k"})
        jobs.append({"name": f"seq_{be}", "kind": "encode_seq", "backend": be, "profile": 0,
                     "format": GAIL_PIX_XYZ12, "frames": ["s0", "s1", "s2"]})
    out = _run(install, jobs, arrays)
    assert "gail_b200" in str(out["cuda_devices"]) or "B200" in str(out["cuda_devices"]), str(out["cuda_devices"])
    assert "(CUDA)" in str(out["x2k_cuda_devices"]), str(out["x2k_cuda_devices"])
    for name in ("x2k", "y4k"):
        a, b = bytes(out[f"{name}_cuda_cs"]), bytes(out[f"{name}_cpu_cs"])
        assert int(out[f"{name}_cuda_compliant"]) == 1 and int(out[f"{name}_cpu_compliant"]) == 1
        assert a != b, "the COM segments should name different devices"
        assert without_comment(a) == without_comment(b), f"{name}: CUDA and CPU codestreams differ"
        assert len(a) <= 1302083
    for i in range(3):
        a, b = bytes(out[f"seq_cuda_cs{i}"]), bytes(out[f"seq_cpu_cs{i}"])
        assert without_comment(a) == without_comment(b), f"sequence frame {i}: CUDA and CPU codestreams differ"
    assert np.all(out["seq_cuda_compliant"] == 1) and np.all(out["seq_cpu_compliant"] == 1)
    np.savez(os.path.join(install, "encoded.npz"), x2k=out["x2k_cuda_cs"], y4k=out["y4k_cuda_cs"])


@pytest.mark.gpu
def test_gail_api_cuda_decoder_within_one_code_of_cpu(install):
    enc = os.path.join(install, "encoded.npz")
    if not os.path.exists(enc):
        pytest.skip("needs the codestreams of the encode test")
    cs = np.load(enc)
    arrays = {"x2k": cs["x2k"], "y4k": cs["y4k"]}
    jobs = []
    for name, (w, h) in (("x2k", (1998, 1080)), ("y4k", (3996, 2160))):
        for reduce in (0, 1):
            for be in ("cuda", "cpu"):
                jobs.append({"name": f"{name}_r{reduce}_{be}", "kind": "decode", "backend": be, "codestream": name,
                             "width": w, "height": h, "reduce": reduce})
    out = _run(install, jobs, arrays)
    assert "(CUDA)" in str(out["x2k_r0_cuda_devices"]), str(out["x2k_r0_cuda_devices"])
    for name in ("x2k", "y4k"):
        for reduce in (0, 1):
            a = out[f"{name}_r{reduce}_cuda_picture"].astype(np.int32)
            b = out[f"{name}_r{reduce}_cpu_picture"].astype(np.int32)
            assert a.shape == b.shape
            d = np.abs(a - b)
            assert d.max() <= 1, f"{name} reduce {reduce}: {np.count_nonzero(d > 1)} codes differ by more than one"
