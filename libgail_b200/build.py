"""Builds the in-tree CUDA library libgail_b200/libgail_cuda13.so for sm_100a.

Every csrc/*.cu and csrc/*.cpp is compiled by nvcc (the CUDA runtime is linked
statically, as a GAIL CUDA plugin is) into one shared object. Objects go to
libgail_b200/_build/ and are rebuilt when their source or any csrc header changed.
No fast-math and no floating-point contraction: the colour and wavelet kernels round
every operation where the CPU reference does.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgail_cuda13.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "--fmad=false",
          "-I", CSRC, "-I", INCLUDE]
# exported: the plugin entry point and the gb_* C API (include/*.h), nothing else (no
# template instantiations of the C++ standard library, nothing of the static CUDA runtime)
EXPORTS = os.path.join(CSRC, "exports.map")


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OUT, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj
    cmd = [_nvcc(), *ARCH, *COMMON, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd[1:1] = ["-x", "cu"]
    if verbose_ptxas and src.endswith(".cu"):
        cmd.append("-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose_ptxas: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max([os.path.getmtime(o) for o in objs] +
                                                             [os.path.getmtime(EXPORTS)]):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lpthread", "-Xlinker",
               f"--version-script={EXPORTS},--exclude-libs,ALL"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
