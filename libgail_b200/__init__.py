"""gail_b200: B200-native JPEG 2000 encode/decode hot path behind GAIL's CUDA plugin ABI.

The product is the shared library libgail_cuda13.so built from csrc/ (hand-written
sm_100a kernels plus the C++ host that implements GAIL's plugin table). This package
loads it with ctypes and mirrors the reference's interfaces for Python callers:
`plugin` (the GailCudaPlugin table: devices, encoder and decoder slots) and the
block-level entry points below. Nothing here falls back to the CPU: without the
library, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgail_cuda13.so")

_lib = None


class GailError(RuntimeError):
    """A failed call: carries the GailCudaStatus and the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status


def lib() -> C.CDLL:
    """The loaded library (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run libgail_b200/build.py (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        L.gb_last_error.restype = C.c_char_p
        L.gb_t1_encode_blocks.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        L.gb_plugin_layout_hash.restype = C.c_uint64
        L.gb_plugin_layout_hash.argtypes = []
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise GailError(status, lib().gb_last_error().decode(errors="replace"))


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def t1_encode_blocks(coeffs: np.ndarray, geom4: np.ndarray, slope: float = 0.0, dist_scale=None,
                     data_stride: int = 65536):
    """Tier-1 encode of n code-blocks on the GPU (t1EncodeRef per block).

    coeffs (n, 1024) uint32 sign-magnitude words; geom4 (n, 4) int32 w, h, orient,
    maxPasses. Returns (info4 (n, 4): nbps, passes, decisions, bytes; pass_len (n, 64);
    pass_dist (n, 64); list of codewords)."""
    c = np.ascontiguousarray(coeffs, np.uint32).reshape(-1, 1024)
    g = np.ascontiguousarray(geom4, np.int32).reshape(-1, 4)
    n = c.shape[0]
    ds = None if dist_scale is None else np.ascontiguousarray(dist_scale, np.float32)
    info = np.zeros((n, 4), np.uint32)
    plen = np.zeros((n, 64), np.uint32)
    pdist = np.zeros((n, 64), np.int32)
    data = np.zeros((n, data_stride), np.uint8)
    check(lib().gb_t1_encode_blocks(_p(c), _p(g), n, C.c_float(slope), _p(ds), _p(info), _p(plen), _p(pdist),
                                    _p(data), data_stride))
    words = [bytes(data[i, : info[i, 3]]) for i in range(n)]
    return info, plen, pdist, words
