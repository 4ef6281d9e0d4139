"""Seeded synthetic frames with the shape and statistics of the benchmark inputs.

One plane: clip(2048 + 900 sin(2 pi f1 x / W + phi) cos(2 pi f2 y / H) + 25 axis-aligned
rectangles with offsets U(-600, 600) + N(0, 30^2), 0, 4095), f1, f2 ~ U(1, 6). The
rectangles' corners and sizes are uniform (widths and heights U(W/40, W/4) and
U(H/40, H/4)), phi ~ U(0, 2 pi); frame i of a sequence uses seed + i and a slow phase
drift of 0.05 rad per frame. Random numbers: numpy PCG64 (default_rng).
"""
from __future__ import annotations

import numpy as np


def plane(width: int, height: int, rng: np.random.Generator, drift: float = 0.0) -> np.ndarray:
    f1, f2 = rng.uniform(1, 6, 2)
    phi = rng.uniform(0, 2 * np.pi) + drift
    x = np.arange(width, dtype=np.float64)
    y = np.arange(height, dtype=np.float64)
    sx = (900.0 * np.sin(2 * np.pi * f1 * x / width + phi)).astype(np.float32)
    cy = np.cos(2 * np.pi * f2 * y / height).astype(np.float32)
    v = rng.standard_normal((height, width), dtype=np.float32)
    v *= np.float32(30.0)
    v += np.float32(2048.0)
    v += cy[:, None] * sx[None, :]
    for _ in range(25):
        rw = int(rng.uniform(width / 40, width / 4))
        rh = int(rng.uniform(height / 40, height / 4))
        x0 = int(rng.uniform(0, width - rw))
        y0 = int(rng.uniform(0, height - rh))
        v[y0:y0 + rh, x0:x0 + rw] += np.float32(rng.uniform(-600, 600))
    np.rint(v, out=v)
    np.clip(v, 0, 4095, out=v)
    return v.astype(np.uint16)


def xyz12_planes(width: int, height: int, seed: int, index: int = 0) -> np.ndarray:
    """(3, H, W) uint16 12-bit X'Y'Z' planes of frame `index` of the sequence `seed`."""
    rng = np.random.default_rng(seed + index)
    return np.stack([plane(width, height, rng, 0.05 * index) for _ in range(3)])


def xyz12_to_rgb48(planes: np.ndarray) -> np.ndarray:
    """The encoder input for 12-bit X'Y'Z': interleaved 16-bit, (v * 65535 + 2047) / 4095
    (the public API's fill, gail_api.cpp:389-394)."""
    v = planes.astype(np.uint32)
    return np.ascontiguousarray(((v * 65535 + 2047) // 4095).astype(np.uint16).transpose(1, 2, 0))


def yuv422p10(width: int, height: int, seed: int, index: int = 0) -> np.ndarray:
    """Planar 10-bit Y'CbCr 4:2:2 (Y in [64, 940], Cb/Cr in [64, 960]) from the same
    generator, as one flat uint16 array Y | Cb | Cr (the layout the encoder takes)."""
    rng = np.random.default_rng(seed + index)
    cw = (width + 1) >> 1

    def scaled(p, span):
        v = p.astype(np.float32)
        v *= np.float32(span / 4095.0)
        v += np.float32(64.0)
        np.rint(v, out=v)
        return v.astype(np.uint16).ravel()

    y = plane(width, height, rng, 0.05 * index)
    cb = plane(cw, height, rng, 0.05 * index)
    cr = plane(cw, height, rng, 0.05 * index)
    return np.concatenate([scaled(y, 876.0), scaled(cb, 896.0), scaled(cr, 896.0)])


def many(fn, count: int, *args, seed: int = 1000, threads: int = 0):
    """fn(*args, seed, i) for i in range(count), generated on a thread pool (numpy releases
    the interpreter lock in the heavy parts)."""
    import concurrent.futures as cf
    import os
    workers = threads or min(16, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda i: fn(*args, seed, i), range(count)))
