"""Seeded ILT targets: centred arrays of square contacts.

A target is the area-averaged (4 x 4 sub-samples per pixel) indicator of a
count_x x count_y array of square holes, value 1 inside, as the reference's
create_target_contact_array builds it (crates/highuvlith-core/src/ilt.rs:336-362).
The workload draws counts in {2..8}, hole size in [16, 24] nm and pitch in
[32, 48] nm with size < pitch, from numpy PCG64 seed base_seed + id.
"""
from __future__ import annotations

import numpy as np


def contact_array(n: int, pixel: float, size: float, pitch_x: float, pitch_y: float, count_x: int,
                  count_y: int) -> np.ndarray:
    half = n * pixel / 2.0
    r = size / 2.0
    s = 4
    sub = (np.arange(s) + 0.5) / s
    coords = -half + (np.arange(n)[:, None] + sub[None, :]) * pixel  # (n, s) sub-sample coordinates
    out = np.zeros((n, n))
    for iy in range(count_y):
        cy = (iy - (count_y - 1) / 2.0) * pitch_y
        fy = (np.abs(coords - cy) <= r).sum(axis=1) / s
        if not fy.any():
            continue
        for ix in range(count_x):
            cx = (ix - (count_x - 1) / 2.0) * pitch_x
            fx = (np.abs(coords - cx) <= r).sum(axis=1) / s
            out = np.maximum(out, fy[:, None] * fx[None, :])
    return out


def gen_contact_targets(count: int, n: int, pixel: float = 1.0, base_seed: int = 2026):
    """(targets float32 (count, n, n), list of (size, pitch, nx, ny))."""
    out = np.zeros((count, n, n), dtype=np.float32)
    meta = []
    for i in range(count):
        rng = np.random.Generator(np.random.PCG64(base_seed + i))
        nx, ny = int(rng.integers(2, 9)), int(rng.integers(2, 9))
        size = float(rng.uniform(16.0, 24.0))
        pitch = float(rng.uniform(32.0, 48.0))
        while size >= pitch:
            size = float(rng.uniform(16.0, 24.0))
        out[i] = contact_array(n, pixel, size, pitch, pitch, nx, ny)
        meta.append((size, pitch, nx, ny))
    return out, meta
