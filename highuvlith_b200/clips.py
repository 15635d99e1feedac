"""Seeded synthetic Manhattan mask clips.

The workloads have no public dataset: clips are drawn from numpy's PCG64
with seed ``base_seed + clip_id``.  A clip is a dark-field binary mask of
clear axis-aligned rectangles with integer-pixel corners (pixel-aligned, so
the raster times the pixel transfer is the exact mask spectrum), added until
the clear-area fraction reaches a target drawn uniformly from
[density_min, density_max].  Rectangles may overlap and are clipped to the
field.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

Rect = Tuple[int, int, int, int]  # x0, y0, w, h in pixels from the field corner


def gen_clip(seed: int, n: int, wmin: int = 10, wmax: int = 80, dmin: float = 0.30,
             dmax: float = 0.50, max_rects: int = 100000) -> Tuple[List[Rect], np.ndarray]:
    """One clip: (rectangles, uint8 raster (n, n))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    target = rng.uniform(dmin, dmax)
    raster = np.zeros((n, n), dtype=np.uint8)
    rects: List[Rect] = []
    covered = 0
    goal = target * n * n
    wmax = min(wmax, n)
    wmin = min(wmin, wmax)
    while covered < goal and len(rects) < max_rects:
        w = int(rng.integers(wmin, wmax + 1))
        h = int(rng.integers(wmin, wmax + 1))
        x0 = int(rng.integers(0, n - w + 1))
        y0 = int(rng.integers(0, n - h + 1))
        sub = raster[y0:y0 + h, x0:x0 + w]
        covered += int(w * h - int(sub.sum()))
        sub[...] = 1
        rects.append((x0, y0, w, h))
    return rects, raster


def gen_batch(n_clips: int, n: int, base_seed: int = 2026, **kw):
    """(list of rect lists, uint8 rasters (n_clips, n, n))."""
    rects, rasters = [], np.zeros((n_clips, n, n), dtype=np.uint8)
    for c in range(n_clips):
        r, img = gen_clip(base_seed + c, n, **kw)
        rects.append(r)
        rasters[c] = img
    return rects, rasters
