"""Parity measures shared by the GPU tests (not a test module).

- ``rel_err``: max|I - I_ref| / max(I_ref), the reference's own convention
  (imaging_validation.rs:209-210);
- ``edge_error_nm``: worst displacement of the threshold crossings found by
  the oracle's restatement of find_crossings (metrics.rs:250-294) along row
  and column cutlines, matched crossing by crossing, plus the count of
  crossings present in one image and not in the other.
"""
from __future__ import annotations

import numpy as np

from oracle import metrics as M


def rel_err(img, ref) -> float:
    return float(np.max(np.abs(np.asarray(img, np.float64) - ref)) / np.max(ref))


def edge_error_nm(img, ref, pixel_nm: float = 1.0, threshold: float = 0.3, step: int = 8):
    n = img.shape[-1]
    x = (-n / 2 + (np.arange(n) + 0.5)) * pixel_nm
    period = n * pixel_nm
    worst, unmatched = 0.0, 0
    for a, b in ((img, ref), (img.T, ref.T)):
        for r in range(0, a.shape[0], step):
            ca = M.find_crossings(list(map(float, a[r])), list(x), threshold, period)
            cb = M.find_crossings(list(map(float, b[r])), list(x), threshold, period)
            if len(ca) != len(cb):
                unmatched += abs(len(ca) - len(cb))
                continue
            for p, q in zip(ca, cb):
                worst = max(worst, abs(p[0] - q[0]))
    return worst, unmatched
