"""Profile metrics of periodic aerial images: threshold crossings, printed CD,
NILS, contrast (crates/highuvlith-core/src/metrics.rs).

Vectorised over the segments of a periodic, uniformly sampled cutline:
node slopes are the five-point central difference (metrics.rs:135-183 on a
uniform periodic grid), each threshold crossing solves the Fritsch-Carlson
limited cubic Hermite segment by bisection (metrics.rs:190-245), features
run from a crossing into the feature tone to the next crossing out of it
(metrics.rs:316-400), and the printed CD / NILS are those of the feature
whose centre is nearest the field centre (metrics.rs:423-471).
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np


def pixel_centres(n: int, field_nm: float) -> np.ndarray:
    """x_j = -L/2 + (j + 1/2) p (types.rs:7-15)."""
    p = field_nm / n
    return -field_nm / 2.0 + (np.arange(n) + 0.5) * p


def centre_profile(image: np.ndarray) -> np.ndarray:
    """The y = 0 cross-section (metrics.rs:520-541): the middle row for odd
    row counts, else the 4-point cubic between the two middle rows."""
    ny = image.shape[0]
    if ny % 2 == 1:
        return np.array(image[ny // 2], dtype=np.float64)
    r0, r1 = ny // 2 - 1, ny // 2
    if ny < 4:
        return 0.5 * (image[r0] + image[r1]).astype(np.float64)
    return (-image[r0 - 1].astype(np.float64) + 9.0 * image[r0] + 9.0 * image[r1] - image[r1 + 1]) / 16.0


def image_contrast(image: np.ndarray) -> float:
    """(max - min) / (max + min) (metrics.rs:620-629)."""
    mx, mn = float(np.max(image)), float(np.min(image))
    return (mx - mn) / (mx + mn) if mx + mn > 0.0 else 0.0


def crossings(profile: np.ndarray, x: np.ndarray, threshold: float,
              periodic: bool = True) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Threshold crossings of a uniform profile: (position, slope, rising),
    in increasing position.  ``periodic``: the profile wraps (the segment
    from the last sample to the first counts, slopes wrap); else it is open
    (metrics.rs:135-183 node slopes: three-point next to the ends,
    one-sided at them)."""
    y = np.asarray(profile, dtype=np.float64)
    n = y.size
    if n < 5:
        raise ValueError("profile needs at least 5 samples")
    h = float(x[1] - x[0])
    m = (-np.roll(y, -2) + 8.0 * np.roll(y, -1) - 8.0 * np.roll(y, 1) + np.roll(y, 2)) / (12.0 * h)
    if not periodic:
        m[[1, n - 2]] = [(y[2] - y[0]) / (2.0 * h), (y[n - 1] - y[n - 3]) / (2.0 * h)]
        m[0], m[n - 1] = (y[1] - y[0]) / h, (y[n - 1] - y[n - 2]) / h
    y0, y1 = y, np.roll(y, -1)
    m0, m1 = m, np.roll(m, -1)
    a0, a1 = y0 >= threshold, y1 >= threshold
    k = np.nonzero(a0 != a1)[0]
    if not periodic:
        k = k[k < n - 1]
    if k.size == 0:
        empty = np.zeros(0)
        return empty, empty, np.zeros(0, dtype=bool)
    y0, y1, m0, m1 = y0[k], y1[k], m0[k], m1[k]
    delta = (y1 - y0) / h
    alpha = np.maximum(m0 / delta, 0.0)
    beta = np.maximum(m1 / delta, 0.0)
    r2 = alpha * alpha + beta * beta
    tau = np.where(r2 > 9.0, 3.0 / np.sqrt(np.maximum(r2, 1e-300)), 1.0)
    m0, m1 = alpha * tau * delta, beta * tau * delta

    def herm(s):
        s2, s3 = s * s, s * s * s
        return ((2 * s3 - 3 * s2 + 1) * y0 + (s3 - 2 * s2 + s) * h * m0 + (-2 * s3 + 3 * s2) * y1
                + (s3 - s2) * h * m1)

    rising = y1 > y0
    lo, hi = np.zeros(k.size), np.ones(k.size)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        up = (herm(mid) >= threshold) == rising
        hi = np.where(up, mid, hi)
        lo = np.where(up, lo, mid)
    s = 0.5 * (lo + hi)
    s2 = s * s
    slope = ((6 * s2 - 6 * s) * y0 + (3 * s2 - 4 * s + 1) * h * m0 + (-6 * s2 + 6 * s) * y1
             + (3 * s2 - 2 * s) * h * m1) / h
    return x[k] + s * h, slope, a1[k]


def _features(profile, x, threshold, tone):
    """(left, width, centre, slope_in, slope_out) of every feature."""
    pos, slope, rising = crossings(profile, x, threshold)
    period = float(x[1] - x[0]) * len(x)
    x_lo = float(x[0]) - 0.5 * float(x[1] - x[0])
    m = pos.size
    out = []
    if m < 2:
        return out, x_lo, period
    starts = ~rising if tone == "dark" else rising
    for i in range(m):
        j = (i + 1) % m
        if not starts[i] or starts[j]:
            continue
        width = pos[j] - pos[i]
        if width <= 0.0:
            width += period
        left = pos[i] if pos[i] < x_lo + period else pos[i] - period
        centre = left + 0.5 * width
        while centre >= x_lo + period:
            centre -= period
        out.append((left, width, centre, slope[i], slope[j]))
    return out, x_lo, period


def _nearest(feats, x_lo, period):
    if not feats:
        return None
    c = x_lo + 0.5 * period

    def ring(a):
        d = (a - c) % period
        return min(d, period - d)

    return min(feats, key=lambda f: ring(f[2]))


def printed_cd(profile, x, threshold: float, tone: str = "dark") -> Optional[float]:
    """Width of the feature nearest the centre (metrics.rs:423-434)."""
    f = _nearest(*_features(profile, x, threshold, tone))
    return None if f is None else float(f[1])


def nils(profile, x, threshold: float, tone: str = "dark", width_nm: Optional[float] = None) -> Optional[float]:
    """width x mean |edge slope| / threshold (metrics.rs:456-471)."""
    if not (threshold > 0.0):
        return None
    f = _nearest(*_features(profile, x, threshold, tone))
    if f is None:
        return None
    ils = 0.5 * (abs(f[3]) + abs(f[4])) / threshold
    return float((width_nm if width_nm is not None else f[1]) * ils)


def features(profile, x, threshold: float, tone: str = "dark"):
    """Every ``tone`` feature of a periodic profile as (left, right, width,
    centre) in nm (metrics.rs:388-421); a feature crossing the field edge has
    ``right`` beyond the field."""
    feats, _, _ = _features(profile, x, threshold, tone)
    return [(float(f[0]), float(f[0] + f[1]), float(f[1]), float(f[2])) for f in feats]


def image_log_slope(profile, x, threshold: float, tone: str = "dark") -> Optional[float]:
    """|d ln I / dx| at the edges of the feature nearest the centre, the two
    edge slopes averaged (metrics.rs:436-449)."""
    if not (threshold > 0.0):
        return None
    f = _nearest(*_features(profile, x, threshold, tone))
    return None if f is None else float(0.5 * (abs(f[3]) + abs(f[4])) / threshold)


def measure_cd_open(profile, x, threshold: float) -> Optional[float]:
    """Width between the consecutive crossings of an open profile whose
    midpoint is nearest the profile centre, whatever its tone
    (metrics.rs:560-580)."""
    pos, _, _ = crossings(profile, x, threshold, periodic=False)
    if pos.size < 2:
        return None
    centre = 0.5 * (float(x[0]) + float(x[-1]))
    i = int(np.argmin(np.abs(0.5 * (pos[:-1] + pos[1:]) - centre)))
    return float(abs(pos[i + 1] - pos[i]))


def nils_open(profile, x, threshold: float) -> Optional[float]:
    """Legacy NILS of an open profile: the slope at the crossing nearest the
    centre times measure_cd_open, over the threshold (metrics.rs:603-617)."""
    if abs(threshold) < 1e-15:
        return None
    pos, slope, _ = crossings(profile, x, threshold, periodic=False)
    if pos.size == 0:
        return None
    centre = 0.5 * (float(x[0]) + float(x[-1]))
    edge = int(np.argmin(np.abs(pos - centre)))
    cd = measure_cd_open(profile, x, threshold)
    return None if cd is None else float(cd * abs(slope[edge]) / abs(threshold))
