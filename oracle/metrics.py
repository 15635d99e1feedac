"""CD / NILS / contrast restatement (metrics.rs) for the parity metric.

TEST INFRASTRUCTURE: the checker, never the product (see ``oracle/__init__``).
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np


def node_slope(profile: Sequence[float], x: Sequence[float], k: int, period: Optional[float]) -> float:
    """metrics.rs:135-183: five-point central difference where the grid is
    locally uniform, else three-point, else one-sided."""
    n = len(profile)
    if n < 2:
        return 0.0

    def at(off: int):
        idx = k + off
        if period is not None:
            wraps = idx // n
            i = idx % n
            return (x[i] + wraps * period, profile[i])
        if idx < 0 or idx >= n:
            return None
        return (x[idx], profile[idx])

    if n >= 5:
        m2, m1, p1, p2 = at(-2), at(-1), at(1), at(2)
        if None not in (m2, m1, p1, p2):
            x0 = at(0)[0]
            h = p1[0] - x0
            uniform = all(abs(d - h) <= 1e-9 * abs(h) for d in (m1[0] - m2[0], x0 - m1[0], p2[0] - p1[0]))
            if h > 0.0 and uniform:
                return (-p2[1] + 8.0 * p1[1] - 8.0 * m1[1] + m2[1]) / (12.0 * h)
    m1, p1 = at(-1), at(1)
    if m1 is not None and p1 is not None:
        return (p1[1] - m1[1]) / (p1[0] - m1[0])
    if m1 is None and p1 is not None:
        x0, y0 = at(0)
        return (p1[1] - y0) / (p1[0] - x0)
    if m1 is not None and p1 is None:
        x0, y0 = at(0)
        return (y0 - m1[1]) / (x0 - m1[0])
    return 0.0


def segment_crossing(x0, x1, y0, y1, m0, m1, t) -> Tuple[float, float]:
    """Fritsch-Carlson limited cubic Hermite crossing (metrics.rs:190-245)."""
    h = x1 - x0
    delta = (y1 - y0) / h
    if delta == 0.0 or not math.isfinite(m0) or not math.isfinite(m1):
        m0 = m1 = delta
    else:
        alpha = max(m0 / delta, 0.0)
        beta = max(m1 / delta, 0.0)
        r2 = alpha * alpha + beta * beta
        if r2 > 9.0:
            tau = 3.0 / math.sqrt(r2)
            alpha *= tau
            beta *= tau
        m0 = alpha * delta
        m1 = beta * delta

    def herm(s):
        s2 = s * s
        s3 = s2 * s
        return ((2 * s3 - 3 * s2 + 1) * y0 + (s3 - 2 * s2 + s) * h * m0
                + (-2 * s3 + 3 * s2) * y1 + (s3 - s2) * h * m1)

    def herm_slope(s):
        s2 = s * s
        return ((6 * s2 - 6 * s) * y0 + (3 * s2 - 4 * s + 1) * h * m0
                + (-6 * s2 + 6 * s) * y1 + (3 * s2 - 2 * s) * h * m1) / h

    rising = y1 > y0
    lo, hi = 0.0, 1.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if (herm(mid) >= t) == rising:
            hi = mid
        else:
            lo = mid
    s = 0.5 * (lo + hi)
    return x0 + s * h, herm_slope(s)


def find_crossings(profile, x, threshold, period=None) -> List[Tuple[float, float, bool]]:
    """metrics.rs:250-294: (x, slope, rising) in increasing x."""
    n = len(profile)
    out = []
    if n < 2 or len(x) != n:
        return out
    n_seg = n if period is not None else n - 1
    for k in range(n_seg):
        k1 = (k + 1) % n
        y0, y1 = profile[k], profile[k1]
        if not (math.isfinite(y0) and math.isfinite(y1)):
            continue
        a0, a1 = y0 >= threshold, y1 >= threshold
        if a0 == a1:
            continue
        x0 = x[k]
        x1 = x[0] + (period or 0.0) if k1 == 0 else x[k1]
        if math.isnan(x1) or x1 <= x0:
            continue
        m0 = node_slope(profile, x, k, period)
        m1 = node_slope(profile, x, k1, period)
        xc, slope = segment_crossing(x0, x1, y0, y1, m0, m1, threshold)
        out.append((xc, slope, a1))
    return out


def _periodic_field(profile, x):
    if len(profile) != len(x) or len(x) < 3:
        return None
    dx = x[1] - x[0]
    if not (math.isfinite(dx) and dx > 0.0):
        return None
    tol = 1e-6 * dx
    if not all(abs((x[i + 1] - x[i]) - dx) <= tol for i in range(len(x) - 1)):
        return None
    return x[0] - 0.5 * dx, dx * len(x)


def periodic_features(profile, x, threshold, tone: str):
    """metrics.rs:316-400: (left, right, width, centre, left_slope, right_slope)."""
    pf = _periodic_field(profile, x)
    if pf is None:
        return []
    x_lo, period = pf
    cr = find_crossings(profile, x, threshold, period)
    m = len(cr)
    out = []
    if m < 2:
        return out

    def starts(c):
        return (not c[2]) if tone == "dark" else c[2]

    for i in range(m):
        start = cr[i]
        if not starts(start):
            continue
        end = cr[(i + 1) % m]
        if starts(end):
            continue
        width = end[0] - start[0]
        if width <= 0.0:
            width += period
        left = start[0]
        if left >= x_lo + period:
            left -= period
        centre = left + 0.5 * width
        while centre >= x_lo + period:
            centre -= period
        out.append((left, left + width, width, centre, start[1], end[1]))
    return out


def _ring_distance(a, b, period):
    d = (a - b) % period
    return min(d, period - d)


def _nearest_centre(features, x_lo, period):
    if not features:
        return None
    centre = x_lo + 0.5 * period
    return min(features, key=lambda f: _ring_distance(f[3], centre, period))


def measure_cd_periodic(profile, x, threshold, tone="dark") -> Optional[float]:
    """metrics.rs:423-434."""
    pf = _periodic_field(profile, x)
    if pf is None:
        return None
    f = _nearest_centre(periodic_features(profile, x, threshold, tone), *pf)
    return None if f is None else f[2]


def nils_periodic(profile, x, threshold, tone="dark", width_nm=None) -> Optional[float]:
    """metrics.rs:456-471."""
    if not (threshold > 0.0):
        return None
    pf = _periodic_field(profile, x)
    if pf is None:
        return None
    f = _nearest_centre(periodic_features(profile, x, threshold, tone), *pf)
    if f is None:
        return None
    ils = 0.5 * (abs(f[4]) + abs(f[5])) / threshold
    return (width_nm if width_nm is not None else f[2]) * ils


def centre_profile(image: np.ndarray) -> np.ndarray:
    """metrics.rs:520-541: y = 0 cross-section (4-point cubic for even rows)."""
    ny = image.shape[0]
    if ny % 2 == 1:
        return image[ny // 2].copy()
    r0, r1 = ny // 2 - 1, ny // 2
    if ny < 4:
        return 0.5 * (image[r0] + image[r1])
    return (-image[r0 - 1] + 9.0 * image[r0] + 9.0 * image[r1] - image[r1 + 1]) / 16.0


def image_contrast(image: np.ndarray) -> float:
    """metrics.rs:620-629."""
    mx, mn = float(np.max(image)), float(np.min(image))
    return (mx - mn) / (mx + mn) if mx + mn > 0.0 else 0.0


def all_edges(image: np.ndarray, x: np.ndarray, threshold: float):
    """Every threshold crossing on every row and every column cutline of a
    periodic image: list of (axis, line, position). Used for the max |d edge|
    CD-error metric on random clips."""
    out = []
    for axis in (0, 1):
        img = image if axis == 0 else image.T
        for r in range(img.shape[0]):
            pf = _periodic_field(img[r], x)
            for c in find_crossings(list(img[r]), list(x), threshold, pf[1]):
                out.append((axis, r, c[0], c[2]))
    return out


def max_edge_error(img: np.ndarray, ref: np.ndarray, x: np.ndarray, threshold: float) -> Tuple[float, int]:
    """Max |edge shift| (nm) between matched threshold crossings of two
    images on all row/column cutlines; returns (max shift, unmatched count).
    Crossings are matched per cutline by order and direction."""
    worst, unmatched = 0.0, 0
    for axis in (0, 1):
        a_img = img if axis == 0 else img.T
        b_img = ref if axis == 0 else ref.T
        period = (x[1] - x[0]) * len(x)
        for r in range(a_img.shape[0]):
            ca = find_crossings(list(a_img[r]), list(x), threshold, period)
            cb = find_crossings(list(b_img[r]), list(x), threshold, period)
            if len(ca) != len(cb):
                unmatched += abs(len(ca) - len(cb))
                continue
            for p, q in zip(ca, cb):
                if p[2] != q[2]:
                    unmatched += 1
                    continue
                worst = max(worst, abs(p[0] - q[0]))
    return worst, unmatched
