"""FP64 numpy restatement of the reference's Hopkins/SOCS imaging path.

TEST INFRASTRUCTURE: the checker, never the product (see ``oracle/__init__``).

Every function names the reference location it restates (paths relative to
``crates/highuvlith-core/src``). FFT conventions follow math/fft2d.rs:11-13:
forward unnormalised, inverse with ``1/N²``, FFT index k -> signed order
``k`` (k < N/2) or ``k - N``. numpy's ``fft2``/``ifft2`` use exactly these
conventions.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# Constants (aerial.rs:284-351)
# ---------------------------------------------------------------------------
MAX_FACTOR_BYTES = 1 << 30
DENSE_FAST_DIM = 320
DENSE_MAX_DIM = 1536
RANDOMIZED_OVERSAMPLE = 16
EIGEN_ZERO_REL = 1e-12
DEGENERACY_REL = 1e-6
DARK_FIELD_FRACTION = 1e-2
PROBE_HALF_WIDTH = 2.0
PROBE_POINTS = 129
ZOOM_POINTS = 129
MAX_ZOOM_LEVELS = 6
SUPPORT_THRESHOLD = 1e-4
RESOLVED_CELLS = 24.0
TARGET_STEP_SIGMA = 0.04
MIN_SOURCE_POINTS = 200.0
SUBCELLS = 8
MAX_REFINE = 8
MAX_REFINE_DEPTH = 3
# Lattice rotation tan(theta) = 1/phi, as (cos, sin) (aerial.rs:345-346).
LATTICE_COS = 0.85065080835204
LATTICE_SIN = 0.5257311121191336
MAX_POINTS_PER_AXIS = 128
COHERENT_EXTENT_FRACTION = 1e-3

ARF_WAVELENGTH_NM = 193.368  # source.rs:285
F2_WAVELENGTH_NM = 157.63
EUV_WAVELENGTH_NM = 13.5
WATER_INDEX_193NM = 1.437  # optics/mod.rs:176


def signed_index(k: int, n: int) -> int:
    """FFT index -> signed order (aerial.rs:976-982, mask.rs:793-799)."""
    return k if k < n // 2 else k - n


def signed_orders(n: int) -> np.ndarray:
    k = np.arange(n)
    return np.where(k < n // 2, k, k - n)


def rust_round(x: float) -> float:
    """f64::round: half away from zero."""
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


# ---------------------------------------------------------------------------
# Grid (types.rs:209-319)
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Grid:
    size: int
    pixel_nm: float

    @property
    def field_nm(self) -> float:
        return self.size * self.pixel_nm

    @property
    def freq_step(self) -> float:
        return 1.0 / self.field_nm

    def pixel_centres(self) -> np.ndarray:
        """x_j = -L/2 + (j + 1/2) p (types.rs:7-15, aerial.rs:1750-1759)."""
        half = self.field_nm / 2.0
        return -half + (np.arange(self.size) + 0.5) * self.pixel_nm


def commensurate_grid(pitch_nm: float, size: int, target_pixel_nm: float) -> Grid:
    """GridConfig::commensurate for one pitch (types.rs:268-298)."""
    cells = max(math.floor(size * target_pixel_nm / pitch_nm + 1e-9), 1.0)
    return Grid(size, cells * pitch_nm / size)


# ---------------------------------------------------------------------------
# Illumination fills (source.rs:1178-1248) and custom fills
# ---------------------------------------------------------------------------
def fill_conventional(sigma: float) -> Callable[[float, float], float]:
    def f(x: float, y: float) -> float:
        rho = math.sqrt(x * x + y * y)
        return 1.0 if rho <= sigma else 0.0
    return f


def fill_annular(inner: float, outer: float) -> Callable[[float, float], float]:
    def f(x: float, y: float) -> float:
        rho = math.sqrt(x * x + y * y)
        return 1.0 if (rho >= inner and rho <= outer) else 0.0
    return f


def fill_dipole(sigma_center: float, sigma_radius: float, orientation_deg: float):
    """Two circular poles at `orient` and `orient + pi` (source.rs:1221-1239)."""
    orient = orientation_deg * (math.pi / 180.0)
    poles = []
    for pole in (orient, orient + math.pi):
        poles.append((sigma_center * math.cos(pole), sigma_center * math.sin(pole)))

    def f(x: float, y: float) -> float:
        for cx, cy in poles:
            dx, dy = x - cx, y - cy
            if math.sqrt(dx * dx + dy * dy) <= sigma_radius:
                return 1.0
        return 0.0
    return f


def fill_quadrupole(sigma_center: float, sigma_radius: float, opening_angle_deg: float):
    """Poles on the axes at 0/90/180/270 deg (source.rs:1198-1220)."""
    half_open = opening_angle_deg / 2.0

    def f(x: float, y: float) -> float:
        angle = math.atan2(y, x) * (180.0 / math.pi)
        for pa in (0.0, 90.0, 180.0, 270.0):
            da = ((angle - pa + 180.0) % 360.0) - 180.0
            cx = sigma_center * math.cos(pa * (math.pi / 180.0))
            cy = sigma_center * math.sin(pa * (math.pi / 180.0))
            if abs(da) <= half_open and math.sqrt((x - cx) ** 2 + (y - cy) ** 2) <= sigma_radius:
                return 1.0
        return 0.0
    return f


def fill_quasar(inner: float, outer: float, opening_deg: float = 45.0):
    """Custom source (not an IlluminationShape): four annular sectors
    inner <= rho <= outer centred at 45 + k*90 deg with the given opening.
    A legal LithographySource::intensity_at (imaging_validation.rs:21-51)."""
    half_open = opening_deg / 2.0

    def f(x: float, y: float) -> float:
        rho = math.sqrt(x * x + y * y)
        if rho < inner or rho > outer:
            return 0.0
        angle = math.atan2(y, x) * (180.0 / math.pi)
        for c in (45.0, 135.0, 225.0, 315.0):
            da = ((angle - c + 180.0) % 360.0) - 180.0
            if abs(da) <= half_open:
                return 1.0
        return 0.0
    return f


def fill_gaussian(sigma: float):
    def f(x: float, y: float) -> float:
        rho = math.sqrt(x * x + y * y)
        if rho <= 1.0 and sigma > 0.0:
            return math.exp(-rho * rho / (2.0 * sigma * sigma))
        return 0.0
    return f


# ---------------------------------------------------------------------------
# Optics (optics/mod.rs:155-171, 310-357; optics/euv.rs:129-160)
# ---------------------------------------------------------------------------
def defocus_phase_in_medium(z: float, na_rho: float, n: float, lam: float,
                            paraxial: bool = False) -> float:
    s = na_rho / n
    s2 = s * s
    if paraxial:
        return math.pi * z * n * s2 / lam
    cos_t = math.sqrt(max(1.0 - s2, 0.0))
    return 2.0 * math.pi * n * z * s2 / ((1.0 + cos_t) * lam)


@dataclass
class ProjectionOptics:
    na: float
    flare_fraction: float = 0.02
    immersion_index: float = 1.0
    paraxial_defocus: bool = False

    @property
    def flare(self) -> float:
        return self.flare_fraction

    def cutoff(self, lam: float) -> float:
        return self.na / lam

    def pupil(self, fx: float, fy: float, z: float, lam: float) -> complex:
        rho2 = fx * fx + fy * fy
        if rho2 > 1.0:
            return 0j
        rho = math.sqrt(rho2)
        ph = 0.0 if z == 0.0 else defocus_phase_in_medium(
            z, self.na * rho, self.immersion_index, lam, self.paraxial_defocus)
        return complex(math.cos(ph), math.sin(ph))

    def pupil_grid(self, fx, fy, z: float, lam: float) -> np.ndarray:
        """Vectorised ``pupil`` (same formulas, elementwise)."""
        rho2 = fx * fx + fy * fy
        inside = rho2 <= 1.0
        rho = np.sqrt(np.where(inside, rho2, 0.0))
        if z == 0.0:
            ph = np.zeros_like(rho)
        else:
            s = self.na * rho / self.immersion_index
            s2 = s * s
            if self.paraxial_defocus:
                ph = np.pi * z * self.immersion_index * s2 / lam
            else:
                c = np.sqrt(np.maximum(1.0 - s2, 0.0))
                ph = 2.0 * np.pi * self.immersion_index * z * s2 / ((1.0 + c) * lam)
        return np.where(inside, np.cos(ph) + 1j * np.sin(ph), 0.0)


@dataclass
class EuvOptics:
    na: float
    central_obscuration: float = 0.0
    flare_fraction: float = 0.0
    transmission: float = 1.0
    paraxial_defocus: bool = False
    immersion_index: float = 1.0

    @property
    def flare(self) -> float:
        return self.flare_fraction

    def cutoff(self, lam: float) -> float:
        return self.na / lam

    def pupil(self, fx: float, fy: float, z: float, lam: float) -> complex:
        rho2 = fx * fx + fy * fy
        if rho2 > 1.0:
            return 0j
        rho = math.sqrt(rho2)
        if rho < self.central_obscuration:
            return 0j
        ph = 0.0 if z == 0.0 else defocus_phase_in_medium(
            z, self.na * rho, 1.0, lam, self.paraxial_defocus)
        amp = math.sqrt(max(self.transmission, 0.0))
        return complex(amp * math.cos(ph), amp * math.sin(ph))

    def pupil_grid(self, fx, fy, z: float, lam: float) -> np.ndarray:
        rho2 = fx * fx + fy * fy
        rho = np.sqrt(np.where(rho2 <= 1.0, rho2, 0.0))
        inside = (rho2 <= 1.0) & ~(rho < self.central_obscuration)
        if z == 0.0:
            ph = np.zeros_like(rho)
        else:
            s2 = (self.na * rho) ** 2
            if self.paraxial_defocus:
                ph = np.pi * z * s2 / lam
            else:
                c = np.sqrt(np.maximum(1.0 - s2, 0.0))
                ph = 2.0 * np.pi * 1.0 * z * s2 / ((1.0 + c) * lam)
        amp = math.sqrt(max(self.transmission, 0.0))
        return np.where(inside, amp * np.cos(ph) + 1j * amp * np.sin(ph), 0.0)


def euv_nxe_033() -> EuvOptics:
    return EuvOptics(0.33, 0.0)


def euv_high_na_055() -> EuvOptics:
    return EuvOptics(0.55, 0.2)


# ---------------------------------------------------------------------------
# Source sampling (aerial.rs:357-947)
# ---------------------------------------------------------------------------
@dataclass
class _Probe:
    bx0: float
    bx1: float
    by0: float
    by1: float
    step_x: float
    step_y: float
    count: int
    cx: float
    cy: float


def _clean(v: float) -> float:
    return v if (math.isfinite(v) and v > 0.0) else 0.0


def _probe_lattice(f, bounds, n: int, centered: bool) -> Optional[_Probe]:
    """aerial.rs:371-433."""
    x0, x1, y0, y1 = bounds
    step_x = (x1 - x0) / (n - 1)
    step_y = (y1 - y0) / (n - 1)
    half = (n - 1) / 2.0

    def coord(lo, step, i):
        return (i - half) * step if centered else lo + i * step

    xs = [coord(x0, step_x, i) for i in range(n)]
    ys = [coord(y0, step_y, i) for i in range(n)]
    values = [[_clean(f(xs[ix], ys[iy])) for ix in range(n)] for iy in range(n)]
    imax = 0.0
    for row in values:
        for v in row:
            imax = max(imax, v)
    if imax <= 0.0:
        return None
    thr = SUPPORT_THRESHOLD * imax
    bx0, bx1, by0, by1 = math.inf, -math.inf, math.inf, -math.inf
    count = 0
    wsum = wx = wy = 0.0
    for iy in range(n):
        y = ys[iy]
        row = values[iy]
        for ix in range(n):
            v = row[ix]
            if v <= 0.0:
                continue
            x = xs[ix]
            wsum += v
            wx += v * x
            wy += v * y
            if v > thr:
                count += 1
                bx0 = min(bx0, x)
                bx1 = max(bx1, x)
                by0 = min(by0, y)
                by1 = max(by1, y)
    return _Probe(bx0, bx1, by0, by1, step_x, step_y, count, wx / wsum, wy / wsum)


@dataclass(frozen=True)
class _Mirror:
    swap: bool
    flip_x: bool
    flip_y: bool

    def apply(self, x, y):
        a, b = (y, x) if self.swap else (x, y)
        return (-a if self.flip_x else a, -b if self.flip_y else b)

    def compose(self, h: "_Mirror") -> "_Mirror":
        hx, hy = (h.flip_y, h.flip_x) if self.swap else (h.flip_x, h.flip_y)
        return _Mirror(self.swap ^ h.swap, self.flip_x ^ hx, self.flip_y ^ hy)


_IDENTITY = _Mirror(False, False, False)
_MX = _Mirror(False, True, False)
_MY = _Mirror(False, False, True)
_MDIAG = _Mirror(True, False, False)


def _generate(gens):
    group = [_IDENTITY]
    k = 0
    while k < len(group):
        for g in gens:
            e = group[k].compose(g)
            if e not in group:
                group.append(e)
        k += 1
    return group


class _CellGeometry:
    """aerial.rs:743-883."""

    def __init__(self, f, center, step, half_box, walls):
        self.f = f
        self.center = center
        self.step = step
        self.half_box = half_box
        self.walls = walls

    def to_xy(self, u, v):
        s = self.step
        return (s * (LATTICE_COS * u - LATTICE_SIN * v), s * (LATTICE_SIN * u + LATTICE_COS * v))

    def in_domain(self, x, y):
        return (abs(x) <= self.half_box[0] and abs(y) <= self.half_box[1]
                and all(inside(x, y) for _, inside in self.walls))

    def eval(self, g, x, y):
        gx, gy = g.apply(x, y)
        return _clean(self.f(self.center[0] + gx, self.center[1] + gy))

    def point(self, g, xy, weight):
        gx, gy = g.apply(xy[0], xy[1])
        return (self.center[0] + gx, self.center[1] + gy, weight)

    def integrate(self, uv0, du, g):
        u0, v0 = uv0
        area = du * du
        centre = self.to_xy(u0 + 0.5 * du, v0 + 0.5 * du)
        corners = [self.to_xy(u0 + a, v0 + b) for a, b in ((0.0, 0.0), (du, 0.0), (0.0, du), (du, du))]
        interior = all(self.in_domain(x, y) for x, y in corners)
        vc = self.eval(g, centre[0], centre[1])
        if interior and all(self.eval(g, x, y) == vc for x, y in corners):
            if vc > 0.0:
                return (self.point(g, centre, vc * area), False, g)
            return None
        sub = float(SUBCELLS)
        mass = mx = my = 0.0
        inside = lit = 0
        vmin, vmax = math.inf, 0.0
        for k in range(SUBCELLS * SUBCELLS):
            a, b = float(k % SUBCELLS), float(k // SUBCELLS)
            x, y = self.to_xy(u0 + (a + 0.5) / sub * du, v0 + (b + 0.5) / sub * du)
            if not self.in_domain(x, y):
                continue
            inside += 1
            v = self.eval(g, x, y)
            vmin = min(vmin, v)
            vmax = max(vmax, v)
            if v > 0.0:
                mass += v
                mx += v * x
                my += v * y
                lit += 1
        if mass <= 0.0:
            return None
        graded = lit == inside and vmin < vmax
        if interior and lit == SUBCELLS * SUBCELLS and vc > 0.0:
            pt = self.point(g, centre, vc * area)
        else:
            pt = self.point(g, (mx / mass, my / mass), mass / (sub * sub) * area)
        return (pt, graded, g)

    def refine(self, uv0, du, cell, target, depth, out):
        pt, graded, image = cell
        if not (graded and pt[2] > target) or depth >= MAX_REFINE_DEPTH:
            out.append(pt)
            return
        r = min(max(int(math.ceil(math.sqrt(pt[2] / target))), 2), MAX_REFINE)
        dc = du / r
        for b in range(r):
            for a in range(r):
                corner = (uv0[0] + a * dc, uv0[1] + b * dc)
                child = self.integrate(corner, dc, image)
                if child is not None:
                    self.refine(corner, dc, child, target, depth + 1, out)


def _lattice_cells(f, center, wh, step, sym):
    """aerial.rs:684-731."""
    w, h = wh
    sx, sy, diag = sym
    walls = []
    if sx and not diag:
        walls.append((_MX, lambda x, y: x > 0.0))
    if sy:
        walls.append((_MY, lambda x, y: y > 0.0))
    if diag:
        walls.append((_MDIAG, lambda x, y: y < x))
    geo = _CellGeometry(f, center, step, (0.5 * w, 0.5 * h), walls)
    margin = step * math.sqrt(2.0)
    reach = math.hypot(w, h) * 0.5 + margin
    n = int(math.ceil(reach / step)) + 1
    cells = []
    for j in range(-n, n):
        for i in range(-n, n):
            x, y = geo.to_xy(i + 0.5, j + 0.5)
            near_domain = ((not sx or diag or x > -margin) and (not sy or y > -margin)
                           and (not diag or y < x + margin))
            near_box = abs(x) <= 0.5 * w + margin and abs(y) <= 0.5 * h + margin
            if near_box and near_domain:
                cells.append((float(i), float(j)))
    group = _generate([wall[0] for wall in walls])
    n_img = len(group)
    coarse = [geo.integrate(cells[k // n_img], 1.0, group[k % n_img])
              for k in range(len(cells) * n_img)]
    total = 0.0
    for c in coarse:
        if c is not None:
            total += c[0][2]
    target = total / MIN_SOURCE_POINTS
    out = []
    for k, c in enumerate(coarse):
        if c is not None:
            geo.refine(cells[k // n_img], 1.0, c, target, 0, out)
    return out


def _normalized_or_centroid(points, cx, cy):
    total = 0.0
    for p in points:
        total += p[2]
    if not points or math.isnan(total) or total <= 0.0:
        return [(cx, cy, 1.0)]
    return [(p[0], p[1], p[2] / total) for p in points]


def sample_source(f, points_per_axis: Optional[int], df_sigma: float) -> List[Tuple[float, float, float]]:
    """sample_intensity (aerial.rs:436-559) / sample_source (941-947)."""
    probe = _probe_lattice(f, (-PROBE_HALF_WIDTH, PROBE_HALF_WIDTH,
                               -PROBE_HALF_WIDTH, PROBE_HALF_WIDTH), PROBE_POINTS, True)
    if probe is None:
        raise ValueError("source pupil fill has no intensity inside |sigma| <= 2")
    for _ in range(MAX_ZOOM_LEVELS):
        rx = probe.bx1 - probe.bx0 >= RESOLVED_CELLS * probe.step_x
        ry = probe.by1 - probe.by0 >= RESOLVED_CELLS * probe.step_y
        if rx and ry:
            break
        b = (probe.bx0 - probe.step_x, probe.bx1 + probe.step_x,
             probe.by0 - probe.step_y, probe.by1 + probe.step_y)
        p = _probe_lattice(f, b, ZOOM_POINTS, False)
        if p is None:
            break
        probe = p
    sym_x = abs(probe.bx0 + probe.bx1) <= 0.5 * probe.step_x
    sym_y = abs(probe.by0 + probe.by1) <= 0.5 * probe.step_y
    if sym_x:
        cx_box, w = 0.0, 2.0 * (max(abs(probe.bx0), abs(probe.bx1)) + probe.step_x)
    else:
        cx_box, w = 0.5 * (probe.bx0 + probe.bx1), probe.bx1 - probe.bx0 + 2.0 * probe.step_x
    if sym_y:
        cy_box, h = 0.0, 2.0 * (max(abs(probe.by0), abs(probe.by1)) + probe.step_y)
    else:
        cy_box, h = 0.5 * (probe.by0 + probe.by1), probe.by1 - probe.by0 + 2.0 * probe.step_y
    if sym_x and sym_y and abs(w - h) <= max(probe.step_x, probe.step_y):
        m = max(w, h)
        w = h = m
    extent = max(w, h)
    if points_per_axis == 1 or extent < COHERENT_EXTENT_FRACTION * df_sigma:
        return [(0.0 if sym_x else probe.cx, 0.0 if sym_y else probe.cy, 1.0)]
    if points_per_axis is not None:
        step = extent / max(points_per_axis, 1)
        nx = max(int(rust_round(w / step)), 1)
        ny = max(int(rust_round(h / step)), 1)
        hx, hy = w / nx, h / ny
        pts = []
        for iy in range(ny):
            y = cy_box + (iy + 0.5 - ny / 2.0) * hy
            for ix in range(nx):
                x = cx_box + (ix + 0.5 - nx / 2.0) * hx
                v = f(x, y)
                if math.isfinite(v) and v > 0.0:
                    pts.append((x, y, v))
        return _normalized_or_centroid(pts, probe.cx, probe.cy)
    area = max(probe.count, 1) * probe.step_x * probe.step_y
    step = max(min(TARGET_STEP_SIGMA, math.sqrt(area / MIN_SOURCE_POINTS)), extent / MAX_POINTS_PER_AXIS)
    sym = (sym_x, sym_y, sym_x and sym_y and w == h)
    pts = _lattice_cells(f, (cx_box, cy_box), (w, h), step, sym)
    return _normalized_or_centroid(pts, probe.cx, probe.cy)


# ---------------------------------------------------------------------------
# Kernel construction (aerial.rs:984-1317)
# ---------------------------------------------------------------------------
def select_kernel_count(values: Sequence[float], trace: float, max_kernels: int, fraction: float) -> int:
    """aerial.rs:992-1029."""
    if len(values) == 0:
        return 0
    lead = values[0]
    if math.isnan(lead) or lead <= 0.0:
        return 0
    tol = EIGEN_ZERO_REL * lead
    n_valid = 0
    for v in values:
        if v > tol:
            n_valid += 1
        else:
            break
    cap = min(max_kernels, n_valid)
    k = cap
    if fraction < 1.0:
        acc = 0.0
        for i in range(cap):
            acc += values[i]
            if acc >= fraction * trace:
                k = i + 1
                break

    def same(a, b):
        return abs(a - b) <= DEGENERACY_REL * max(abs(a), abs(b))

    if 0 < k < n_valid and same(values[k - 1], values[k]):
        end = k
        while end < n_valid and same(values[end - 1], values[end]):
            end += 1
        if end <= max_kernels:
            k = end
        else:
            while k > 0 and same(values[k - 1], values[k]):
                k -= 1
            if k == 0:
                k = end
    return k


@dataclass
class KernelSet:
    """SparseKernelSet (aerial.rs:955-973): kernels on the support only."""
    n: int
    support: np.ndarray          # flat indices i*n + j
    eigenvalues: np.ndarray      # raw (absolute), decreasing
    values: np.ndarray           # (K, S) complex128
    trace: float
    clear_field: float
    pupil_peak: float
    method: str
    num_columns: int
    support_exceeds_nyquist: bool

    @property
    def captured_energy_fraction(self) -> float:
        return float(np.sum(self.eigenvalues) / self.trace)

    def divisor(self, normalization: str = "clear_field") -> Optional[float]:
        """normalization_divisor (aerial.rs:1727-1733)."""
        bright = self.clear_field > 0.0 and self.clear_field >= DARK_FIELD_FRACTION * self.pupil_peak
        if normalization == "clear_field" and bright:
            return self.clear_field
        return None

    def dense(self) -> np.ndarray:
        """kernels(z) materialisation (aerial.rs:1912-1942): (K, n, n)."""
        k = self.values.shape[0]
        out = np.zeros((k, self.n * self.n), dtype=np.complex128)
        out[:, self.support] = self.values
        return out.reshape(k, self.n, self.n)


def build_kernels(points, optics, grid: Grid, lam: float, max_kernels: int,
                  fraction: float = 1.0, defocus_nm: float = 0.0,
                  method: Optional[str] = None) -> KernelSet:
    """KernelBuilder::build (aerial.rs:1041-1317), dense eigensolvers only.

    The reference switches to a randomized solver for large problems
    (aerial.rs:1116-1128); the oracle always solves densely (exact), which
    bounds the reference's randomized result to within its own tested
    1e-5 image tolerance (aerial.rs:2648-2675)."""
    n = grid.size
    df = grid.freq_step
    cutoff = optics.cutoff(lam)
    sigma_max = 0.0
    for sx, sy, _ in points:
        sigma_max = max(sigma_max, math.hypot(sx, sy))
    radius = cutoff * (1.0 + sigma_max)
    r2 = (radius / df) ** 2 * (1.0 + 1e-12)
    exceeds = radius > (n // 2) * df
    cand = []
    for i in range(n):
        ky = float(signed_index(i, n))
        if ky * ky > r2:
            continue
        for j in range(n):
            kx = float(signed_index(j, n))
            if kx * kx + ky * ky <= r2:
                cand.append((i * n + j, kx * df / cutoff, ky * df / cutoff))
    n_cand, n_pts = len(cand), len(points)
    if n_cand == 0 or n_pts == 0:
        raise ValueError("no diffraction orders")
    if n_cand * n_pts * 16 > MAX_FACTOR_BYTES:
        raise ValueError("pupil sampling too dense")
    amp = np.sqrt(np.array([w for _, _, w in points]))
    fxn = np.array([c[1] for c in cand])[:, None]
    fyn = np.array([c[2] for c in cand])[:, None]
    sxs = np.array([p[0] for p in points])[None, :]
    sys_ = np.array([p[1] for p in points])[None, :]
    a = optics.pupil_grid(fxn + sxs, fyn + sys_, defocus_nm, lam) * amp[None, :]
    clear_field = float(np.sum(np.abs(a[0]) ** 2))
    pupil_peak = float(np.max(np.abs(a) ** 2 / np.array([w for _, _, w in points])[None, :]))
    col_nz = np.any(a != 0, axis=0)
    if method is None:
        method = "dense_tcc" if n_cand <= n_pts else "dense_gram"
    if method == "dense_tcc":
        row_nz = np.any(a[:, col_nz] != 0, axis=1)
        x = a[row_nz][:, col_nz]
        support = np.array([c[0] for c, keep in zip(cand, row_nz) if keep], dtype=np.int64)
        trace = float(np.sum(np.abs(x) ** 2))
        tcc = x @ x.conj().T
        vals, vecs = np.linalg.eigh(tcc)
        order = np.argsort(-vals, kind="stable")
        vals, vecs = vals[order], vecs[:, order]
        k = select_kernel_count(list(vals), trace, max_kernels, fraction)
        values = vecs[:, :k].T.copy()
        eig = vals[:k].copy()
        n_eff = int(np.sum(col_nz))
    else:
        a_eff = a[:, col_nz]
        support = np.array([c[0] for c in cand], dtype=np.int64)
        trace = float(np.sum(np.abs(a_eff) ** 2))
        gram = a_eff.conj().T @ a_eff
        vals, vecs = np.linalg.eigh(gram)
        order = np.argsort(-vals, kind="stable")
        vals, vecs = vals[order], vecs[:, order]
        k = select_kernel_count(list(vals), trace, max_kernels, fraction)
        u = a_eff @ (vecs[:, :k] / np.sqrt(vals[:k])[None, :])
        values = u.T.copy()
        eig = vals[:k].copy()
        n_eff = a_eff.shape[1]
    if k == 0 or not (trace > 0.0):
        raise ValueError("no diffraction orders")
    return KernelSet(n, support, eig, values, trace, clear_field, pupil_peak, method, n_eff, exceeds)


# ---------------------------------------------------------------------------
# Mask spectrum (mask.rs:28-36, 616-657, 783-815, 910-972, 1439-1503)
# ---------------------------------------------------------------------------
def sinc(u):
    u = np.asarray(u, dtype=np.float64)
    small = np.abs(u) < 1e-6
    safe = np.where(small, 1.0, u)
    return np.where(small, 1.0 - u * u / 6.0, np.sin(safe) / safe)


def pixel_transfer(n: int) -> np.ndarray:
    """sinc(pi m / N) per FFT index (mask.rs:804-815)."""
    return sinc(np.pi * signed_orders(n) / n)


def spectrum_from_raster(t: np.ndarray, pixel_transfer_on: bool = True) -> np.ndarray:
    """Raster path of Mask::spectrum: FFT(t) x sinc x sinc (mask.rs:630-635);
    without the transfer it is compute_from_transmittance's FFT (aerial.rs:1789-1798)."""
    s = np.fft.fft2(np.asarray(t, dtype=np.complex128))
    if pixel_transfer_on:
        tr = pixel_transfer(t.shape[0])
        s = s * tr[:, None] * tr[None, :]
    return s


def axis_coefficients_finite(intervals, grid: Grid) -> np.ndarray:
    """N X(m) exp(-i pi m (N-1)/N) of a union of intervals (mask.rs:1462-1475)."""
    n = grid.size
    nf = float(n)
    L = 2.0 * (grid.field_nm / 2.0)
    m = signed_orders(n).astype(np.float64)
    acc = np.zeros(n, dtype=np.complex128)
    for a, b in intervals:
        w = b - a
        amp = w / L * sinc(np.pi * m * w / L)
        acc += amp * np.exp(-1j * np.pi * m * (a + b) / L)
    return acc * (nf * np.exp(-1j * np.pi * m * (nf - 1.0) / nf))


def axis_coefficients_full(grid: Grid) -> np.ndarray:
    out = np.zeros(grid.size, dtype=np.complex128)
    out[0] = grid.size
    return out


def axis_coefficients_grating(width, pitch, offset, periods, grid: Grid) -> np.ndarray:
    """Commensurate grating (mask.rs:1447-1461)."""
    n = grid.size
    nf = float(n)
    out = np.zeros(n, dtype=np.complex128)
    for k in range(n):
        m = signed_index(k, n)
        if m % periods != 0:
            continue
        q = m // periods
        amp = width / pitch * float(sinc(np.pi * q * width / pitch))
        phase = -2.0 * np.pi * q * offset / pitch - np.pi * m * (nf - 1.0) / nf
        out[k] = nf * amp * np.exp(1j * phase)
    return out


def _interval_axis(a: float, b: float, grid: Grid):
    half = grid.field_nm / 2.0
    lo, hi = max(a, -half), min(b, half)
    if hi - lo <= 0.0:
        return None
    eps = 1e-9 * grid.field_nm
    if lo <= -half + eps and hi >= half - eps:
        return ("full",)
    return ("finite", [(lo, hi)])


def _grating_axis(width, pitch, offset, grid: Grid):
    """mask.rs:910-972. Returns (axis, fraction)."""
    if width >= pitch:
        return ("full",), 1.0
    L = grid.field_nm
    half = L / 2.0
    periods = L / pitch
    m = rust_round(periods)
    commensurate = m >= 1.0 and abs(periods - m) <= 1e-9 * periods
    k_lo = math.floor((-half - offset - width / 2.0) / pitch)
    k_hi = math.ceil((half - offset + width / 2.0) / pitch)
    intervals = []
    for k in range(k_lo, k_hi + 1):
        c = offset + k * pitch
        lo = max(c - width / 2.0, -half)
        hi = min(c + width / 2.0, half)
        if hi > lo:
            intervals.append((lo, hi))
    if commensurate:
        return ("grating", width, pitch, offset, int(m)), 1.0
    return ("finite", intervals), 1.0


def _axis_coeffs(axis, grid: Grid) -> np.ndarray:
    if axis[0] == "full":
        return axis_coefficients_full(grid)
    if axis[0] == "grating":
        return axis_coefficients_grating(axis[1], axis[2], axis[3], axis[4], grid)
    return axis_coefficients_finite(axis[1], grid)


@dataclass
class Mask:
    """Subset of mask.rs: rectangles, line/space gratings and rect arrays on a
    binary or attenuated-PSM mask. ``spectrum`` evaluates non-overlapping
    separable features in closed form (mask.rs:636-644, 1479-1503)."""
    features: list = field(default_factory=list)   # ("rect", x, y, w, h) | ("ls", cd, pitch, orient, offset) | ("array", w, h, px, py, ox, oy)
    dark_field: bool = False
    absorber: complex = 0j

    @staticmethod
    def line_space(cd, pitch, orientation="vertical", offset=0.0) -> "Mask":
        return Mask([("ls", cd, pitch, orientation, offset)], dark_field=False)

    @property
    def bg(self) -> complex:
        return self.absorber if self.dark_field else 1.0 + 0j

    @property
    def fg(self) -> complex:
        return 1.0 + 0j if self.dark_field else self.absorber

    def _terms(self, grid: Grid):
        bg, fg = self.bg, self.fg
        terms = []
        for feat in self.features:
            kind = feat[0]
            if kind == "rect":
                _, x, y, w, h = feat
                ax = _interval_axis(x - w / 2.0, x + w / 2.0, grid)
                ay = _interval_axis(y - h / 2.0, y + h / 2.0, grid)
                if ax is None or ay is None:
                    continue
                terms.append((fg, ax, ay))
            elif kind == "ls":
                _, cd, pitch, orient, offset = feat
                g, frac = _grating_axis(cd, pitch, offset, grid)
                value = bg + (fg - bg) * frac
                if orient == "vertical":
                    terms.append((value, g, ("full",)))
                else:
                    terms.append((value, ("full",), g))
            elif kind == "array":
                _, w, h, px, py, ox, oy = feat
                gx, fx = _grating_axis(w, px, ox, grid)
                gy, fy = _grating_axis(h, py, oy, grid)
                terms.append((bg + (fg - bg) * (fx * fy), gx, gy))
            else:
                raise ValueError(kind)
        return terms

    def spectrum(self, grid: Grid) -> np.ndarray:
        n = grid.size
        spec = np.zeros((n, n), dtype=np.complex128)
        spec[0, 0] = self.bg * (n * n)
        for value, ax, ay in self._terms(grid):
            w = value - self.bg
            if w == 0:
                continue
            xc = w * _axis_coeffs(ax, grid)
            yc = _axis_coeffs(ay, grid)
            spec += yc[:, None] * xc[None, :]
        return spec

    def rasterize(self, grid: Grid) -> np.ndarray:
        """Area-averaged raster of non-overlapping separable features
        (mask.rs:1505-1571)."""
        n = grid.size
        out = np.full((n, n), self.bg, dtype=np.complex128)
        for value, ax, ay in self._terms(grid):
            w = value - self.bg
            cx = _axis_coverage(ax, grid)
            cy = _axis_coverage(ay, grid)
            out += w * cy[:, None] * cx[None, :]
        return out


def rects_union_spectrum(rects, grid: Grid, feature: complex = 1.0, background: complex = 0.0) -> np.ndarray:
    """Exact FFT-layout spectrum of the union of rectangles (x, y, w, h; centre
    and size in nm, field-centred), amplitude ``feature`` on ``background``.
    Overlaps are resolved into disjoint cells by coordinate compression (the
    reference's compress, mask.rs:1365-1437); each covered cell contributes
    its separable closed form (axis_coefficients_finite, mask.rs:1462-1475)."""
    n = grid.size
    half = grid.field_nm / 2.0
    boxes = []
    for x, y, w, h in rects:
        x0, x1 = max(x - w / 2.0, -half), min(x + w / 2.0, half)
        y0, y1 = max(y - h / 2.0, -half), min(y + h / 2.0, half)
        if x1 > x0 and y1 > y0:
            boxes.append((x0, x1, y0, y1))
    spec = np.zeros((n, n), dtype=np.complex128)
    spec[0, 0] = complex(background) * n * n
    if not boxes:
        return spec
    xe = np.unique([b[0] for b in boxes] + [b[1] for b in boxes])
    ye = np.unique([b[2] for b in boxes] + [b[3] for b in boxes])
    cover = np.zeros((len(ye) - 1, len(xe) - 1), dtype=bool)
    for x0, x1, y0, y1 in boxes:
        e0, e1 = np.searchsorted(xe, x0), np.searchsorted(xe, x1)
        f0, f1 = np.searchsorted(ye, y0), np.searchsorted(ye, y1)
        cover[f0:f1, e0:e1] = True
    cx = np.array([axis_coefficients_finite([(xe[e], xe[e + 1])], grid) for e in range(len(xe) - 1)])
    cy = np.array([axis_coefficients_finite([(ye[f], ye[f + 1])], grid) for f in range(len(ye) - 1)])
    rows = cover.astype(np.float64) @ cx  # (F-1, N): per y cell, sum of covered x cells
    spec += (complex(feature) - complex(background)) * (cy.T @ rows)
    return spec


def _axis_coverage(axis, grid: Grid) -> np.ndarray:
    n, p = grid.size, grid.pixel_nm
    half = grid.field_nm / 2.0
    if axis[0] == "full":
        return np.ones(n)
    if axis[0] == "grating":
        _, width, pitch, offset, _ = axis
        k_lo = math.floor((-half - offset - width / 2.0) / pitch)
        k_hi = math.ceil((half - offset + width / 2.0) / pitch)
        intervals = []
        for k in range(k_lo, k_hi + 1):
            c = offset + k * pitch
            lo, hi = max(c - width / 2.0, -half), min(c + width / 2.0, half)
            if hi > lo:
                intervals.append((lo, hi))
    else:
        intervals = axis[1]
    cov = np.zeros(n)
    edges = -half + np.arange(n + 1) * p
    for a, b in intervals:
        o = np.minimum(b, edges[1:]) - np.maximum(a, edges[:-1])
        cov += np.clip(o, 0.0, None) / p
    return cov


# ---------------------------------------------------------------------------
# SOCS sum, normalisation, flare (aerial.rs:1682-1748)
# ---------------------------------------------------------------------------
def socs_intensity(ks: KernelSet, spectrum: np.ndarray) -> np.ndarray:
    """Sum_k lambda_k |IFFT(u_k . M)|^2, raw eigenvalues (aerial.rs:1682-1721)."""
    n = ks.n
    m_s = spectrum.reshape(-1)[ks.support]
    acc = np.zeros((n, n))
    buf = np.zeros(n * n, dtype=np.complex128)
    for k in range(ks.values.shape[0]):
        buf[:] = 0
        buf[ks.support] = ks.values[k] * m_s
        e = np.fft.ifft2(buf.reshape(n, n))
        acc += ks.eigenvalues[k] * (e.real ** 2 + e.imag ** 2)
    return acc


def apply_flare(image: np.ndarray, phi: float) -> np.ndarray:
    """aerial.rs:1741-1748 / opc.rs:464-471."""
    if phi > 0.0 and image.size:
        mean = float(np.sum(image)) / image.size
        return image * (1.0 - phi) + phi * mean
    return image


def image_from_spectrum(ks: KernelSet, spectrum: np.ndarray, flare: float,
                        normalization: str = "clear_field") -> np.ndarray:
    """compute_from_spectrum (aerial.rs:1805-1816)."""
    img = socs_intensity(ks, spectrum)
    d = ks.divisor(normalization)
    if d is not None:
        img = img / d
    return apply_flare(img, flare)


def abbe_image(points, optics, grid: Grid, spectrum: np.ndarray, z: float, lam: float) -> np.ndarray:
    """Independent direct Abbe sum over all grid frequencies
    (imaging_validation.rs:171-198). Absolute intensity, no flare."""
    n = grid.size
    df = grid.freq_step
    fc = optics.cutoff(lam)
    so = signed_orders(n).astype(np.float64)
    total = np.zeros((n, n))
    for sx, sy, w in points:
        fx = so[None, :] * df / fc + sx
        fy = so[:, None] * df / fc + sy
        pup = np.zeros((n, n), dtype=np.complex128)
        for i in range(n):
            for j in range(n):
                pup[i, j] = optics.pupil(fx[0, j], fy[i, 0], z, lam)
        e = np.fft.ifft2(pup * spectrum)
        total += w * np.abs(e) ** 2
    return total


# ---------------------------------------------------------------------------
# Engine facade (aerial.rs:1495-1816): source sampling + in-focus kernels
# ---------------------------------------------------------------------------
@dataclass
class Engine:
    fill: Callable[[float, float], float]
    optics: object
    grid: Grid
    wavelength_nm: float
    max_kernels: int = 48
    fraction: float = 1.0
    points_per_axis: Optional[int] = None
    normalization: str = "clear_field"
    points: list = field(default_factory=list)
    _sets: dict = field(default_factory=dict)

    def __post_init__(self):
        cutoff = self.optics.cutoff(self.wavelength_nm)
        df_sigma = self.grid.freq_step / cutoff
        self.points = sample_source(self.fill, self.points_per_axis, df_sigma)

    def kernel_set(self, z: float = 0.0) -> KernelSet:
        key = 0.0 if z == 0.0 else z
        if key not in self._sets:
            self._sets[key] = build_kernels(self.points, self.optics, self.grid, self.wavelength_nm,
                                            self.max_kernels, self.fraction, key)
        return self._sets[key]

    def compute_from_spectrum(self, spectrum: np.ndarray, z: float = 0.0) -> np.ndarray:
        return image_from_spectrum(self.kernel_set(z), spectrum, self.optics.flare, self.normalization)

    def compute(self, mask: Mask, z: float = 0.0) -> np.ndarray:
        return self.compute_from_spectrum(mask.spectrum(self.grid), z)

    def compute_from_transmittance(self, t: np.ndarray, z: float = 0.0) -> np.ndarray:
        return self.compute_from_spectrum(np.fft.fft2(np.asarray(t, dtype=np.complex128)), z)

    def clear_field_intensity(self, z: float = 0.0) -> float:
        return self.kernel_set(z).clear_field


def paint_rects(grid: Grid, rects, dark_field: bool = True, absorber: complex = 0j) -> np.ndarray:
    """Painter's-rule raster of rectangles (x, y, w, h in nm, centred field
    coordinates): later rectangles win overlaps (mask.rs:1-9). Exact area
    coverage per rectangle; for pixel-aligned edges (coverage 0 or 1) this is
    the reference's exact raster."""
    n, p = grid.size, grid.pixel_nm
    half = grid.field_nm / 2.0
    bg = absorber if dark_field else 1.0 + 0j
    fg = 1.0 + 0j if dark_field else absorber
    out = np.full((n, n), bg, dtype=np.complex128)
    edges = -half + np.arange(n + 1) * p
    for x, y, w, h in rects:
        cx = np.clip(np.minimum(x + w / 2, edges[1:]) - np.maximum(x - w / 2, edges[:-1]), 0, None) / p
        cy = np.clip(np.minimum(y + h / 2, edges[1:]) - np.maximum(y - h / 2, edges[:-1]), 0, None) / p
        cov = cy[:, None] * cx[None, :]
        out = out * (1.0 - cov) + fg * cov
    return out
