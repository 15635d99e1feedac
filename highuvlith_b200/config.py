"""TOML front end: the imaging sections of the reference CLI's configuration
(crates/highuvlith-cli/src/config.rs: [source], [illumination], [optics],
[mask], [grid], [process], [imaging]) mapped onto this engine.

Covered: vuv presets or an explicit wavelength with a conventional sigma or
an [illumination] shape; refractive (optionally immersion), EUV projection
and Schwarzschild optics; line/space, contact-hole and rectangle masks
(binary or attenuated PSM) imaged through their exact analytic spectrum;
the commensurate-grid pixel adjustment; monochromatic scalar imaging with
exact defocus.  Anything outside that raises ``ConfigError`` rather than
being approximated.
"""
from __future__ import annotations

import cmath
import math
import tomllib
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

from .api import (ARF_WAVELENGTH_NM, EUV_WAVELENGTH_NM, F2_WAVELENGTH_NM, GridConfig, OpticsConfig,
                  SimulationEngine, SourceConfig)


class ConfigError(ValueError):
    """A configuration this front end does not support or cannot parse."""


# vuv presets (source.rs:327-440)
VUV_PRESETS = {"f2": F2_WAVELENGTH_NM, "ar2": 126.0, "arf": ARF_WAVELENGTH_NM, "krf": 248.3,
               "hg_i": 365.0153, "i_line": 365.0153, "hg_h": 404.6563, "h_line": 404.6563, "hg_g": 435.8328,
               "g_line": 435.8328}


@dataclass
class Scene:
    """One simulate scene: engine inputs, the mask as rectangles, process."""
    source: SourceConfig
    optics: OpticsConfig
    grid: GridConfig
    rects: List[Tuple[float, float, float, float]]
    feature: complex
    background: complex
    tone: str                      # "dark" (opaque features) or "bright" (clear features)
    orientation: str               # measurement cutline: "vertical" lines -> along x
    focus_nm: float = 0.0
    dose: float = 30.0
    nominal_dose: float = 30.0
    threshold: float = 0.3
    imaging: dict = field(default_factory=dict)
    notes: List[str] = field(default_factory=list)

    def engine(self, device: int = 0, kernel_build: str = "host") -> SimulationEngine:
        im = self.imaging
        return SimulationEngine(self.source, self.optics, grid=self.grid, max_kernels=int(im.get("max_kernels", 20)),
                                kernel_energy_fraction=float(im.get("kernel_energy_fraction", 1.0)),
                                source_points_per_axis=im.get("source_points_per_axis"),
                                normalization=im.get("normalization", "clear_field"),
                                kernel_cache_capacity=int(im.get("kernel_cache_capacity", 32)), device=device,
                                kernel_build=kernel_build)


def _source(cfg: dict) -> SourceConfig:
    s = cfg.get("source", {})
    kind = s.get("type", "vuv")
    if kind not in ("vuv", "euv"):
        raise ConfigError(f"[source] type '{kind}' is outside the imaging front end (vuv, euv)")
    if kind == "euv":
        lam = float(s.get("wavelength_nm", EUV_WAVELENGTH_NM))
    elif "preset" in s:
        if s["preset"] not in VUV_PRESETS:
            raise ConfigError(f"unknown vuv preset '{s['preset']}'")
        lam = float(s.get("wavelength_nm", VUV_PRESETS[s["preset"]]))
    else:
        lam = float(s.get("wavelength_nm", F2_WAVELENGTH_NM))
    sigma = float(s.get("sigma", 0.7))
    ill = cfg.get("illumination", s.get("illumination"))
    if not ill:
        return SourceConfig(lam, "conventional", (sigma,))
    shape = ill.get("shape")
    if shape == "conventional":
        return SourceConfig(lam, "conventional", (float(ill.get("sigma", sigma)),))
    if shape == "annular":
        return SourceConfig(lam, "annular", (float(ill["sigma_inner"]), float(ill["sigma_outer"])))
    if shape == "dipole":
        return SourceConfig(lam, "dipole", (float(ill["sigma_center"]), float(ill["sigma_radius"]),
                                            float(ill.get("orientation_deg", 0.0))))
    if shape == "quadrupole":
        return SourceConfig(lam, "quadrupole", (float(ill["sigma_center"]), float(ill["sigma_radius"]),
                                                float(ill.get("opening_angle_deg", 30.0))))
    if shape == "coherent_gaussian":
        return SourceConfig(lam, "gaussian", (float(ill.get("sigma", sigma)),))
    raise ConfigError(f"unknown [illumination] shape '{shape}'")


def _optics(cfg: dict, lam: float) -> OpticsConfig:
    o = cfg.get("optics", {})
    kind = o.get("type", "refractive")
    preset = o.get("preset")
    if kind == "refractive":
        na, n_imm = 0.75, 1.0
        if preset == "immersion_193i":
            na, n_imm = 1.35, 1.437
        elif preset is not None:
            raise ConfigError(f"unknown refractive preset '{preset}'")
        return OpticsConfig(float(o.get("na", na)), float(o.get("flare_fraction", 0.02)),
                            float(o.get("immersion_index", n_imm)), "projection")
    if kind == "euv_projection":
        na, eps = {"nxe": (0.33, 0.0), "high_na": (0.55, 0.2), None: (0.33, 0.0)}[preset]
        return OpticsConfig(float(o.get("na", na)), float(o.get("flare_fraction", 0.0)), 1.0, "euv",
                            float(o.get("central_obscuration", eps)), 1.0)
    if kind == "schwarzschild":
        # SchwarzschildObjective::euv_standard (optics/schwarzschild.rs:62-72):
        # two Mo/Si mirrors of reflectivity 0.67 -> transmission 0.67^2
        if preset not in (None, "euv"):
            raise ConfigError(f"schwarzschild preset '{preset}' is outside the imaging front end")
        refl = float(o.get("mirror_reflectivity", 0.67))
        return OpticsConfig(float(o.get("na", 0.33)), float(o.get("flare_fraction", 0.03)), 1.0, "euv",
                            float(o.get("central_obscuration", 0.25)), refl * refl)
    raise ConfigError(f"[optics] type '{kind}' is outside the imaging front end")


def _mask(cfg: dict, field_nm: float):
    """(rects, feature amplitude, background amplitude, tone, orientation, cell)."""
    m = cfg.get("mask", {})
    pattern = m.get("pattern", "line_space" if "features" not in m else "features")
    mask_type = m.get("mask_type", "binary")
    if mask_type == "binary":
        absorber = 0.0
    elif mask_type == "att_psm":
        absorber = math.sqrt(float(m.get("transmission", 0.06))) * cmath.exp(
            1j * math.radians(float(m.get("phase_deg", 180.0))))
    else:
        raise ConfigError(f"unknown mask_type '{mask_type}'")
    half = field_nm / 2.0
    rects: List[Tuple[float, float, float, float]] = []

    def lines(cd, pitch, orient, offset):
        k0 = math.floor((-half - offset - cd) / pitch)
        k1 = math.ceil((half - offset + cd) / pitch)
        for k in range(k0, k1 + 1):
            c = offset + k * pitch
            rects.append((c, 0.0, cd, 2.0 * field_nm) if orient == "vertical" else (0.0, c, 2.0 * field_nm, cd))

    orientation = "vertical"
    if pattern == "line_space":
        cd, pitch = float(m.get("cd_nm", 65.0)), float(m.get("pitch_nm", 180.0))
        orientation = m.get("orientation", "vertical")
        lines(cd, pitch, orientation, float(m.get("offset_nm", 0.0)))
        dark_field = bool(m.get("dark_field", False))
        cell = pitch
    elif pattern == "contact_holes":
        d = float(m.get("diameter_nm", 60.0))
        px = float(m.get("pitch_nm", 180.0))
        py = float(m.get("pitch_y_nm", px))
        for i in range(math.floor(-half / px) - 1, math.ceil(half / px) + 2):
            for j in range(math.floor(-half / py) - 1, math.ceil(half / py) + 2):
                rects.append((i * px, j * py, d, d))
        dark_field = bool(m.get("dark_field", True))
        cell = px if abs(px - py) <= 1e-12 * px else None
    elif pattern == "features":
        for f in m.get("features", []):
            t = f.get("type")
            if t == "rect":
                rects.append((float(f["x"]), float(f["y"]), float(f["w"]), float(f["h"])))
            elif t == "line_space":
                lines(float(f["cd"]), float(f["pitch"]), f.get("orientation", "vertical"), float(f.get("offset", 0.0)))
            else:
                raise ConfigError(f"[[mask.features]] type '{t}' is outside the imaging front end")
        dark_field = bool(m.get("dark_field", False))
        cell = None
    else:
        raise ConfigError(f"unknown mask pattern '{pattern}'")
    # Bright field: clear background, features are absorber; dark field: the reverse.
    feature, background = (1.0 + 0j, complex(absorber)) if dark_field else (complex(absorber), 1.0 + 0j)
    tone = "bright" if dark_field else "dark"
    return rects, feature, background, tone, orientation, cell


def load(text_or_path: str, is_text: bool = False) -> Scene:
    """Parse a simulate configuration (TOML text or a path)."""
    if is_text:
        cfg = tomllib.loads(text_or_path)
    else:
        with open(text_or_path, "rb") as f:
            cfg = tomllib.load(f)
    im = dict(cfg.get("imaging", {}))
    if im.get("defocus_model", "exact") != "exact":
        raise ConfigError("[imaging] defocus_model: only 'exact' is on the device path")
    if im.get("spectrum", "monochromatic") != "monochromatic":
        raise ConfigError("[imaging] spectrum: only 'monochromatic' is on the device path")
    if "vector" in im:
        raise ConfigError("[imaging.vector]: vector imaging is outside the device path")
    src = _source(cfg)
    opt = _optics(cfg, src.wavelength_nm)
    g = cfg.get("grid", {})
    size, pixel = int(g.get("size", 256)), float(g.get("pixel_nm", 1.0))
    notes = []
    field_nm = size * pixel
    _, _, _, _, _, cell = _mask(cfg, field_nm)
    if g.get("commensurate", True) and cell:
        periods = max(1, round(field_nm / cell))
        new_pixel = periods * cell / size
        if abs(new_pixel - pixel) > 1e-12 * pixel:
            notes.append(f"pixel {pixel} nm -> {new_pixel:.6f} nm so the {periods * cell:.3f} nm field holds "
                         f"{periods} whole period(s) of the {cell} nm mask cell")
            pixel = new_pixel
            field_nm = size * pixel
    rects, feature, background, tone, orientation, _ = _mask(cfg, field_nm)
    p = cfg.get("process", {})
    nominal = float(p.get("dose_mj_cm2", 30.0))
    return Scene(src, opt, GridConfig(size, pixel), rects, feature, background, tone, orientation,
                 float(p.get("focus_nm", 0.0)), nominal, nominal, float(p.get("threshold", 0.3)), im, notes)


def simulate(scene: Scene, focus_nm: Optional[float] = None, dose: Optional[float] = None, device: int = 0,
             kernel_build: str = "host") -> dict:
    """The reference CLI's simulate pipeline (commands/simulate.rs) on the
    device: image, contrast, printed CD and NILS at the dose-scaled
    constant threshold I = threshold * nominal / dose."""
    import numpy as np
    from . import metrics
    z = scene.focus_nm if focus_nm is None else float(focus_nm)
    d = scene.dose if dose is None else float(dose)
    if not (math.isfinite(d) and d > 0.0):
        raise ConfigError("dose must be finite and > 0")
    thr = scene.threshold * scene.nominal_dose / d
    eng = scene.engine(device, kernel_build)
    img = eng.compute_batch_rects_host([scene.rects], feature=scene.feature, background=scene.background,
                                       focus_nm=z)[0].astype(np.float64)
    x = metrics.pixel_centres(scene.grid.size, scene.grid.field_nm)
    prof = metrics.centre_profile(img if scene.orientation == "vertical" else img.T)
    return {"image": img, "contrast": metrics.image_contrast(img), "threshold": thr,
            "printed_cd_nm": metrics.printed_cd(prof, x, thr, scene.tone),
            "nils": metrics.nils(prof, x, thr, scene.tone), "focus_nm": z, "dose_mj_cm2": d,
            "pixel_nm": scene.grid.pixel_nm, "notes": scene.notes, "max_intensity": float(img.max()),
            "min_intensity": float(img.min())}
