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


def coverage_raster(scene: Scene) -> "np.ndarray":
    """The drawn mask's clear area as an N x N raster of exact area coverage
    (the reference's ILT target, Mask::rasterize_intensity of the binary
    mask, mask.rs:600-603): per pixel, the fraction covered by the clear
    parts (the features on a dark field, the background on a bright one).
    Features must not overlap (ConfigError otherwise)."""
    import numpy as np
    n, p = scene.grid.size, scene.grid.pixel_nm
    half = n * p / 2.0
    edges = -half + np.arange(n + 1) * p
    boxes = [(x - w / 2.0, x + w / 2.0, y - h / 2.0, y + h / 2.0) for x, y, w, h in scene.rects]
    for i, a in enumerate(boxes):
        for b in boxes[i + 1:]:
            if min(a[1], b[1]) > max(a[0], b[0]) and min(a[3], b[3]) > max(a[2], b[2]):
                raise ConfigError("ILT target: overlapping [mask] features are not supported")
    cov = np.zeros((n, n))
    for x0, x1, y0, y1 in boxes:
        cx = np.clip(np.minimum(x1, edges[1:]) - np.maximum(x0, edges[:-1]), 0.0, None) / p
        cy = np.clip(np.minimum(y1, edges[1:]) - np.maximum(y0, edges[:-1]), 0.0, None) / p
        cov += cy[:, None] * cx[None, :]
    cov = np.clip(cov, 0.0, 1.0)
    return cov if scene.tone == "bright" else 1.0 - cov


# [optimize] keys of method = "ilt" this front end maps onto the device
# optimizer (optimize.rs:579-700); the rest raise ConfigError.
_ILT_KEYS = {"method", "cost", "threshold", "steepness", "max_iterations", "learning_rate", "tv_weight",
             "convergence_tol", "sigmoid_steepness", "binarization_weight", "init", "init_level", "gradient",
             "optimizer"}


def optimize_ilt(cfg_text_or_path: str, is_text: bool = False, device: int = 0, kernel_build: str = "host") -> dict:
    """The reference CLI's ``optimize`` with ``method = "ilt"``
    (optimize.rs:579-700) on the device: target = the drawn mask's clear
    area, theta_0 = Z - 1/2 (or the uniform logit), CG Polak-Ribiere+ with
    Armijo backtracking (huv_ilt_optimize); misprinted-pixel counts of the
    drawn, optimized and binarised masks at the print threshold
    (ilt.rs:267-275, 920-931)."""
    import numpy as np
    import torch
    from . import ilt
    if is_text:
        cfg = tomllib.loads(cfg_text_or_path)
    else:
        with open(cfg_text_or_path, "rb") as f:
            cfg = tomllib.load(f)
    scene = load(cfg_text_or_path, is_text)
    o = dict(cfg.get("optimize", {}))
    if o.get("method") != "ilt":
        raise ConfigError(f"[optimize] method '{o.get('method')}': only 'ilt' is on the device path")
    extra = sorted(set(o) - _ILT_KEYS)
    if extra:
        raise ConfigError(f"[optimize] keys outside the device ILT: {', '.join(extra)}")
    if o.get("gradient", "adjoint") != "adjoint" or o.get("optimizer", "cg") != "cg":
        raise ConfigError("[optimize]: the device ILT runs the exact adjoint with conjugate gradient")
    cost = o.get("cost", "image")
    if cost not in ("image", "resist"):
        raise ConfigError(f"[optimize] cost must be 'image' or 'resist', got '{cost}'")
    threshold = float(o.get("threshold", scene.threshold))
    if not (math.isfinite(threshold) and threshold > 0.0):
        raise ConfigError("[optimize] threshold must be finite and > 0")
    print_t = threshold if cost == "resist" else 0.5
    if scene.feature != 1.0 + 0j and scene.background != 1.0 + 0j:
        raise ConfigError("ILT needs a binary or att_psm mask")
    absorber = scene.background if scene.tone == "bright" else scene.feature
    if absorber.imag != 0.0 or not (0.0 <= absorber.real < 1.0):
        raise ConfigError("the device ILT takes a real absorber amplitude in [0, 1)")
    st = ilt.IltSettings(cost=cost, threshold=threshold, steepness=float(o.get("steepness", 50.0)),
                         sigmoid_steepness=float(o.get("sigmoid_steepness", 4.0)),
                         regularization=float(o.get("tv_weight", 0.01)),
                         binarization_weight=float(o.get("binarization_weight", 0.0)), absorber=absorber.real,
                         defocus_nm=scene.focus_nm, max_iterations=int(o.get("max_iterations", 50)),
                         learning_rate=float(o.get("learning_rate", 0.5)),
                         convergence_tol=float(o.get("convergence_tol", 1e-4)))
    target = coverage_raster(scene)
    init = o.get("init", "target")
    if init == "target":
        theta0 = target - 0.5
    elif init == "uniform":
        m0 = min(max(float(o.get("init_level", 0.5)), 0.01), 0.99)
        theta0 = np.full_like(target, math.log(m0 / (1.0 - m0)) / st.sigmoid_steepness)
    else:
        raise ConfigError(f"[optimize] init must be 'target' or 'uniform', got '{init}'")
    eng = scene.engine(device, kernel_build)
    dev = torch.device("cuda", device)
    theta = torch.from_numpy(theta0.astype(np.float32)[None]).to(dev)
    tgt = torch.from_numpy(target.astype(np.float32)[None]).to(dev)
    res = ilt.optimize(eng, theta, tgt, st)
    m = 1.0 / (1.0 + np.exp(-st.sigmoid_steepness * theta.cpu().numpy()[0].astype(np.float64)))
    a = st.absorber

    def image(mask):
        t = torch.from_numpy((a + (1.0 - a) * mask).astype(np.float32)[None]).to(dev)
        return eng.compute_batch(t, focus_nm=scene.focus_nm, pixel_transfer=False).cpu().numpy()[0]

    def misprinted(mask):
        return int(np.sum((image(mask) > print_t) != (target > 0.5)))

    hist = res["cost_history"][0]
    hist = [float(c) for c in hist[:int(res["iterations"][0]) + 1]]
    iters = int(res["iterations"][0])
    return {"method": "ilt", "gradient": "adjoint", "optimizer": "cg", "cost": cost, "print_threshold": print_t,
            "iterations": iters,
            "termination": "max_iterations" if iters >= st.max_iterations else "stopped",
            "initial_cost": hist[0], "final_cost": float(res["final_cost"][0]), "cost_history": hist,
            "drawn_pattern_error": misprinted(target), "pattern_error": misprinted(m),
            "binary_pattern_error": misprinted((m > 0.5).astype(np.float64)),
            "grid": {"size": scene.grid.size, "pixel_nm": scene.grid.pixel_nm}, "mask_transmittance": m,
            "notes": scene.notes}


def parse_range(spec: str) -> List[float]:
    """``start,stop,steps`` -> steps evenly spaced values, inclusive
    (commands/sweep.rs:15-40)."""
    parts = spec.split(",")
    if len(parts) != 3:
        raise ConfigError("range must be 'start,stop,steps' (e.g. '-200,200,21')")
    start, stop, steps = float(parts[0]), float(parts[1]), int(parts[2])
    if not (math.isfinite(start) and math.isfinite(stop)):
        raise ConfigError("range start and stop must be finite")
    if steps > 1 and start > stop:
        raise ConfigError(f"invalid range: start ({start}) > stop ({stop})")
    if steps < 2:
        return [start]
    return [start + i * (stop - start) / (steps - 1) for i in range(steps)]


def sweep(scene: Scene, focuses: List[float], doses: Optional[List[float]] = None, device: int = 0,
          kernel_build: str = "host") -> dict:
    """The reference CLI's ``sweep`` grid (commands/sweep.rs:63-200) on the
    device: one aerial image per focus (exact rectangle spectrum, kernels
    built and cached per plane), and for every (dose, focus) the printed CD
    of the measurement cutline at the constant-threshold resist's intensity
    threshold t * nominal / dose, with the image contrast per focus.  The
    process-window summary (best focus, DOF, exposure latitude) belongs to
    the reference's process module and is not computed here."""
    import numpy as np
    from . import metrics
    doses = list(doses) if doses else [scene.nominal_dose]
    for d in doses:
        if not (math.isfinite(d) and d > 0.0):
            raise ConfigError("doses must be finite and > 0")
    eng = scene.engine(device, kernel_build)
    x = metrics.pixel_centres(scene.grid.size, scene.grid.field_nm)
    contrast, profiles = [], []
    for z in focuses:
        img = eng.compute_batch_rects_host([scene.rects], feature=scene.feature, background=scene.background,
                                           focus_nm=float(z))[0].astype(np.float64)
        contrast.append(metrics.image_contrast(img))
        profiles.append(metrics.centre_profile(img if scene.orientation == "vertical" else img.T))
    results = []
    for d in doses:
        t = scene.threshold * scene.nominal_dose / d
        for z, c, prof in zip(focuses, contrast, profiles):
            cd = metrics.printed_cd(prof, x, t, scene.tone)
            results.append({"dose_mj_cm2": d, "focus_nm": float(z), "intensity_threshold": t, "contrast": c,
                            "cd_nm": cd})
    return {"config": {"wavelength_nm": scene.source.wavelength_nm, "na": scene.optics.numerical_aperture,
                       "grid_size": scene.grid.size, "pixel_nm": scene.grid.pixel_nm, "tone": scene.tone},
            "focuses": [float(z) for z in focuses], "doses": doses, "results": results, "notes": scene.notes}
