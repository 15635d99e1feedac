"""Python face of the engine, mirroring the reference's imaging call.

``SimulationEngine`` follows the reference's PyO3 class of the same name
(crates/highuvlith-py/src/py_simulation.rs:89-566): it is built once from a
source, optics and grid (FP64 source sampling + SOCS kernels on the host),
then images many masks.  Images come back as FP32 on the engine grid, indexed
``[y, x]`` with pixel centres ``x_j = -L/2 + (j + 1/2) p``.  Device memory and
streams are torch tensors; all arithmetic runs in the library's own CUDA
kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L

ARF_WAVELENGTH_NM = 193.368
F2_WAVELENGTH_NM = 157.63
EUV_WAVELENGTH_NM = 13.5
WATER_INDEX_193NM = 1.437


@dataclass(frozen=True)
class SourceConfig:
    """Wavelength + pupil fill (source.rs:57-186).  ``fill`` is one of
    conventional, annular, quadrupole, dipole, gaussian, quasar."""
    wavelength_nm: float
    fill: str = "conventional"
    params: Tuple[float, ...] = (0.7,)

    @staticmethod
    def arf_laser(sigma: float = 0.7) -> "SourceConfig":
        return SourceConfig(ARF_WAVELENGTH_NM, "conventional", (sigma,))

    @staticmethod
    def f2_laser(sigma: float = 0.7) -> "SourceConfig":
        return SourceConfig(F2_WAVELENGTH_NM, "conventional", (sigma,))

    @staticmethod
    def euv(sigma: float = 0.5) -> "SourceConfig":
        return SourceConfig(EUV_WAVELENGTH_NM, "conventional", (sigma,))

    def with_illumination(self, fill: str, *params: float) -> "SourceConfig":
        if fill not in L.FILL:
            raise ValueError(f"unknown illumination {fill!r}")
        return replace(self, fill=fill, params=tuple(float(p) for p in params))

    def _c(self) -> L.Source:
        s = L.Source()
        s.wavelength_nm = self.wavelength_nm
        s.fill = L.FILL[self.fill]
        for i, p in enumerate(self.params[:4]):
            s.p[i] = p
        return s


@dataclass(frozen=True)
class OpticsConfig:
    """ProjectionOptics (optics/mod.rs:193-357) or EuvProjectionOptics
    (optics/euv.rs:51-160), scalar pupil, no aberrations."""
    numerical_aperture: float
    flare_fraction: float = 0.02
    immersion_index: float = 1.0
    kind: str = "projection"
    central_obscuration: float = 0.0
    transmission: float = 1.0
    paraxial_defocus: bool = False

    @staticmethod
    def immersion(na: float, index: float = WATER_INDEX_193NM) -> "OpticsConfig":
        return OpticsConfig(na, 0.02, index)

    @staticmethod
    def euv(na: float, central_obscuration: float = 0.0) -> "OpticsConfig":
        return OpticsConfig(na, 0.0, 1.0, "euv", central_obscuration)

    @staticmethod
    def euv_nxe_033() -> "OpticsConfig":
        return OpticsConfig.euv(0.33, 0.0)

    @staticmethod
    def euv_high_na_055() -> "OpticsConfig":
        return OpticsConfig.euv(0.55, 0.2)

    def _c(self) -> L.Optics:
        o = L.Optics()
        o.kind = L.OPTICS_EUV if self.kind == "euv" else L.OPTICS_PROJECTION
        o.na = self.numerical_aperture
        o.flare_fraction = self.flare_fraction
        o.immersion_index = self.immersion_index
        o.central_obscuration = self.central_obscuration
        o.transmission = self.transmission
        o.paraxial_defocus = int(self.paraxial_defocus)
        return o


@dataclass(frozen=True)
class GridConfig:
    size: int = 256
    pixel_nm: float = 1.0

    @property
    def field_nm(self) -> float:
        return self.size * self.pixel_nm

    def pixel_centres(self) -> np.ndarray:
        return -self.field_nm / 2 + (np.arange(self.size) + 0.5) * self.pixel_nm


@dataclass
class MaskConfig:
    """A binary Manhattan mask: pixel-aligned rectangles (x0, y0, w, h) in
    pixels from the field corner, clear on a dark field (``dark_field=True``)
    or opaque on a clear field."""
    rects: list = field(default_factory=list)
    dark_field: bool = True

    def rasterize(self, grid: GridConfig) -> np.ndarray:
        n = grid.size
        bg, fg = (0, 1) if self.dark_field else (1, 0)
        out = np.full((n, n), bg, dtype=np.uint8)
        for x0, y0, w, h in self.rects:
            out[max(y0, 0):min(y0 + h, n), max(x0, 0):min(x0 + w, n)] = fg
        return out


class AerialImageResult:
    """One aerial image and its measurements, the reference's Python result
    (crates/highuvlith-py/src/py_results.rs:15-238): ``intensity`` (ny, nx)
    indexed [y, x] (FP32, read-only), the field extent, and CD / NILS /
    contrast of the y = 0 cross-section (metrics.rs).  Also usable as an
    array (``np.asarray(result)``)."""

    __slots__ = ("_i", "x_min_nm", "x_max_nm", "y_min_nm", "y_max_nm")

    def __init__(self, intensity: np.ndarray, field_nm: float):
        i = np.asarray(intensity)
        i.flags.writeable = False
        self._i = i
        self.x_min_nm, self.x_max_nm = -field_nm / 2.0, field_nm / 2.0
        self.y_min_nm, self.y_max_nm = -field_nm / 2.0, field_nm / 2.0

    @property
    def intensity(self) -> np.ndarray:
        return self._i

    def __array__(self, dtype=None, copy=None):
        return self._i if dtype is None else self._i.astype(dtype)

    @property
    def shape(self):
        return self._i.shape

    @property
    def pixel_nm(self) -> float:
        return (self.x_max_nm - self.x_min_nm) / self._i.shape[1]

    @property
    def x_nm(self) -> np.ndarray:
        return self.x_min_nm + (np.arange(self._i.shape[1]) + 0.5) * self.pixel_nm

    @property
    def y_nm(self) -> np.ndarray:
        py = (self.y_max_nm - self.y_min_nm) / self._i.shape[0]
        return self.y_min_nm + (np.arange(self._i.shape[0]) + 0.5) * py

    @property
    def extent_nm(self):
        return (self.x_min_nm, self.x_max_nm, self.y_min_nm, self.y_max_nm)

    def cross_section(self, y_nm: float = 0.0):
        """(x_nm, intensity) of the row nearest y_nm."""
        ny = self._i.shape[0]
        py = (self.y_max_nm - self.y_min_nm) / ny
        row = int(min(max(round((y_nm - self.y_min_nm) / py - 0.5), 0), ny - 1))
        return self.x_nm, np.array(self._i[row], dtype=np.float64)

    def _profile(self):
        from . import metrics
        return metrics, self.x_nm, metrics.centre_profile(self._i)

    def image_contrast(self) -> float:
        from . import metrics
        return metrics.image_contrast(self._i)

    def cd(self, threshold: float = 0.3, tone: str = "dark") -> Optional[float]:
        m, x, p = self._profile()
        return m.printed_cd(p, x, threshold, _tone(tone))

    def nils_periodic(self, threshold: float = 0.3, tone: str = "dark",
                      width_nm: Optional[float] = None) -> Optional[float]:
        m, x, p = self._profile()
        return m.nils(p, x, threshold, _tone(tone), width_nm)

    def nils(self, threshold: float = 0.3) -> Optional[float]:
        """Legacy open-profile NILS (metrics.rs:603-617)."""
        m, x, p = self._profile()
        return m.nils_open(p, x, threshold)

    def image_log_slope(self, threshold: float = 0.3, tone: str = "dark") -> Optional[float]:
        m, x, p = self._profile()
        return m.image_log_slope(p, x, threshold, _tone(tone))

    def features(self, threshold: float = 0.3, tone: str = "dark"):
        m, x, p = self._profile()
        return m.features(p, x, threshold, _tone(tone))

    def __eq__(self, other) -> bool:
        if not isinstance(other, AerialImageResult):
            return NotImplemented
        return (np.allclose(self.extent_nm, other.extent_nm, rtol=0, atol=1e-9) and self.shape == other.shape
                and bool(np.all(np.abs(self._i.astype(np.float64) - other._i) < 1e-12)))

    def __repr__(self) -> str:
        return (f"AerialImageResult({self._i.shape[0]}x{self._i.shape[1]}, x=[{self.x_min_nm:.1f}, "
                f"{self.x_max_nm:.1f}]nm, y=[{self.y_min_nm:.1f}, {self.y_max_nm:.1f}]nm)")


def _tone(tone: str) -> str:
    t = tone.lower()
    if t not in ("dark", "bright"):
        raise ValueError(f"tone must be 'dark' or 'bright', got {tone!r}")
    return t


_NORMALIZATION = {"clear_field": 0, "absolute": 1}
# Where the FP64 kernel set is built: host C++ (dense), the GPU (dense), or the
# GPU with the reference's solver rule (randomized subspace iteration for
# large problems, aerial.rs:1116-1128).
_KERNEL_BUILD = {"host": 0, "device": 1, "device_reference_rule": 2}


class SimulationEngine:
    """Hopkins/SOCS imaging engine on one B200 (py_simulation.rs:115-164).

    Construction samples the source and builds the in-focus FP64 kernel set
    (``max_kernels`` as in the reference's Python default, 30)."""

    def __init__(self, source: SourceConfig, optics: OpticsConfig, mask: Optional[MaskConfig] = None,
                 grid: Optional[GridConfig] = None, max_kernels: int = 30,
                 kernel_energy_fraction: float = 1.0, source_points_per_axis: Optional[int] = None,
                 normalization: str = "clear_field", kernel_cache_capacity: int = 32, device: int = 0,
                 kernel_build: str = "host"):
        if normalization not in _NORMALIZATION:
            raise ValueError(f"normalization must be one of {sorted(_NORMALIZATION)}")
        if source_points_per_axis is not None and source_points_per_axis < 1:
            raise ValueError("source_points_per_axis must be >= 1 (or None for adaptive sampling)")
        self.source, self.optics = source, optics
        self.grid = grid or GridConfig()
        self.mask = mask
        self.device = device
        st = L.Settings()
        st.max_kernels = max_kernels
        st.kernel_energy_fraction = kernel_energy_fraction
        st.source_points_per_axis = source_points_per_axis or 0
        st.normalization = _NORMALIZATION[normalization]
        st.kernel_cache_capacity = kernel_cache_capacity
        if kernel_build not in _KERNEL_BUILD:
            raise ValueError(f"kernel_build must be one of {sorted(_KERNEL_BUILD)}")
        st.kernel_build = _KERNEL_BUILD[kernel_build]
        g = L.Grid(self.grid.size, self.grid.pixel_nm)
        h = C.c_void_p()
        L.check(L.lib().huv_engine_create(C.byref(source._c()), C.byref(optics._c()), C.byref(g),
                                          C.byref(st), device, C.byref(h)))
        self._h = h
        self._destroy = L.lib().huv_engine_destroy

    @classmethod
    def from_kernel_set(cls, eigenvalues, kernels, flare_fraction: float = 0.0, defocus_nm: float = 0.0,
                        pixel_nm: float = 1.0, wavelength_nm: float = 0.0, captured_energy_fraction: float = 1.0,
                        device: int = 0) -> "SimulationEngine":
        """An engine over a caller-built kernel set for one focus plane, in
        the layout ``kernels(z)`` returns (the reference's KernelSet,
        aerial.rs:216-228, 1912-1942): ``eigenvalues`` (K,) non-increasing
        with the normalisation folded in, ``kernels`` complex (K, n, n) in
        FFT layout.  Images at that plane only (huv_kernelset_create)."""
        ev = np.ascontiguousarray(np.asarray(eigenvalues, dtype=np.float64).reshape(-1))
        ker = np.ascontiguousarray(np.asarray(kernels, dtype=np.complex128))
        if ker.ndim != 3 or ker.shape[1] != ker.shape[2] or ker.shape[0] != ev.size:
            raise ValueError("kernels must be complex (K, n, n) with K = len(eigenvalues)")
        ks = L.KernelSetDesc(ker.shape[1], float(pixel_nm), ev.size, ev.ctypes.data, ker.ctypes.data,
                             float(defocus_nm), float(wavelength_nm), float(captured_energy_fraction),
                             float(flare_fraction))
        h = C.c_void_p()
        L.check(L.lib().huv_kernelset_create(C.byref(ks), device, C.byref(h)))
        self = cls.__new__(cls)
        self.source = self.optics = self.mask = None
        self.grid = GridConfig(ker.shape[1], float(pixel_nm))
        self.device = device
        self._h = h
        self._destroy = L.lib().huv_engine_destroy
        return self

    def __del__(self):
        # The destroy function is bound at construction: at interpreter exit
        # module globals may already be gone.
        h, destroy = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and destroy is not None:
            destroy(h)
            self._h = None

    @property
    def handle(self) -> int:
        return self._h.value

    # ---------------------------------------------------------- host queries
    def source_points(self) -> np.ndarray:
        n = C.c_int32()
        L.check(L.lib().huv_engine_source_points(self._h, None, 0, C.byref(n)))
        out = np.zeros((n.value, 3))
        L.check(L.lib().huv_engine_source_points(self._h, out.ctypes.data, n.value, C.byref(n)))
        return out

    def imaging_diagnostics(self, focus_nm: float = 0.0) -> dict:
        d = L.Diagnostics()
        L.check(L.lib().huv_engine_diagnostics(self._h, focus_nm, C.byref(d)))
        return {
            "num_kernels": d.num_kernels, "captured_energy_fraction": d.captured_energy_fraction,
            "num_frequencies": d.num_frequencies, "num_columns": d.num_columns,
            "method": ["dense_tcc", "dense_gram", "randomized", "supplied"][d.method],
            "support_exceeds_nyquist": bool(d.support_exceeds_nyquist),
            "clear_field_intensity": d.clear_field_intensity, "normalized": bool(d.normalized),
            "band_half_width": d.band_half_width, "num_source_points": d.num_source_points,
            "imaging_model": "scalar", "defocus_model": "exact",
        }

    def clear_field_intensity(self, focus_nm: float = 0.0) -> float:
        v = C.c_double()
        L.check(L.lib().huv_engine_clear_field(self._h, focus_nm, C.byref(v)))
        return v.value

    def kernels(self, focus_nm: float = 0.0) -> Tuple[np.ndarray, np.ndarray]:
        """(eigenvalues, kernels complex128 (k, n, n)) in FFT layout, unit norm;
        I = sum_k lambda_k |ifft2(K_k * spectrum)|^2 before flare."""
        k = C.c_int32()
        L.check(L.lib().huv_engine_kernels(self._h, focus_nm, None, None, 0, C.byref(k)))
        n = self.grid.size
        ev = np.zeros(k.value)
        ker = np.zeros((k.value, n, n), dtype=np.complex128)
        L.check(L.lib().huv_engine_kernels(self._h, focus_nm, ev.ctypes.data, ker.ctypes.data, k.value,
                                           C.byref(k)))
        return ev, ker

    def device_status(self, stream=None) -> None:
        """Synchronise and raise HuvError(DEVICE_TIMEOUT) if a bounded device
        wait of an earlier call gave up."""
        st = stream.cuda_stream if stream is not None else None
        L.check(L.lib().huv_device_status(self._h, st))

    # ---------------------------------------------------------- measurement
    def profile(self, on: bool = True) -> None:
        """Turn live timing of the dominant kernel on or off (resets counters)."""
        L.check(L.lib().huv_profile_enable(self._h, int(on)))

    def profile_read(self) -> dict:
        """{'kernel', 'ms', 'launches', 'total_launches', 'regions'} since the
        last read; 'kernel' is the region with the largest total time and
        'regions' maps every timed region to (launches, total ms)."""
        import json as _json
        buf = C.create_string_buffer(8192)
        L.check(L.lib().huv_profile_regions(self._h, buf, 8192))
        regions = {k: tuple(v) for k, v in _json.loads(buf.value.decode()).items()}
        ms, nl, tot = C.c_double(), C.c_int32(), C.c_int64()
        name = C.create_string_buffer(64)
        L.check(L.lib().huv_profile_read(self._h, C.byref(ms), C.byref(nl), C.byref(tot), name, 64))
        return {"kernel": name.value.decode(), "ms": ms.value, "launches": nl.value,
                "total_launches": tot.value, "regions": regions}

    # ---------------------------------------------------------- device calls
    @staticmethod
    def _kind(t) -> int:
        import torch
        if t.dtype == torch.uint8:
            return L.INPUT_U8
        if t.dtype == torch.float32:
            return L.INPUT_F32
        if t.dtype == torch.complex64:
            return L.INPUT_C64
        raise TypeError(f"unsupported mask dtype {t.dtype} (uint8, float32 or complex64)")

    def compute_batch(self, rasters, focus_nm: float = 0.0, pixel_transfer: bool = True,
                      form: str = "auto", eval_grid: int = 0, out=None, stream=None):
        """Images of a batch of rasters resident on the engine's device.

        ``rasters``: torch tensor (B, N, N) uint8 / float32 / complex64 on the
        device.  ``pixel_transfer=True`` gives ``compute(mask)`` of the
        pixel-aligned mask the raster depicts (Mask::spectrum, mask.rs:616-657);
        ``False`` gives ``compute_from_transmittance`` (aerial.rs:1789-1798).
        ``form``: "fft" (FP32 register-radix FFTs throughout), "tc" (split-BF16x3
        tcgen05 y-contraction and band interpolation), "tc_rows" (row
        transforms on tcgen05 too), "hybrid" (FP32 FFT field pass on the
        coarse grid, then the exact band interpolation I_N = P I_M P^T as two
        split-FP16x3 tcgen05 GEMMs) or "auto" (hybrid where its kernels
        apply, else fft).
        Returns a float32 (B, N, N) tensor; ``out``, if given, must be a
        contiguous float32 (B, N, N) tensor on the rasters' device."""
        import torch
        n = self.grid.size
        if rasters.dim() == 2:
            rasters = rasters.unsqueeze(0)
        if rasters.shape[-2:] != (n, n):
            raise ValueError(f"rasters must be (B, {n}, {n}), got {tuple(rasters.shape)}")
        if not rasters.is_cuda:
            raise ValueError("rasters must live on the CUDA device; use compute_batch_host for host arrays")
        rasters = rasters.contiguous()
        if out is None:
            out = torch.empty((rasters.shape[0], n, n), dtype=torch.float32, device=rasters.device)
        elif (out.dtype != torch.float32 or out.device != rasters.device or not out.is_contiguous()
              or tuple(out.shape) != (rasters.shape[0], n, n)):
            raise ValueError(f"out must be a contiguous float32 ({rasters.shape[0]}, {n}, {n}) tensor on "
                             f"{rasters.device}")
        b = L.Batch(rasters.shape[0], self._kind(rasters), rasters.data_ptr(), int(pixel_transfer),
                    float(focus_nm), L.FORM[form], int(eval_grid))
        st = (stream or torch.cuda.current_stream(rasters.device)).cuda_stream
        L.check(L.lib().huv_image_batch(self._h, C.byref(b), out.data_ptr(), st))
        return out

    def compute_batch_host(self, rasters: np.ndarray, focus_nm: float = 0.0, pixel_transfer: bool = True,
                           form: str = "auto", eval_grid: int = 0, out: Optional[np.ndarray] = None,
                           stream=None) -> np.ndarray:
        """Same as ``compute_batch`` from host memory to host memory (copies
        included; pinned buffers make them faster).  ``out``, if given, must
        be a writeable C-contiguous float32 (B, N, N) array."""
        n = self.grid.size
        r = np.ascontiguousarray(rasters)
        if r.ndim == 2:
            r = r[None]
        kind = {np.dtype(np.uint8): L.INPUT_U8, np.dtype(np.float32): L.INPUT_F32,
                np.dtype(np.complex64): L.INPUT_C64}.get(r.dtype)
        if kind is None:
            raise TypeError(f"unsupported mask dtype {r.dtype}")
        if r.shape[-2:] != (n, n):
            raise ValueError(f"rasters must be (B, {n}, {n})")
        if out is None:
            out = np.empty((r.shape[0], n, n), dtype=np.float32)
        elif (not isinstance(out, np.ndarray) or out.dtype != np.float32 or out.shape != (r.shape[0], n, n)
              or not out.flags.c_contiguous or not out.flags.writeable):
            raise ValueError(f"out must be a writeable C-contiguous float32 ({r.shape[0]}, {n}, {n}) array")
        b = L.Batch(r.shape[0], kind, r.ctypes.data, int(pixel_transfer), float(focus_nm), L.FORM[form],
                    int(eval_grid))
        st = 0
        if stream is not None:
            st = stream.cuda_stream
        L.check(L.lib().huv_image_batch_host(self._h, C.byref(b), out.ctypes.data, st))
        return out

    def compute_aerial_image(self, focus_nm: float = 0.0, mask: Optional[MaskConfig] = None) -> AerialImageResult:
        """Image of ``mask`` (or the engine's own mask) at ``focus_nm``
        (py_simulation.rs:169-179), as an AerialImageResult."""
        m = mask or self.mask
        if m is None:
            raise ValueError("no mask given")
        img = self.compute_batch_host(m.rasterize(self.grid), focus_nm, pixel_transfer=True)[0]
        return AerialImageResult(img, self.grid.field_nm)

    @staticmethod
    def _rect_clips(clips, feature, background):
        """ctypes view of rectangle clips (centre x, y and size w, h in nm,
        field-centred coordinates); keeps the arrays alive on the view."""
        flat = [tuple(map(float, r)) for c in clips for r in c]
        rects = np.ascontiguousarray(np.asarray(flat, dtype=np.float64).reshape(-1, 4))
        offs = np.zeros(len(clips) + 1, dtype=np.int32)
        offs[1:] = np.cumsum([len(c) for c in clips])
        f, bgd = complex(feature), complex(background)
        view = L.RectClips(rects.ctypes.data if rects.size else None, offs.ctypes.data, f.real, f.imag, bgd.real,
                           bgd.imag)
        view._keep = (rects, offs)
        return view

    def compute_batch_rects(self, clips, feature: complex = 1.0, background: complex = 0.0, focus_nm: float = 0.0,
                            form: str = "auto", eval_grid: int = 0, out=None, stream=None):
        """Images of rectangle clips from their exact analytic spectrum
        (Mask::spectrum, mask.rs:616-657; overlaps resolved into disjoint
        cells, sub-pixel positions exact).  ``clips``: sequence of sequences
        of (x, y, w, h) in nm, centre and size, field-centred.  Each clip is
        the union of its rectangles with amplitude ``feature`` on
        ``background`` (dark field: 1 on 0).  Returns float32 (B, N, N) on the
        device."""
        import torch
        n = self.grid.size
        view = self._rect_clips(clips, feature, background)
        if out is None:
            out = torch.empty((len(clips), n, n), dtype=torch.float32, device=f"cuda:{self.device}")
        elif (out.dtype != torch.float32 or not out.is_cuda or not out.is_contiguous()
              or tuple(out.shape) != (len(clips), n, n)):
            raise ValueError(f"out must be a contiguous float32 ({len(clips)}, {n}, {n}) CUDA tensor")
        b = L.Batch(len(clips), L.INPUT_RECTS, C.addressof(view), 0, float(focus_nm), L.FORM[form], int(eval_grid))
        st = (stream or torch.cuda.current_stream(out.device)).cuda_stream
        L.check(L.lib().huv_image_batch(self._h, C.byref(b), out.data_ptr(), st))
        return out

    def compute_batch_rects_host(self, clips, feature: complex = 1.0, background: complex = 0.0,
                                 focus_nm: float = 0.0, form: str = "auto", eval_grid: int = 0) -> np.ndarray:
        """``compute_batch_rects`` into host memory (images copied out in
        chunks overlapped with the imaging)."""
        n = self.grid.size
        view = self._rect_clips(clips, feature, background)
        out = np.empty((len(clips), n, n), dtype=np.float32)
        b = L.Batch(len(clips), L.INPUT_RECTS, C.addressof(view), 0, float(focus_nm), L.FORM[form], int(eval_grid))
        L.check(L.lib().huv_image_batch_host(self._h, C.byref(b), out.ctypes.data, None))
        return out

    def compute_through_focus(self, focus_nm: Sequence[float],
                              mask: Optional[MaskConfig] = None) -> List[AerialImageResult]:
        """Images of ``mask`` at several focus planes (py_simulation.rs:319-330,
        aerial.rs:1820-1825): kernels of uncached planes built concurrently,
        every plane imaged on the device (huv_image_focus_sweep)."""
        import torch
        m = mask or self.mask
        if m is None:
            raise ValueError("no mask given")
        r = torch.from_numpy(np.ascontiguousarray(m.rasterize(self.grid))[None]).to(f"cuda:{self.device}")
        return [AerialImageResult(img[0], self.grid.field_nm)
                for img in self.compute_batch_through_focus(r, focus_nm).cpu().numpy()]

    def compute_batch_through_focus(self, rasters, focus_nm: Sequence[float], pixel_transfer: bool = True,
                                    form: str = "auto", eval_grid: int = 0, out=None, stream=None):
        """process::batch_defocus (process.rs:1303-1313) for a batch of device
        rasters: returns float32 (planes, B, N, N) on the device."""
        import torch
        n = self.grid.size
        if rasters.dim() == 2:
            rasters = rasters.unsqueeze(0)
        if not rasters.is_cuda or rasters.shape[-2:] != (n, n):
            raise ValueError(f"rasters must be (B, {n}, {n}) on the CUDA device")
        rasters = rasters.contiguous()
        z = np.ascontiguousarray(np.asarray(focus_nm, dtype=np.float64).reshape(-1))
        if out is None:
            out = torch.empty((len(z), rasters.shape[0], n, n), dtype=torch.float32, device=rasters.device)
        elif (out.dtype != torch.float32 or out.device != rasters.device or not out.is_contiguous()
              or tuple(out.shape) != (len(z), rasters.shape[0], n, n)):
            raise ValueError(f"out must be a contiguous float32 ({len(z)}, {rasters.shape[0]}, {n}, {n}) tensor "
                             f"on {rasters.device}")
        b = L.Batch(rasters.shape[0], self._kind(rasters), rasters.data_ptr(), int(pixel_transfer), 0.0,
                    L.FORM[form], int(eval_grid))
        st = (stream or torch.cuda.current_stream(rasters.device)).cuda_stream
        L.check(L.lib().huv_image_focus_sweep(self._h, C.byref(b), z.ctypes.data, len(z), out.data_ptr(), st))
        return out

    def compute_from_transmittance(self, transmittance, focus_nm: float = 0.0) -> AerialImageResult:
        """Image of a complex transmittance map (n, n) [y, x]
        (py_simulation.rs:375-393); the spectrum is the plain FFT."""
        t = np.asarray(transmittance)
        n = self.grid.size
        if t.shape != (n, n):
            raise ValueError(f"transmittance must be ({n}, {n}) to match the grid, got {t.shape}")
        t = t.astype(np.complex64) if np.iscomplexobj(t) else t.astype(np.float32)
        return AerialImageResult(self.compute_batch_host(t, focus_nm, pixel_transfer=False)[0], self.grid.field_nm)


def rasterize_rects(n: int, clips: Sequence[Sequence[Tuple[int, int, int, int]]], dark_field: bool = True,
                    device=None):
    """Device rasters (B, n, n) uint8 of pixel-aligned rectangle clips, drawn
    by the library's rasteriser kernel."""
    import torch
    device = device or torch.device("cuda")
    flat = [r for c in clips for r in c]
    offs = np.zeros(len(clips) + 1, dtype=np.int32)
    offs[1:] = np.cumsum([len(c) for c in clips])
    rects = torch.tensor(np.asarray(flat, dtype=np.int32).reshape(-1, 4) if flat else np.zeros((1, 4), np.int32),
                         device=device)
    offsets = torch.tensor(offs, device=device)
    out = torch.empty((len(clips), n, n), dtype=torch.uint8, device=device)
    st = torch.cuda.current_stream(device).cuda_stream
    L.check(L.lib().huv_rasterize_rects(n, len(clips), rects.data_ptr(), offsets.data_ptr(),
                                        int(dark_field), out.data_ptr(), st))
    return out


class UnevenPlan:
    """Many clips of different grids, sources and kernel budgets imaged by one
    CUDA-graph launch (huv_plan_*).  ``clips``: sequence of
    (engine, max_kernels, input_tensor (N, N) on the device, output_tensor
    (N, N) float32 on the device).  Group-contiguous storage (clips of the
    same engine and budget adjacent in one tensor) avoids staging copies."""

    def __init__(self, clips, pixel_transfer: bool = True, autotune: bool = True):
        arr = (L.Clip * len(clips))()
        self._keep = []
        for i, (eng, kmax, inp, out) in enumerate(clips):
            arr[i] = L.Clip(eng.handle, int(kmax), SimulationEngine._kind(inp), inp.data_ptr(), out.data_ptr())
            self._keep.append((eng, inp, out))
        h = C.c_void_p()
        L.check(L.lib().huv_plan_create(arr, len(clips), int(pixel_transfer), int(autotune), C.byref(h)))
        self._h = h
        self._destroy = L.lib().huv_plan_destroy

    def launch(self, stream=None):
        import torch
        st = (stream or torch.cuda.current_stream()).cuda_stream
        L.check(L.lib().huv_plan_launch(self._h, st))

    def describe(self):
        import json
        buf = C.create_string_buffer(1 << 16)
        L.check(L.lib().huv_plan_describe(self._h, buf, 1 << 16))
        return json.loads(buf.value.decode())

    def __del__(self):
        # The destroy function is bound at construction: at interpreter exit
        # module globals may already be gone.
        h, destroy = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and destroy is not None:
            destroy(h)
            self._h = None
