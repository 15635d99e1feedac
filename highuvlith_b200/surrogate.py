"""FNO image surrogate: training on SOCS-generated pairs, and surrogate-assisted ILT.

The workload is High-NA EUV (lambda 13.5 nm, NA 0.55, central obscuration
0.2 -- the EuvProjectionOptics preset, optics/euv.rs:123-125), annular
sigma 0.3/0.8, 48 SOCS kernels, 512 x 512 pixels of 1 nm.  Anamorphic 4x/8x
reduction is not modelled by the reference; the Manhattan clips are drawn
directly at wafer scale (features 15-60 nm, clear-area density 20-60 %),
which is the mask-side x/4, y/8 scaling already applied.

Training pairs are (transmittance map, SOCS image of that map) with images
from the engine's own device path (``compute_batch`` with
``pixel_transfer=False``, the map ILT images).  Half of each batch is binary
clips, half "soft" clips: sigmoid(beta (r - 1/2 + noise)) with beta in
[2, 8], the grey-level masks that ILT iterates pass through.

``optimize_with_surrogate`` is the ILT stage loop with costs and gradients
from the FNO, exact SOCS judging every ``judge_every`` iterations and taking
over when the surrogate's relative image error passes ``error_bound``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib as L
from .api import GridConfig, OpticsConfig, SimulationEngine, SourceConfig
from .clips import gen_clip
from .fno import FnoSurrogate
from .ilt import IltSettings


def high_na_engine(grid: int = 512, pixel_nm: float = 1.0, max_kernels: int = 48, device: int = 0) -> SimulationEngine:
    """High-NA EUV engine: NA 0.55, obscuration 0.2, annular 0.3/0.8."""
    return SimulationEngine(SourceConfig(13.5, "annular", (0.3, 0.8)), OpticsConfig.euv_high_na_055(),
                            grid=GridConfig(grid, pixel_nm), max_kernels=max_kernels, device=device)


@dataclass
class PairSource:
    """Seeded stream of (mask, image) training pairs on the device."""
    engine: SimulationEngine
    seed: int = 7
    wmin: int = 15
    wmax: int = 60
    dmin: float = 0.20
    dmax: float = 0.60
    soft_fraction: float = 0.5
    _next: int = 0

    def clips(self, count: int) -> np.ndarray:
        n = self.engine.grid.size
        px = self.engine.grid.pixel_nm
        lo, hi = max(1, int(round(self.wmin / px))), max(1, int(round(self.wmax / px)))
        out = np.zeros((count, n, n), dtype=np.uint8)
        for i in range(count):
            _, out[i] = gen_clip(self.seed * 1_000_003 + self._next, n, lo, hi, self.dmin, self.dmax)
            self._next += 1
        return out

    def batch(self, count: int):
        """(masks float32 (count, N, N), images float32 (count, N, N)) on the device."""
        import torch
        dev = f"cuda:{self.engine.device}"
        r = torch.from_numpy(self.clips(count)).to(dev).float()
        g = torch.Generator(device=dev)
        g.manual_seed(self.seed * 7919 + self._next)
        n_soft = int(round(self.soft_fraction * count))
        if n_soft:
            beta = 2.0 + 6.0 * torch.rand((n_soft, 1, 1), generator=g, device=dev)
            noise = 0.15 * torch.randn((n_soft, r.shape[1], r.shape[2]), generator=g, device=dev)
            r[:n_soft] = torch.sigmoid(beta * (r[:n_soft] - 0.5 + noise))
        masks = r.contiguous()
        images = self.engine.compute_batch(masks, pixel_transfer=False)
        return masks, images


def train(fno: FnoSurrogate, pairs: PairSource, steps: int, batch: int = 8, lr: float = 1e-3,
          lr_final: float = 1e-4, weight_decay: float = 0.0) -> List[float]:
    """Adam on the MSE between FNO and SOCS images, fresh pairs every step,
    cosine learning-rate decay from lr to lr_final.  Returns the losses."""
    losses = []
    for s in range(steps):
        masks, images = pairs.batch(batch)
        a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * s / max(1, steps)))
        losses.append(fno.train_step(masks, images, lr=float(a), weight_decay=weight_decay))
    return losses


def relative_image_error(fno: FnoSurrogate, engine: SimulationEngine, masks) -> np.ndarray:
    """Per mask max|I_fno - I_socs| / max|I_socs| (the judge's measure)."""
    socs = engine.compute_batch(masks, pixel_transfer=False)
    pred = fno.forward(masks)
    err = (pred - socs).abs().amax(dim=(1, 2)) / socs.abs().amax(dim=(1, 2)).clamp_min(1e-30)
    return err.double().cpu().numpy()


@dataclass
class SurrogateReport:
    final_cost: np.ndarray
    iterations: np.ndarray
    cost_history: np.ndarray
    surrogate_iterations: int
    exact_iterations: int
    takeover_iteration: int
    judge_errors: List[float] = field(default_factory=list)


def optimize_with_surrogate(engine: SimulationEngine, fno: FnoSurrogate, theta, target, settings: IltSettings,
                            judge_every: int = 5, error_bound: float = 0.05, stream=None) -> SurrogateReport:
    """ILT with FNO costs/gradients, exact SOCS judge every ``judge_every``
    iterations and takeover past ``error_bound``; theta is updated in place.
    ``final_cost`` is the exact SOCS cost; ``cost_history`` holds the costs
    the optimizer saw (surrogate ones until a takeover)."""
    import torch
    b = theta.shape[0]
    fc = np.zeros(b)
    its = np.zeros(b, dtype=np.int32)
    hist = np.zeros((b, settings.max_iterations + 1))
    opt = L.IltOpt(settings.max_iterations, settings.learning_rate, settings.convergence_tol)
    sur = L.SurrogateIlt()
    sur.judge_every = judge_every
    sur.error_bound = error_bound
    st = (stream or torch.cuda.current_stream(theta.device)).cuda_stream
    L.check(L.lib().huv_ilt_optimize_surrogate(engine.handle, fno.handle, C.byref(settings._params()), C.byref(opt),
                                               b, theta.data_ptr(), target.contiguous().data_ptr(), C.byref(sur),
                                               fc.ctypes.data, its.ctypes.data, hist.ctypes.data, st))
    return SurrogateReport(fc, its, hist, sur.surrogate_iterations, sur.exact_iterations, sur.takeover_iteration,
                           [sur.judge_errors[i] for i in range(min(sur.n_judges, 64))])
