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


def _clip_block(args) -> np.ndarray:
    """Rasters of clips first, first + 1, ... (a process-pool task)."""
    first, count, n, lo, hi, dmin, dmax = args
    out = np.zeros((count, n, n), dtype=np.uint8)
    for i in range(count):
        _, out[i] = gen_clip(first + i, n, lo, hi, dmin, dmax)
    return out


@dataclass
class PairSource:
    """Seeded stream of (mask, image) training pairs on the device.

    Clip i of the stream is ``gen_clip(seed * 1000003 + i, ...)``.  With
    ``workers > 0`` the clips are drawn ahead by a spawn-started process pool
    (the generator is Python-bound); the stream is the same either way."""
    engine: SimulationEngine
    seed: int = 7
    wmin: int = 15
    wmax: int = 60
    dmin: float = 0.20
    dmax: float = 0.60
    soft_fraction: float = 0.5
    workers: int = 0
    _next: int = 0
    _pool: object = None
    _ahead: list = field(default_factory=list)

    def _args(self, first: int, count: int):
        n = self.engine.grid.size
        px = self.engine.grid.pixel_nm
        lo, hi = max(1, int(round(self.wmin / px))), max(1, int(round(self.wmax / px)))
        return (self.seed * 1_000_003 + first, count, n, lo, hi, self.dmin, self.dmax)

    def clips(self, count: int) -> np.ndarray:
        if self.workers <= 0:
            out = _clip_block(self._args(self._next, count))
            self._next += count
            return out
        if self._pool is None:
            import multiprocessing as mp
            self._pool = mp.get_context("spawn").Pool(self.workers)
            self._queued = self._next
        # keep 2 * workers blocks of `count` clips in flight, in stream order
        while len(self._ahead) < 2 * self.workers:
            self._ahead.append(self._pool.apply_async(_clip_block, (self._args(self._queued, count),)))
            self._queued += count
        out = self._ahead.pop(0).get()
        self._next += count
        return out

    def close(self) -> None:
        if self._pool is not None:
            self._pool.terminate()
            self._pool = None
            self._ahead = []

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


def train_timed(fno: FnoSurrogate, pairs: PairSource, pairs_total: int, batch: int = 16, lr: float = 2e-3,
                lr_final: float = 1e-4, log_every: int = 200, log=print):
    """Training on ``pairs_total`` fresh pairs with progress lines; returns
    (losses, dict of timings)."""
    import time
    import torch
    steps = max(1, pairs_total // batch)
    losses = []
    t0 = time.perf_counter()
    t_gen = 0.0
    for s in range(steps):
        g0 = time.perf_counter()
        masks, images = pairs.batch(batch)
        t_gen += time.perf_counter() - g0
        a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * s / steps))
        losses.append(fno.train_step(masks, images, lr=float(a)))
        if log_every and (s + 1) % log_every == 0:
            el = time.perf_counter() - t0
            log({"step": s + 1, "pairs": (s + 1) * batch, "loss": float(np.mean(losses[-log_every:])),
                 "elapsed_s": round(el, 1), "pairs_per_s": round((s + 1) * batch / el, 1)})
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    return losses, {"steps": steps, "pairs": steps * batch, "elapsed_s": el, "pairs_per_s": steps * batch / el,
                    "pair_s": t_gen}


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
    from .ilt import _masks_on_device
    theta, target = _masks_on_device(engine, theta, target, in_place=True)
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
                                               b, theta.data_ptr(), target.data_ptr(), C.byref(sur),
                                               fc.ctypes.data, its.ctypes.data, hist.ctypes.data, st))
    return SurrogateReport(fc, its, hist, sur.surrogate_iterations, sur.exact_iterations, sur.takeover_iteration,
                           [sur.judge_errors[i] for i in range(min(sur.n_judges, 64))])


def _time_step(b: int) -> int:
    """Two warm-up training steps, then one timed step and one timed forward
    (CUDA events) of batch b on seeded random 512^2 maps."""
    import json
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    masks = (torch.rand((b, 512, 512), generator=g, device="cuda") > 0.5).float()
    targets = torch.rand((b, 512, 512), generator=g, device="cuda")
    fno = FnoSurrogate(512, 16, 4, seed=1)
    for _ in range(2):
        fno.train_step(masks, targets, lr=1e-3)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    fno.train_step(masks, targets, lr=1e-3)
    e1.record()
    fno.forward(masks)
    e2.record()
    torch.cuda.synchronize()
    print(json.dumps({"batch": b, "grid": 512, "train_step_ms": e0.elapsed_time(e1),
                      "forward_ms": e1.elapsed_time(e2)}))
    return 0


def main(argv=None) -> int:
    """Train the FNO surrogate on SOCS pairs of the High-NA workload, then
    compare surrogate-assisted ILT with exact ILT; one JSON line per report."""
    import argparse
    import json
    import time
    import torch
    from .targets import gen_contact_targets
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--pairs", type=int, default=200_000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--workers", type=int, default=0, help="clip-generator processes (0: host cores - 2, at most 32)")
    ap.add_argument("--out", default="", help="save the trained parameters (.npz)")
    ap.add_argument("--log-every", type=int, default=500)
    ap.add_argument("--time-step", type=int, default=0, metavar="B",
                    help="only time one training step and one forward of batch B on random 512^2 maps")
    a = ap.parse_args(argv)
    if a.time_step:
        return _time_step(a.time_step)
    import os
    workers = a.workers or max(1, min(32, (os.cpu_count() or 2) - 2))
    say = lambda d: print(json.dumps(d), flush=True)  # noqa: E731
    eng = high_na_engine()
    fno = FnoSurrogate(512, 16, 4, seed=3)
    src = PairSource(eng, seed=11, workers=workers)
    losses, tm = train_timed(fno, src, a.pairs, batch=a.batch, lr=a.lr, log_every=a.log_every, log=say)
    src.close()
    tm.update({"workers": workers, "final_loss": float(np.mean(losses[-50:]))})
    say({"training": tm})
    if a.out:
        fno.save(a.out)
    held, _ = PairSource(eng, seed=99).batch(32)
    err = relative_image_error(fno, eng, held)
    say({"held_out_rel_err": {"median": float(np.median(err)), "max": float(np.max(err)),
                              "binary_median": float(np.median(err[16:])), "soft_median": float(np.median(err[:16]))}})
    tg_np, _ = gen_contact_targets(8, 512, 1.0, base_seed=5)
    tg = torch.from_numpy(tg_np).cuda()
    st = IltSettings(cost="resist", threshold=0.25, steepness=50.0, max_iterations=20)
    from . import ilt
    th0 = ilt.initial_theta_from_target(tg).contiguous()
    c0, _ = ilt.cost_and_gradient(eng, th0, tg, st, want_gradient=False)
    res = {"initial_cost": float(np.mean(c0))}
    # warm-up: the optimizer's and the judge's kernels and buffers, so that no
    # method below pays first-call set-up
    ilt.optimize(eng, th0.clone(), tg, IltSettings(cost="resist", threshold=0.25, steepness=50.0, max_iterations=1))
    optimize_with_surrogate(eng, fno, th0.clone(), tg, IltSettings(cost="resist", threshold=0.25, steepness=50.0,
                                                                   max_iterations=1), judge_every=1, error_bound=0.05)
    th = th0.clone()
    torch.cuda.synchronize()
    t = time.perf_counter()
    r = ilt.optimize(eng, th, tg, st)
    torch.cuda.synchronize()
    res["exact"] = {"final_cost": float(np.mean(r["final_cost"])), "s": time.perf_counter() - t}
    for name, bound in (("surrogate_judged", 0.05), ("surrogate_only", 1e9)):
        th = th0.clone()
        torch.cuda.synchronize()
        t = time.perf_counter()
        rep = optimize_with_surrogate(eng, fno, th, tg, st, judge_every=5, error_bound=bound)
        torch.cuda.synchronize()
        res[name] = {"final_cost": float(np.mean(rep.final_cost)), "s": time.perf_counter() - t,
                     "surrogate_iterations": rep.surrogate_iterations, "exact_iterations": rep.exact_iterations,
                     "takeover_iteration": rep.takeover_iteration, "judge_errors": rep.judge_errors}
    say({"ilt_8_contact_targets_512": res})
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
