"""FP64 restatement of the reference's pixel ILT objective and optimizer.

TEST INFRASTRUCTURE: the checker, never the product (see ``oracle/__init__``).
Follows crates/highuvlith-core/src/ilt.rs: mask parametrisation 538-550,
data_term 564-603, regularization 606-645, cost 648-659,
cost_and_gradient_with 667-738, run_stage 755-866, optimize_ilt 881-951,
create_target_contact_array 336-362; and opc.rs:432-471 (kernel fields,
intensity, flare).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np


@dataclass
class IltConfig:
    cost: str = "resist"          # "resist" (ResistContour) or "image" (ImageFidelity)
    threshold: float = 0.25
    steepness: float = 50.0
    beta: float = 4.0             # sigmoid steepness of the mask parametrisation
    tv_weight: float = 0.01
    tv_eps: float = 0.01
    bin_weight: float = 0.0
    dose: float = 1.0
    weight: float = 1.0
    flare: float = 0.0
    absorber: complex = 0j
    learning_rate: float = 0.5
    convergence_tol: float = 1e-4


class IltProblem:
    """One condition; kernels = dense (K, n, n) in FFT layout, eigenvalues
    already divided by the clear field (AerialImageEngine::kernels)."""

    def __init__(self, eigenvalues, kernels, target, cfg: IltConfig):
        self.lam = np.asarray(eigenvalues, dtype=np.float64)
        self.ker = np.asarray(kernels, dtype=np.complex128)
        self.target = np.asarray(target, dtype=np.float64)
        self.cfg = cfg

    def mask(self, theta):
        return 1.0 / (1.0 + np.exp(-self.cfg.beta * theta))

    def spectrum(self, m):
        a = self.cfg.absorber
        return np.fft.fft2(a + (1.0 - a) * m)

    def fields(self, spec):
        return [np.fft.ifft2(k * spec) for k in self.ker]

    def image(self, m):
        spec = self.spectrum(m)
        img = sum(l * np.abs(f) ** 2 for l, f in zip(self.lam, self.fields(spec)))
        return self._flare(img)

    def _flare(self, img):
        phi = self.cfg.flare
        if phi > 0.0:
            return img * (1.0 - phi) + phi * img.mean()
        return img

    def data_term(self, img, want_grad):
        c = self.cfg
        inv_n = 1.0 / img.size
        if c.cost == "image":
            r = c.dose * img - self.target
            g = 2.0 * r * c.dose * inv_n if want_grad else None
        else:
            rr = 1.0 / (1.0 + np.exp(-c.steepness * (c.dose * img - c.threshold)))
            r = rr - self.target
            g = 2.0 * r * c.steepness * rr * (1.0 - rr) * c.dose * inv_n if want_grad else None
        return float(np.sum(r * r)) * inv_n, g

    def regularization(self, m):
        c = self.cfg
        inv_n = 1.0 / m.size
        cost = 0.0
        grad = np.zeros_like(m)
        if c.tv_weight > 0.0:
            gx = np.roll(m, -1, axis=1) - m
            gy = np.roll(m, -1, axis=0) - m
            s = np.sqrt(gx * gx + gy * gy + c.tv_eps ** 2)
            cost += c.tv_weight * float(np.sum(s - c.tv_eps)) * inv_n
            g = -(gx + gy) / s + np.roll(gx / s, 1, axis=1) + np.roll(gy / s, 1, axis=0)
            grad += c.tv_weight * g * inv_n
        if c.bin_weight > 0.0:
            cost += c.bin_weight * float(np.sum(4.0 * m * (1.0 - m))) * inv_n
            grad += c.bin_weight * 4.0 * (1.0 - 2.0 * m) * inv_n
        return cost, grad

    def cost(self, theta):
        m = self.mask(theta)
        img = self.image(m)
        return self.cfg.weight * self.data_term(img, False)[0] + self.regularization(m)[0]

    def cost_and_gradient(self, theta):
        c = self.cfg
        m = self.mask(theta)
        spec = self.spectrum(m)
        fields = self.fields(spec)
        img = self._flare(sum(l * np.abs(f) ** 2 for l, f in zip(self.lam, fields)))
        cost, g = self.data_term(img, True)
        total = c.weight * cost
        g0 = (1.0 - c.flare) * g + c.flare * g.sum() / g.size
        conj_c = np.conj(1.0 - c.absorber)
        dcdm = np.zeros_like(m)
        for lam, k, a in zip(self.lam, self.ker, fields):
            v = np.fft.ifft2(np.conj(k) * np.fft.fft2(a * g0)) * lam
            dcdm += 2.0 * c.weight * np.real(conj_c * v)
        rc, rg = self.regularization(m)
        total += rc
        dcdm += rg
        return total, dcdm * c.beta * m * (1.0 - m)


def contact_array_target(n: int, pixel: float, size: float, pitch_x: float, pitch_y: float,
                         count_x: int, count_y: int) -> np.ndarray:
    """create_target_contact_array, square holes, 4x4 supersampling (ilt.rs:336-362, 300-324)."""
    half = n * pixel / 2.0
    centres = [((ix - (count_x - 1) / 2.0) * pitch_x, (iy - (count_y - 1) / 2.0) * pitch_y)
               for iy in range(count_y) for ix in range(count_x)]
    r = size / 2.0
    s = 4
    sub = (np.arange(s) + 0.5) / s
    ys = -half + (np.arange(n)[:, None] + sub[None, :]) * pixel   # (n, s)
    xs = ys.copy()
    out = np.zeros((n, n))
    for cx, cy in centres:
        inx = (np.abs(xs - cx) <= r).astype(float).sum(axis=1) / s   # fraction per column pixel
        iny = (np.abs(ys - cy) <= r).astype(float).sum(axis=1) / s
        out = np.maximum(out, iny[:, None] * inx[None, :])
    return out


def run_stage(problem: IltProblem, theta, max_iterations: int, lr: float, tol: float):
    """CG Polak-Ribiere+ with Armijo backtracking on the unit-max-norm
    direction (ilt.rs:755-866).  Returns (theta, cost history)."""
    armijo, backtracks = 1e-4, 25
    cost, grad = problem.cost_and_gradient(theta)
    hist = [cost]
    direction = -grad
    step = lr
    small = 0
    for _ in range(max_iterations):
        accepted = None
        for attempt in range(2):
            d_max = float(np.max(np.abs(direction)))
            if d_max == 0.0:
                break
            unit = direction / d_max
            slope = float(np.sum(grad * unit))
            if slope >= 0.0:
                direction = -grad
                continue
            s = step
            for _ in range(backtracks):
                trial = theta + s * unit
                ct = problem.cost(trial)
                if ct <= cost + armijo * s * slope and math.isfinite(ct):
                    accepted = (ct, trial, s)
                    break
                s *= 0.5
            if accepted is not None or attempt == 1:
                break
            direction = -grad
        if accepted is None:
            return theta, hist
        _, theta, s_used = accepted
        c_new, g_new = problem.cost_and_gradient(theta)
        prev = cost
        cost = c_new
        hist.append(cost)
        gg = float(np.sum(grad * grad))
        beta_pr = max((float(np.sum(g_new * g_new)) - float(np.sum(g_new * grad))) / gg, 0.0) if gg > 0 else 0.0
        direction = -g_new + beta_pr * direction
        grad = g_new
        step = min(s_used * 1.5, 10.0 * lr)
        rel = (prev - cost) / prev if prev > 0 else 0.0
        small = small + 1 if rel < tol else 0
        if small >= 3 or cost == 0.0:
            return theta, hist
    return theta, hist
