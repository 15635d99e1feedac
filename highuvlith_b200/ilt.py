"""Batched pixel ILT on the device (crates/highuvlith-core/src/ilt.rs).

``IltSettings`` mirrors ILTConfig's fields that apply to one process
condition; ``cost_and_gradient`` is IltProblem::cost_and_gradient_with for a
batch of masks; ``optimize`` runs the CG (Polak-Ribiere+) / Armijo stage loop
for every mask concurrently.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class IltSettings:
    cost: str = "resist"            # "resist" (ResistContour) | "image" (ImageFidelity)
    threshold: float = 0.25
    steepness: float = 50.0
    sigmoid_steepness: float = 4.0
    regularization: float = 0.01    # TV weight
    tv_epsilon: float = 0.01
    binarization_weight: float = 0.0
    dose: float = 1.0
    weight: float = 1.0
    absorber: float = 0.0
    defocus_nm: float = 0.0
    max_iterations: int = 50
    learning_rate: float = 0.5
    convergence_tol: float = 1e-4

    def _params(self) -> L.IltParams:
        return L.IltParams(1 if self.cost == "resist" else 0, self.threshold, self.steepness,
                           self.sigmoid_steepness, self.regularization, self.tv_epsilon,
                           self.binarization_weight, self.dose, self.weight, self.absorber, self.defocus_nm)


def initial_theta_from_target(target):
    """IltInit::Target: theta = Z - 1/2 (ilt.rs:518-520)."""
    return target - 0.5


def _masks_on_device(engine, theta, target, in_place: bool):
    """theta (B, N, N) float32 CUDA tensor (kept as given when it is updated
    in place, else converted), target converted to match it."""
    import torch
    n = engine.grid.size
    if theta.dim() != 3 or tuple(theta.shape[1:]) != (n, n) or not theta.is_cuda:
        raise ValueError(f"theta must be a (B, {n}, {n}) CUDA tensor")
    if in_place:
        if theta.dtype != torch.float32 or not theta.is_contiguous():
            raise ValueError("theta is updated in place: it must be a contiguous float32 tensor")
    else:
        theta = theta.to(dtype=torch.float32).contiguous()
    target = torch.as_tensor(target).to(device=theta.device, dtype=torch.float32).contiguous()
    if tuple(target.shape) != tuple(theta.shape):
        raise ValueError(f"target must have theta's shape {tuple(theta.shape)}, got {tuple(target.shape)}")
    return theta, target


def cost_and_gradient(engine, theta, target, settings: IltSettings, want_gradient: bool = True, stream=None):
    """theta, target: torch tensors (B, N, N) on the engine's device (float32
    is used; other dtypes are converted).  Returns (costs numpy (B,),
    gradient tensor or None)."""
    import torch
    theta, target = _masks_on_device(engine, theta, target, in_place=False)
    b = theta.shape[0]
    cost = np.zeros(b)
    grad = torch.empty_like(theta) if want_gradient else None
    st = (stream or torch.cuda.current_stream(theta.device)).cuda_stream
    L.check(L.lib().huv_ilt_cost_grad(engine.handle, C.byref(settings._params()), b, theta.data_ptr(),
                                      target.data_ptr(), cost.ctypes.data,
                                      grad.data_ptr() if grad is not None else None, st))
    return cost, grad


def optimize(engine, theta, target, settings: IltSettings, stream=None):
    """Run the ILT stage loop on every mask; theta (a contiguous float32
    (B, N, N) CUDA tensor) is updated in place.
    Returns dict(final_cost, iterations, cost_history)."""
    import torch
    theta, target = _masks_on_device(engine, theta, target, in_place=True)
    b = theta.shape[0]
    fc = np.zeros(b)
    its = np.zeros(b, dtype=np.int32)
    hist = np.zeros((b, settings.max_iterations + 1))
    opt = L.IltOpt(settings.max_iterations, settings.learning_rate, settings.convergence_tol)
    st = (stream or torch.cuda.current_stream(theta.device)).cuda_stream
    L.check(L.lib().huv_ilt_optimize(engine.handle, C.byref(settings._params()), C.byref(opt), b,
                                     theta.data_ptr(), target.data_ptr(), fc.ctypes.data,
                                     its.ctypes.data, hist.ctypes.data, st))
    return {"final_cost": fc, "iterations": its, "cost_history": hist}
