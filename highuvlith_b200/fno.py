"""FNO surrogate of the aerial image (device kernels in csrc/cuda/fno.cu).

A 4-layer Fourier neural operator (width 64, 16 x 16 retained modes, GELU)
mapping a transmittance map to the normalised aerial image, trained on the
GPU on image pairs that the SOCS engine itself produces.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class FnoSurrogate:
    def __init__(self, grid: int = 512, modes: int = 16, layers: int = 4, width: int = 64, proj: int = 128,
                 seed: int = 2026, device: int = 0):
        self.grid, self.modes, self.layers = grid, modes, layers
        h = C.c_void_p()
        L.check(L.lib().huv_fno_create(grid, width, modes, layers, proj, seed, device, C.byref(h)))
        self._h = h
        self._destroy = L.lib().huv_fno_destroy

    def __del__(self):
        # The destroy function is bound at construction: at interpreter exit
        # module globals may already be gone.
        h, destroy = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and destroy is not None:
            destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h.value

    def num_params(self) -> int:
        n = C.c_int64()
        L.check(L.lib().huv_fno_params(self._h, None, 0, C.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        n = self.num_params()
        out = np.zeros(n, dtype=np.float32)
        L.check(L.lib().huv_fno_params(self._h, out.ctypes.data, n, None))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        L.check(L.lib().huv_fno_set_params(self._h, p.ctypes.data, p.size))

    def save(self, path: str) -> None:
        np.savez(path, params=self.get_params(), grid=self.grid, modes=self.modes, layers=self.layers)

    def load(self, path: str) -> None:
        self.set_params(np.load(path)["params"])

    def _maps(self, t, name: str):
        """A (B, grid, grid) float32 contiguous CUDA copy (or the tensor itself)."""
        g = self.grid
        if t.dim() != 3 or tuple(t.shape[1:]) != (g, g) or not t.is_cuda:
            raise ValueError(f"{name} must be a (B, {g}, {g}) CUDA tensor")
        return t.float().contiguous()

    def forward(self, masks, out=None, stream=None):
        import torch
        masks = self._maps(masks, "masks")
        if out is None:
            out = torch.empty_like(masks)
        elif (out.dtype != torch.float32 or out.device != masks.device or not out.is_contiguous()
              or tuple(out.shape) != tuple(masks.shape)):
            raise ValueError(f"out must be a contiguous float32 {tuple(masks.shape)} tensor on {masks.device}")
        st = (stream or torch.cuda.current_stream()).cuda_stream
        L.check(L.lib().huv_fno_forward(self._h, masks.shape[0], masks.data_ptr(), out.data_ptr(), st))
        return out

    def device_status(self, stream=None) -> None:
        """Synchronise the stream; raises HuvError (DEVICE_TIMEOUT) if a bounded
        device-side wait of an earlier forward gave up (its images are then not
        valid).  backward and train_step check this themselves."""
        import torch
        st = (stream or torch.cuda.current_stream()).cuda_stream
        L.check(L.lib().huv_fno_device_status(self._h, st))

    def backward(self, masks, targets=None, dout=None, want_param_grad=True, want_input_grad=False, stream=None):
        import torch
        masks = self._maps(masks, "masks")
        targets = self._maps(targets, "targets") if targets is not None else None
        dout = self._maps(dout, "dout") if dout is not None else None
        for name, t in (("targets", targets), ("dout", dout)):
            if t is not None and tuple(t.shape) != tuple(masks.shape):
                raise ValueError(f"{name} must have the masks' shape {tuple(masks.shape)}")
        pg = torch.empty(self.num_params(), dtype=torch.float32, device=masks.device) if want_param_grad else None
        dm = torch.empty_like(masks) if want_input_grad else None
        loss = C.c_float(0.0)
        st = (stream or torch.cuda.current_stream()).cuda_stream
        L.check(L.lib().huv_fno_backward(self._h, masks.shape[0], masks.data_ptr(),
                                         targets.data_ptr() if targets is not None else None,
                                         dout.data_ptr() if dout is not None else None,
                                         pg.data_ptr() if pg is not None else None,
                                         dm.data_ptr() if dm is not None else None, C.byref(loss), st))
        return loss.value, pg, dm

    def train_step(self, masks, targets, lr: float = 1e-3, weight_decay: float = 0.0, stream=None) -> float:
        import torch
        masks, targets = self._maps(masks, "masks"), self._maps(targets, "targets")
        if tuple(targets.shape) != tuple(masks.shape):
            raise ValueError(f"targets must have the masks' shape {tuple(masks.shape)}")
        loss = C.c_float(0.0)
        st = (stream or torch.cuda.current_stream()).cuda_stream
        L.check(L.lib().huv_fno_train_step(self._h, masks.shape[0], masks.data_ptr(),
                                           targets.data_ptr(), lr, weight_decay, C.byref(loss), st))
        return loss.value
