"""ctypes driver of the C restatement (oracle/socs_cpu.c).

TEST INFRASTRUCTURE: the checker and the timed CPU baseline, never the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build_cpu import build

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.socs_cpu_batch.restype = C.c_int
        _lib.socs_cpu_batch.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]
    return _lib


def images(ks, rasters: np.ndarray, flare: float, pixel_transfer: bool = True, threads: int = 0,
           normalization: str = "clear_field", want_output: bool = True):
    """Images of uint8 rasters (B, n, n) with an oracle KernelSet, FP64 inside,
    FP32 out.  threads = 0 uses every host core."""
    r = np.ascontiguousarray(rasters, dtype=np.uint8)
    if r.ndim == 2:
        r = r[None]
    b, n = r.shape[0], r.shape[1]
    support = np.ascontiguousarray(ks.support, dtype=np.int64)
    vals = np.ascontiguousarray(ks.values, dtype=np.complex128)
    eig = np.ascontiguousarray(ks.eigenvalues, dtype=np.float64)
    d = ks.divisor(normalization) or 0.0
    out = np.zeros((b, n, n), dtype=np.float32) if want_output else None
    t = threads or os.cpu_count() or 1
    lib().socs_cpu_batch(n, b, r.ctypes.data, int(pixel_transfer), vals.shape[0], vals.shape[1], support.ctypes.data,
                         vals.ctypes.data, eig.ctypes.data, d, flare, t, out.ctypes.data if want_output else None)
    return out
