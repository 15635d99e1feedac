"""FP64 CPU restatement of the reference's per-image imaging loop on pocketfft.

TEST INFRASTRUCTURE: the second timed CPU baseline series, never the product.

The same algorithm as ``oracle/socs_cpu.c`` (and the reference's
``socs_intensity``, crates/highuvlith-core/src/aerial.rs:1682-1721, with the
row-pruned inverse transform of math/fft2d.rs:166-170 and the normalisation
and flare of aerial.rs:1727-1748), with the FFTs done by ``scipy.fft``
(pocketfft, a mixed-radix FFT of the same class as the rustfft 6.4.1 the
reference calls) instead of the C port's radix-2 transform:

- the mask spectrum is the forward 2-D FFT of the raster times the separable
  pixel transfer sinc(pi m / N) (mask.rs:630-635, 804-815);
- kernels are processed in at most 16 fixed contiguous groups whose
  workspace stays under 256 MiB (aerial.rs:1690-1720); within a group the
  inverse transform runs along x on the band rows only, then along y on
  every column (on the transposed field, so the transforms run along
  contiguous rows), and lambda_k |E_k|^2 is accumulated in kernel order.

Images of a batch run concurrently on a thread pool (scipy.fft and numpy's
ufuncs release the GIL); each image's transforms use one worker, so the
whole batch uses ``threads`` host cores.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft


def _ptx(n: int) -> np.ndarray:
    m = np.fft.fftfreq(n, 1.0 / n)
    u = np.pi * m / n
    small = np.abs(u) < 1e-6
    return np.where(small, 1.0 - u * u / 6.0, np.sin(np.where(small, 1.0, u)) / np.where(small, 1.0, u))


class Prepared:
    """Kernel set laid out for the pruned transform: band rows, the support's
    (row slot, column) positions, values and eigenvalues."""

    def __init__(self, ks, normalization: str = "clear_field", flare: float = 0.0):
        n = ks.n
        self.n = n
        rows = np.unique(ks.support // n)
        self.rows = rows
        slot = {int(r): i for i, r in enumerate(rows)}
        self.slot = np.array([slot[int(s // n)] for s in ks.support], dtype=np.int64)
        self.col = (ks.support % n).astype(np.int64)
        self.support = ks.support
        self.values = ks.values
        self.eig = ks.eigenvalues
        d = ks.divisor(normalization)
        self.divisor = d if d else 1.0
        self.flare = flare
        self.ptx2 = np.outer(_ptx(n), _ptx(n))
        k = ks.values.shape[0]
        per_group = n * n * (8 + 16)
        groups = max(1, min(16, (256 << 20) // per_group, k))
        per = -(-k // groups)
        self.groups = [(g, min(g + per, k)) for g in range(0, k, per)]

    def image(self, raster: np.ndarray) -> np.ndarray:
        n = self.n
        spec = sfft.fft2(raster.astype(np.float64), workers=1) * self.ptx2
        ms = spec.reshape(-1)[self.support]
        acc_t = np.zeros((n, n))  # the image transposed, [x, y]
        nr = len(self.rows)
        full = np.zeros((n, n), dtype=np.complex128)
        for k0, k1 in self.groups:
            band = np.zeros((k1 - k0, nr, n), dtype=np.complex128)
            band[:, self.slot, self.col] = self.values[k0:k1] * ms[None, :]
            band = sfft.ifft(band, axis=-1, workers=1)  # pruned: band rows only
            for j in range(k1 - k0):
                # the column pass on the transposed field, so it runs along
                # contiguous rows; zero rows stay zero
                full[:, self.rows] = band[j].T
                e = sfft.ifft(full, axis=-1, workers=1)
                v = e.view(np.float64)
                v *= v
                acc_t += self.eig[k0 + j] * (v[:, 0::2] + v[:, 1::2])
        img = acc_t.T / self.divisor
        if self.flare > 0.0:
            img = img * (1.0 - self.flare) + self.flare * img.mean()
        return img


def images(prep: Prepared, rasters: np.ndarray, threads: int = 0, want_output: bool = True):
    """Images (B, N, N) of u8 rasters, FP64 inside, FP32 out; ``threads``
    images in flight at once (0: every host core)."""
    t = threads or os.cpu_count() or 1
    out = np.zeros(rasters.shape, dtype=np.float32) if want_output else None

    def one(i):
        img = prep.image(rasters[i])
        if out is not None:
            out[i] = img

    with ThreadPoolExecutor(max_workers=t) as pool:
        list(pool.map(one, range(rasters.shape[0])))
    return out
