"""The separable band interpolation the hybrid form runs on tensor cores,
checked in FP64 on the CPU: an intensity whose spectrum lies in |f| <= 2h
per axis, sampled on any grid of M > 4h points, is reproduced exactly on the
N-point grid by I_N = P I_M P^T with the real Dirichlet matrix

    P(Y, m) = (1/M) sum_{|f| <= 2h} exp(2 pi i f (Y/N - m/M))
            = sin((4h + 1) pi t) / (M sin(pi t)),  t = Y/N - m/M,

the closed form the engine builds on the host.  The intensities are sums of
|E_k|^2 over random fields band-limited to |f| <= h (the SOCS structure)."""
import numpy as np
import pytest


def dirichlet_matrix(n: int, m: int, h2: int) -> np.ndarray:
    y = np.arange(n)[:, None].astype(np.int64)
    c = np.arange(m)[None, :].astype(np.int64)
    q = y * m - c * n  # t = q / (n m), |q| < n m
    t = q / float(n * m)
    with np.errstate(invalid="ignore", divide="ignore"):
        p = np.where(q == 0, float(2 * h2 + 1), np.sin((2 * h2 + 1) * np.pi * t) / np.sin(np.pi * t))
    return p / m


def band_limited_intensity(n: int, h: int, k: int, seed: int) -> np.ndarray:
    """sum_k |E_k|^2 on the n x n grid, E_k with random orders |f| <= h."""
    rng = np.random.default_rng(seed)
    f = np.fft.fftfreq(n, 1.0 / n)
    band = (np.abs(f)[:, None] <= h) & (np.abs(f)[None, :] <= h)
    out = np.zeros((n, n))
    for j in range(k):
        s = np.zeros((n, n), complex)
        s[band] = (rng.normal(size=band.sum()) + 1j * rng.normal(size=band.sum())) / (1 + j)
        out += np.abs(np.fft.ifft2(s) * n * n) ** 2
    return out / out.max()


def resample(img: np.ndarray, m: int, h2: int) -> np.ndarray:
    """The band-limited image at the m x m grid points Y = j n / m, from its
    Fourier series (orders |f| <= h2)."""
    n = img.shape[0]
    c = np.fft.fft2(img) / (n * n)
    f = np.fft.fftfreq(n, 1.0 / n).astype(int)
    keep = np.abs(f) <= h2
    fk = f[keep]
    ck = c[np.ix_(keep, keep)]
    e = np.exp(2j * np.pi * np.outer(np.arange(m), fk) / m)  # [m][f]
    return np.real(e @ ck @ e.T)


@pytest.mark.parametrize("n,h,m", [(256, 9, 40), (256, 9, 64), (1024, 37, 160), (1024, 37, 192)])
def test_dirichlet_matrix_interpolates_band_limited_intensity_exactly(n, h, m):
    assert m > 4 * h
    img = band_limited_intensity(n, h, k=6, seed=n + m)
    p = dirichlet_matrix(n, m, 2 * h)
    coarse = resample(img, m, 2 * h)
    rebuilt = p @ coarse @ p.T
    assert np.max(np.abs(rebuilt - img)) < 1e-11


def test_dirichlet_rows_sum_to_one():
    """A constant (the flare term) passes unchanged: each row of P sums to 1
    (only the f = 0 order survives the sum over m)."""
    for n, m, h2 in ((1024, 160, 74), (1024, 192, 94), (256, 40, 18)):
        p = dirichlet_matrix(n, m, h2)
        assert np.max(np.abs(p.sum(axis=1) - 1.0)) < 1e-12
