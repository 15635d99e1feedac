"""Pin the FP64 oracle to the reference's own known-answer tests.

Each test names the reference test or published number it reproduces
(paths relative to the reference checkout).
"""
import math

import numpy as np
import pytest

from oracle import hopkins as H
from oracle import metrics as M

PATTERN_2D = [(-64.0, 16.0, 96.0, 224.0), (24.0, -80.0, 176.0, 64.0), (120.0, 120.0, 48.0, 48.0)]


def _abbe_check(fill, optics, grid, ppa, zs, lam=100.0, tol=1e-8):
    eng = H.Engine(fill, optics, grid, lam, max_kernels=100000, points_per_axis=ppa)
    raster = H.paint_rects(grid, PATTERN_2D, dark_field=True)
    spec = H.spectrum_from_raster(raster)
    for z in zs:
        socs = eng.compute_from_spectrum(spec, z) * eng.clear_field_intensity(z)
        abbe = H.abbe_image(eng.points, optics, grid, spec, z, lam)
        err = np.max(np.abs(socs - abbe)) / np.max(abbe)
        assert err <= tol, (z, err)


def test_socs_equals_abbe_conventional():
    """crates/highuvlith-core/tests/imaging_validation.rs:222-238."""
    _abbe_check(H.fill_conventional(0.7), H.ProjectionOptics(0.5, flare_fraction=0.0),
                H.Grid(64, 8.0), 13, [0.0, 250.0, -400.0])


def test_socs_equals_abbe_annular_euv_obscured():
    """Same identity for an annular fill through an obscured EUV-style pupil
    (imaging_validation.rs:200-216 tolerance)."""
    _abbe_check(H.fill_annular(0.5, 0.9), H.EuvOptics(0.6, 0.2), H.Grid(64, 8.0), 15, [0.0, 150.0])


def test_clear_field_is_unity():
    """imaging_validation.rs:292-326: clear mask images to 1 +- 1e-12, and a
    truncated set stays within the dropped-trace bound."""
    optics = H.ProjectionOptics(0.5, flare_fraction=0.0)
    grid = H.Grid(32, 12.5)
    clear = H.Mask([], dark_field=False)
    for fill in (H.fill_conventional(0.7), H.fill_annular(0.5, 0.9)):
        exact = H.Engine(fill, optics, grid, 100.0, max_kernels=100000)
        trunc = H.Engine(fill, optics, grid, 100.0, max_kernels=6)
        for z in (0.0, 200.0, -1000.0):
            v = exact.compute(clear, z)
            assert np.max(np.abs(v - 1.0)) < 1e-12
            ks = trunc.kernel_set(z)
            kept = np.sum(ks.eigenvalues)
            dropped = (kept / ks.captured_energy_fraction - kept) / ks.clear_field
            vt = trunc.compute(clear, z)
            assert np.all(vt <= 1.0 + 1e-12) and np.all(1.0 - vt <= dropped + 1e-12)


def test_coherent_three_beam_closed_form():
    """analytical_validation.rs:228-293: coherent on-axis grating whose +-1
    orders pass the pupil images to |c0 + (c1 e^ix + c-1 e^-ix) e^{i phi(z)}|^2."""
    wl, na, pitch, pixel, periods = 100.0, 0.5, 300.0, 10.0, 4
    n = int(pitch * periods / pixel)
    grid = H.Grid(n, pixel)
    field = n * pixel
    rects = [(-field / 2 + (k + 0.5) * pitch, 0.0, pitch / 2, field) for k in range(periods)]
    raster = H.paint_rects(grid, rects, dark_field=False)
    spec = H.spectrum_from_raster(raster)
    optics = H.ProjectionOptics(na, flare_fraction=0.0)
    eng = H.Engine(H.fill_conventional(0.7), optics, grid, wl, points_per_axis=1)
    norm = float(n * n)
    c0, c1, cm1 = spec[0, 0] / norm, spec[0, periods] / norm, spec[0, n - periods] / norm
    for z in (0.0, 400.0, -900.0):
        phi = H.defocus_phase_in_medium(z, wl / pitch, 1.0, wl)
        tilt = complex(math.cos(phi), math.sin(phi))
        img = eng.compute_from_spectrum(spec, z)
        for j in range(n):
            x = 2.0 * math.pi * j / (n / periods)
            e = c0 + (c1 * complex(math.cos(x), math.sin(x)) + cm1 * complex(math.cos(x), -math.sin(x))) * tilt
            for i in (0, n // 3):
                assert abs(img[i, j] - abs(e) ** 2) < 1e-12


def test_readme_f2_line_space_published_numbers():
    """README.md:106,132,338-340: F2 157.63 nm, sigma 0.7, NA 0.75 (2 % flare),
    65/180 nm lines on the commensurate 256 grid, 20 kernels -> contrast 0.4545,
    printed CD 41.20 nm at I = 0.3, NILS 0.654."""
    g = H.commensurate_grid(180.0, 256, 1.0)
    eng = H.Engine(H.fill_conventional(0.7), H.ProjectionOptics(0.75), g, 157.63, max_kernels=20)
    img = eng.compute(H.Mask.line_space(65.0, 180.0))
    prof, x = list(M.centre_profile(img)), list(g.pixel_centres())
    assert round(M.image_contrast(img), 4) == 0.4545
    assert round(M.measure_cd_periodic(prof, x, 0.3, "dark"), 2) == 41.20
    assert round(M.nils_periodic(prof, x, 0.3, "dark"), 3) == 0.654


def test_sim_arf_published_cd_and_nils():
    """examples/sim_arf.toml:19: ArF NA 0.93 sigma 0.7, 80/160 nm, 128 x 2.5 nm
    -> printed CD 85.7 nm, NILS 1.32 (contrast printed as 0.412; the
    monochromatic image gives 0.4115)."""
    g = H.Grid(128, 2.5)
    eng = H.Engine(H.fill_conventional(0.7), H.ProjectionOptics(0.93), g, 193.368, max_kernels=20)
    img = eng.compute(H.Mask.line_space(80.0, 160.0))
    prof, x = list(M.centre_profile(img)), list(g.pixel_centres())
    assert round(M.measure_cd_periodic(prof, x, 0.3, "dark"), 1) == 85.7
    assert round(M.nils_periodic(prof, x, 0.3, "dark"), 2) == 1.32
    assert abs(M.image_contrast(img) - 0.412) < 1e-3


def test_mask_spectrum_identities():
    """mask.rs:1979 (clear DC = N^2), 2071 (pixel-aligned raster x pixel
    transfer == analytic spectrum), 2552 (line centred on the origin)."""
    g = H.Grid(64, 4.0)
    clear = H.Mask([], dark_field=False)
    assert abs(clear.spectrum(g)[0, 0] - 64 * 64) < 1e-9
    rect = H.Mask([("rect", 8.0, -12.0, 40.0, 24.0)], dark_field=True)
    ana = rect.spectrum(g)
    ras = H.spectrum_from_raster(rect.rasterize(g))
    assert np.max(np.abs(ana - ras)) / (64 * 64) < 1e-12
    # A line centred at x = 0 images symmetric about x = 0.
    eng = H.Engine(H.fill_conventional(0.5), H.ProjectionOptics(0.75, flare_fraction=0.0),
                   H.Grid(64, 4.0), 157.63, max_kernels=16)
    img = eng.compute(H.Mask([("rect", 0.0, 0.0, 40.0, 256.0)], dark_field=True))
    assert np.max(np.abs(img - img[:, ::-1])) < 1e-12


def test_source_sampling_properties():
    """aerial.rs:2220-2447: weights sum to 1, symmetric fills give mirror-
    symmetric point sets, typical sizes (sigma 0.7 disk ~1180 points,
    annulus 0.5-0.9 ~1310), second moments within 1 %."""
    for fill, n_expect, m2 in ((H.fill_conventional(0.7), 1180, 0.7 ** 2 / 4),
                               (H.fill_annular(0.5, 0.9), 1310, (0.9 ** 4 - 0.5 ** 4) / (4 * (0.9 ** 2 - 0.5 ** 2)))):
        pts = np.array(H.sample_source(fill, None, 1e-3))
        assert abs(np.sum(pts[:, 2]) - 1.0) < 1e-12
        assert abs(len(pts) - n_expect) < 0.1 * n_expect
        mx = np.sum(pts[:, 2] * pts[:, 0] ** 2)
        assert abs(mx - m2) / m2 < 0.01
        s = {(round(x, 12), round(y, 12)) for x, y, _ in pts}
        assert all((round(-x, 12), round(y, 12)) in s and (round(y, 12), round(x, 12)) in s for x, y, _ in pts)


def test_select_kernel_count_clusters():
    """aerial.rs:2541-2555: cuts never split a degenerate cluster."""
    vals = [4.0, 2.0, 2.0, 1.0, 0.5]
    assert H.select_kernel_count(vals, 9.5, 2, 1.0) == 1
    assert H.select_kernel_count(vals, 9.5, 3, 1.0) == 3
    assert H.select_kernel_count(vals, 9.5, 10, 0.5) == 3
    assert H.select_kernel_count([3.0, 3.0, 3.0], 9.0, 2, 1.0) == 3
    assert H.select_kernel_count([1.0, 1e-13], 1.0, 5, 1.0) == 1


def test_cd_cosine_fixture_closed_form():
    """metrics.rs:819-836 style fixture: a cosine profile I = a + b cos(2 pi x/P)
    has closed-form crossings; CD and NILS from the finder match them."""
    period, n, a, b, t = 200.0, 256, 0.5, 0.4, 0.3
    dx = period / n
    x = [-period / 2 + (j + 0.5) * dx for j in range(n)]
    prof = [a + b * math.cos(2 * math.pi * xi / period) for xi in x]
    # dark feature: I < t around x = +-P/2 ; edges where cos = (t - a)/b
    x_edge = period / (2 * math.pi) * math.acos((t - a) / b)
    cd_exact = period - 2 * x_edge
    slope = b * 2 * math.pi / period * math.sin(2 * math.pi * x_edge / period)
    nils_exact = cd_exact * slope / t
    cd = M.measure_cd_periodic(prof, x, t, "dark")
    assert abs(cd - cd_exact) < 2e-3
    assert abs(M.nils_periodic(prof, x, t, "dark") - nils_exact) / nils_exact < 1e-3


def test_union_spectrum_of_overlapping_pixel_aligned_rects_equals_raster_spectrum():
    """Pixel-transfer exactness (mask.rs:2071) extended to overlapping
    rectangles: the closed-form spectrum of the union's disjoint cells equals
    FFT(raster) x sinc x sinc when every edge sits on a pixel edge."""
    g = H.Grid(64, 1.0)
    rng = np.random.default_rng(0)
    rects, ras = [], np.zeros((64, 64))
    for _ in range(12):
        w, h = rng.integers(3, 20, 2)
        x0, y0 = rng.integers(0, 44, 2)
        rects.append((x0 - 32 + w / 2, y0 - 32 + h / 2, float(w), float(h)))
        ras[y0:y0 + h, x0:x0 + w] = 1
    a = H.rects_union_spectrum(rects, g)
    b = H.spectrum_from_raster(ras)
    assert np.max(np.abs(a - b)) < 1e-12 * np.max(np.abs(b))
    # a clear field with opaque features: background 1, feature 0
    c = H.rects_union_spectrum(rects, g, feature=0.0, background=1.0)
    d = H.spectrum_from_raster(1.0 - ras)
    assert np.max(np.abs(c - d)) < 1e-12 * np.max(np.abs(d))


def test_cpu_ports_match_the_numpy_oracle():
    """The two timed CPU restatements (the C port with its radix-2 FFT and
    the pocketfft series) image like oracle.hopkins, flare included."""
    from highuvlith_b200.clips import gen_batch
    from oracle import cpu, socs_scipy
    for fill, optics, lam, kmax in ((H.fill_conventional(0.5), H.euv_nxe_033(), 13.5, 16),
                                    (H.fill_dipole(0.8, 0.1, 0.0), H.ProjectionOptics(1.35, immersion_index=1.437),
                                     193.368, 12)):
        eng = H.Engine(fill, optics, H.Grid(128, 1.0), lam, max_kernels=kmax)
        ks = eng.kernel_set(0.0)
        _, r = gen_batch(2, 128, base_seed=31, wmin=4, wmax=24)
        a = cpu.images(ks, r, optics.flare)
        b = socs_scipy.images(socs_scipy.Prepared(ks, flare=optics.flare), r)
        for c in range(2):
            ref = eng.compute_from_spectrum(H.spectrum_from_raster(r[c]))
            assert np.max(np.abs(a[c] - ref)) / ref.max() < 1e-6
            assert np.max(np.abs(b[c] - ref)) / ref.max() < 1e-6
