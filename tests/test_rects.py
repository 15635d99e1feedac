"""Exact analytic spectrum of rectangle clips on the device (Mask::spectrum,
mask.rs:616-657, 1439-1503; overlaps resolved like compress, mask.rs:1365-1437)
against the FP64 oracle, and against the raster path where both are exact."""
import numpy as np
import pytest

import highuvlith_b200 as HB
from oracle import hopkins as H

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _engine(n=128, kmax=24):
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(n, 1.0),
                              max_kernels=kmax)
    oeng = H.Engine(H.fill_conventional(0.5), H.euv_nxe_033(), H.Grid(n, 1.0), 13.5, max_kernels=kmax)
    return eng, oeng


def _random_clip(rng, n, count, subpixel):
    out = []
    for _ in range(count):
        w, h = rng.uniform(4, 30, 2) if subpixel else rng.integers(4, 30, 2).astype(float)
        x, y = rng.uniform(-n / 2 + 16, n / 2 - 16, 2) if subpixel else rng.integers(-n // 2 + 16, n // 2 - 16, 2)
        if not subpixel:  # corners on pixel edges
            x, y = x + (w % 2) / 2.0, y + (h % 2) / 2.0
        out.append((float(x), float(y), float(w), float(h)))
    return out


@pytest.mark.parametrize("form", ["fft", "tc"])
def test_pixel_aligned_rects_match_raster_path(form):
    import torch
    n = 128
    eng, _ = _engine(n)
    rng = np.random.default_rng(1)
    clips = [_random_clip(rng, n, 15, False) for _ in range(3)]
    ras = np.zeros((3, n, n), dtype=np.uint8)
    for c, clip in enumerate(clips):
        for x, y, w, h in clip:
            x0, y0 = int(round(x - w / 2 + n / 2)), int(round(y - h / 2 + n / 2))
            assert 0 <= x0 and x0 + int(w) <= n and 0 <= y0 and y0 + int(h) <= n
            ras[c, y0:y0 + int(h), x0:x0 + int(w)] = 1
    a = eng.compute_batch_rects(clips, form=form).cpu().numpy()
    b = eng.compute_batch(torch.from_numpy(ras).cuda(), form=form).cpu().numpy()
    tol = 2e-6 if form == "fft" else 2e-5  # the TC form carries ~1e-5 of split-BF16 rounding
    for c in range(3):
        assert _rel(a[c], b[c]) < tol, (c, _rel(a[c], b[c]))


@pytest.mark.parametrize("form,tol", [("fft", 1e-5), ("tc", 1e-3)])
def test_subpixel_overlapping_rects_match_oracle(form, tol):
    n = 128
    eng, oeng = _engine(n)
    rng = np.random.default_rng(2)
    clips = [_random_clip(rng, n, 20, True) for _ in range(3)]
    out = eng.compute_batch_rects(clips, form=form).cpu().numpy()
    for c, clip in enumerate(clips):
        ref = oeng.compute_from_spectrum(H.rects_union_spectrum(clip, H.Grid(n, 1.0)))
        assert _rel(out[c], ref) < tol, (c, _rel(out[c], ref))


def test_attenuated_clear_field_and_host_path():
    """Opaque-feature clear field with an attenuated-PSM absorber amplitude
    (0.245 at phase pi), at a defocus plane; host-buffer call == device call."""
    n = 128
    eng, oeng = _engine(n)
    rng = np.random.default_rng(3)
    clips = [_random_clip(rng, n, 10, True) for _ in range(5)] + [[]]
    feat = 0.245 * np.exp(1j * np.pi)
    dev = eng.compute_batch_rects(clips, feature=feat, background=1.0, focus_nm=40.0, form="fft").cpu().numpy()
    host = eng.compute_batch_rects_host(clips, feature=feat, background=1.0, focus_nm=40.0, form="fft")
    np.testing.assert_array_equal(dev, host)
    for c, clip in enumerate(clips):
        spec = H.rects_union_spectrum(clip, H.Grid(n, 1.0), feature=feat, background=1.0)
        ref = oeng.compute_from_spectrum(spec, 40.0)
        assert _rel(dev[c], ref) < 1e-5, (c, _rel(dev[c], ref))
    # the empty clip images uniformly (the truncated clear field, checked
    # against the oracle above)
    assert np.ptp(dev[-1]) < 1e-6


def test_rect_input_rejects_bad_tables():
    import ctypes as C
    from highuvlith_b200 import _lib as L
    eng, _ = _engine(64, 8)
    with pytest.raises(HB.HuvError):
        eng.compute_batch_rects([[(0.0, 0.0, -5.0, 3.0)]])
    offs = np.array([0, 2, 1], dtype=np.int32)
    rects = np.zeros((2, 4))
    view = L.RectClips(rects.ctypes.data, offs.ctypes.data, 1.0, 0.0, 0.0, 0.0)
    b = L.Batch(2, L.INPUT_RECTS, C.addressof(view), 0, 0.0, 0, 0)
    import torch
    out = torch.empty((2, 64, 64), device="cuda")
    assert L.lib().huv_image_batch(eng.handle, C.byref(b), out.data_ptr(), None) == 1


@pytest.mark.parametrize("form,tol", [("fft", 1e-5), ("tc", 1e-3)])
def test_c1_line_space_on_incommensurate_field(form, tol):
    """C1: ArF dry 193.368 nm, NA 0.93, annular 0.60/0.85, K = 24, 256^2 at
    2 nm, 65 nm opaque lines on a 130 nm pitch (512 / 130 = 3.94 periods, so
    the grating is truncated at the field edge) -- exact spectrum vs the
    oracle's Mask.line_space, and the printed CD."""
    from oracle import metrics as M
    n, p = 256, 2.0
    eng = HB.SimulationEngine(HB.SourceConfig.arf_laser(0.7).with_illumination("annular", 0.6, 0.85),
                              HB.OpticsConfig(0.93), grid=HB.GridConfig(n, p), max_kernels=24)
    oeng = H.Engine(H.fill_annular(0.6, 0.85), H.ProjectionOptics(0.93), H.Grid(n, p), 193.368, max_kernels=24)
    half = n * p / 2
    lines = [(c, 0.0, 65.0, 2 * n * p) for c in np.arange(-130.0 * 3, 130.0 * 4, 130.0) if abs(c) < half + 65]
    img = eng.compute_batch_rects([lines], feature=0.0, background=1.0, form=form).cpu().numpy()[0]
    ref = oeng.compute(H.Mask.line_space(65.0, 130.0))
    assert _rel(img, ref) < tol, _rel(img, ref)
    x = -half + (np.arange(n) + 0.5) * p
    cd = M.measure_cd_periodic(list(M.centre_profile(img)), list(x), 0.3, "dark")
    cd_ref = M.measure_cd_periodic(list(M.centre_profile(ref)), list(x), 0.3, "dark")
    assert cd is not None and abs(cd - cd_ref) < 0.2
