"""Through-focus imaging (compute_through_focus, aerial.rs:1820-1825;
process::batch_defocus, process.rs:1303-1313) against the FP64 oracle at
every plane, and against per-plane single calls."""
import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200.clips import gen_batch
from oracle import hopkins as H

pytestmark = pytest.mark.gpu

FOCUS = [-150.0, -50.0, 0.0, 37.5, 120.0]


def _rel(img, ref):
    return float(np.max(np.abs(img - ref)) / np.max(ref))


@pytest.mark.parametrize("form", ["fft", "tc"])
def test_focus_sweep_matches_oracle_every_plane(form):
    import torch
    n = 256
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.7), HB.OpticsConfig.euv_nxe_033(),
                              grid=HB.GridConfig(n, 1.0), max_kernels=20)
    oeng = H.Engine(H.fill_conventional(0.7), H.euv_nxe_033(), H.Grid(n, 1.0), 13.5, max_kernels=20)
    _, rasters = gen_batch(3, n, base_seed=31, wmin=8, wmax=40, dmin=0.2, dmax=0.6)
    d = torch.from_numpy(rasters).cuda()
    out = eng.compute_batch_through_focus(d, FOCUS, form=form).cpu().numpy()
    assert out.shape == (len(FOCUS), 3, n, n)
    tol = 1e-5 if form == "fft" else 1e-3
    for p, z in enumerate(FOCUS):
        for c in range(3):
            ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]), z)
            assert _rel(out[p, c], ref) < tol, (z, c, _rel(out[p, c], ref))
    # identical to imaging each plane on its own (same kernels, same path)
    for p, z in enumerate(FOCUS):
        one = eng.compute_batch(d, focus_nm=z, form=form).cpu().numpy()
        np.testing.assert_array_equal(out[p], one)


def test_through_focus_single_mask_api():
    eng = HB.SimulationEngine(HB.SourceConfig.f2_laser(0.7), HB.OpticsConfig(0.75),
                              mask=HB.MaskConfig(rects=[(x0, 0, 32, 256) for x0 in (10, 100, 190)], dark_field=False),
                              grid=HB.GridConfig(256, 2.0), max_kernels=20)
    imgs = eng.compute_through_focus([-100.0, 0.0, 100.0])
    assert len(imgs) == 3
    for z, img in zip([-100.0, 0.0, 100.0], imgs):
        np.testing.assert_allclose(img, eng.compute_aerial_image(z), rtol=0, atol=1e-6)
    # defocus is symmetric for an aberration-free pupil
    np.testing.assert_allclose(imgs[0], imgs[2], atol=1e-4)


def test_focus_sweep_rejects_bad_planes():
    import torch
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(64, 1.0),
                              max_kernels=8)
    d = torch.zeros((1, 64, 64), dtype=torch.uint8, device="cuda")
    with pytest.raises(HB.HuvError):
        eng.compute_batch_through_focus(d, [0.0, float("nan")])
