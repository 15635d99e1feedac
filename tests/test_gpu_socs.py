"""Device SOCS path vs the FP64 oracle, through the C ABI.

Tolerance (stated by the task): max relative intensity error
max|I - I_ref| / max(I_ref) <= 1e-3 against the FP64 oracle, and edge
(CD) error <= 0.2 nm on every row and column cutline at I = 0.3.  The FP32
FFT path lands near 1e-6.
"""
import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200.clips import gen_batch
from oracle import hopkins as H
from oracle import metrics as M

pytestmark = pytest.mark.gpu

REL_TOL = 1e-3
CD_TOL_NM = 0.2


def _torch():
    import torch
    return torch


def rel_err(img, ref):
    return float(np.max(np.abs(img - ref)) / np.max(ref))


def _oracle_engine(fill, optics, grid, lam, kmax):
    return H.Engine(fill, optics, H.Grid(grid.size, grid.pixel_nm), lam, max_kernels=kmax)


SMALL = [
    # C1-like: ArF dry NA 0.93 annular 0.60/0.85, 2 nm pixels
    ("c1_64", HB.SourceConfig(193.368, "annular", (0.6, 0.85)), HB.OpticsConfig(0.93), HB.GridConfig(64, 2.0), 24,
     H.fill_annular(0.6, 0.85), H.ProjectionOptics(0.93)),
    # EUV NA 0.33 sigma 0.5 at 1 nm (C2 optics) on 128^2
    ("euv_128", HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(128, 1.0), 32,
     H.fill_conventional(0.5), H.euv_nxe_033()),
    # ArF immersion dipole (C3 source A)
    ("arfi_dipole_128", HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)), HB.OpticsConfig.immersion(1.35),
     HB.GridConfig(128, 1.0), 16, H.fill_dipole(0.8, 0.1, 0.0), H.ProjectionOptics(1.35, immersion_index=1.437)),
    # EUV quasar (C3 source B)
    ("euv_quasar_256", HB.SourceConfig(13.5, "quasar", (0.7, 0.9, 45.0)), HB.OpticsConfig.euv_nxe_033(),
     HB.GridConfig(256, 1.0), 48, H.fill_quasar(0.7, 0.9, 45.0), H.euv_nxe_033()),
]


@pytest.mark.parametrize("case", SMALL, ids=[c[0] for c in SMALL])
@pytest.mark.parametrize("eval_grid", ["full", "auto"])
def test_fft_form_matches_oracle(case, eval_grid):
    torch = _torch()
    _, src, opt, grid, kmax, fill, oopt = case
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax)
    oeng = _oracle_engine(fill, oopt, grid, src.wavelength_nm, kmax)
    n = grid.size
    rects, rasters = gen_batch(3, n, base_seed=11, wmin=max(2, n // 40), wmax=max(4, n // 8), dmin=0.2, dmax=0.6)
    d = torch.from_numpy(rasters).cuda()
    eg = n if eval_grid == "full" else 0
    for z in (0.0, 40.0):
        out = eng.compute_batch(d, focus_nm=z, pixel_transfer=True, form="fft", eval_grid=eg).cpu().numpy()
        for c in range(3):
            ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]), z)
            assert rel_err(out[c], ref) < 1e-5, (c, z, rel_err(out[c], ref))


def test_transmittance_inputs_agree():
    """u8, f32 and complex64 rasters image alike; pixel_transfer=0 is
    compute_from_transmittance (plain FFT spectrum).  u8 rows take the exact
    integer tensor-core band, f32 / complex64 rows the FP32 FFT."""
    torch = _torch()
    src, opt, grid = HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(128, 1.0)
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=16)
    oeng = _oracle_engine(H.fill_conventional(0.5), H.euv_nxe_033(), grid, 13.5, 16)
    _, rasters = gen_batch(2, 128, base_seed=3, wmin=4, wmax=20)
    u8 = torch.from_numpy(rasters).cuda()
    f32 = u8.float()
    c64 = f32.to(torch.complex64)
    a = eng.compute_batch(u8, pixel_transfer=False, form="fft")
    b = eng.compute_batch(f32, pixel_transfer=False, form="fft")
    c = eng.compute_batch(c64, pixel_transfer=False, form="fft")
    assert torch.max(torch.abs(a - b)).item() < 5e-6 * torch.max(a).item()
    assert torch.max(torch.abs(b - c)).item() < 1e-6 * torch.max(a).item()
    ref = oeng.compute_from_transmittance(rasters[0])
    assert rel_err(a[0].cpu().numpy(), ref) < 1e-5
    # complex transmittance (attenuated PSM-like) through the host entry point
    t = np.where(rasters[1] > 0, 1.0 + 0j, 0.245 * np.exp(1j * np.pi))
    res = eng.compute_from_transmittance(t)
    assert isinstance(res, HB.AerialImageResult) and res.shape == (128, 128)
    assert rel_err(res.intensity, oeng.compute_from_transmittance(t)) < 1e-5


@pytest.mark.parametrize("form", ["fft", "tc"])
def test_u8_levels_tensor_rows_match_fft_rows_and_oracle(form, monkeypatch):
    """Grey-level u8 rasters (0..255, not only 0/1): the exact integer
    tensor-core row band against the FP32 FFT rows (HUV_MASK_ROWS=fft) and
    the FP64 oracle, at several grid sizes."""
    torch = _torch()
    src, opt = HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033()
    rng = np.random.default_rng(21)
    for n, kmax in ((128, 16), (256, 24), (512, 24)):
        grid = HB.GridConfig(n, 1.0)
        rasters = rng.integers(0, 256, size=(3, n, n), dtype=np.uint8)
        rasters[1] = (rasters[1] > 127).astype(np.uint8)  # a binary one
        rasters[2] = 255  # a clear field at full scale
        d = torch.from_numpy(rasters).cuda()
        monkeypatch.delenv("HUV_MASK_ROWS", raising=False)
        a = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax).compute_batch(d, form=form)
        monkeypatch.setenv("HUV_MASK_ROWS", "fft")
        b = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax).compute_batch(d, form=form)
        monkeypatch.delenv("HUV_MASK_ROWS")
        a, b = a.cpu().numpy(), b.cpu().numpy()
        oeng = _oracle_engine(H.fill_conventional(0.5), H.euv_nxe_033(), grid, 13.5, kmax)
        # the TC form's split-BF16 GEMMs round at ~1e-5, so a 1e-7 change of
        # the mask band moves its image by up to that much
        tol_ab = 5e-6 if form == "fft" else 3e-5
        for c in range(3):
            assert rel_err(a[c], b[c]) < tol_ab, (n, c, rel_err(a[c], b[c]))
            if n <= 256:
                ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]), 0.0)
                tol = 1e-5 if form == "fft" else 5e-5
                assert rel_err(a[c], ref) < tol, (n, c, rel_err(a[c], ref))


@pytest.mark.parametrize("form", ["fft", "hybrid"])
@pytest.mark.parametrize("eval_grid", [160, 192])
def test_mixed_radix_eval_grids_match_oracle(form, eval_grid):
    """Evaluation on the mixed-radix 160 (16 x 10) and 192 (16 x 12) point
    grids, requested explicitly, against the FP64 oracle on the full grid."""
    torch = _torch()
    case = SMALL[3]  # EUV quasar on 256^2
    _, src, opt, grid, kmax, fill, oopt = case
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax)
    oeng = _oracle_engine(fill, oopt, grid, src.wavelength_nm, kmax)
    n = grid.size
    _, rasters = gen_batch(3, n, base_seed=17, wmin=6, wmax=32, dmin=0.2, dmax=0.6)
    d = torch.from_numpy(rasters).cuda()
    out = eng.compute_batch(d, form=form, eval_grid=eval_grid).cpu().numpy()
    tol = 1e-5 if form == "fft" else 1e-4
    for c in range(3):
        ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]))
        assert rel_err(out[c], ref) < tol, (c, rel_err(out[c], ref))


@pytest.mark.parametrize("normalization", ["clear_field", "absolute"])
def test_hybrid_fp16_planes_on_extreme_clips(normalization):
    """The separable interpolation carries I / (16 mean) in FP16 planes: a
    lone contact in a dark field (peak far above the mean), an opaque clip
    (mean 0: the image must stay exactly 0), a clear clip and a random clip,
    under both normalisations, against the FP32 FFT form and the oracle."""
    torch = _torch()
    _, src, opt, grid, kmax, fill, oopt = SMALL[3]  # EUV quasar on 256^2
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax, normalization=normalization)
    n = grid.size
    clips = np.zeros((4, n, n), np.uint8)
    clips[0, n // 2 - 4:n // 2 + 4, n // 2 - 4:n // 2 + 4] = 1  # one 8 x 8 contact
    clips[2] = 1
    _, rnd = gen_batch(1, n, base_seed=29, wmin=6, wmax=32, dmin=0.2, dmax=0.6)
    clips[3] = rnd[0]
    d = torch.from_numpy(clips).cuda()
    hyb = eng.compute_batch(d, form="hybrid", eval_grid=160).cpu().numpy()
    fft = eng.compute_batch(d, form="fft", eval_grid=160).cpu().numpy()
    assert np.all(np.isfinite(hyb))
    assert np.max(np.abs(hyb[1])) == 0.0
    for c in (0, 2, 3):
        assert rel_err(hyb[c], fft[c]) < 2e-5, (c, rel_err(hyb[c], fft[c]))
    assert np.max(hyb[0]) / max(float(np.mean(hyb[0])), 1e-30) > 50  # the dark-field case is one
    if normalization == "clear_field":  # (a truncated kernel set images a clear clip slightly below 1)
        oeng = _oracle_engine(fill, oopt, grid, src.wavelength_nm, kmax)
        for c in (0, 2):
            ref = oeng.compute_from_spectrum(H.spectrum_from_raster(clips[c]))
            assert rel_err(hyb[c], ref) < 1e-4, (c, rel_err(hyb[c], ref))


def test_clear_and_dark_masks():
    """Clear mask images to 1 (flare keeps it 1); an opaque mask to 0."""
    torch = _torch()
    eng = HB.SimulationEngine(HB.SourceConfig.arf_laser(0.7), HB.OpticsConfig(0.93), grid=HB.GridConfig(64, 2.0),
                              max_kernels=100000)
    ones = torch.ones((1, 64, 64), dtype=torch.uint8, device="cuda")
    zeros = torch.zeros((1, 64, 64), dtype=torch.uint8, device="cuda")
    assert torch.max(torch.abs(eng.compute_batch(ones, form="fft") - 1.0)).item() < 1e-5
    assert torch.max(torch.abs(eng.compute_batch(zeros, form="fft"))).item() == 0.0
    empty = torch.zeros((0, 64, 64), dtype=torch.uint8, device="cuda")
    assert eng.compute_batch(empty, form="fft").shape == (0, 64, 64)


def test_deterministic_run_to_run():
    torch = _torch()
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(256, 1.0),
                              max_kernels=32)
    _, rasters = gen_batch(4, 256, base_seed=7, wmin=5, wmax=40)
    d = torch.from_numpy(rasters).cuda()
    a = eng.compute_batch(d, form="fft").clone()
    b = eng.compute_batch(d, form="fft")
    assert torch.equal(a, b)


def test_rasterizer_matches_numpy():
    torch = _torch()
    rects, rasters = gen_batch(5, 256, base_seed=99, wmin=10, wmax=80)
    dev = HB.rasterize_rects(256, rects, dark_field=True)
    assert torch.equal(dev.cpu(), torch.from_numpy(rasters))
    bright = HB.rasterize_rects(256, rects[:2], dark_field=False)
    assert torch.equal(bright.cpu(), torch.from_numpy(1 - rasters[:2]))


def test_rasterizer_matches_oracle_paint_rects():
    """huv_rasterize_rects against the oracle's painter's-rule raster
    (Mask::rasterize, mask.rs:1717-1741) for pixel-aligned rectangles, some
    of them running past the field edge, on both field tones and at 2 nm
    pixels."""
    torch = _torch()
    n = 256
    rects, _ = gen_batch(3, n, base_seed=123, wmin=6, wmax=70)
    rects[1] = rects[1] + [(-20, 40, 50, 30), (230, 200, 60, 90), (100, -10, 12, 300)]
    for pixel in (1.0, 2.0):
        g = H.Grid(n, pixel)
        for dark in (True, False):
            dev = HB.rasterize_rects(n, rects, dark_field=dark).cpu().numpy()
            for c, clip in enumerate(rects):
                nm = [((x0 + w / 2.0) * pixel - n * pixel / 2.0, (y0 + h / 2.0) * pixel - n * pixel / 2.0,
                       w * pixel, h * pixel) for x0, y0, w, h in clip]
                ref = H.paint_rects(g, nm, dark_field=dark)
                assert np.array_equal(ref.imag, np.zeros_like(ref.imag))
                assert np.array_equal(dev[c], ref.real.astype(np.uint8)), (pixel, dark, c)


def test_c2_clips_full_size_parity_and_cd():
    """C2 (EUV NA 0.33, sigma 0.5, K = 32 requested, 1024^2 at 1 nm): seeded
    Manhattan clips; max relative error and CD (edge) error vs the FP64
    oracle on every row/column cutline at I = 0.3."""
    torch = _torch()
    grid = HB.GridConfig(1024, 1.0)
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=grid, max_kernels=32)
    oeng = _oracle_engine(H.fill_conventional(0.5), H.euv_nxe_033(), grid, 13.5, 32)
    _, rasters = gen_batch(2, 1024, base_seed=2026)
    d = torch.from_numpy(rasters).cuda()
    x = grid.pixel_centres()
    for eg in (1024, 0):
        out = eng.compute_batch(d, form="fft", eval_grid=eg).cpu().numpy()
        for c in range(2):
            ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]))
            assert rel_err(out[c], ref) < REL_TOL
            if c == 0:
                sub = slice(0, 1024, 16)
                worst, unmatched = M.max_edge_error(out[c][sub], ref[sub], x, 0.3)
                assert unmatched == 0 and worst < CD_TOL_NM, (worst, unmatched)


TC_CASES = [c for c in SMALL if c[3].size >= 128]


@pytest.mark.parametrize("form", ["tc", "tc_rows", "hybrid"])
@pytest.mark.parametrize("case", TC_CASES, ids=[c[0] for c in TC_CASES])
def test_tc_form_matches_oracle(case, form):
    """Split-BF16x3 tcgen05 form vs the FP64 oracle (tolerance 1e-3; the
    split products carry ~2^-16 relative precision); row transforms as FFTs
    ("tc"), as tensor-core DFT-GEMMs too ("tc_rows"), or the FP32 FFT field
    pass with only the band interpolation on tensor cores ("hybrid")."""
    torch = _torch()
    _, src, opt, grid, kmax, fill, oopt = case
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax)
    oeng = _oracle_engine(fill, oopt, grid, src.wavelength_nm, kmax)
    n = grid.size
    _, rasters = gen_batch(3, n, base_seed=13, wmin=max(2, n // 40), wmax=max(4, n // 8), dmin=0.2, dmax=0.6)
    d = torch.from_numpy(rasters).cuda()
    out = eng.compute_batch(d, form=form).cpu().numpy()
    eng.device_status()
    for c in range(3):
        ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]))
        assert rel_err(out[c], ref) < 1e-4, (c, rel_err(out[c], ref))


def test_tc_form_c2_full_size():
    """C2 at full size through the tensor-core form: parity and CD error."""
    torch = _torch()
    grid = HB.GridConfig(1024, 1.0)
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=grid, max_kernels=32)
    oeng = _oracle_engine(H.fill_conventional(0.5), H.euv_nxe_033(), grid, 13.5, 32)
    _, rasters = gen_batch(3, 1024, base_seed=2026)
    d = torch.from_numpy(rasters).cuda()
    out = eng.compute_batch(d, form="tc").cpu().numpy()
    eng.device_status()
    fft = eng.compute_batch(d, form="fft").cpu().numpy()
    hyb = eng.compute_batch(d).cpu().numpy()  # auto: the hybrid form
    x = grid.pixel_centres()
    for c in range(3):
        ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]))
        assert rel_err(out[c], ref) < REL_TOL
        assert rel_err(out[c], fft[c]) < REL_TOL
        assert rel_err(hyb[c], ref) < 1e-4, rel_err(hyb[c], ref)
    worst, unmatched = M.max_edge_error(out[0], oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[0])), x, 0.3)
    assert unmatched == 0 and worst < CD_TOL_NM, (worst, unmatched)


@pytest.mark.parametrize("form", ["fft", "hybrid"])
def test_fused_field_pass_matches_oracle(form, monkeypatch):
    """The fused field-pass kernel (HUV_FIELD_PASS=fused: row and column
    transforms of each kernel in one CTA) on the 160- and 128-point grids,
    narrow bands included (ArF dipole, B = 7, whose output staging is larger
    than its working set), one and several kernel groups (K <= 8 and K > 8),
    against the FP64 oracle."""
    torch = _torch()
    monkeypatch.setenv("HUV_FIELD_PASS", "fused")
    cases = [(SMALL[1], 128, 8), (SMALL[2], 128, 16), (SMALL[3], 160, 48), (SMALL[3], 128, 12)]
    for (name, src, opt, grid, _, fill, oopt), eg, kmax in cases:
        eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax)
        oeng = _oracle_engine(fill, oopt, grid, src.wavelength_nm, kmax)
        n = grid.size
        if 4 * eng.imaging_diagnostics()["band_half_width"] >= eg:
            continue
        _, rasters = gen_batch(3, n, base_seed=61, wmin=max(2, n // 40), wmax=max(4, n // 8), dmin=0.2, dmax=0.6)
        out = eng.compute_batch(torch.from_numpy(rasters).cuda(), form=form, eval_grid=eg).cpu().numpy()
        for c in range(3):
            ref = oeng.compute_from_spectrum(H.spectrum_from_raster(rasters[c]))
            tol = 1e-5 if form == "fft" else 1e-4
            assert rel_err(out[c], ref) < tol, (name, eg, kmax, c, rel_err(out[c], ref))
