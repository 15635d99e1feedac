"""Host FP64 half of the engine (source sampling, pupils, kernel build)
checked against the oracle on the CPU, and the C ABI surface."""
import ctypes
import os
import re

import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200 import _lib
from oracle import hopkins as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    """Every function declared in include/huv_b200.h is exported by the .so."""
    hdr = open(os.path.join(ROOT, "include", "huv_b200.h")).read()
    declared = set(re.findall(r"\b(huv_[a-z0-9_]+)\s*\(", hdr))
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [d for d in declared if not hasattr(lib, d)]
    assert not missing, missing
    assert declared <= set(_lib.SIGNATURES), declared - set(_lib.SIGNATURES)


FILLS = [
    ("conventional", (0.7,), H.fill_conventional(0.7)),
    ("annular", (0.6, 0.85), H.fill_annular(0.6, 0.85)),
    ("dipole", (0.8, 0.1, 0.0), H.fill_dipole(0.8, 0.1, 0.0)),
    ("quasar", (0.7, 0.9, 45.0), H.fill_quasar(0.7, 0.9, 45.0)),
    ("gaussian", (0.05,), H.fill_gaussian(0.05)),
    ("quadrupole", (0.7, 0.15, 30.0), H.fill_quadrupole(0.7, 0.15, 30.0)),
]


@pytest.mark.parametrize("name,params,fill", FILLS, ids=[f[0] for f in FILLS])
@pytest.mark.parametrize("ppa", [None, 17])
def test_source_points_match_oracle(name, params, fill, ppa):
    eng = HB.SimulationEngine(HB.SourceConfig(193.368, name, params), HB.OpticsConfig(0.93),
                              grid=HB.GridConfig(64, 4.0), max_kernels=4, source_points_per_axis=ppa)
    got = eng.source_points()
    cutoff = 0.93 / 193.368
    ref = np.array(H.sample_source(fill, ppa, (1.0 / 256.0) / cutoff))
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) < 1e-13


CASES = [
    # (source, optics, grid, max_kernels, oracle fill, oracle optics)
    (HB.SourceConfig(193.368, "annular", (0.6, 0.85)), HB.OpticsConfig(0.93), HB.GridConfig(64, 4.0), 24,
     H.fill_annular(0.6, 0.85), H.ProjectionOptics(0.93)),
    (HB.SourceConfig(13.5, "conventional", (0.5,)), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(128, 1.0), 32,
     H.fill_conventional(0.5), H.euv_nxe_033()),
    (HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)), HB.OpticsConfig.immersion(1.35), HB.GridConfig(128, 1.0),
     16, H.fill_dipole(0.8, 0.1, 0.0), H.ProjectionOptics(1.35, immersion_index=1.437)),
    (HB.SourceConfig(13.5, "quasar", (0.7, 0.9, 45.0)), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(128, 1.0),
     48, H.fill_quasar(0.7, 0.9, 45.0), H.euv_nxe_033()),
    (HB.SourceConfig(13.5, "annular", (0.3, 0.8)), HB.OpticsConfig.euv_high_na_055(), HB.GridConfig(64, 1.0), 48,
     H.fill_annular(0.3, 0.8), H.euv_high_na_055()),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("z", [0.0, 37.5])
def test_kernel_build_matches_oracle(case, z):
    src, opt, grid, kmax, fill, oopt = CASES[case]
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax)
    ev, ker = eng.kernels(z)
    oeng = H.Engine(fill, oopt, H.Grid(grid.size, grid.pixel_nm), src.wavelength_nm, max_kernels=kmax)
    ks = oeng.kernel_set(z)
    d = ks.divisor()
    assert len(ev) == len(ks.eigenvalues)
    np.testing.assert_allclose(ev, ks.eigenvalues / d, rtol=1e-9, atol=1e-14 * ev[0])
    diag = eng.imaging_diagnostics(z)
    assert diag["method"] == ks.method
    assert abs(diag["clear_field_intensity"] - ks.clear_field) < 1e-12 * ks.clear_field
    # Kernels within degenerate clusters may differ by a unitary mixing; the
    # image they produce may not.  Compare images of a random band-limited mask.
    rng = np.random.default_rng(5)
    n = grid.size
    t = (rng.random((n, n)) > 0.6).astype(float)
    spec = H.spectrum_from_raster(t)
    img_ref = H.image_from_spectrum(ks, spec, 0.0)
    acc = np.zeros((n, n))
    for lam, k in zip(ev, ker):
        nrm = np.sum(np.abs(k) ** 2)
        assert abs(nrm - 1.0) < 1e-10
        e = np.fft.ifft2(k * spec)
        acc += lam * np.abs(e) ** 2
    assert np.max(np.abs(acc - img_ref)) / np.max(img_ref) < 1e-10


def test_invalid_inputs_return_status():
    """Bad parameters map to the reference's error variants (error.rs:1-72)."""
    with pytest.raises(HB.HuvError) as e:
        HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(100, 1.0))
    assert e.value.status == 2  # GridSizeNotPowerOfTwo
    with pytest.raises(HB.HuvError) as e:
        HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(64, 1.0),
                            max_kernels=0)
    assert e.value.status == 1
    with pytest.raises(HB.HuvError) as e:
        HB.SimulationEngine(HB.SourceConfig(193.0, "annular", (0.9, 0.5)), HB.OpticsConfig(0.9),
                            grid=HB.GridConfig(64, 1.0))
    assert e.value.status == 1  # no light in the fill
    with pytest.raises(HB.HuvError) as e:
        HB.SimulationEngine(HB.SourceConfig.arf_laser(0.7), HB.OpticsConfig(1.2), grid=HB.GridConfig(64, 1.0))
    assert e.value.status == 1  # NA above the medium index
    with pytest.raises(HB.HuvError) as e:
        HB.SimulationEngine(HB.SourceConfig.arf_laser(0.7), HB.OpticsConfig(0.93), grid=HB.GridConfig(2048, 10.0))
    assert e.value.status == 4  # PupilSamplingTooDense
    lib = _lib.lib()
    assert lib.huv_image_batch(None, None, None, None) == 1
    assert lib.huv_engine_destroy(None) is None


def test_misaligned_device_buffers_are_rejected_before_any_launch():
    """The device entry points read rasters with TMA / vector loads and write
    images with vector stores, so input and out must be 16-byte aligned; a
    misaligned pointer is refused on the host (no CUDA call is made)."""
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(),
                              grid=HB.GridConfig(64, 1.0), max_kernels=4)
    lib = _lib.lib()
    buf = np.zeros(64 * 64 * 2 + 16, np.float32)
    base = (buf.ctypes.data + 15) & ~15
    b = _lib.Batch(1, 0, base, 1, 0.0, 0, 0)
    for fn in (lib.huv_image_batch, lib.huv_image_batch_noalloc):
        assert fn(eng.handle, ctypes.byref(b), ctypes.c_void_p(base + 4), None) == 1
        assert b"16-byte aligned" in lib.huv_last_error()
    b.input = base + 1
    assert lib.huv_image_batch(eng.handle, ctypes.byref(b), ctypes.c_void_p(base), None) == 1
    assert b"16-byte aligned" in lib.huv_last_error()


def test_host_output_buffer_is_validated_before_the_call():
    """compute_batch_host writes through the output's raw pointer, so a
    wrong dtype, shape or layout is refused in Python first."""
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(),
                              grid=HB.GridConfig(64, 1.0), max_kernels=4)
    masks = np.zeros((2, 64, 64), np.uint8)
    bad = [np.empty((2, 64, 64), np.float64), np.empty((1, 64, 64), np.float32),
           np.empty((2, 64, 128), np.float32)[:, :, ::2]]
    ro = np.empty((2, 64, 64), np.float32)
    ro.flags.writeable = False
    bad.append(ro)
    for out in bad:
        with pytest.raises(ValueError):
            eng.compute_batch_host(masks, out=out)


def test_ilt_inputs_are_validated_before_the_call():
    """The ILT wrappers pass raw device pointers: a theta of the wrong grid,
    a host tensor, or a target of another shape is refused in Python."""
    import torch
    from highuvlith_b200 import ilt
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(),
                              grid=HB.GridConfig(64, 1.0), max_kernels=4)
    st = ilt.IltSettings(max_iterations=1)
    for theta in (torch.zeros((1, 32, 32)), torch.zeros((1, 64, 64)), torch.zeros((64, 64))):
        with pytest.raises(ValueError):
            ilt.cost_and_gradient(eng, theta, theta, st)
        with pytest.raises(ValueError):
            ilt.optimize(eng, theta, theta, st)


def test_c2_kernel_set_shape():
    """C2: EUV NA 0.33, sigma 0.5, 1024 x 1 nm -> r = 37.55, h = 37, S = 4429, K = 32."""
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(),
                              grid=HB.GridConfig(1024, 1.0), max_kernels=32)
    d = eng.imaging_diagnostics()
    pts = eng.source_points()
    sigma_max = float(np.max(np.hypot(pts[:, 0], pts[:, 1])))
    r = 0.33 / 13.5 * (1 + sigma_max) * 1024.0
    o = np.arange(-40, 41)
    s_expect = int(np.sum(o[:, None] ** 2 + o[None, :] ** 2 <= r * r * (1 + 1e-12)))
    assert d["band_half_width"] == 37
    assert d["num_frequencies"] == s_expect  # sampled sigma_max < 0.5, so S < 4429
    # max_kernels = 32 cuts inside a degenerate pair, so the rule of
    # select_kernel_count (aerial.rs:992-1029) keeps 31.
    assert d["num_kernels"] == 31 and d["method"] == "dense_gram"
