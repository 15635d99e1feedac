"""FP64 kernel construction on the device (KernelBuilder::build,
aerial.rs:1041-1317) against the host build, and the randomized solver the
reference's rule picks for large problems (aerial.rs:1116-1128) against the
dense one, with the reference's own bounds (aerial.rs:2622-2675)."""
import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200.clips import gen_batch

pytestmark = pytest.mark.gpu

CASES = [
    ("arf_annular_64", HB.SourceConfig(193.368, "annular", (0.6, 0.85)), HB.OpticsConfig(0.93),
     HB.GridConfig(64, 2.0), 24),
    ("euv_128", HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(128, 1.0), 32),
    ("arfi_dipole_128", HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)), HB.OpticsConfig.immersion(1.35),
     HB.GridConfig(128, 1.0), 16),
    ("high_na_64", HB.SourceConfig(13.5, "annular", (0.3, 0.8)), HB.OpticsConfig.euv_high_na_055(),
     HB.GridConfig(64, 1.0), 48),
]


def _images(eng, rasters, z):
    import torch
    d = torch.from_numpy(rasters).cuda()
    return eng.compute_batch(d, focus_nm=z, form="fft").cpu().numpy()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("z", [0.0, 37.5])
def test_device_build_matches_host_build(case, z):
    _, src, opt, grid, kmax = case
    host = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax)
    dev = HB.SimulationEngine(src, opt, grid=grid, max_kernels=kmax, kernel_build="device")
    ev_h, _ = host.kernels(z)
    ev_d, _ = dev.kernels(z)
    assert len(ev_h) == len(ev_d)
    np.testing.assert_allclose(ev_d, ev_h, rtol=1e-9, atol=1e-13 * ev_h[0])
    dh, dd = host.imaging_diagnostics(z), dev.imaging_diagnostics(z)
    for key in ("num_kernels", "num_frequencies", "num_columns", "method", "band_half_width"):
        assert dh[key] == dd[key], key
    assert abs(dh["clear_field_intensity"] - dd["clear_field_intensity"]) < 1e-12
    n = grid.size
    _, rasters = gen_batch(2, n, base_seed=3, wmin=max(2, n // 40), wmax=max(4, n // 8), dmin=0.2, dmax=0.6)
    a, b = _images(host, rasters, z), _images(dev, rasters, z)
    assert np.max(np.abs(a - b)) / np.max(a) < 1e-6


@pytest.mark.parametrize("z", [0.0, 90.0])
def test_randomized_rule_matches_dense_within_reference_bounds(z):
    """EUV 256^2 at 1 nm, sigma 0.7: 349 orders > 320 and 3 (6 + 16) < 349, so
    the reference's rule takes the randomized solver.  Six kernels, as in the
    reference's own test (aerial.rs:2650-2675): each eigenvalue within 10 x
    (lambda_{l+1} / lambda_k)^(2q+1) of the dense one, images within 1e-5."""
    src, opt, grid = HB.SourceConfig.euv(0.7), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(256, 1.0)
    dense = HB.SimulationEngine(src, opt, grid=grid, max_kernels=6)
    rnd = HB.SimulationEngine(src, opt, grid=grid, max_kernels=6, kernel_build="device_reference_rule")
    assert rnd.imaging_diagnostics(z)["method"] == "randomized"
    assert dense.imaging_diagnostics(z)["method"] == "dense_tcc"
    ev_d, _ = dense.kernels(z)
    ev_r, _ = rnd.kernels(z)
    assert len(ev_r) == len(ev_d) == 6
    full = HB.SimulationEngine(src, opt, grid=grid, max_kernels=1000)
    ev_all, _ = full.kernels(z)
    l = 6 + 16
    for k in range(6):
        bound = max((ev_all[l] / ev_all[k]) ** 7, 1e-13)
        assert abs(ev_r[k] / ev_d[k] - 1.0) <= 10.0 * bound, (k, ev_r[k], ev_d[k], bound)
    _, rasters = gen_batch(2, 256, base_seed=9, wmin=8, wmax=40, dmin=0.2, dmax=0.6)
    a, b = _images(dense, rasters, z), _images(rnd, rasters, z)
    assert np.max(np.abs(a - b)) < 1e-5


def test_reference_rule_keeps_dense_for_small_problems():
    """min(orders, columns) <= 320: the rule solves densely (as the host)."""
    src, opt, grid = HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), HB.GridConfig(128, 1.0)
    eng = HB.SimulationEngine(src, opt, grid=grid, max_kernels=16, kernel_build="device_reference_rule")
    assert eng.imaging_diagnostics()["method"] in ("dense_tcc", "dense_gram")
