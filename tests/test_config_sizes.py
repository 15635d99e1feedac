"""The ILT and surrogate workloads' own sizes against the FP64 oracle.

- ILT gradient (EUV NA 0.33, conventional sigma 0.5, K = 31 of 32 requested,
  1024^2 at 1 nm, resist threshold 0.25 / steepness 50, seeded contact-array
  targets): the device's batched cost and exact adjoint on the 160-point
  evaluation grid against oracle/ilt.py on the full grid.  Tolerance: cost
  within 1e-4 relative, gradient within 2e-3 of its largest magnitude (FP32
  sums over 1024^2 pixels), and a cosine above 0.9999.
- High-NA EUV image (NA 0.55, central obscuration 0.2, annular 0.3/0.8,
  K = 48, 512^2 at 1 nm, seeded Manhattan clips of 15-60 nm at 20-60 %
  density): every form against the oracle's C restatement of the image loop.
  Tolerance: the task's 1e-3 max relative intensity error and 0.2 nm edge
  error; the FP32 FFT form is held to 2e-5.
"""
import numpy as np
import pytest

from highuvlith_b200.clips import gen_batch
from oracle import cpu
from oracle import hopkins as H
from oracle import ilt as OI

from parity import edge_error_nm, rel_err

pytestmark = pytest.mark.gpu


def test_ilt_gradient_at_1024_with_31_kernels():
    import torch
    import highuvlith_b200 as HB
    from highuvlith_b200 import ilt
    from highuvlith_b200.targets import gen_contact_targets
    n = 1024
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(n, 1.0),
                              max_kernels=32)
    assert eng.imaging_diagnostics()["num_kernels"] == 31
    targets, _ = gen_contact_targets(2, n)
    rng = np.random.default_rng(11)
    theta = (targets - 0.5 + 0.2 * rng.standard_normal(targets.shape)).astype(np.float32)
    st = ilt.IltSettings(cost="resist", threshold=0.25, steepness=50.0)
    c_dev, g_dev = ilt.cost_and_gradient(eng, torch.from_numpy(theta).cuda(), torch.from_numpy(targets).cuda(), st)
    g_dev = g_dev.cpu().numpy()
    ev, ker = eng.kernels(0.0)
    cfg = OI.IltConfig(cost="resist", threshold=0.25, steepness=50.0, flare=0.0, tv_weight=0.01, bin_weight=0.0)
    for i in range(2):
        c_ref, g_ref = OI.IltProblem(ev, ker, targets[i].astype(np.float64), cfg).cost_and_gradient(
            theta[i].astype(np.float64))
        assert abs(c_dev[i] - c_ref) <= 1e-4 * abs(c_ref), (i, c_dev[i], c_ref)
        err = np.max(np.abs(g_dev[i] - g_ref)) / np.max(np.abs(g_ref))
        cos = float(np.sum(g_dev[i] * g_ref) / (np.linalg.norm(g_dev[i]) * np.linalg.norm(g_ref)))
        assert err <= 2e-3 and cos > 0.9999, (i, err, cos)


def test_high_na_image_every_form_at_k48():
    import torch
    from highuvlith_b200.surrogate import high_na_engine
    n = 512
    eng = high_na_engine(n, 1.0, max_kernels=48)
    oeng = H.Engine(H.fill_annular(0.3, 0.8), H.euv_high_na_055(), H.Grid(n, 1.0), 13.5, max_kernels=48)
    ks = oeng.kernel_set(0.0)
    assert eng.imaging_diagnostics()["num_kernels"] == ks.values.shape[0]
    _, rasters = gen_batch(2, n, base_seed=5050, wmin=15, wmax=60, dmin=0.2, dmax=0.6)
    refs = cpu.images(ks, rasters, 0.0)
    d = torch.from_numpy(rasters).cuda()
    for form, eg in (("fft", 0), ("fft", n), ("tc", 0), ("hybrid", 0), ("auto", 0)):
        out = eng.compute_batch(d, form=form, eval_grid=eg).cpu().numpy()
        for c in range(2):
            e = rel_err(out[c], refs[c])
            assert e < (2e-5 if form == "fft" else 1e-3), (form, eg, c, e)
            cd, unmatched = edge_error_nm(out[c], refs[c], step=8)
            assert cd < 0.2 and unmatched <= 2, (form, eg, c, cd, unmatched)
