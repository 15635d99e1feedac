"""The give-up path of the tensor-core kernels' bounded waits.

huv_debug_probe_wait makes every tensor-core GEMM wait, before its first
MMA, on a barrier that nothing arrives at, for a short time: the wait runs
out, the kernel records the failure, drains its in-flight copies, frees its
tensor memory and returns, and huv_device_status reports
HUV_ERR_DEVICE_TIMEOUT.  Nothing faults or hangs: the probe is a bounded
wait, and the context stays usable, which the clean run afterwards checks
against the FP64 oracle.
"""
import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200 import _lib as L
from highuvlith_b200.clips import gen_batch
from oracle import hopkins as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["tc", "hybrid"])
def test_probe_wait_runs_out_and_is_reported(form):
    import torch
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(256, 1.0),
                              max_kernels=16)
    _, r = gen_batch(2, 256, base_seed=404, wmin=8, wmax=40)
    d = torch.from_numpy(r).cuda()
    eng.compute_batch(d, form=form)  # warm: operands built, module loaded
    eng.device_status()
    L.check(L.lib().huv_debug_probe_wait(200_000))  # 0.2 ms
    try:
        eng.compute_batch(d, form=form)
        with pytest.raises(HB.HuvError) as ex:
            eng.device_status()
        assert ex.value.status == 10  # HUV_ERR_DEVICE_TIMEOUT
        # the host entry point reports it on its own
        with pytest.raises(HB.HuvError) as ex:
            eng.compute_batch_host(r, form=form)
        assert ex.value.status == 10
    finally:
        L.check(L.lib().huv_debug_probe_wait(0))
    eng.device_status()  # the flag was cleared by the report
    out = eng.compute_batch(d, form=form).cpu().numpy()
    eng.device_status()
    oeng = H.Engine(H.fill_conventional(0.5), H.euv_nxe_033(), H.Grid(256, 1.0), 13.5, max_kernels=16)
    for c in range(2):
        ref = oeng.compute_from_spectrum(H.spectrum_from_raster(r[c]))
        assert np.max(np.abs(out[c] - ref)) / np.max(ref) < 1e-4
