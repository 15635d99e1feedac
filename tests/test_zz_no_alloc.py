"""The allocation-free entry point, huv_image_batch_noalloc.

It exists for callers that cannot call cudaMalloc (an application whose own
memory pool already owns the device, or a latency-critical loop that cannot
take cudaMalloc's device-wide synchronisation).  It must image exactly like
huv_image_batch, call after call, using only its fixed 32 MiB device array,
and reject a grid whose single clip does not fit that array.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200 import _lib as L
from highuvlith_b200.clips import gen_batch

pytestmark = pytest.mark.gpu


def _noalloc(eng, rasters, out, eval_grid=0, form="fft"):
    import torch
    b = L.Batch(rasters.shape[0], L.INPUT_U8, rasters.data_ptr(), 1, 0.0, L.FORM[form], eval_grid)
    st = torch.cuda.current_stream().cuda_stream
    return L.lib().huv_image_batch_noalloc(eng.handle, C.byref(b), out.data_ptr(), st)


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(256, 1.0),
                              max_kernels=32)
    _, rasters = gen_batch(6, 256, base_seed=2026, wmin=5, wmax=40)
    d = torch.from_numpy(rasters).cuda()
    ref = eng.compute_batch(d, form="fft").clone()
    for _ in range(2):  # two calls in a row share (and overwrite) the same array
        out = torch.full_like(ref, float("nan"))
        L.check(_noalloc(eng, d, out))
        torch.cuda.synchronize()
        err = torch.max(torch.abs(out - ref)).item() / torch.max(ref).item()
        assert err < 1e-5, err


def test_noalloc_rejects_clips_beyond_its_scratch():
    import torch
    # ArF immersion dipole on 4096 x 1 nm, full-grid evaluation: one clip's
    # row transforms alone take 16 x 109 x 4096 complex values (57 MiB).
    eng = HB.SimulationEngine(HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)), HB.OpticsConfig.immersion(1.35),
                              grid=HB.GridConfig(4096, 1.0), max_kernels=16)
    d = torch.zeros((1, 4096, 4096), dtype=torch.uint8, device="cuda")
    out = torch.empty((1, 4096, 4096), dtype=torch.float32, device="cuda")
    status = _noalloc(eng, d, out, eval_grid=4096)
    assert status == 1
    assert b"fixed maximum of 32 MiB" in L.lib().huv_last_error()


def test_noalloc_rejects_tensor_core_forms():
    import torch
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(256, 1.0),
                              max_kernels=8)
    d = torch.zeros((1, 256, 256), dtype=torch.uint8, device="cuda")
    out = torch.empty((1, 256, 256), dtype=torch.float32, device="cuda")
    for form in ("tc", "tc_rows", "hybrid"):
        assert _noalloc(eng, d, out, form=form) != 0
        assert b"FP32 FFT form only" in L.lib().huv_last_error()
