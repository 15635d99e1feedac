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


def _noalloc(eng, rasters, out, eval_grid=0, form="fft", z=0.0):
    import torch
    b = L.Batch(rasters.shape[0], L.INPUT_U8, rasters.data_ptr(), 1, float(z), L.FORM[form], eval_grid)
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


def test_noalloc_defocus_planes_allocate_nothing_and_match_oracle():
    """A defocused plane on a host-build engine (built on the host for the
    call, never cached) and a cached plane on a device-build engine with a
    one-plane cache: the device's free memory is unchanged across each call
    after the first, the images match huv_image_batch and the FP64 oracle,
    and an uncached plane on the device-build engine is rejected without
    building anything."""
    import torch
    from oracle import hopkins as H
    n, z = 128, 35.0
    _, rasters = gen_batch(2, n, base_seed=77, wmin=4, wmax=24)
    d = torch.from_numpy(rasters).cuda()
    oeng = H.Engine(H.fill_conventional(0.5), H.euv_nxe_033(), H.Grid(n, 1.0), 13.5, max_kernels=16)
    ref = np.stack([oeng.compute_from_spectrum(H.spectrum_from_raster(r), z) for r in rasters])
    for build, capacity in (("host", 32), ("device", 1)):
        eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(n, 1.0),
                                  max_kernels=16, kernel_build=build, kernel_cache_capacity=capacity)
        out = torch.full((2, n, n), float("nan"), device="cuda")
        if build == "device":
            # the plane must be held by the engine: an uncached one is refused
            free0 = torch.cuda.mem_get_info()[0]
            assert _noalloc(eng, d, out, z=z) == 11  # HUV_ERR_UNSUPPORTED
            assert b"not cached" in L.lib().huv_last_error()
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0
            eng.compute_batch(d, focus_nm=z, form="fft")  # caches the plane (allocates, as it may)
        L.check(_noalloc(eng, d, out, z=z))  # first call: set-up of the array's address
        torch.cuda.synchronize()
        want = eng.compute_batch(d, focus_nm=z, form="fft").cpu().numpy()
        for _ in range(2):
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            L.check(_noalloc(eng, d, out, z=z))
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0, build
            got = out.cpu().numpy()
            assert np.max(np.abs(got - want)) / np.max(want) < 1e-5, build
            for c in range(2):
                assert np.max(np.abs(got[c] - ref[c])) / np.max(ref[c]) < 1e-5, (build, c)


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
