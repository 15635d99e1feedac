"""Uneven batches through one CUDA-graph launch (huv_plan_*): every clip
must image exactly like a single-clip call on an engine built with that
clip's own kernel budget."""
import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200.clips import gen_batch

pytestmark = pytest.mark.gpu


def test_plan_matches_per_clip_engines():
    import torch
    euv = lambda n: HB.SimulationEngine(HB.SourceConfig(13.5, "quasar", (0.7, 0.9, 45.0)),
                                        HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(n, 1.0), max_kernels=48)
    arfi = lambda n: HB.SimulationEngine(HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)),
                                         HB.OpticsConfig.immersion(1.35), grid=HB.GridConfig(n, 1.0), max_kernels=48)
    engines = {("euv", 128): euv(128), ("euv", 256): euv(256), ("arfi", 256): arfi(256)}
    spec = [("euv", 128, 16), ("euv", 128, 16), ("euv", 128, 48), ("euv", 256, 32), ("arfi", 256, 16),
            ("euv", 256, 32), ("arfi", 256, 48), ("euv", 128, 16)]
    clips, refs = [], []
    # group-contiguous storage for the two (euv,128,16) clips at the front
    _, r128 = gen_batch(4, 128, base_seed=50, wmin=4, wmax=30)
    inp128 = torch.from_numpy(r128).cuda()
    out128 = torch.zeros((4, 128, 128), dtype=torch.float32, device="cuda")
    k128 = 0
    for i, (src, n, kmax) in enumerate(spec):
        if n == 128:
            inp, out = inp128[k128], out128[k128]
            raster = r128[k128]
            k128 += 1
        else:
            _, r = gen_batch(1, n, base_seed=100 + i, wmin=5, wmax=40)
            raster = r[0]
            inp = torch.from_numpy(r[0]).cuda()
            out = torch.zeros((n, n), dtype=torch.float32, device="cuda")
        clips.append((engines[(src, n)], kmax, inp, out))
        refs.append((src, n, kmax, raster))
    plan = HB.UnevenPlan(clips, autotune=True)
    for _ in range(2):
        for _, _, _, out in clips:
            out.zero_()
        plan.launch()
        torch.cuda.synchronize()
    groups = plan.describe()
    # (arfi, 256) has only 8 kernels: budgets 16 and 48 share one group
    assert len(groups) == 4 and sum(g["clips"] for g in groups) == len(spec)
    for (src, n, kmax, raster), (_, _, _, out) in zip(refs, clips):
        ref_eng = euv(n) if src == "euv" else arfi(n)
        ref_eng = HB.SimulationEngine(ref_eng.source, ref_eng.optics, grid=HB.GridConfig(n, 1.0), max_kernels=kmax)
        ref = ref_eng.compute_batch(torch.from_numpy(raster).cuda(), form="fft").cpu().numpy()[0]
        got = out.cpu().numpy()
        assert np.max(np.abs(got - ref)) / np.max(ref) < 1e-4, (src, n, kmax)


def test_plan_group_merged_from_two_stores():
    """ArF immersion dipole at 256^2 keeps 8 kernels for budgets 16 and 48, so
    the two budgets' clips form one group; each budget's clips sit in a
    store of their own (two contiguous runs), which the plan gathers and
    scatters run by run.  Every clip against a single-clip call."""
    import torch
    arfi = HB.SimulationEngine(HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)),
                               HB.OpticsConfig.immersion(1.35), grid=HB.GridConfig(256, 1.0), max_kernels=48)
    stores = []
    for seed in (300, 400):
        _, r = gen_batch(3, 256, base_seed=seed, wmin=5, wmax=40)
        stores.append((r, torch.from_numpy(r).cuda(), torch.zeros((3, 256, 256), dtype=torch.float32, device="cuda")))
    clips = [(arfi, kmax, inp[i], out[i]) for kmax, (_, inp, out) in zip((16, 48), stores) for i in range(3)]
    plan = HB.UnevenPlan(clips, autotune=True)
    groups = plan.describe()
    assert len(groups) == 1 and groups[0]["clips"] == 6 and groups[0]["contiguous"] == 0
    plan.launch()
    torch.cuda.synchronize()
    for kmax, (r, _, out) in zip((16, 48), stores):
        ref_eng = HB.SimulationEngine(arfi.source, arfi.optics, grid=HB.GridConfig(256, 1.0), max_kernels=kmax)
        ref = ref_eng.compute_batch(torch.from_numpy(r).cuda(), form="fft").cpu().numpy()
        got = out.cpu().numpy()
        assert np.max(np.abs(got - ref)) / np.max(ref) < 1e-4, kmax
