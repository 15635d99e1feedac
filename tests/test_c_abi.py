"""The C ABI as a reference-side binding sees it.

A plain C program (tests/c_caller.c) is compiled against include/huv_b200.h
with every struct's size and field offsets from the ctypes mirror
(highuvlith_b200/_lib.py) as static assertions, then linked against the
library and run: engine creation and diagnostics on the host, and (on a GPU)
huv_image_batch_host against the Python entry point and the FP64 oracle.
The caller-supplied kernel set (huv_kernelset_create) is checked against
the engine's own kernels.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

import highuvlith_b200 as HB
from highuvlith_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {"huv_source": L.Source, "huv_optics": L.Optics, "huv_grid": L.Grid, "huv_settings": L.Settings,
           "huv_diagnostics": L.Diagnostics, "huv_rect": L.Rect, "huv_rect_clips": L.RectClips,
           "huv_batch": L.Batch, "huv_kernel_set": L.KernelSetDesc, "huv_clip": L.Clip,
           "huv_ilt_params": L.IltParams, "huv_ilt_opt": L.IltOpt, "huv_surrogate_ilt": L.SurrogateIlt}


def _defines(override=None):
    out = []
    for cname, ct in STRUCTS.items():
        out.append(f"-DHUV_EXPECT_{cname}_SIZE={C.sizeof(ct)}")
        for f in ct._fields_:
            off = getattr(ct, f[0]).offset
            if override and override[0] == (cname, f[0]):
                off = override[1]
            out.append(f"-DHUV_EXPECT_{cname}_{f[0]}={off}")
    return out


def _compile(tmp_path, override=None):
    L.lib()  # the library must be built
    exe = str(tmp_path / "c_caller")
    libdir = os.path.join(ROOT, "highuvlith_b200")
    cmd = ["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), *_defines(override),
           os.path.join(ROOT, "tests", "c_caller.c"), "-o", exe, os.path.join(libdir, "libhuv_b200.so"),
           f"-Wl,-rpath,{libdir}"]
    return subprocess.run(cmd, capture_output=True, text=True), exe


def test_c_caller_layout_matches_the_ctypes_binding(tmp_path):
    res, exe = _compile(tmp_path)
    assert res.returncode == 0, res.stderr
    sizes = json.loads(subprocess.run([exe, "layout"], capture_output=True, text=True, check=True).stdout)
    assert sizes == {k: C.sizeof(v) for k, v in STRUCTS.items()}


def test_a_wrong_offset_fails_the_build(tmp_path):
    """The static assertions bite: one field offset off by 4 bytes."""
    res, _ = _compile(tmp_path, override=(("huv_settings", "kernel_build"), 16))
    assert res.returncode != 0 and "kernel_build" in res.stderr


def test_c_caller_creates_an_engine_on_the_host(tmp_path):
    res, exe = _compile(tmp_path)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([exe, "create"], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    got = json.loads(run.stdout)
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(128, 1.0),
                              max_kernels=16)
    d = eng.imaging_diagnostics()
    assert (got["num_kernels"], got["band_half_width"], got["num_frequencies"]) == (
        d["num_kernels"], d["band_half_width"], d["num_frequencies"])
    assert got["clear_field"] == d["clear_field_intensity"]


def _c_caller_clips():
    r = np.zeros((2, 128, 128), dtype=np.uint8)
    r[0, 48:80, 48:80] = 1
    r[1, :, 40:56] = 1
    r[1, :, 72:88] = 1
    return r


@pytest.mark.gpu
def test_c_caller_images_like_python_and_the_oracle(tmp_path):
    from oracle import hopkins as H
    res, exe = _compile(tmp_path)
    assert res.returncode == 0, res.stderr
    out = tmp_path / "img.bin"
    run = subprocess.run([exe, "image", str(out)], capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    img = np.fromfile(out, dtype=np.float32).reshape(2, 128, 128)
    r = _c_caller_clips()
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(128, 1.0),
                              max_kernels=16)
    py = eng.compute_batch_host(r)
    assert np.max(np.abs(img - py)) <= 1e-6 * np.max(py)
    oeng = H.Engine(H.fill_conventional(0.5), H.euv_nxe_033(), H.Grid(128, 1.0), 13.5, max_kernels=16)
    for c in range(2):
        ref = oeng.compute_from_spectrum(H.spectrum_from_raster(r[c]))
        assert np.max(np.abs(img[c] - ref)) / np.max(ref) < 1e-4


def test_kernel_set_engine_round_trip_and_validation():
    eng = HB.SimulationEngine(HB.SourceConfig.euv(0.5), HB.OpticsConfig.euv_nxe_033(), grid=HB.GridConfig(64, 1.0),
                              max_kernels=8)
    ev, ker = eng.kernels()
    sup = HB.SimulationEngine.from_kernel_set(ev, ker)
    ev2, ker2 = sup.kernels()
    assert np.array_equal(ev, ev2) and np.array_equal(ker, ker2)
    d = sup.imaging_diagnostics()
    assert d["method"] == "supplied" and d["band_half_width"] == eng.imaging_diagnostics()["band_half_width"]
    with pytest.raises(L.HuvError) as ex:
        sup.kernels(25.0)
    assert ex.value.status == 11  # another focus plane: UNSUPPORTED
    for bad, status in ((dict(eigenvalues=ev[::-1]), 1), (dict(kernels=ker * np.nan), 1),
                        (dict(kernels=ker * 0), 3), (dict(flare_fraction=1.0), 1)):
        kw = dict(eigenvalues=ev, kernels=ker)
        kw.update(bad)
        with pytest.raises(L.HuvError) as ex:
            HB.SimulationEngine.from_kernel_set(**kw)
        assert ex.value.status == status, bad
    with pytest.raises(ValueError):
        HB.SimulationEngine.from_kernel_set(ev[:3], ker)


@pytest.mark.gpu
@pytest.mark.parametrize("defocus", [0.0, 30.0])
def test_kernel_set_engine_images_like_the_engine(defocus):
    """A kernel set exported by kernels(z) and handed back through
    huv_kernelset_create images like the engine that built it (ArF
    immersion dipole with 2 % flare, so the flare path is covered)."""
    import torch
    from highuvlith_b200.clips import gen_batch
    eng = HB.SimulationEngine(HB.SourceConfig(193.368, "dipole", (0.8, 0.1, 0.0)), HB.OpticsConfig.immersion(1.35),
                              grid=HB.GridConfig(256, 1.0), max_kernels=16)
    ev, ker = eng.kernels(defocus)
    sup = HB.SimulationEngine.from_kernel_set(ev, ker, flare_fraction=0.02, defocus_nm=defocus)
    _, r = gen_batch(3, 256, base_seed=5, wmin=10, wmax=60, dmin=0.2, dmax=0.6)
    d = torch.from_numpy(r).cuda()
    for form in ("fft", "auto"):
        a = eng.compute_batch(d, focus_nm=defocus, form=form)
        b = sup.compute_batch(d, focus_nm=defocus, form=form)
        assert torch.max(torch.abs(a - b)).item() <= 1e-6 * torch.max(a).item(), form
    # the host entry point and the set's own plane named as 0
    h = sup.compute_batch_host(r, focus_nm=0.0)
    assert np.max(np.abs(h - a.cpu().numpy())) <= 1e-6 * float(a.max())
