"""The C-ABI library loads and exports every entry point include/tlfr.h declares;
host-only entry points (parameters, sample-buffer IO, scene generator) work
without a GPU; device entry points fail with a status, not a crash, when no CUDA
device is present."""
import ctypes
import os
import re

import numpy as np
import pytest

import tlfr
from tlfr_testutil import ROOT

HEADER = os.path.join(ROOT, "include", "tlfr.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tlfr_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = tlfr.load_library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_params_default_matches_reference_ctor():
    lib = tlfr.load_library()
    p = tlfr._Params()
    lib.tlfr_params_default(ctypes.byref(p))
    assert (p.aperture_adjust, p.focus_adjust, p.lens_filter, p.time_filter, p.override_uvt, p.output_spp) == \
        (1.0, 1.0, 0, 0, 0, 0)


def test_synth_scene_deterministic():
    a, ca = tlfr.synth_scene(tlfr.SCENE_CARDS, 40, 30, 4, 5)
    b, cb = tlfr.synth_scene(tlfr.SCENE_CARDS, 40, 30, 4, 5)
    assert np.array_equal(a, b) and ca == cb
    assert np.all(a[..., 3] > 0)                 # w > 0: no sample is discarded
    assert np.all(a[..., 10] == 1.0)
    assert np.all((a[..., 4] >= -1) & (a[..., 4] <= 1) & (a[..., 6] >= 0) & (a[..., 6] <= 1))
    px = a[..., 0] - np.arange(40)[None, :, None]
    assert np.all((px >= 0) & (px < 1))


def test_buffer_from_host_forces_alpha():
    rec, coc = tlfr.synth_scene(tlfr.SCENE_PLANES, 8, 6, 2, 1)
    rec[..., 10] = 0.25
    b = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    assert b.info()[:3] == (8, 6, 2)
    assert np.all(b.records()[..., 10] == 1.0)


@pytest.mark.parametrize("binary", [True, False])
def test_serialize_load_roundtrip(tmp_path, binary):
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, 12, 9, 2, 2)
    b = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    path = str(tmp_path / "buf.bin")
    b.serialize(path, separate_header=True, binary=binary)
    assert os.path.exists(path + ".header")
    c = tlfr.UVTSampleBuffer(path)
    W, H, S, cc = c.info()
    assert (W, H, S) == (12, 9, 2)
    got = c.records()
    if binary:
        exp = rec.copy()
        exp[..., 10] = 1.0
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))
    else:
        # text records carry 6 decimals ("%f")
        assert np.allclose(got[..., :10], rec[..., :10], atol=2e-6 * np.maximum(1, np.abs(rec[..., :10])).max())


def test_binary_needs_separate_header(tmp_path):
    rec, coc = tlfr.synth_scene(tlfr.SCENE_PLANES, 4, 4, 1, 1)
    b = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    with pytest.raises(tlfr.TlfrError) as e:
        b.serialize(str(tmp_path / "x.bin"), separate_header=False, binary=True)
    assert e.value.status == 1


def test_load_errors(tmp_path):
    with pytest.raises(tlfr.TlfrError) as e:
        tlfr.UVTSampleBuffer(str(tmp_path / "missing.bin"))
    assert e.value.status == 2
    p = tmp_path / "bad.txt"
    p.write_text("Version 1.2\nWidth 2\nHeight 2\nSamples per pixel 1\n")
    with pytest.raises(tlfr.TlfrError) as e:
        tlfr.UVTSampleBuffer(str(p))
    assert e.value.status == 3
    p2 = tmp_path / "trunc.bin"
    open(str(p2), "wb").write(b"\0" * 64)
    (tmp_path / "trunc.bin.header").write_text(
        "Version 1.3\nWidth 2\nHeight 2\nSamples per pixel 1\n"
        "CoC coefficients (coc radius = C0/w+C1): -1.0,2.0\nEncoding = binary\nx,y\n")
    with pytest.raises(tlfr.TlfrError) as e:
        tlfr.UVTSampleBuffer(str(p2))
    assert e.value.status == 3


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_create_without_device_reports_status():
    rec, coc = tlfr.synth_scene(tlfr.SCENE_PLANES, 8, 8, 1, 1)
    b = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    with pytest.raises(tlfr.TlfrError) as e:
        tlfr.TreeGather(b)
    assert e.value.status == 8
