"""The reference's GPU-toggle algorithm (CameraParams::enableCuda, tlfr_params::
enable_cuda) on the GPU against the reference's own CPU restatement of it
(CudaReconstruction::reconstructCPUSingle / reconstructCPU, ReconstructionCuda.cpp:
261-872, compiled by oracle/build_ref.sh): every checked output sample's colour
bit for bit, every pixel within 1e-4 relative (the reference normalises a
pixel by dividing by alpha, this library multiplies by its reciprocal)."""
import numpy as np
import pytest

import tlfr
from tlfr_testutil import CpuRecon, ref_available, rel_err, sample_queries

pytestmark = pytest.mark.gpu

SCENES = [
    ("cards", tlfr.SCENE_CARDS, 64, 48, 4, 81, {}),
    ("large", tlfr.SCENE_CARDS_LARGE, 96, 64, 8, 82, {}),
    ("planes", tlfr.SCENE_PLANES, 48, 40, 16, 83, {}),
    ("cards_1spp", tlfr.SCENE_CARDS, 48, 32, 1, 84, {}),
    ("refocus", tlfr.SCENE_CARDS, 56, 40, 2, 85, {"aperture": 1.5, "focus": 0.8}),
    ("pinhole", tlfr.SCENE_CARDS, 64, 48, 4, 86, {"uvt": (0.0, 0.0, 1.0)}),
]


@pytest.mark.parametrize("name,preset,W,H,spp,seed,p", SCENES, ids=[s[0] for s in SCENES])
def test_gpu_toggle_matches_reference(name, preset, W, H, spp, seed, p):
    if not ref_available():
        pytest.skip("reference build absent")
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    aperture, focus, uvt = p.get("aperture", 1.0), p.get("focus", 1.0), p.get("uvt")
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc), tlfr.CameraParams(enableCuda=True, overrideUVT=uvt),
                        aperture, focus)
    img = g.reconstructDofMotion()
    samples = g.output_sample_buffer().records()
    r = CpuRecon("ref", rec, coc, aperture=aperture, focus=focus, uvt=uvt)
    M = samples.shape[2]
    q = sample_queries(W, H, M, 500, seed)
    want = r.gpu_toggle_queries(q)
    got = samples[q[:, 1], q[:, 0], q[:, 2], 7:11]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    ref = r.gpu_toggle_image()
    assert rel_err(img, ref).max() <= 1e-4
    # a different algorithm from the default (Filterer) one
    plain = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc), tlfr.CameraParams(overrideUVT=uvt),
                            aperture, focus).reconstructDofMotion()
    assert np.array_equal(plain.view(np.uint32), r.reconstruct().view(np.uint32))
