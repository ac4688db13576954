"""Shadow reconstruction (TreeGather::reconstructShadows, Reconstruction.cpp:302-344):
light-space query samples through the Filterer in shadow mode on the GPU, against
the reference build's own reconstructShadows, every query's colour bit for bit."""
import numpy as np
import pytest

import tlfr
from tlfr_testutil import CpuRecon, ref_available

pytestmark = pytest.mark.gpu


def _scene(preset, W, H, spp, qspp, seed):
    rng = np.random.default_rng(seed)
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    # depth gradients of the light-space samples (the generator's are zero)
    rec[..., 14] = rng.uniform(-0.05, 0.05, rec.shape[:3]).astype(np.float32)
    rec[..., 15] = rng.uniform(-0.05, 0.05, rec.shape[:3]).astype(np.float32)
    q, _ = tlfr.synth_scene(preset, W, H, qspp, seed)
    # queries in front of, at, and behind the light-visible surface
    q[..., 3] *= rng.choice(np.float32([0.7, 1.0, 1.0, 1.3]), q.shape[:3])
    q[..., 0] += rng.uniform(-0.3, 0.3, q.shape[:3]).astype(np.float32)
    q[..., 1] += rng.uniform(-0.3, 0.3, q.shape[:3]).astype(np.float32)
    density = rng.uniform(0.5, 2.0, q.shape[:3]).astype(np.float32)
    return rec, coc, q, density


@pytest.mark.parametrize("preset,W,H,spp,qspp,seed", [
    (tlfr.SCENE_CARDS, 48, 32, 4, 2, 90),
    (tlfr.SCENE_CARDS_LARGE, 64, 40, 8, 4, 91),
    (tlfr.SCENE_PLANES, 40, 30, 16, 1, 92),
])
def test_gpu_shadows_match_reference(preset, W, H, spp, qspp, seed):
    if not ref_available():
        pytest.skip("reference build absent")
    rec, coc, q, density = _scene(preset, W, H, spp, qspp, seed)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    got = g.reconstructShadows(q, density)
    want = CpuRecon("ref", rec, coc).shadows(q, density)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the queries behind the surface are (partly) shadowed, the ones in front lit
    lum = got[..., :3].sum(-1)
    assert (lum == 0).any() and (lum > 0).any()
