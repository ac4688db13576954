"""Batches: several sample buffers of uneven resolution and spp reconstructed as
one CUDA graph give the same images, bit for bit, as reconstructing each
context on its own (the per-output-sample results do not depend on the grid the
autotuner picks)."""
import numpy as np
import pytest

import route_ref as R
import tlfr

pytestmark = pytest.mark.gpu

FRAMES = [
    (tlfr.SCENE_CARDS, 64, 48, 4, 61),
    (tlfr.SCENE_CARDS_LARGE, 96, 64, 8, 62),
    (tlfr.SCENE_PLANES, 40, 30, 16, 63),
    (tlfr.SCENE_CARDS, 50, 40, 1, 64),
    (tlfr.SCENE_CARDS_LARGE, 120, 80, 2, 65),
]


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def test_batch_matches_single_frames():
    torch = _torch()
    trees, want = [], []
    fast = tlfr.Router(0, seed=1)
    p = fast.params()
    p[R.OFF_W3:R.OFF_B3] = 0
    p[R.OFF_B3] = 50.0          # every pixel on the fast path
    fast.set_params(p)
    for k, (preset, W, H, S, seed) in enumerate(FRAMES):
        rec, coc = tlfr.synth_scene(preset, W, H, S, seed)
        g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
        if k == 1:
            g.set_routing(fast, 0.5)
        want.append(g.reconstructDofMotion())
        trees.append(g)
    outs = [torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda") for (_, W, H, _, _) in FRAMES]
    batch = tlfr.Batch(trees, [o.data_ptr() for o in outs], autotune=True)
    blocks = batch.light_blocks()
    assert len(blocks) == len(FRAMES) and (blocks > 0).all()
    for run in range(2):
        for o in outs:
            o.fill_(float("nan"))
        batch.run()
        ms = batch.sync()
        assert ms > 0
        for k, (o, w) in enumerate(zip(outs, want)):
            got = o.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), w.view(np.uint32)), (run, k)
    batch.close()
    trees[1].set_routing(None)
    fast.close()


def test_batch_rejects_bad_arguments():
    _torch()
    with pytest.raises(tlfr.TlfrError):
        tlfr.Batch([], [])
