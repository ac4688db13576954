"""Batches: sample buffers of uneven resolution and spp, and sweeps of output
settings over one hierarchy, reconstructed as one CUDA graph with one persistent
launch per pass per chunk of frames.  Every frame equals the oracle's image and
the single-frame GPU path bit for bit, whatever tile shape the autotuner picks
and however the frames are split into chunks."""
import numpy as np
import pytest

import route_ref as R
import tlfr
from tlfr_testutil import CpuRecon

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


def _fast_router():
    fast = tlfr.Router(0, seed=1)
    p = fast.params()
    p[R.OFF_W3:R.OFF_B3] = 0
    p[R.OFF_B3] = 50.0          # every pixel on the fast path
    fast.set_params(p)
    return fast


@pytest.mark.parametrize("budget", [0, 3 << 20], ids=["one_chunk", "chunks"])
def test_batch_matches_oracle_and_single_frames(budget):
    torch = _torch()
    trees, want, oracle = [], [], []
    fast = _fast_router()
    for k, (preset, W, H, S, seed) in enumerate(FRAMES):
        rec, coc = tlfr.synth_scene(preset, W, H, S, seed)
        g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
        if k == 1:
            g.set_routing(fast, 0.5)
        else:
            oracle.append((k, CpuRecon("orc", rec, coc).reconstruct()))
        want.append(g.reconstructDofMotion())
        trees.append(g)
    outs = [torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda") for (_, W, H, _, _) in FRAMES]
    batch = tlfr.Batch(trees, [o.data_ptr() for o in outs], autotune=True, budget_bytes=budget)
    shapes = batch.tile_shapes()
    chunks, launches = batch.layout()
    assert len(shapes) == len(FRAMES) and ((shapes >= 0) & (shapes < len(tlfr.TILE_SHAPES))).all()
    if budget:
        assert chunks.max() >= 2, chunks          # several chunks share the storage
    else:
        assert chunks.max() == 0
    assert launches > 0
    for run in range(2):
        for o in outs:
            o.fill_(float("nan"))
        batch.run()
        ms = batch.sync()
        assert ms > 0
        got = [o.cpu().numpy() for o in outs]
        for k, w in enumerate(want):
            assert np.array_equal(got[k].view(np.uint32), w.view(np.uint32)), (run, k)
        for k, ref in oracle:
            assert np.array_equal(got[k].view(np.uint32), ref.view(np.uint32)), (run, k)
    batch.close()
    trees[1].set_routing(None)
    fast.close()


def test_batch_retry_tier_matches_oracle():
    """The benchmark scene at 960x540x8 beside a small frame: output samples of the large
    frame outgrow the first light tier (the single-frame path reports them) and the batch's
    retry launch runs them; both frames equal the oracle's images bit for bit."""
    torch = _torch()
    import os
    specs = [(tlfr.SCENE_CARDS_LARGE, 960, 540, 8, 6), (tlfr.SCENE_CARDS, 64, 48, 4, 61)]
    trees, refs, outs = [], [], []
    for preset, W, H, S, seed in specs:
        rec, coc = tlfr.synth_scene(preset, W, H, S, seed)
        g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
        trees.append(g)
        refs.append(CpuRecon("orc", rec, coc, nthreads=os.cpu_count() or 8).reconstruct())
        outs.append(torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda"))
    trees[0].reconstructDofMotion()
    assert trees[0].stats().num_retried_queries > 0
    batch = tlfr.Batch(trees, [o.data_ptr() for o in outs], autotune=False)
    batch.run()
    batch.sync()
    for o, ref in zip(outs, refs):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    batch.close()


def test_batch_sweep_over_one_hierarchy():
    """A (u,v,t) movie of one buffer (the reference's export path builds a new
    TreeGather per frame, App.cpp:616-694): one hierarchy, one frame per output
    setting, each equal to the oracle's image for that setting."""
    torch = _torch()
    W, H, S = 48, 32, 4
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, W, H, S, 66)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    settings = [tlfr.CameraParams(overrideUVT=((u + 0.5) / 2, (v + 0.5) / 2, 0.5)) for v in range(2) for u in range(2)]
    settings.append(tlfr.CameraParams(overrideUVT=(0.0, 0.0, 1.0)))          # the t=1 pinhole image
    settings.append(tlfr.CameraParams(outputSpp=64))
    outs = [torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda") for _ in settings]
    batch = tlfr.Batch([g] * len(settings), [o.data_ptr() for o in outs], autotune=False, params=settings)
    batch.run()
    batch.sync()
    for p, o in zip(settings, outs):
        ref = CpuRecon("orc", rec, coc, uvt=p.overrideUVT, output_spp=p.outputSpp).reconstruct()
        got = o.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), p.overrideUVT
    batch.close()


def test_batch_rejects_bad_arguments():
    _torch()
    with pytest.raises(tlfr.TlfrError):
        tlfr.Batch([], [])


def test_trim_keeps_the_hierarchy():
    """tlfr_trim frees the build's working storage: reconstructions after it, and
    after a rebuild that allocates it again, give the same image."""
    _torch()
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS_LARGE, 64, 40, 8, 67)
    buf = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    g = tlfr.TreeGather(buf)
    want = g.reconstructDofMotion()
    g.trim()
    assert np.array_equal(g.reconstructDofMotion().view(np.uint32), want.view(np.uint32))
    g.rebuild_from(buf)
    assert np.array_equal(g.reconstructDofMotion().view(np.uint32), want.view(np.uint32))
    g.close()
