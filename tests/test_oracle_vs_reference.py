"""Pins the CPU restatement to the reference's own CPU code (oracle/_ref, built
from the reference sources by oracle/build_ref.sh) on fresh seeded scenes:
identical hierarchy, output pattern, per-query surfaces and every pixel."""
import numpy as np
import pytest

import tlfr
from tlfr_testutil import CpuRecon, compare_trees, ref_available, sample_queries

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference build oracle/_ref not present")

SCENES = [
    (tlfr.SCENE_PLANES, 40, 32, 4, 11, {}),
    (tlfr.SCENE_CARDS, 64, 40, 4, 12, {}),
    (tlfr.SCENE_CARDS, 48, 32, 2, 13, {"aperture": 0.6, "focus": 1.3}),
    (tlfr.SCENE_CARDS, 48, 36, 4, 14, {"uvt": (0.25, -0.5, 1.0)}),
    (tlfr.SCENE_CARDS_LARGE, 64, 48, 8, 15, {}),
    (tlfr.SCENE_CARDS_LARGE, 40, 24, 16, 16, {"lens": 1, "time": 1}),
    (tlfr.SCENE_CARDS, 20, 16, 1, 17, {}),
    (tlfr.SCENE_PLANES, 12, 10, 3, 18, {}),          # spp rounded up to 4
]


@pytest.mark.parametrize("preset,W,H,spp,seed,p", SCENES)
def test_restatement_equals_reference(preset, W, H, spp, seed, p):
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    kw = dict(aperture=p.get("aperture", 1.0), focus=p.get("focus", 1.0), uvt=p.get("uvt"),
              lens=p.get("lens", 0), time=p.get("time", 0))
    r = CpuRecon("ref", rec, coc, **kw)
    o = CpuRecon("orc", rec, coc, **kw)
    assert (o.spp_pow2, o.out_spp) == (r.spp_pow2, r.out_spp)
    assert o.coc_adjusted.view(np.uint32).tolist() == r.coc_adjusted.view(np.uint32).tolist()
    assert compare_trees(o.tree(), r.tree()) == []
    assert np.array_equal(o.output_samples().view(np.uint32), r.output_samples().view(np.uint32))
    for x, y, i in sample_queries(W, H, r.out_spp, 300, seed):
        ca, ta = r.query(int(x), int(y), int(i))
        cb, tb = o.query(int(x), int(y), int(i))
        assert np.array_equal(ta, tb) and np.array_equal(ca.view(np.uint32), cb.view(np.uint32))
    assert np.array_equal(o.reconstruct().view(np.uint32), r.reconstruct().view(np.uint32))


@pytest.mark.skipif(not ref_available(m64=True), reason="64-output-sample reference build not present")
def test_restatement_equals_reference_64_outputs():
    rec, coc = tlfr.synth_scene(tlfr.SCENE_PLANES, 32, 24, 16, 21)
    r = CpuRecon("ref", rec, coc, m64=True)
    o = CpuRecon("orc", rec, coc, output_spp=64)
    assert r.out_spp == 64 and o.out_spp == 64
    assert np.array_equal(o.output_samples().view(np.uint32), r.output_samples().view(np.uint32))
    assert np.array_equal(o.reconstruct().view(np.uint32), r.reconstruct().view(np.uint32))
