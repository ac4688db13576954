"""CUDA path (libtlfr.so through its C ABI) against the CPU checkers.

Bar: the hierarchy is identical node for node (bounds bitwise, same sample order);
every traced output sample accepts the same samples into the same surfaces and
returns the same colour bit for bit; pixels agree within 1e-4 relative per
channel (the frame sums output samples in a different order only when a query ran
in the large-capacity pass)."""
import numpy as np
import pytest

import tlfr
from tlfr_testutil import GOLDEN, CpuRecon, compare_trees, rel_err, sample_queries, tree_digest

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def gpu_recon(rec, coc, aperture=1.0, focus=1.0, uvt=None, lens=0, time=0, output_spp=0):
    buf = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    p = tlfr.CameraParams(lensFilter=lens, timeFilter=time, overrideUVT=uvt, outputSpp=output_spp)
    return tlfr.TreeGather(buf, p, aperture, focus)


def check_tree(g, o):
    gt = g.tree_export()
    ot = o.tree()
    assert compare_trees(gt, ot) == []
    # same sample layout as the reference (task order, preorder, sorted within leaves)
    assert np.array_equal(gt[3], ot[3])
    n, s, _root, height = g.tree_info()
    assert s == o.num_samples
    assert height >= 1


def check_queries(g, o, W, H, M, n, seed):
    q = sample_queries(W, H, M, n, seed)
    rgba, tr = g.trace_queries(q, stride=8192)
    for k, (x, y, i) in enumerate(q):
        oc, ot = o.query(int(x), int(y), int(i), 8192)
        row = tr[k]
        assert row[1] != -1, "trace truncated"
        assert np.array_equal(row[:len(ot)], ot), f"query ({x},{y},{i}) surfaces differ"
        assert np.array_equal(rgba[k].view(np.uint32), oc.view(np.uint32)), f"query ({x},{y},{i}) colour"


SCENES = [
    ("planes", tlfr.SCENE_PLANES, 64, 48, 4, 31, {}),
    ("cards", tlfr.SCENE_CARDS, 96, 64, 4, 32, {}),
    ("cards_refocus", tlfr.SCENE_CARDS, 80, 48, 2, 33, {"aperture": 1.5, "focus": 0.8}),
    ("cards_pinhole", tlfr.SCENE_CARDS, 96, 64, 4, 34, {"uvt": (0.0, 0.0, 1.0)}),
    ("cards_uvt", tlfr.SCENE_CARDS, 64, 48, 4, 35, {"uvt": (-0.3, 0.6, 0.25)}),
    ("large", tlfr.SCENE_CARDS_LARGE, 128, 80, 8, 36, {}),
    ("planes_m64", tlfr.SCENE_PLANES, 64, 64, 16, 37, {"output_spp": 64}),
    ("cards_1spp", tlfr.SCENE_CARDS, 64, 40, 1, 38, {}),
    ("planes_spp3", tlfr.SCENE_PLANES, 30, 20, 3, 39, {}),
]


@pytest.mark.parametrize("name,preset,W,H,spp,seed,p", SCENES, ids=[s[0] for s in SCENES])
def test_gpu_matches_oracle(name, preset, W, H, spp, seed, p):
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    kw = dict(aperture=p.get("aperture", 1.0), focus=p.get("focus", 1.0), uvt=p.get("uvt"),
              lens=p.get("lens", 0), time=p.get("time", 0), output_spp=p.get("output_spp", 0))
    g = gpu_recon(rec, coc, **kw)
    o = CpuRecon("orc", rec, coc, **kw)
    check_tree(g, o)
    assert np.array_equal(g.output_samples().view(np.uint32), o.output_samples().view(np.uint32))
    check_queries(g, o, W, H, o.out_spp, 400, seed)
    img = g.reconstructDofMotion()
    ref = o.reconstruct()
    assert rel_err(img, ref).max() <= RTOL
    # every output sample's colour is exact and pixels sum them in sample order,
    # as the reference does, so the frame is bit-identical
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))


def test_gpu_gaussian_filters():
    """Lens/time Gaussian weights use powf on both sides (RO.cpp:354-355): within tolerance."""
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS_LARGE, 48, 32, 8, 40)
    g = gpu_recon(rec, coc, lens=1, time=1)
    o = CpuRecon("orc", rec, coc, lens=1, time=1)
    check_tree(g, o)
    img = g.reconstructDofMotion()
    assert rel_err(img, o.reconstruct()).max() <= RTOL


def test_gpu_stats_match_oracle_counters():
    """Device counters equal the reference Stats sums (the roofline's algorithmic bytes)."""
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS_LARGE, 64, 48, 8, 41)
    g = gpu_recon(rec, coc)
    o = CpuRecon("orc", rec, coc)
    _img, st = g.reconstructDofMotion(stats=True)
    o.reconstruct()
    s = o.last_stats
    assert st.num_output_samples == s[1]
    assert st.num_leaf_nodes == s[0]
    assert st.num_samples_in_leaf_nodes == s[2]
    assert st.num_samples_within_1r == s[4]
    assert st.num_samples_fetched == s[6]
    assert st.num_surfaces == s[8]
    assert st.num_2r == s[10]
    assert st.num_surfaces_merged == s[12]
    assert st.num_at_least_one == s[14]


@pytest.mark.parametrize("path", sorted(__import__("glob").glob(GOLDEN + "/*.npz")))
def test_gpu_matches_reference_golden(path):
    g0 = np.load(path)
    uvt = g0["uvt"]
    kw = dict(aperture=float(g0["aperture"]), focus=float(g0["focus"]),
              uvt=None if np.isnan(uvt).any() else tuple(float(v) for v in uvt),
              lens=int(g0["lens"]), time=int(g0["time"]), output_spp=int(g0["output_spp"]))
    g = gpu_recon(g0["records"], tuple(g0["coc"]), **kw)
    digest, nreach = tree_digest(g.tree_export())
    assert (digest, nreach) == (g0["tree_digest"].item().decode(), int(g0["tree_nodes"]))
    assert np.array_equal(g.output_samples().view(np.uint32), g0["pattern"].view(np.uint32))
    rgba, tr = g.trace_queries(g0["queries"], stride=g0["query_traces"].shape[1])
    gauss = kw["lens"] or kw["time"]
    for k in range(len(g0["queries"])):
        ref_tr = g0["query_traces"][k]
        n = int(np.argmax(ref_tr == -2)) if (ref_tr == -2).any() else len(ref_tr)
        assert np.array_equal(tr[k][:n], ref_tr[:n])
        if gauss:
            # Gaussian output-sample weights use powf (Reconstruction.hpp:378); the
            # device powf and the host libm powf may differ in the last bit
            assert rel_err(rgba[k], g0["query_rgba"][k]).max() <= 1e-6
        else:
            assert np.array_equal(rgba[k].view(np.uint32), g0["query_rgba"][k].view(np.uint32))
    img = g.reconstructDofMotion()
    assert rel_err(img, g0["image"]).max() <= RTOL


def test_gpu_set_output_reuses_hierarchy():
    """Refocus/animation loop: change (u,v,t) without rebuilding (App.cpp:616-694)."""
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, 64, 40, 4, 42)
    g = gpu_recon(rec, coc)
    for uvt in [(0.0, 0.0, 1.0), (0.5, -0.5, 0.0)]:
        g.set_output(tlfr.CameraParams(overrideUVT=uvt))
        o = CpuRecon("orc", rec, coc, uvt=uvt)
        assert rel_err(g.reconstructDofMotion(), o.reconstruct()).max() <= RTOL


def test_gpu_repeatable():
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, 64, 48, 4, 43)
    g = gpu_recon(rec, coc)
    a = g.reconstructDofMotion()
    b = g.reconstructDofMotion()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.isfinite(a).all() and np.all(a[..., 3] == 1.0)


@pytest.mark.slow
def test_gpu_full_size_band_matches_oracle():
    """1920x1080, 8 spp, strong blur and motion (the benchmark frame): identical
    hierarchy, 2000 traced output samples, and a band of full rows."""
    W, H, spp = 1920, 1080, 8
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS_LARGE, W, H, spp, 2)
    g = gpu_recon(rec, coc)
    o = CpuRecon("orc", rec, coc, nthreads=16)
    check_tree(g, o)
    check_queries(g, o, W, H, 128, 2000, 7)
    img = g.reconstructDofMotion()
    for y0 in (0, 537, 1076):
        band = o.reconstruct_rows(y0, y0 + 4)
        assert rel_err(img[y0:y0 + 4], band).max() <= RTOL


EDGE = [
    ("one_row", tlfr.SCENE_CARDS, 17, 1, 4, 41),
    ("one_column", tlfr.SCENE_CARDS_LARGE, 2, 9, 8, 42),
    ("tiny_16spp", tlfr.SCENE_PLANES, 3, 2, 16, 43),
]


@pytest.mark.parametrize("name,preset,W,H,spp,seed", EDGE, ids=[e[0] for e in EDGE])
def test_gpu_degenerate_frames_match_oracle(name, preset, W, H, spp, seed):
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    g = gpu_recon(rec, coc)
    o = CpuRecon("orc", rec, coc)
    check_tree(g, o)
    img = g.reconstructDofMotion()
    assert np.array_equal(img.view(np.uint32), o.reconstruct().view(np.uint32))


def test_gpu_all_samples_discarded_reports_empty():
    # a 1x1 frame whose only sample reprojects off screen: the reference fails with
    # "All samples were discarded" (Reconstruction.cpp:587-588); here TLFR_EMPTY
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, 1, 1, 1, 5)
    with pytest.raises(RuntimeError):
        CpuRecon("orc", rec, coc)
    with pytest.raises(tlfr.TlfrError) as e:
        gpu_recon(rec, coc)
    assert e.value.status == 9   # TLFR_EMPTY


FULL_FRAMES = [
    # the 256x256, 16 spp three-plane frame with 64 output samples per pixel
    ("planes_256x256x16_m64", tlfr.SCENE_PLANES, 256, 256, 16, 3, {"output_spp": 64}),
    # the 962x543, 4 spp 64-card frame (defocus and motion), blurred and as the t=1 pinhole image
    ("cards_962x543x4", tlfr.SCENE_CARDS, 962, 543, 4, 4, {}),
    ("cards_962x543x4_pinhole", tlfr.SCENE_CARDS, 962, 543, 4, 4, {"uvt": (0.0, 0.0, 1.0)}),
    # the benchmark scene (256 cards and 64 disks, strong blur and motion) at 960x540x8: output
    # samples outgrow the first light tier and are run again by the retry tier
    ("cards_large_960x540x8", tlfr.SCENE_CARDS_LARGE, 960, 540, 8, 6, {}),
]


@pytest.mark.parametrize("name,preset,W,H,spp,seed,p", FULL_FRAMES, ids=[s[0] for s in FULL_FRAMES])
def test_gpu_full_frame_matches_oracle(name, preset, W, H, spp, seed, p):
    """Whole frames of the stated workload sizes, every pixel against the oracle."""
    import os
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    kw = dict(uvt=p.get("uvt"), output_spp=p.get("output_spp", 0))
    g = gpu_recon(rec, coc, **kw)
    img = g.reconstructDofMotion()
    if name.startswith("cards_large"):
        st = g.stats()      # counts of the reconstruction that made img (not a statistics run)
        assert st.num_retried_queries > 0 and st.num_heavy_queries > 0
    o = CpuRecon("orc", rec, coc, nthreads=os.cpu_count() or 8, **kw)
    ref = o.reconstruct()
    assert rel_err(img, ref).max() <= RTOL
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))


def test_gpu_output_sample_buffer_matches_oracle(tmp_path):
    """The output-sample dump (the reference's m_obuf): every record holds its
    output sample's position, lens and time coordinates and the colour the oracle
    computes for it; the dump survives a text save and load."""
    W, H, spp = 24, 16, 4
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, W, H, spp, 42)
    g = gpu_recon(rec, coc)
    g.reconstructDofMotion()
    ob = g.output_sample_buffer()
    M = 128
    r = ob.records()
    assert r.shape == (H, W, M, 16)
    o = CpuRecon("orc", rec, coc)
    pat = o.output_samples().reshape(64, M, 5)
    from tlfr_testutil import hash_pattern
    rng = np.random.default_rng(43)
    for _ in range(200):
        x, y, i = int(rng.integers(0, W)), int(rng.integers(0, H)), int(rng.integers(0, M))
        pp = pat[hash_pattern(x, y), i]
        want = np.float32([pp[0] + x, pp[1] + y, 1, 1, pp[2], pp[3], pp[4]])
        assert np.array_equal(r[y, x, i, :7].view(np.uint32), want.view(np.uint32))
        col, _ = o.query(x, y, i)
        assert np.array_equal(r[y, x, i, 7:11].view(np.uint32), col.view(np.uint32))
    path = str(tmp_path / "outputSamples.txt")
    ob.serialize(path, separate_header=False, binary=False)
    back = tlfr.UVTSampleBuffer(path).records()
    # text round trip keeps positions and colours (alpha is forced to 1 on load)
    assert np.allclose(back[..., :10], r[..., :10], rtol=1e-6, atol=1e-6)
