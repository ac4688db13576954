"""Learned routing: the network's forward and backward kernels against the CPU
restatement (tests/route_ref.py), and what the trained router gains over the
method without it."""
import numpy as np
import pytest

import route_ref as R
import tlfr


def test_reference_backward_matches_finite_differences():
    # pins the CPU restatement's backward formulas (no rounding, float64)
    rng = np.random.default_rng(0)
    p = R.init_params(3).astype(np.float64)
    f = rng.normal(size=(37, 8)).astype(np.float32)
    lab = (rng.random(37) < 0.5).astype(np.float64)
    g = R.gradient(p, f, lab, bf=False)
    eps = 1e-6
    for i in [0, 5, 70, R.OFF_B1 + 3, R.OFF_W2 + 17, R.OFF_W2 + 1000, R.OFF_B2 + 9, R.OFF_W3 + 4, R.OFF_B3]:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (R.loss(pp, f, lab, bf=False) - R.loss(pm, f, lab, bf=False)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.1415926], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125) and r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-7


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


@pytest.mark.gpu
def test_router_kernels_match_reference():
    torch = _torch()
    rng = np.random.default_rng(5)
    n = 1000   # not a multiple of the 16-row tiles
    feats = rng.normal(size=(n, 8)).astype(np.float32) * 2 + 1
    labels = (rng.random(n) < 0.4).astype(np.float32)
    mean = feats.mean(0)
    inv_std = 1.0 / feats.std(0)
    router = tlfr.Router(0, seed=11, mean=mean, inv_std=inv_std)
    p = router.params()
    assert p.size == R.NUM_PARAMS
    assert np.all(p[R.OFF_W1:R.OFF_B1].reshape(64, 16)[:, 8:] == 0)
    d_f = torch.from_numpy(feats).cuda()
    d_l = torch.from_numpy(labels).cuda()
    d_p = torch.empty(n, dtype=torch.float32, device="cuda")
    router.predict(d_f.data_ptr(), n, d_p.data_ptr())
    torch.cuda.synchronize()
    want = R.forward(p, feats)["p"]
    assert np.abs(d_p.cpu().numpy() - want).max() < 2e-3
    g, loss = router.gradient(d_f.data_ptr(), d_l.data_ptr(), n)
    gr = R.gradient(p, feats, labels)
    assert abs(loss - R.loss(p, feats, labels)) < 1e-3
    scale = np.abs(gr).max()
    assert np.linalg.norm(g - gr) <= 1e-2 * np.linalg.norm(gr), np.linalg.norm(g - gr) / np.linalg.norm(gr)
    assert np.abs(g - gr).max() <= 2e-2 * scale
    # every block is exercised
    for a, b in [(R.OFF_W1, R.OFF_B1), (R.OFF_B1, R.OFF_W2), (R.OFF_W2, R.OFF_B2), (R.OFF_B2, R.OFF_W3),
                 (R.OFF_W3, R.OFF_B3)]:
        assert np.abs(g[a:b]).max() > 0
    # parameters round-trip
    q = p.copy()
    q[R.OFF_B3] += 0.5
    router.set_params(q)
    assert router.params()[R.OFF_B3] == q[R.OFF_B3]
    router.close()


def _frames(torch, seeds, W, H, S):
    """(features, labels, plain image, tree) for the config-2 scene generator at a small size."""
    out = []
    for seed in seeds:
        rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS_LARGE, W, H, S, seed)
        g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
        f = torch.empty((H * W, 8), dtype=torch.float32, device="cuda")
        lab = torch.empty(H * W, dtype=torch.float32, device="cuda")
        img = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
        g.route_features(f.data_ptr())
        g.route_labels(lab.data_ptr(), img.data_ptr())
        out.append((f, lab, img, g))
    return out


@pytest.mark.gpu
def test_router_learns_and_routes():
    torch = _torch()
    W, H, S = 320, 180, 8
    train = _frames(torch, range(100, 106), W, H, S)
    held = _frames(torch, [140, 141], W, H, S)
    feats = torch.cat([t[0] for t in train])
    labels = torch.cat([t[1] for t in train])
    fh = feats.cpu().numpy()
    router = tlfr.Router(0, seed=3, mean=fh.mean(0), inv_std=1.0 / np.maximum(fh.std(0), 1e-6))
    n = feats.shape[0]
    loss0 = router.gradient(feats.data_ptr(), labels.data_ptr(), n)[1]
    loss = router.train(feats.data_ptr(), labels.data_ptr(), n, steps=600, batch=4096, lr=3e-3)
    print(f"train: {n} pixels, label mean {labels.mean().item():.3f}, loss {loss0:.4f} -> {loss:.4f}")
    assert loss < loss0 * 0.8, (loss0, loss)
    # held-out: routing sends a good share of pixels to the fast path while the image
    # stays much closer to the plain method than with every pixel on the fast path
    for f, lab, plain, g in held:
        prob = torch.empty(W * H, dtype=torch.float32, device="cuda")
        router.predict(f.data_ptr(), W * H, prob.data_ptr())
        pr, lb = prob.cpu().numpy(), lab.cpu().numpy()
        acc = float(((pr > 0.5) == (lb > 0.5)).mean())
        sel = pr > 0.8
        precision = float(lb[sel].mean()) if sel.any() else 1.0
        print(f"held-out: label mean {lb.mean():.3f} accuracy {acc:.3f} precision@0.8 {precision:.3f}")
        # routed reconstruction
        g.set_routing(router, 0.8)
        routed = np.empty((H, W, 4), np.float32)
        g.reconstructDofMotion(routed)
        fast = float((pr > 0.8).mean())
        # everything on the fast path (the method without the network's abstention)
        g.set_routing(_always_fast(router), 0.5)
        allfast = np.empty((H, W, 4), np.float32)
        g.reconstructDofMotion(allfast)
        g.set_routing(None)
        pl = plain.cpu().numpy()
        p_routed, p_all = R.psnr(routed, pl), R.psnr(allfast, pl)
        print(f"held-out: fast {fast:.3f} psnr routed {p_routed:.2f} all-fast {p_all:.2f} "
              f"max err {np.abs(routed - pl)[..., :3].max():.4f}")
        assert fast > 0.2, fast
        assert p_routed > p_all + 0.5, (p_routed, p_all)
        assert p_routed > 42.0, p_routed
    router.close()


_ALWAYS = {}


def _always_fast(router):
    """A router whose output is 1 everywhere (large output bias): the fast path without the network."""
    if "r" not in _ALWAYS:
        r = tlfr.Router(0, seed=1)
        p = r.params()
        p[R.OFF_W3:R.OFF_B3] = 0
        p[R.OFF_B3] = 50.0
        r.set_params(p)
        _ALWAYS["r"] = r
    return _ALWAYS["r"]

