"""Shadow reconstruction (TreeGather::reconstructShadows, Reconstruction.cpp:302-344):
light-space query samples through the Filterer in shadow mode on the GPU, against
the reference build's own reconstructShadows, every query's colour bit for bit."""
import numpy as np
import pytest

import tlfr
from tlfr_testutil import CpuRecon, ref_available, rel_err

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


def _perspective(fov_deg, aspect, near, far):
    f = 1.0 / np.tan(np.radians(fov_deg) / 2)
    return np.array([[f / aspect, 0, 0, 0],
                     [0, f, 0, 0],
                     [0, 0, (far + near) / (near - far), 2 * far * near / (near - far)],
                     [0, 0, -1, 0]], np.float64)


def _pose(yaw_deg, t):
    a = np.radians(yaw_deg)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = np.cos(a), np.sin(a), -np.sin(a), np.cos(a)
    m[:3, 3] = t
    return m


def _dms_scene(W, H, spp, seed, cam_far, light_offset, density, filters=False, cam_preset=tlfr.SCENE_PLANES):
    """A camera buffer (the planes scene, w in 2..12, or the moving cards) and a light-space
    buffer of the same size (the planes scene), both with random depth gradients, the two
    cameras (the light shifted and turned; the camera with Gaussian lens and time filters
    when filters), and the camera buffer's light-space density channel (or None)."""
    rng = np.random.default_rng(seed)
    cam_rec, cam_coc = tlfr.synth_scene(cam_preset, W, H, spp, seed)
    light_rec, light_coc = tlfr.synth_scene(tlfr.SCENE_PLANES, W, H, spp, seed + 1)
    for r in (cam_rec, light_rec):
        r[..., 14:16] = rng.uniform(-0.04, 0.04, r.shape[:3] + (2,)).astype(np.float32)
    proj = _perspective(60.0, W / H, 0.1, 100.0).astype(np.float32)
    c2w = _pose(0.0, (0.0, 0.0, 0.0))
    l2w = _pose(8.0, light_offset)
    cam = tlfr.CameraParams(projection=proj, cameraToWorld=c2w.astype(np.float32),
                            worldToCamera=np.linalg.inv(c2w).astype(np.float32), far=cam_far,
                            windowSize=(W, H), apertureRadius=0.05, focusDistance=5.0,
                            lensFilter=tlfr.LENS_GAUSSIAN if filters else tlfr.LENS_BOX,
                            timeFilter=tlfr.TIME_GAUSSIAN if filters else tlfr.TIME_BOX)
    light = tlfr.CameraParams(projection=proj, cameraToWorld=l2w.astype(np.float32),
                              worldToCamera=np.linalg.inv(l2w).astype(np.float32), far=100.0,
                              windowSize=(W, H), apertureRadius=0.5, focusDistance=5.0)
    dens = rng.uniform(0.5, 2.0, cam_rec.shape[:3]).astype(np.float32) if density else None
    return cam_rec, cam_coc, cam, light_rec, light_coc, light, dens


_dms_scene.cases = [
    (40, 24, 4, 93, 100.0, (0.3, 0.2, 0.0), True),
    (48, 32, 8, 94, 7.0, (-0.5, 0.1, 0.3), False),
    # moving cards seen through Gaussian lens and time filters
    (44, 28, 4, 95, 100.0, (0.2, -0.3, 0.1), True, True, tlfr.SCENE_CARDS),
]


@pytest.mark.parametrize("case", _dms_scene.cases)
def test_gpu_dof_motion_shadows_match_reference(case):
    """TreeGather::reconstructDofMotionShadows (Reconstruction.cpp:355-433, 723-829) on the
    GPU against the reference build's, every pixel bit for bit (within 1e-4 with Gaussian
    lens and time filters)."""
    if not ref_available():
        pytest.skip("reference build absent")
    cam_rec, cam_coc, cam, light_rec, light_coc, light, dens = _dms_scene(*case)
    cg = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=cam_rec, coc=cam_coc), cam)
    lg = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=light_rec, coc=light_coc), light)
    got = cg.reconstructDofMotionShadows(lg, dens)
    filt = 1 if len(case) > 7 and case[7] else 0
    c = CpuRecon("ref", cam_rec, cam_coc, density=dens, lens=filt, time=filt)
    l = CpuRecon("ref", light_rec, light_coc)
    c.set_view(cam)
    l.set_view(light)
    want = c.dof_motion_shadows(l)
    if filt:
        # the Gaussian lens and time weights are powf on both sides (RO.cpp:354-355), which
        # CUDA and the host library may round differently: within 1e-4 relative per channel
        assert rel_err(got, want).max() <= 1e-4
    else:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the shading changed the camera's image
    plain = cg.reconstructDofMotion()
    assert (np.abs(got - plain).max(-1) > 1e-3).mean() > 0.2
