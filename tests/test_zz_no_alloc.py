"""tlfr_query_samples_noalloc: output-sample queries for callers that cannot
allocate device memory while they run.  Its per-query working storage is a fixed
device array inside the library, so the call allocates nothing; the caller passes
device buffers for the queries, the colours and the overflow count.

Checked against the allocating entry point (tlfr_trace_queries) and the CPU
oracle on the same output samples, on two calls in a row (the shared array keeps
the previous call's contents, which must not matter); plus the edge cases: no
queries, no overflow counter, out-of-range (x, y, i) entries, a misaligned colour
pointer, an oversized call, and a full call's rate.  This file is collected last."""
import ctypes
import time

import numpy as np
import pytest

import tlfr
from tlfr_testutil import CpuRecon, sample_queries

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


@pytest.mark.parametrize("preset,W,H,spp,seed", [
    (tlfr.SCENE_CARDS_LARGE, 96, 64, 8, 51),
    (tlfr.SCENE_CARDS, 64, 48, 4, 52),
])
def test_noalloc_matches_allocating_path(preset, W, H, spp, seed):
    torch = _torch()
    lib = tlfr.load_library()
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    q = sample_queries(W, H, 128, 600, seed)
    want, _trace = g.trace_queries(q, stride=8192)
    d_q = torch.from_numpy(q).cuda()
    d_out = torch.empty((len(q), 4), dtype=torch.float32, device="cuda")
    d_ovf = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
    for _call in range(2):
        d_out.fill_(float("nan"))
        st = lib.tlfr_query_samples_noalloc(g.handle, ctypes.c_void_p(d_q.data_ptr()), len(q),
                                            ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_ovf.data_ptr()))
        assert st == 0, lib.tlfr_last_error(g.handle)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        ok = got[:, 3] >= 0
        assert int(d_ovf.item()) == int((~ok).sum())
        assert ok.mean() > 0.99
        # per-sample colours are exact in both paths
        assert np.array_equal(got[ok].view(np.uint32), want[ok].view(np.uint32))
    # and equal to the CPU oracle's output samples
    o = CpuRecon("orc", rec, coc)
    ref = np.stack([o.query(int(x), int(y), int(i))[0] for x, y, i in q])
    o.close()
    assert np.array_equal(got[ok].view(np.uint32), ref[ok].view(np.uint32))


def test_noalloc_edge_cases():
    torch = _torch()
    lib = tlfr.load_library()
    W, H = 48, 32
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, W, H, 4, 54)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    # no queries: the counter is still cleared
    d_ovf = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    d_q = torch.zeros((1, 3), dtype=torch.int32, device="cuda")
    d_out = torch.zeros((1, 4), dtype=torch.float32, device="cuda")
    st = lib.tlfr_query_samples_noalloc(g.handle, ctypes.c_void_p(d_q.data_ptr()), 0,
                                        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_ovf.data_ptr()))
    assert st == 0
    torch.cuda.synchronize()
    assert int(d_ovf.item()) == 0
    # out-of-range entries among valid ones give (0, 0, 0, -1) and are counted;
    # with and without the overflow counter
    q = sample_queries(W, H, 128, 64, 55)
    bad = np.array([[-1, 0, 0], [W, 0, 0], [0, H, 0], [0, -3, 0], [0, 0, 128], [1, 1, -1]], np.int32)
    qq = np.concatenate([q[:20], bad, q[20:]])
    want, _ = g.trace_queries(q, stride=8192)
    d_q = torch.from_numpy(qq).cuda()
    d_out = torch.empty((len(qq), 4), dtype=torch.float32, device="cuda")
    for with_counter in (True, False):
        d_out.fill_(float("nan"))
        ptr = ctypes.c_void_p(d_ovf.data_ptr()) if with_counter else None
        st = lib.tlfr_query_samples_noalloc(g.handle, ctypes.c_void_p(d_q.data_ptr()), len(qq),
                                            ctypes.c_void_p(d_out.data_ptr()), ptr)
        assert st == 0, lib.tlfr_last_error(g.handle)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.array_equal(got[20:20 + len(bad)], np.tile(np.float32([0, 0, 0, -1]), (len(bad), 1)))
        good = np.concatenate([got[:20], got[20 + len(bad):]])
        assert (good[:, 3] >= 0).all()
        assert np.array_equal(good.view(np.uint32), want.view(np.uint32))
        if with_counter:
            assert int(d_ovf.item()) == len(bad)
    # a colour pointer that is not 16-byte aligned is refused before any launch
    st = lib.tlfr_query_samples_noalloc(g.handle, ctypes.c_void_p(d_q.data_ptr()), 4,
                                        ctypes.c_void_p(d_out.data_ptr() + 4), None)
    assert st == 1
    assert b"aligned" in lib.tlfr_last_error(g.handle)


def test_noalloc_full_call():
    """A call at the cap (262144 output samples of the 8-spp strong-blur scene)
    finishes, agrees with the allocating path on a sample of its queries, and
    reports its rate."""
    torch = _torch()
    lib = tlfr.load_library()
    W, H, S = 256, 192, 8
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS_LARGE, W, H, S, 56)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    n = 1 << 18
    q = sample_queries(W, H, 128, n, 57)
    d_q = torch.from_numpy(q).cuda()
    d_out = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    d_ovf = torch.zeros(1, dtype=torch.int32, device="cuda")
    args = (g.handle, ctypes.c_void_p(d_q.data_ptr()), n, ctypes.c_void_p(d_out.data_ptr()),
            ctypes.c_void_p(d_ovf.data_ptr()))
    assert lib.tlfr_query_samples_noalloc(*args) == 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    assert lib.tlfr_query_samples_noalloc(*args) == 0
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    print(f"noalloc: {n} output samples in {dt * 1e3:.1f} ms ({n / dt / 1e6:.2f} M/s)")
    got = d_out.cpu().numpy()
    pick = np.arange(0, n, 997)
    want, _ = g.trace_queries(q[pick], stride=8192)
    ok = got[pick, 3] >= 0
    assert ok.mean() > 0.99
    assert np.array_equal(got[pick][ok].view(np.uint32), want[ok].view(np.uint32))


def test_noalloc_rejects_oversized_call():
    torch = _torch()
    lib = tlfr.load_library()
    rec, coc = tlfr.synth_scene(tlfr.SCENE_PLANES, 16, 12, 2, 53)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    d = torch.zeros(3, dtype=torch.int32, device="cuda")
    o = torch.zeros(4, dtype=torch.float32, device="cuda")
    st = lib.tlfr_query_samples_noalloc(g.handle, ctypes.c_void_p(d.data_ptr()), (1 << 18) + 1,
                                        ctypes.c_void_p(o.data_ptr()), None)
    assert st == 1
    assert b"num_queries" in lib.tlfr_last_error(g.handle)
