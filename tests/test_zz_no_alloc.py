"""tlfr_query_samples_noalloc: output-sample queries for callers that cannot
allocate device memory while they run.  Its per-query working storage is a fixed
device array inside the library, so the call allocates nothing; the caller passes
device buffers for the queries, the colours and the overflow count.

Checked against the allocating entry point (tlfr_trace_queries) on the same output
samples, on two calls in a row (the shared array keeps the previous call's
contents, which must not matter).  This file is collected last."""
import ctypes

import numpy as np
import pytest

import tlfr
from tlfr_testutil import sample_queries

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


def test_noalloc_rejects_oversized_call():
    torch = _torch()
    lib = tlfr.load_library()
    rec, coc = tlfr.synth_scene(tlfr.SCENE_PLANES, 16, 12, 2, 53)
    g = tlfr.TreeGather(tlfr.UVTSampleBuffer(records=rec, coc=coc))
    d = torch.zeros(3, dtype=torch.int32, device="cuda")
    o = torch.zeros(4, dtype=torch.float32, device="cuda")
    st = lib.tlfr_query_samples_noalloc(g.handle, ctypes.c_void_p(d.data_ptr()), (1 << 22) + 1,
                                        ctypes.c_void_p(o.data_ptr()), None)
    assert st == 1
    assert b"num_queries" in lib.tlfr_last_error(g.handle)
