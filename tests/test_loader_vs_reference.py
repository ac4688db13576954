"""The library's loader reads files exactly as the reference loader
(UVTSampleBuffer(const char*), SampleBuffer.cpp:230-387) does, for binary and text
encodings, with and without a separate header."""
import ctypes
import os

import numpy as np
import pytest

import tlfr
from tlfr_testutil import f32p, ref_available, ref_lib

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference build oracle/_ref not present")


def ref_load(path):
    lib = ref_lib()
    h = ctypes.c_void_p()
    bs = ctypes.c_double()
    r = lib.ref_create_from_file(os.fsencode(path), ctypes.c_float(1), ctypes.c_float(1), None, 0, 0,
                                 ctypes.byref(h), ctypes.byref(bs))
    assert r == 0
    W, H, S = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    c0, c1 = ctypes.c_float(), ctypes.c_float()
    lib.ref_buffer_info(h, ctypes.byref(W), ctypes.byref(H), ctypes.byref(S), ctypes.byref(c0), ctypes.byref(c1))
    rec = np.zeros((H.value, W.value, S.value, 16), np.float32)
    lib.ref_buffer_records(h, f32p(rec))
    lib.ref_destroy(h)
    return rec, (c0.value, c1.value)


@pytest.mark.parametrize("binary,separate", [(True, True), (False, True), (False, False)])
def test_loader_matches_reference(tmp_path, binary, separate):
    rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, 10, 8, 2, 3)
    path = str(tmp_path / "s.bin")
    tlfr.UVTSampleBuffer(records=rec, coc=coc).serialize(path, separate_header=separate, binary=binary)
    mine = tlfr.UVTSampleBuffer(path)
    got = mine.records()
    ref, rcoc = ref_load(path)
    assert mine.info()[3] == rcoc
    # z and dw gradients are not part of the reference's in-memory sample for these
    # fields' comparison; compare every field the reference stores
    fields = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15]
    assert np.array_equal(got[..., fields].view(np.uint32), ref[..., fields].view(np.uint32))
