"""The CPU restatement (oracle/tlfr_oracle.c) reproduces the reference's own
outputs stored in tests/golden/ (generated by tests/golden/make_golden.py from the
reference build): hierarchy digest, output sampling pattern, per-query surfaces
and colours, and every pixel, all bit for bit."""
import glob
import os

import numpy as np
import pytest

from tlfr_testutil import GOLDEN, CpuRecon, tree_digest

CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def _params(g):
    uvt = g["uvt"]
    return dict(aperture=float(g["aperture"]), focus=float(g["focus"]),
                uvt=None if np.isnan(uvt).any() else tuple(float(v) for v in uvt),
                lens=int(g["lens"]), time=int(g["time"]), output_spp=int(g["output_spp"]))


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_oracle_matches_reference_golden(path):
    g = np.load(path)
    rec, coc = g["records"], tuple(g["coc"])
    o = CpuRecon("orc", rec, coc, **_params(g))
    digest, nreach = tree_digest(o.tree())
    assert nreach == int(g["tree_nodes"])
    assert digest == g["tree_digest"].item().decode()
    assert o.output_samples().view(np.uint32).tobytes() == g["pattern"].view(np.uint32).tobytes()
    for k, (x, y, i) in enumerate(g["queries"]):
        rgba, tr = o.query(int(x), int(y), int(i), g["query_traces"].shape[1])
        ref_tr = g["query_traces"][k]
        ref_tr = ref_tr[:np.argmax(ref_tr == -2)] if (ref_tr == -2).any() else ref_tr
        assert np.array_equal(tr, ref_tr), f"query {k} ({x},{y},{i}) surfaces differ"
        assert np.array_equal(rgba.view(np.uint32), g["query_rgba"][k].view(np.uint32)), f"query {k} colour"
    img = o.reconstruct()
    assert np.array_equal(img.view(np.uint32), g["image"].view(np.uint32))
