"""Generate the golden fixtures in tests/golden/ from the reference's own CPU code.

The reference ships no tests, fixtures or known-answer vectors for the
reconstruction path.  These fixtures are outputs of the reference itself, built
on Linux by oracle/build_ref.sh (oracle/_ref/libtlfr_ref*.so), on small seeded
synthetic scenes (libtlfr.so's tlfr_synth_scene).  Each .npz holds the input
records and parameters, the reconstructed image, a digest of the hierarchy, the
output sampling pattern and traces of a set of output samples.

Run from the repository root after `bash oracle/build_ref.sh` and building
libtlfr.so:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "temporal-lightfield-reconstruction_b200"))

import tlfr  # noqa: E402
from tlfr_testutil import CpuRecon, ref_available, sample_queries, tree_digest  # noqa: E402

CASES = [
    # name, preset, W, H, spp, seed, dict(params)
    ("planes_24x20x4", tlfr.SCENE_PLANES, 24, 20, 4, 3, {}),
    ("planes_m64_20x16x16", tlfr.SCENE_PLANES, 20, 16, 16, 4, {"output_spp": 64}),
    ("cards_32x24x4", tlfr.SCENE_CARDS, 32, 24, 4, 5, {}),
    ("cards_pinhole_32x24x4", tlfr.SCENE_CARDS, 32, 24, 4, 6, {"uvt": (0.0, 0.0, 1.0)}),
    ("cards_refocus_28x20x2", tlfr.SCENE_CARDS, 28, 20, 2, 7, {"aperture": 1.5, "focus": 0.8}),
    ("large_36x24x8", tlfr.SCENE_CARDS_LARGE, 36, 24, 8, 8, {}),
    ("large_gauss_24x16x8", tlfr.SCENE_CARDS_LARGE, 24, 16, 8, 9, {"lens": 1, "time": 1}),
    ("cards_1spp_40x30x1", tlfr.SCENE_CARDS, 40, 30, 1, 10, {}),
]
NQ = 48
TRACE_CAP = 4096


def make(name, preset, W, H, spp, seed, p):
    rec, coc = tlfr.synth_scene(preset, W, H, spp, seed)
    m64 = p.get("output_spp", 0) == 64
    r = CpuRecon("ref", rec, coc, aperture=p.get("aperture", 1.0), focus=p.get("focus", 1.0), uvt=p.get("uvt"),
                 lens=p.get("lens", 0), time=p.get("time", 0), m64=m64)
    img = r.reconstruct()
    digest, nreach = tree_digest(r.tree())
    pattern = r.output_samples()
    q = sample_queries(W, H, r.out_spp, NQ, seed)
    rgba = np.zeros((NQ, 4), np.float32)
    traces = np.full((NQ, TRACE_CAP), -2, np.int32)
    for k, (x, y, i) in enumerate(q):
        c, t = r.query(int(x), int(y), int(i), TRACE_CAP)
        rgba[k] = c
        traces[k, :len(t)] = t
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), records=rec, coc=np.array(coc, np.float32),
        aperture=np.float32(p.get("aperture", 1.0)), focus=np.float32(p.get("focus", 1.0)),
        uvt=np.array(p.get("uvt", (np.nan, np.nan, np.nan)), np.float32), lens=np.int32(p.get("lens", 0)),
        time=np.int32(p.get("time", 0)), output_spp=np.int32(r.out_spp), image=img, tree_digest=np.bytes_(digest),
        tree_nodes=np.int32(nreach), pattern=pattern, queries=q, query_rgba=rgba, query_traces=traces)
    print(f"{name}: {nreach} reachable nodes, {r.num_samples} samples")


if __name__ == "__main__":
    if not ref_available() or not ref_available(m64=True):
        sys.exit("reference build missing: run `bash oracle/build_ref.sh` first")
    for c in CASES:
        make(*c)
