"""Multi-rank logic of bench.py on CPU: the max-over-ranks time reduction with two
gloo ranks, and the reference arm's rule that only rank 0 runs and prints."""
import contextlib
import io
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        # each rank measured a different time; every rank must see the largest
        got = bench.max_over_ranks(10.0 * (rank + 1) + 0.25, dist, device="cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 20.25, 1: 20.25}


def test_max_over_ranks_without_group():
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5


def test_reference_arm_runs_on_rank0_only():
    import bench

    class A:
        width, height, spp, steps, warmup, cpu_rows = 8, 8, 1, 1, 0, 2
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.run_reference(A(), 1, 2) is None
    assert buf.getvalue() == ""


def test_reference_scene_generator_matches_package():
    """The reference arm generates its inputs with the reference build's copy of
    the scene generator (so it loads no library of the package); both copies
    give the same records bit for bit."""
    import numpy as np
    import pytest
    import tlfr
    import bench
    from tlfr_testutil import ref_available
    if not ref_available():
        pytest.skip("reference build absent")
    a, ca = bench.ref_scene(40, 24, 4, 7)
    b, cb = tlfr.synth_scene(bench.PRESET, 40, 24, 4, 7)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert tuple(np.float32(ca)) == tuple(np.float32(cb))


def test_cpu_rows_spread_over_the_frame():
    import bench
    ys = bench.cpu_rows(1080, 8, 0)
    assert len(ys) == 8 and ys == sorted(ys) and ys[0] < 135 and ys[-1] >= 945
    assert bench.cpu_rows(1080, 8, 1) != ys
