"""Benchmark: temporal light field reconstruction of one 1920x1080, 8 spp frame.

Workload: 1920x1080 pixels, 8 input samples per pixel (16.6 M samples of 64 B),
strong defocus (C0=-30, C1=40) and motion up to 60 px, 256 textured rectangles
+ 64 disks at depths log-uniform in [0.5, 100] (the seeded analytic scene
TLFR_SCENE_CARDS_LARGE), 128 output samples per pixel (265 M output samples).

A step is one full reconstruction of the frame from sample records resident in
HBM: hierarchy build + per-output-sample query + pixel resolve.
  value  Mpix/s over all ranks (W*H per rank per step / max-over-ranks step time)
  e2e    the same through the public C ABI with host buffers: page-locked host
         records -> device (tlfr_rebuild), build, reconstruct, RGBA image -> host
  roofline   the query kernel's algorithmic bytes (64 B per leaf node tested,
         32 B per sample tested, 16 B per sample accepted, summed over fetch
         passes; + 16 B per output pixel) per launch / its CUDA-event duration,
         against the measured HBM copy bandwidth.
  cpu_baseline   the reference's own CPU reconstruction (oracle/_ref, or the C
         restatement when the reference build is absent) on this host's cores:
         full hierarchy build + a band of rows, extrapolated to the frame.
  routed the same frame and timing with the learned router on (trained first,
         untimed, on plain-method labels of frames with seeds 100+), with its
         PSNR and max error against the plain image.
  batch  uneven sample buffers (resolution and spp drawn per buffer) built as
         contexts and reconstructed as one CUDA graph per run, router on;
         Mpix/s over all buffers.  --batch-scale 1 is the full-size mix.

Multi-GPU: one process per GPU, each reconstructs its own frame (replicas; the
path has no exchange step), timed with CUDA events, max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "temporal-lightfield-reconstruction_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "recon Mpix/s on 1 B200: learned-routed vs plain GPU at <=0.1 dB loss; HBM GB/s"
W, H, SPP, M = 1920, 1080, 8, 128
PRESET = 2
WORKLOAD = "1920x1080 8spp defocus+motion, 256 rects + 64 disks, 128 output samples/px"
DATA = "synthetic (seeded analytic scene)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-rows", type=int, default=32, help="rows per CPU sample (spread over the frame)")
    ap.add_argument("--width", type=int, default=W)
    ap.add_argument("--height", type=int, default=H)
    ap.add_argument("--spp", type=int, default=SPP)
    ap.add_argument("--route-frames", type=int, default=32, help="router training frames, seeds 100.. (0: no routed run)")
    ap.add_argument("--route-eval", type=int, default=8, help="held-out evaluation frames, seeds 200..")
    ap.add_argument("--route-steps", type=int, default=600)
    ap.add_argument("--route-threshold", type=float, default=0.8)
    ap.add_argument("--route-labels", default="gt", choices=["gt", "plain"],
                    help="router labels against the scene's ground truth or the plain image")
    ap.add_argument("--route-tol", type=float, default=0.0,
                    help="label tolerance: squared RGB error above the plain pixel's (gt) or channel difference")
    ap.add_argument("--gt-samples", type=int, default=1024, help="ground-truth samples per pixel")
    ap.add_argument("--batch-frames", type=int, default=48, help="uneven-buffer batch size (0: no batch run)")
    ap.add_argument("--batch-scale", type=int, default=1, help="linear downscale of the batch's resolutions")
    ap.add_argument("--profile-frame", action="store_true",
                    help="time the query passes of one frame (--width/--height/--spp, --steps/--warmup) and print "
                         "one JSON line; the entry point for profiler captures")
    ap.add_argument("--scene", type=int, default=PRESET, help="scene preset of --profile-frame")
    ap.add_argument("--enable-cuda", action="store_true",
                    help="--profile-frame with the reference's GPU-toggle algorithm (CameraParams.enableCuda)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def ncu_traffic():
    """DRAM bytes per query-kernel launch from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "query_kernel_traffic.json")) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch")
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_rows(height, rows, step):
    """`rows` rows spread evenly over the frame, the comb shifted per step (golden
    ratio), so that successive samples cover different rows."""
    stride = height / rows
    off = (0.5 + 0.6180339887 * step) % 1.0
    return sorted({min(height - 1, int((j + off) * stride)) for j in range(rows)})


def ref_scene(width, height, spp, seed):
    """The seeded scene from the reference build's own copy of the generator
    (oracle/_ref), so that the reference's CPU runs load no library of this
    package; the package's generator when the reference build is absent."""
    import ctypes
    import numpy as np
    from tlfr_testutil import ref_available, ref_lib
    if not ref_available():
        import tlfr
        return tlfr.synth_scene(PRESET, width, height, spp, seed)
    lib = ref_lib()
    rec = np.empty((height, width, spp, 16), np.float32)
    coc = np.zeros(2, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    st = lib.ref_synth_scene(PRESET, width, height, spp, ctypes.c_ulonglong(seed), rec.ctypes.data_as(fp),
                             coc.ctypes.data_as(fp))
    if st != 0:
        raise RuntimeError(f"ref_synth_scene failed ({st})")
    return rec, (float(coc[0]), float(coc[1]))


class CpuSampler:
    """The reference's own CPU reconstruction (oracle/_ref; the C restatement
    when the reference build is absent) of one frame on this host's cores: the
    full hierarchy build once, then per sample a comb of rows spread over the
    frame, reconstructed in one call (the reference runs one task per scanline,
    so the rows run in parallel on its threads).  The frame time is estimated as build + (query time of the rows) x
    height / rows.  Both the reference arm and the GPU arm's cpu_baseline use it."""

    def __init__(self, rec, coc, threads):
        from tlfr_testutil import CpuRecon, ref_available
        self.kind = "reference" if ref_available() else "port"
        os.environ["TLFR_REF_THREADS"] = str(threads)
        self.threads = threads
        self.r = CpuRecon("ref" if self.kind == "reference" else "orc", rec, coc, nthreads=threads)
        self.H, self.W = rec.shape[0], rec.shape[1]
        self.build_s = self.r.build_seconds

    def sample(self, rows, step):
        ys = cpu_rows(self.H, rows, step)
        img = self.r.reconstruct_rowlist(ys)
        t = self.r.last_seconds
        imgs = {y: img[k] for k, y in enumerate(ys)}
        est = self.build_s + t * self.H / len(ys)
        return est, t, ys, imgs

    def close(self):
        self.r.close()


def cpu_baseline_sample(rec, coc, rows, threads, gpu_img=None):
    """cpu_baseline of the GPU arm, plus a parity check of the timed GPU frame:
    the sampled rows of the reference's CPU image against the same rows of the
    GPU image (outside every timed region)."""
    import numpy as np
    cs = CpuSampler(rec, coc, threads)
    est, t, ys, imgs = cs.sample(rows, 0)
    cs.close()
    out = {
        "value": (cs.W * cs.H / est) / 1e6, "unit": "Mpix/s", "cores": threads, "kind": cs.kind,
        "sample": f"full {cs.W}x{cs.H} hierarchy build ({cs.build_s:.2f} s) + {len(ys)} rows spread over the frame "
                  f"({t:.2f} s), extrapolated to {cs.H} rows",
        "build_s": cs.build_s, "rows_s": t, "rows": ys,
    }
    if gpu_img is not None:
        cpu = np.stack([imgs[y] for y in ys])
        gpu = np.stack([gpu_img[y] for y in ys])
        rel = np.abs(gpu - cpu) / np.maximum(np.abs(cpu), 1e-6)
        out["parity"] = {"rows": ys, "pixels": int(cpu.shape[0] * cpu.shape[1]),
                         "bit_exact": bool(np.array_equal(gpu.view(np.uint32), cpu.view(np.uint32))),
                         "max_rel_err": float(rel.max()), "tolerance": 1e-4, "ok": bool(rel.max() <= 1e-4)}
    return out


def psnr(img, ref):
    """PSNR in dB of the RGB channels of img against ref (peak 1)."""
    import numpy as np
    mse = float(np.mean((img[..., :3].astype(np.float64) - ref[..., :3].astype(np.float64)) ** 2))
    return 10 * float(np.log10(1.0 / mse)) if mse > 0 else float("inf")


def train_router(args, device, W, H, S):
    """The learned router trained on plain-method labels of args.route_frames
    frames of the strong-blur scene (seeds 100, 101, ...), untimed."""
    import numpy as np
    import torch
    import tlfr
    feats, labels = [], []
    t0 = time.perf_counter()
    for seed in range(100, 100 + args.route_frames):
        rec, coc = tlfr.synth_scene(PRESET, W, H, S, seed)
        d = torch.from_numpy(rec).cuda()
        g = tlfr.TreeGather(None, tlfr.CameraParams(device=device), device_records=(d.data_ptr(), (W, H, S), coc))
        f = torch.empty((H * W, 8), dtype=torch.float32, device="cuda")
        lab = torch.empty(H * W, dtype=torch.float32, device="cuda")
        img = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
        g.route_features(f.data_ptr())
        if args.route_labels == "gt":
            gt = torch.from_numpy(tlfr.synth_reference_image(PRESET, W, H, args.gt_samples, seed)).cuda()
            g.route_labels(lab.data_ptr(), img.data_ptr(), args.route_tol, d_ref=gt.data_ptr())
            del gt
        else:
            g.route_labels(lab.data_ptr(), img.data_ptr(), args.route_tol)
        feats.append(f)
        labels.append(lab)
        g.close()
        del d
    label_s = time.perf_counter() - t0
    F = torch.cat(feats)
    L = torch.cat(labels)
    del feats, labels
    fh = F[::97].cpu().numpy()
    router = tlfr.Router(device, seed=3, mean=fh.mean(0), inv_std=1.0 / np.maximum(fh.std(0), 1e-6))
    n = F.shape[0]
    loss0 = router.gradient(F.data_ptr(), L.data_ptr(), min(n, 1 << 20))[1]
    t0 = time.perf_counter()
    loss = router.train(F.data_ptr(), L.data_ptr(), n, steps=args.route_steps, batch=8192, lr=3e-3)
    info = {"frames": args.route_frames, "seeds": [100, 100 + args.route_frames - 1], "pixels": n,
            "label_mean": float(L.mean().item()), "label_tolerance": args.route_tol, "label_reference":
            "ground truth (fast pixel's squared RGB error at most tol above the plain pixel's)"
            if args.route_labels == "gt" else "plain method (max channel difference at most tol)",
            "steps": args.route_steps,
            "loss_initial": loss0, "loss_final": loss, "train_s": time.perf_counter() - t0, "labels_s": label_s}
    del F, L
    torch.cuda.empty_cache()
    return router, info


def routing_eval(args, device, router, W, H, S, thresholds=None):
    """The router on held-out frames (seeds 200, 201, ...): per seed the plain
    method, the routed form and every pixel on the fast path (no network), each
    timed over full steps (hierarchy build + reconstruction, CUDA events), and
    each image's PSNR against the scene's ground truth (tlfr.synth_reference_image)."""
    import numpy as np
    import torch
    import tlfr
    stream = torch.cuda.current_stream()
    rows = []
    thresholds = sorted(set(thresholds or [args.route_threshold, 0.5]))
    for seed in range(200, 200 + args.route_eval):
        rec, coc = tlfr.synth_scene(PRESET, W, H, S, seed)
        d = torch.from_numpy(rec).cuda()
        g = tlfr.TreeGather(None, tlfr.CameraParams(device=device), stream=stream.cuda_stream,
                            device_records=(d.data_ptr(), (W, H, S), coc))
        out = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")

        def timed(router_, thr, k=2):
            g.set_routing(router_, thr)
            g.rebuild(d.data_ptr())
            g.reconstruct_to_device(out.data_ptr())
            ms = []
            for _ in range(k):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                g.rebuild(d.data_ptr())
                g.reconstruct_to_device(out.data_ptr())
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            return statistics.median(ms), out.cpu().numpy()

        ms_plain, plain = timed(None, 0.8)
        ms_all, allfast = timed(router, 0.0)
        feats = torch.empty((H * W, 8), dtype=torch.float32, device="cuda")
        prob = torch.empty(H * W, dtype=torch.float32, device="cuda")
        g.route_features(feats.data_ptr())
        router.predict(feats.data_ptr(), W * H, prob.data_ptr())
        gt = tlfr.synth_reference_image(PRESET, W, H, args.gt_samples, seed)
        p_plain, p_all = psnr(plain, gt), psnr(allfast, gt)
        row = {"seed": seed, "plain_ms": ms_plain, "all_fast_ms": ms_all, "psnr_plain_db": p_plain,
               "psnr_all_fast_db": p_all, "psnr_loss_all_fast_db": p_plain - p_all, "thresholds": {}}
        for thr in thresholds:
            ms_r, routed = timed(router, thr)
            p_r = psnr(routed, gt)
            row["thresholds"][str(thr)] = {
                "routed_ms": ms_r, "speedup": ms_plain / ms_r,
                "fast_pixel_fraction": float((prob > thr).float().mean().item()),
                "psnr_routed_db": p_r, "psnr_loss_db": p_plain - p_r,
                "max_abs_err_vs_plain": float(np.abs(routed[..., :3] - plain[..., :3]).max()),
                "psnr_routed_vs_plain_db": psnr(routed, plain)}
        g.set_routing(None)
        g.close()
        del d
        rows.append(row)
    med = lambda f: statistics.median(f(r) for r in rows)
    summary = {}
    for thr in thresholds:
        k = str(thr)
        summary[k] = {
            "speedup_median": med(lambda r: r["thresholds"][k]["speedup"]),
            "psnr_loss_db_max": max(r["thresholds"][k]["psnr_loss_db"] for r in rows),
            "psnr_loss_db_median": med(lambda r: r["thresholds"][k]["psnr_loss_db"]),
            "fast_pixel_fraction_median": med(lambda r: r["thresholds"][k]["fast_pixel_fraction"]),
            "value": (W * H / (med(lambda r: r["thresholds"][k]["routed_ms"]) / 1e3)) / 1e6, "unit": "Mpix/s"}
    main = summary[str(args.route_threshold)]
    return {
        "seeds": [r["seed"] for r in rows], "per_seed": rows, "threshold": args.route_threshold,
        "value": main["value"], "unit": "Mpix/s", "speedup_median": main["speedup_median"],
        "psnr_loss_db_max": main["psnr_loss_db_max"], "psnr_loss_db_median": main["psnr_loss_db_median"],
        "fast_pixel_fraction_median": main["fast_pixel_fraction_median"], "by_threshold": summary,
        "no_network": {"plain_value": (W * H / (med(lambda r: r["plain_ms"]) / 1e3)) / 1e6,
                       "all_fast_speedup_median": med(lambda r: r["plain_ms"] / r["all_fast_ms"]),
                       "all_fast_psnr_loss_db_median": med(lambda r: r["psnr_loss_all_fast_db"])},
        "psnr_plain_db_median": med(lambda r: r["psnr_plain_db"]), "gt_samples_per_pixel": args.gt_samples,
        "timing": "median of 2 full steps (hierarchy build + reconstruction) per seed after one warm-up, CUDA events",
    }


def max_over_ranks(value, dist, device="cuda"):
    """The largest value over all ranks (a time measured on every rank); the value itself
    without a process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


BATCH_RES = [(320, 240), (640, 480), (962, 543), (1280, 720), (1920, 1080)]
BATCH_SPP = [1, 2, 4, 8, 16]


def run_batch(args, device, router, steps, warmup):
    """Uneven buffers (resolution and spp drawn per frame, the 64-rectangle scene
    generator per seed) reconstructed as one CUDA graph, router on."""
    import numpy as np
    import torch
    import tlfr
    rng = np.random.default_rng(4)
    trees, outs, recs, pix = [], [], [], 0
    shapes = []
    for k in range(args.batch_frames):
        Wr, Hr = BATCH_RES[rng.integers(len(BATCH_RES))]
        Wb, Hb = max(8, Wr // args.batch_scale), max(8, Hr // args.batch_scale)
        Sb = int(BATCH_SPP[rng.integers(len(BATCH_SPP))])
        rec, coc = tlfr.synth_scene(tlfr.SCENE_CARDS, Wb, Hb, Sb, 1000 + k)
        d = torch.from_numpy(rec).cuda()
        g = tlfr.TreeGather(None, tlfr.CameraParams(device=device), device_records=(d.data_ptr(), (Wb, Hb, Sb), coc))
        g.trim()
        if router is not None:
            g.set_routing(router, args.route_threshold)
        recs.append(d)
        trees.append(g)
        outs.append(torch.empty((Hb, Wb, 4), dtype=torch.float32, device="cuda"))
        shapes.append((Wb, Hb, Sb))
        pix += Wb * Hb
    t0 = time.perf_counter()
    batch = tlfr.Batch(trees, [o.data_ptr() for o in outs], autotune=True)
    create_s = time.perf_counter() - t0
    for _ in range(warmup):
        batch.run()
        batch.sync()
    ms = []
    for _ in range(steps):
        batch.run()
        ms.append(batch.sync())
    shapes = batch.tile_shapes()
    chunks, launches = batch.layout()
    batch.close()
    for g in trees:
        g.close()
    t = statistics.median(ms)
    return {
        "config": f"{args.batch_frames} buffers, resolutions drawn from {BATCH_RES} divided by {args.batch_scale}, "
                  f"spp drawn from {BATCH_SPP}, 64-rectangle scene per seed, 128 output samples/px, "
                  f"router {'on' if router is not None else 'off'}",
        "frames": args.batch_frames, "pixels": pix, "output_samples": pix * 128,
        "value": pix / (t / 1e3) / 1e6, "unit": "Mpix/s", "ms_per_run": t, "runs": steps,
        "create_s": create_s,
        "tile_shapes": {tlfr.TILE_SHAPES[k]: int((shapes == k).sum()) for k in sorted(set(int(x) for x in shapes))},
        "chunks": int(chunks.max()) + 1, "launches_per_run": int(launches),
        "launch": "one CUDA graph per run; per chunk one persistent launch per pass over all its frames",
    }


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation on the host cores."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    rec, coc = ref_scene(args.width, args.height, args.spp, 2)
    cs = CpuSampler(rec, coc, threads)
    rows = max(1, args.cpu_rows)
    ests, ts = [], []
    for k in range(args.warmup + args.steps):
        est, t, ys, _ = cs.sample(rows, k)
        if k >= args.warmup:
            ests.append(est)
            ts.append(t)
    cs.close()
    est = statistics.median(ests)
    value = (args.width * args.height / est) / 1e6
    sample = (f"full {args.width}x{args.height} hierarchy build ({cs.build_s:.2f} s, once) + per step {rows} rows "
              f"spread over the frame (comb shifted per step); frame time = build + rows' time x "
              f"{args.height}/{rows}; ms_per_step = the rows' measured time")
    line = {
        "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(ts) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA, "impl": "reference",
        "config": bench_config(args), "frame_s_estimate": est,
        "cpu_baseline": {"value": value, "unit": "Mpix/s", "cores": threads, "kind": cs.kind, "sample": sample},
        "e2e": {"value": value, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_config(args):
    """The workload both arms report (identical dicts)."""
    return {"workload": WORKLOAD, "width": args.width, "height": args.height, "spp": args.spp, "output_spp": M}


def run_profile_frame(args):
    """One frame reconstructed from device-resident records: hierarchy build and
    query passes timed with CUDA events per step (no CPU baseline, no router,
    no batch).  Used for profiler captures of single kernels."""
    import torch
    import tlfr
    torch.cuda.set_device(0)
    Wd, Hd, S = args.width, args.height, args.spp
    rec, coc = tlfr.synth_scene(args.scene, Wd, Hd, S, 2)
    d_rec = torch.from_numpy(rec).cuda()
    stream = torch.cuda.current_stream()
    tg = tlfr.TreeGather(None, tlfr.CameraParams(device=0, enableCuda=args.enable_cuda), stream=stream.cuda_stream,
                         device_records=(d_rec.data_ptr(), (Wd, Hd, S), coc))
    out = torch.empty((Hd, Wd, 4), dtype=torch.float32, device="cuda")
    rows = []
    for k in range(args.warmup + args.steps):
        tg.rebuild(d_rec.data_ptr())
        b = tg.stats().build_ms
        tg.reconstruct_to_device(out.data_ptr())
        st = tg.stats()
        if k >= args.warmup:
            rows.append((b, st.light_ms, st.heavy_ms, st.query_kernel_ms, st.num_heavy_queries))
    torch.cuda.synchronize()
    med = lambda i: statistics.median(r[i] for r in rows)
    line = {"profile_frame": f"{Wd}x{Hd}x{S}", "scene": args.scene, "steps": args.steps, "warmup": args.warmup,
            "algorithm": "gpu toggle (enableCuda)" if args.enable_cuda else "filterer",
            "build_ms": med(0), "light_ms": med(1), "heavy_ms": med(2), "query_kernel_ms": med(3),
            "heavy_queries": int(rows[-1][4]), "output_samples": Wd * Hd * M,
            "checksum": float(out.double().sum().item())}
    tg.close()
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.profile_frame:
        run_profile_frame(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    import tlfr

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist:
            dist.barrier()

    Wd, Hd, S = args.width, args.height, args.spp
    rec, coc = tlfr.synth_scene(PRESET, Wd, Hd, S, 2 + rank)
    stream = torch.cuda.current_stream()
    d_rec = torch.from_numpy(rec).cuda()
    params = tlfr.CameraParams(device=local_rank)
    tg = tlfr.TreeGather(None, params, stream=stream.cuda_stream,
                         device_records=(d_rec.data_ptr(), (Wd, Hd, S), coc))
    out = torch.empty((Hd, Wd, 4), dtype=torch.float32, device="cuda")

    def step():
        tg.rebuild(d_rec.data_ptr())
        tg.reconstruct_to_device(out.data_ptr())

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    # counters for the algorithmic-byte roofline (untimed run)
    st = tg.reconstruct_to_device(out.data_ptr(), stats=True)
    alg_bytes = 64.0 * st.num_leaf_nodes + 32.0 * st.num_samples_in_leaf_nodes + 16.0 * st.num_samples_fetched \
        + 16.0 * Wd * Hd

    # timed region: inputs (1 GB records, ~1 GB hierarchy) exceed the 126 MB L2
    clocks = ClockSampler(local_rank)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    q_ms, b_ms, l_ms, h_ms, launches = [], [], [], [], 0
    e0.record(stream)
    for _ in range(args.steps):
        tg.rebuild(d_rec.data_ptr())
        sb = tg.stats()
        s2 = tg.reconstruct_to_device(out.data_ptr(), stats=False)
        sq = tg.stats()
        b_ms.append(sb.build_ms)
        q_ms.append(sq.query_kernel_ms)
        l_ms.append(sq.light_ms)
        h_ms.append(sq.heavy_ms)
        launches += int(sb.build_launches + sq.query_launches)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = e0.elapsed_time(e1)
    total_ms = max_over_ranks(total_ms, dist)
    ms_per_step = total_ms / args.steps
    value = (world * Wd * Hd * args.steps / (total_ms / 1e3)) / 1e6
    plain_host = out.cpu().numpy()          # the timed frame, for the parity check of cpu_baseline

    # learned routing: trained on route_frames plain-method frames (seeds 100+),
    # evaluated on route_eval held-out frames (seeds 200+) against ground truth
    routed = None
    router = None
    if args.route_frames > 0:
        router, rinfo = train_router(args, local_rank, Wd, Hd, S)
        routed = routing_eval(args, local_rank, router, Wd, Hd, S)
        routed["train"] = rinfo

    # uneven-buffer batch (one CUDA graph), learned routing on
    batch = None
    if args.batch_frames > 0:
        batch = run_batch(args, local_rank, router if args.route_frames > 0 else None, max(1, min(args.steps, 5)),
                          max(1, min(args.warmup, 3)))
    if args.route_frames > 0:
        router.close()

    # end to end through the public API with host buffers (pinned records in,
    # RGBA image out); every rank runs it, timed by its own clock, max over ranks
    buf = tlfr.UVTSampleBuffer(records=rec, coc=coc)
    img = np.empty((Hd, Wd, 4), np.float32)
    tg.rebuild_from(buf)
    tg.reconstructDofMotion(img)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        tg.rebuild_from(buf)
        tg.reconstructDofMotion(img)
    e2e_s = (time.perf_counter() - t0) / max(1, args.e2e_steps)
    e2e_s = max_over_ranks(e2e_s, dist)
    e2e = {"value": (world * Wd * Hd / e2e_s) / 1e6, "unit": "Mpix/s", "ms_per_step": e2e_s * 1e3,
           "h2d_bytes_per_step": int(rec.nbytes), "d2h_bytes_per_step": int(img.nbytes)}

    peaks, peak_kind = measured_peaks()
    q_mean = statistics.mean(q_ms)
    achieved = alg_bytes / (q_mean / 1e3) / 1e9
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
        "frac": achieved / peaks["hbm_gbs"], "traffic": ncu_traffic(), "kernel": "k_query",
        "peak_source": f"{peak_kind} HBM copy bandwidth", "algorithmic_bytes_per_launch": alg_bytes,
        "query_kernel_ms": q_mean,
    }

    line = {
        "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": DATA + ", records resident in HBM",
        "config": bench_config(args),
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "l2": "inputs larger than L2 (1.06 GB records, ~1 GB hierarchy)",
        "build_ms": statistics.mean(b_ms), "query_kernel_ms": q_mean,
        "light_pass_ms": statistics.mean(l_ms), "heavy_pass_ms": statistics.mean(h_ms),
        "heavy_queries": sq.num_heavy_queries,
        "recon_samples_per_s": world * Wd * Hd * M * args.steps / (total_ms / 1e3),
        "query_stats": {"leaf_nodes_per_query": st.num_leaf_nodes / st.num_output_samples,
                        "samples_tested_per_query": st.num_samples_in_leaf_nodes / st.num_output_samples,
                        "samples_fetched_per_query": st.num_samples_fetched / st.num_output_samples,
                        "frac_2r": st.num_2r / st.num_output_samples,
                        "overflow_queries": st.num_overflow_queries},
        "e2e": e2e, "roofline": roofline, "gpu_launches": launches, "clocks": clk,
        "routed": routed, "batch": batch,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(rec, coc, args.cpu_rows, os.cpu_count() or 1,
                                                   gpu_img=plain_host)
    tg.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
