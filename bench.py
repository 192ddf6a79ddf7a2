"""Benchmark: the plain forward of the splat tile rasteriser at 1M splats, 1920x1080.

Workload (the configuration the headline metric is quoted on): 1,000,000 seeded
synthetic Gaussians (means N(0,1), log-scales N(-4.5,0.5), uniform rotations,
opacity sigmoid(N(0,1)), SH degree 3 with DC N(0,0.5) and rest N(0,0.05)),
1920x1080, 16x16 tiles, 0.3 px Mip-Splatting 2D filter, 60 degree vertical field
of view, camera orbiting the origin at radius 4 over 20 frames. A step is one
frame (one view) of the orbit through the rasteriser's public call.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's algorithm on the host cores: the
reference's own kernels are Slang, which cannot run here, so its CPU arm is
the oracle (oracle/, a C++ restatement of those kernels), multithreaded.
Under torchrun each rank renders its own views of the orbit (replicas: the
frames are independent, there is no data exchange); value is whole-job ms per
view = max-over-ranks time / (steps x ranks).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ms/view @1M splats 1080p: plain fwd vs batched fwd+bwd; sort GB/s vs HBM"
UNIT = "ms/view"
SPLATS = 1_000_000
WIDTH, HEIGHT = 1920, 1080
FRAMES = 20
RADIUS = 4.0
SEED = 1
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + written) of one launch, from ncu (`dram__bytes_read.sum +
# dram__bytes_write.sum`) on one frame of this orbit; the capture and its command
# are summarised under profiles/ (blend_1M_1080p.md).
PROFILED_DRAM_BYTES = {"blend": 53.549312e6 + 7.519232e6}
# The blend is bound by instruction issue, not by HBM: its issue-active
# fraction (`smsp__issue_active.avg.pct_of_peak_sustained_active`) from the
# same capture, the secondary roofline its HBM fraction is read beside.
PROFILED_ISSUE_ACTIVE = {"blend": 0.9007}


def orbit_camera(L, k: int):
    th = 2.0 * math.pi * (k % FRAMES) / FRAMES
    eye = (RADIUS * math.sin(th), 0.0, RADIUS * math.cos(th))
    return L.square_pixel_camera(eye, (0.0, 0.0, 0.0), WIDTH, HEIGHT, 60.0, 0.01)


def workload_config(world: int) -> dict:
    """The workload, the same in both arms."""
    return {"workload": "plain forward, 1M splats, 1920x1080, 20-frame orbit at radius 4",
            "splats": SPLATS, "width": WIDTH, "height": HEIGHT, "frames": FRAMES, "tile": 16, "sh_degree": 3,
            "seed": SEED, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "flushed before every device-timed step (256 MB write); the end-to-end steps run back to back "
                  "with a 283 MB working set per frame, larger than L2"}


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock samples (every 20 ms) for the whole run; `summary`
    keeps the samples taken inside the timed windows (widened by 0.25 s, since
    one timed region can be shorter than the sampling period)."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.windows = []
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def window(self, t0: float, t1: float) -> None:
        self.windows.append((t0, t1))

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        inside = [r for r in rows if any(a - 0.25 <= r[0] <= b + 0.25 for a, b in self.windows)]
        sm = [r[1] for r in inside]
        reasons = sorted({n for r in inside for n, v in zip(names, r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max((r[2] for r in rows), default=None), "reasons": reasons,
                "samples": len(sm), "samples_whole_run": len(rows)}


def cpu_reference_frames(frame_ids, threads: int) -> tuple[float, list]:
    """The oracle (CPU restatement of the reference's kernels) rendering full
    frames of the orbit. The scene and the cameras are built by the oracle
    too (oracle/bench_workload.py): this leg imports nothing from the package."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import bench_workload as W
    cloud = W.packed_cloud(SPLATS, SEED)
    times = W.time_frames(cloud, frame_ids, FRAMES, RADIUS, WIDTH, HEIGHT, threads)
    return float(np.mean(times)), times


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    cpu_reference_frames(range(args.warmup), threads)
    mean_ms, _ = cpu_reference_frames(range(args.steps), threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(mean_ms, 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean_ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.gpus),
        "reference_arm": "the oracle: a C++ restatement of the reference's Slang raster kernels (the Slang itself "
                         "cannot run here), on the host cores; scene and cameras built by the oracle",
        "cpu_baseline": {"value": round(mean_ms, 3), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"frames 0-{args.steps - 1} of the orbit, {threads} threads"},
        "e2e": {"value": round(mean_ms, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


BATCH_SPLATS = 2_000_000
BATCH_VIEWS = 64
BATCH_SIZES = [(256, 256), (640, 480), (1280, 720), (1920, 1080)]


def batch_views(L, seed: int):
    """64 cameras looking at the origin from directions uniform on the sphere,
    at radius U(3, 6), each with a resolution drawn uniformly from four."""
    rng = np.random.Generator(np.random.Philox(seed))
    views = []
    for _ in range(BATCH_VIEWS):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        r = rng.uniform(3.0, 6.0)
        w, h = BATCH_SIZES[int(rng.integers(len(BATCH_SIZES)))]
        up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.99 else (1.0, 0.0, 0.0)
        views.append((L.square_pixel_camera(tuple(d * r), (0.0, 0.0, 0.0), w, h, 60.0, 0.01, up), w, h))
    return views


def run_batch(L, torch, dev, rank, raster, args, clocks) -> dict:
    """2M splats, 64 views of mixed resolution: one lrt_rast_render_batch call
    per step against 64 sequential lrt_rast_render calls, ms per view, with
    the batched images checked equal to the sequential ones bit for bit."""
    packed = L.pack_splats(L.synthetic_records(BATCH_SPLATS, SEED + 1), 15, 3)
    cloud = L.to_device(packed, dev)
    instances = [L.SplatInstance(cloud)]
    settings = L.RenderSettings()
    views = batch_views(L, SEED + rank)
    projections = [(L.projection_for(c, w, h), w, h) for c, w, h in views]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    singles = [L.RenderTargets(w, h, device=dev) for _, w, h in views]
    batched = [L.RenderTargets(w, h, device=dev) for _, w, h in views]

    def sequential():
        for (p, w, h), t in zip(projections, singles):
            st = L.RenderSettings(width=w, height=h)
            raster.render(p, instances, st, t, stream)

    def one_batch():
        return raster.render_batch(projections, instances, settings, batched, stream)[1]

    for _ in range(2):
        sequential()
    stats = None
    for _ in range(3):          # tune, capture, replay
        stats = one_batch()
    torch.cuda.synchronize(dev)
    steps = max(3, args.steps // 4)
    seq_ms = bat_ms = 0.0
    w0 = time.time()
    for _ in range(steps):
        flush.fill_(1.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sequential()
        b.record(stream)
        b.synchronize()
        seq_ms += a.elapsed_time(b)
        flush.fill_(2.0)
        a.record(stream)
        stats = one_batch()
        b.record(stream)
        b.synchronize()
        bat_ms += a.elapsed_time(b)
    clocks.window(w0, time.time())
    equal = all(torch.equal(x.colour, y.colour) and torch.equal(x.depth, y.depth) for x, y in zip(singles, batched))
    per_seq = seq_ms / (steps * BATCH_VIEWS)
    per_bat = bat_ms / (steps * BATCH_VIEWS)
    out = {"workload": "2M splats, 64 views on a sphere of radius U(3,6), resolutions uniform over 256x256, "
                       "640x480, 1280x720, 1920x1080", "steps": steps,
           "batched_ms_per_view": round(per_bat, 4), "sequential_ms_per_view": round(per_seq, 4),
           "speedup": round(per_seq / per_bat, 3), "images_equal_bit_for_bit": bool(equal),
           "pairs_per_batch": int(stats.pairs), "views_per_chunk": int(stats.views_per_chunk),
           "blend_blocks_per_sm": int(stats.blend_blocks_per_sm), "graph_replayed": int(stats.graph_replayed)}
    del cloud, instances, singles, batched
    out["fwd_bwd"] = run_batch_train(L, torch, dev, raster, views, projections, flush, stream, steps, per_seq, clocks)
    return out


def run_batch_train(L, torch, dev, raster, views, projections, flush, stream, steps, per_plain, clocks) -> dict:
    """The 64 views' forward+backward: one lrt_rast_train_batch call per step
    (each view's L1 loss against a seeded uniform target, gradients of their
    sum over the same 2M splats' raw parameters) against 64 sequential
    single-view steps (rasterize + l1_loss + backward), in ms per view."""
    raw = L.synthetic_records(BATCH_SPLATS, SEED + 1)
    keep = raw.shape[0]
    sh = np.zeros((keep, 16, 3), np.float32)
    sh[:, 0, :] = raw[:, 11:14]
    for c in range(3):
        sh[:, 1:, c] = raw[:, 14 + 15 * c:14 + 15 * (c + 1)]
    sh = sh.astype(np.float16).astype(np.float32)
    params = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in (
        ("means", raw[:, 0:3]), ("log_scales", raw[:, 4:7]), ("quats", raw[:, 7:11]), ("logits", raw[:, 3]),
        ("sh", sh))}
    sh16 = params["sh"].reshape(keep, 48).half().contiguous()
    gen = torch.Generator(device=dev).manual_seed(SEED)
    tviews = [(p, torch.rand((h, w, 3), generator=gen, device=dev)) for p, w, h in projections]
    ordered = [params[k] for k in ("means", "log_scales", "quats", "logits", "sh")]

    def batch_step():
        return L.train_batch(*ordered, tviews, L.RenderSettings(), raster, sh_storage=sh16, stream=stream)

    leaves = {k: v.clone().requires_grad_(True) for k, v in params.items()}
    lordered = [leaves[k] for k in ("means", "log_scales", "quats", "logits", "sh")]

    def sequential_steps():
        for p, target in tviews:
            for v in lordered:
                v.grad = None
            h, w = target.shape[:2]
            colour, _ = L.rasterize(*lordered, p, L.RenderSettings(width=w, height=h), raster, sh_storage=sh16)
            L.l1_loss(colour, target, raster).backward()

    for _ in range(2):
        stats = batch_step()[4]
        sequential_steps()
    torch.cuda.synchronize(dev)
    bat_ms = seq_ms = 0.0
    w0 = time.time()
    for _ in range(steps):
        flush.fill_(3.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats = batch_step()[4]
        b.record(stream)
        b.synchronize()
        bat_ms += a.elapsed_time(b)
        flush.fill_(4.0)
        a.record(stream)
        sequential_steps()
        b.record(stream)
        b.synchronize()
        seq_ms += a.elapsed_time(b)
    clocks.window(w0, time.time())
    per_bat = bat_ms / (steps * BATCH_VIEWS)
    per_seq = seq_ms / (steps * BATCH_VIEWS)
    return {"workload": "the same 64 views and 2M splats as raw parameters; per view an L1 loss against a seeded "
                        "uniform [0,1]^3 target; gradients of the views' summed loss",
            "batched_ms_per_view": round(per_bat, 4), "sequential_fwd_bwd_ms_per_view": round(per_seq, 4),
            "speedup_vs_sequential_fwd_bwd": round(per_seq / per_bat, 3),
            "ratio_to_sequential_plain_forward": round(per_bat / per_plain, 3),
            "views_per_chunk": int(stats.views_per_chunk), "chunks": int(stats.chunks),
            "pairs_per_batch": int(stats.pairs)}


def time_device(torch, stream, fn, reps: int) -> float:
    """Mean ms of `fn` over `reps` calls, CUDA events on `stream`, after one warm call."""
    fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def run_next_rows(L, torch, dev, raster, packed, cloud, peak) -> dict:
    """The rows around the hot path: device decode of the benchmark cloud's
    raw records, the composite frame (the same splats with a million point
    discs, and over an under layer), and the on-device image metric."""
    stream = torch.cuda.current_stream(dev)
    raw = L.synthetic_records(SPLATS, SEED)
    raw_dev = torch.from_numpy(raw).to(dev)
    enc = L.ply_encoding(15)
    decode_ms = time_device(torch, stream, lambda: raster.decode_splats(raw_dev, enc, 15, stream), 5)
    decode_bytes = raw.nbytes + SPLATS * (16 + 16 + 4 * 23)
    rng = np.random.default_rng(SEED)
    pts_raw = np.concatenate([rng.normal(0.0, 1.0, (SPLATS, 3)), rng.uniform(0.0, 1.0, (SPLATS, 3))], 1)
    points = raster.decode_points(torch.from_numpy(pts_raw.astype(np.float32)).to(dev), 2, 1.0, stream)
    settings = L.RenderSettings(width=WIDTH, height=HEIGHT)
    cam = orbit_camera(L, 0)
    inst = [L.SplatInstance(cloud)]
    pinst = [L.PointInstance(points, np.eye(4), L.PointStyle(size_mode=0, size=0.004))]
    layer, out = L.RenderTargets(WIDTH, HEIGHT, device=dev), L.RenderTargets(WIDTH, HEIGHT, device=dev)
    raster.render(cam, [], settings, layer, stream, points=pinst)
    mixed_ms = time_device(torch, stream, lambda: raster.render(cam, inst, settings, out, stream, points=pinst), 5)
    under_ms = time_device(torch, stream, lambda: raster.render(cam, inst, settings, out, stream, under=layer), 5)
    plain_ms = time_device(torch, stream, lambda: raster.render(cam, inst, settings, out, stream), 5)
    cmp_ms = time_device(torch, stream, lambda: raster.compare_images(out.colour, layer.colour, stream), 5)
    cmp_bytes = 2 * WIDTH * HEIGHT * 16
    lod = run_lod(L, torch, stream, raster, cloud, settings, peak)
    return {
        "lod": lod,
        "decode": {"workload": "1M raw 3DGS PLY records (236 B) to the packed layout, on the device",
                   "ms": round(decode_ms, 4), "gbs": round(decode_bytes / (decode_ms * 1e-3) / 1e9, 1),
                   "frac_of_hbm": round(decode_bytes / (decode_ms * 1e-3) / 1e9 / peak, 4)},
        "composite": {"workload": "frame 0 of the orbit, 1M splats: alone, with 1M point discs (0.004 world units), "
                                  "and over an under layer of those discs; 1920x1080",
                      "plain_ms": round(plain_ms, 4), "with_discs_ms": round(mixed_ms, 4),
                      "over_layer_ms": round(under_ms, 4)},
        "compare_images": {"workload": "two 1920x1080 float4 images, 8-bit code histogram on the device",
                           "ms": round(cmp_ms, 4), "gbs": round(cmp_bytes / (cmp_ms * 1e-3) / 1e9, 1)},
    }


def run_lod(L, torch, stream, raster, cloud, settings, peak) -> dict:
    """Levels of detail of the benchmark cloud: the build, and per frame the
    cut (one kernel and one count read) at a far view, 30 units out, where the
    finest cells span 9-12 pixels; the frame drawn from each cut."""
    import time
    builder, selector = L.LodBuilder.create(raster), L.CutSelector.create(raster)
    builds = []
    for _ in range(3):
        t0 = time.perf_counter()
        lod = builder.build(cloud, stream=stream)
        builds.append((time.perf_counter() - t0) * 1e3)
        if len(builds) < 3:
            lod.close()
    far = L.projection_for(L.Camera.looking_at((6.0, 4.0, 30.0), (0.0, 0.0, 0.0)), WIDTH, HEIGHT)
    out = L.RenderTargets(WIDTH, HEIGHT, device=cloud.positions.device)
    full_ms = time_device(torch, stream, lambda: raster.render(far, [L.SplatInstance(cloud)], settings, out, stream), 5)
    shw = cloud.sh_words
    cuts = []
    for threshold in (0.0, 10.0, 20.0, 40.0):
        stats = []
        inst = [L.LodInstance(lod)]
        cut_ms = time_device(torch, stream, lambda: selector.select(far, inst, threshold, stats, stream), 5)
        drawn = selector.select(far, inst, threshold, stats, stream)
        frame_ms = time_device(torch, stream, lambda: raster.render(far, drawn, settings, out, stream), 5)
        n_drawn = stats[0].splats + stats[0].merged
        moved = (lod.merged_gaussians() + lod.count) * 4 + 2 * n_drawn * (32 + 4 * shw)
        cuts.append({"threshold_px": threshold, "splats": stats[0].splats, "merged": stats[0].merged,
                     "select_ms": round(cut_ms, 4), "select_gbs": round(moved / (cut_ms * 1e-3) / 1e9, 1),
                     "frame_ms": round(frame_ms, 4)})
    return {"workload": "the 1M-splat benchmark cloud (SH degree 3): LodBuilder.build, then CutSelector.select "
                        "from (6, 4, 30) at 1920x1080 and the frame drawn from each cut",
            "build_ms": round(float(np.median(builds)), 3), "levels": [lv.gaussians.count for lv in lod.levels],
            "full_frame_ms": round(full_ms, 4), "cuts": cuts,
            "select_bytes": "cells + codes read, drawn records read and written (32 + 4 sh_words B each); "
                            "select_ms includes its one count read back"}


def sort_bytes(slots: float, pairs: float, tiles: int) -> dict:
    """Algorithmic bytes of a frame's two sorts: the depth sort of one 8-byte
    word per slot on 24 key bits, and the stable sort of one 8-byte word per
    pair on the tile bits; per 8-bit pass 8 B read + 8 B written per word (the
    digit counts come from the kernels that write the keys)."""
    tile_bits = max(1, math.ceil(math.log2(tiles)))
    depth_passes, tile_passes = 3, math.ceil(tile_bits / 8)
    return {"depth": 16 * depth_passes * slots, "tile": 16 * tile_passes * pairs,
            "depth_passes": depth_passes, "tile_passes": tile_passes}


def run_standin(L, torch, dev, raster, cloud, frames: int) -> dict:
    """The same orbit frames through the stand-in for the reference's GPU
    path (baseline/standin: the reference's stage sequence and launch shapes
    in CUDA -- one thread per chunk in its scans and radix sorts, a blocking
    count readback, a per-pixel blend reading a 48-byte record per pair from
    global memory), device-timed per frame after two warm-up frames, with the
    last image checked equal to the product's."""
    sys.path.insert(0, str(ROOT / "baseline" / "standin"))
    import standin as S
    s = S.Standin(dev.index or 0)
    try:
        settings = L.RenderSettings(width=WIDTH, height=HEIGHT)
        theirs = L.RenderTargets(WIDTH, HEIGHT, device=dev)
        stream = torch.cuda.current_stream(dev)
        times, stages = [], []
        for k in range(frames + 2):
            pr = L.projection_for(orbit_camera(L, k), WIDTH, HEIGHT)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            st = s.render(pr.struct(), cloud.struct(), settings.struct(), theirs.struct(), stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            if k >= 2:
                times.append(a.elapsed_time(b))
                stages.append(st)
        ours = L.RenderTargets(WIDTH, HEIGHT, device=dev)
        raster.render(pr, [L.SplatInstance(cloud)], settings, ours, stream)
        torch.cuda.synchronize(dev)
        equal = torch.equal(ours.colour, theirs.colour) and torch.equal(ours.depth, theirs.depth)
        return {"label": "stand-in for the reference's Slang kernels on this GPU (they cannot run here): "
                         "its stage sequence and launch shapes in CUDA, the same arithmetic",
                "frames": frames, "ms_per_view": round(float(np.mean(times)), 4),
                "stages_ms": {k: round(float(np.mean([x[k] for x in stages])), 4) for k in S.STAGES},
                "images_equal_to_product": bool(equal)}
    finally:
        s.close()


HEAVY_SPLATS = 6_000_000
HEAVY_WIDTH, HEAVY_HEIGHT = 3840, 2160
HEAVY_SEED = 7


def run_sort_heavy(L, torch, dev, raster, peak, clocks, steps: int, splats: int = HEAVY_SPLATS) -> dict:
    """The sort-heavy frame: 6M splats with means N(0,2) and log-scales
    N(-3.5,0.7), 3840x2160, 16x16 tiles, camera 4 units out. Per-stage ms
    from the frame's own events, pairs, and the pair sort's algorithmic bytes
    per second against the HBM peak. The cloud is decoded on the device from
    its raw records (the same bytes as the host packing). The working set
    (about 4 GB of pair words) is far larger than L2, so no flush is needed."""
    raw = L.synthetic_records(splats, HEAVY_SEED, mean_sigma=2.0, log_scale_mean=-3.5, log_scale_sigma=0.7)
    raw_dev = torch.from_numpy(raw).to(dev)
    del raw
    stream = torch.cuda.current_stream(dev)
    cloud = raster.decode_splats(raw_dev, L.ply_encoding(15), 15, stream)
    del raw_dev
    cam = L.square_pixel_camera((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), HEAVY_WIDTH, HEAVY_HEIGHT, 60.0, 0.01)
    proj = L.projection_for(cam, HEAVY_WIDTH, HEAVY_HEIGHT)
    settings = L.RenderSettings(width=HEAVY_WIDTH, height=HEAVY_HEIGHT, time_stages=True)
    targets = L.RenderTargets(HEAVY_WIDTH, HEAVY_HEIGHT, device=dev)
    inst = [L.SplatInstance(cloud)]
    for _ in range(2):
        raster.render(proj, inst, settings, targets, stream)
    torch.cuda.synchronize(dev)
    frame_ms, st = [], []
    w0 = time.time()
    for _ in range(steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st.append(raster.render(proj, inst, settings, targets, stream))
        b.record(stream)
        b.synchronize()
        frame_ms.append(a.elapsed_time(b))
    clocks.window(w0, time.time())
    pairs = float(np.mean([x.pairs for x in st]))
    tiles = ((HEAVY_WIDTH + 15) // 16) * ((HEAVY_HEIGHT + 15) // 16)
    sb = sort_bytes(splats, pairs, tiles)
    sort_ms = float(np.mean([x.depth_sort_ms + x.tile_sort_ms for x in st]))
    gbs = (sb["depth"] + sb["tile"]) / (sort_ms * 1e-3) / 1e9
    out = {"workload": f"{splats / 1e6:g}M splats, means N(0,2), log-scales N(-3.5,0.7), 3840x2160, 16x16 tiles, "
                       "eye (0, 0, 4)",
           "steps": steps, "ms_per_frame": round(float(np.mean(frame_ms)), 4),
           "stages_ms": {k: round(float(np.mean([getattr(x, k) for x in st])), 4)
                         for k in ("project_ms", "depth_sort_ms", "emit_ms", "tile_sort_ms", "blend_ms")},
           "pairs": int(pairs), "visible": int(np.mean([x.visible for x in st])),
           "sort_passes": {"depth": sb["depth_passes"], "tile": sb["tile_passes"]},
           "sort_bytes": "depth sort: 8 B words per slot, tile sort: 8 B words per pair; per 8-bit pass 8 B read "
                         "+ 8 B written per word (the digit counts come from the kernels that write the keys); "
                         "tile_sort_ms also holds the ranges pass",
           "sort_gbs": round(gbs, 1), "sort_frac_of_hbm": round(gbs / peak, 4)}
    del cloud, inst, targets
    torch.cuda.empty_cache()
    return out


def run_heavy_only(args) -> None:
    """Only the sort-heavy frame (for profiling that workload, or a smaller
    one of the same distributions with --heavy-splats)."""
    import torch
    import lucabrtrender_b200 as L
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    clocks = Clocks(0).start()
    raster = L.TileRasterizer.create(0)
    heavy = run_sort_heavy(L, torch, dev, raster, measured_peaks()[0], clocks, args.steps, args.heavy_splats)
    clocks.stop()
    heavy["clocks"] = clocks.summary()
    print(json.dumps(heavy), flush=True)
    raster.close()


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist
    import lucabrtrender_b200 as L
    from lucabrtrender_b200 import _abi
    from lucabrtrender_b200.replicas import GradientBucket

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    clocks = Clocks(local).start()
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    packed = L.pack_splats(L.synthetic_records(SPLATS, SEED), 15, 3)
    cloud = L.to_device(packed, dev)
    instances = [L.SplatInstance(cloud)]
    raster = L.TileRasterizer.create(local)
    settings = L.RenderSettings(width=WIDTH, height=HEIGHT)
    targets = L.RenderTargets(WIDTH, HEIGHT, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    projections = [L.projection_for(orbit_camera(L, k), WIDTH, HEIGHT) for k in range(FRAMES)]

    def frame(k: int, stages: bool = False):
        settings.time_stages = stages
        return raster.render(projections[(k + rank * 7) % FRAMES], instances, settings, targets, stream)

    for k in range(max(3, args.warmup)):
        frame(k)
    torch.cuda.synchronize(dev)

    # --- device-timed steps: inputs resident, L2 flushed before every step ---
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stats_list = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    w0 = time.time()
    for k in range(args.steps):
        flush.fill_(float(k))
        starts[k].record(stream)
        stats_list.append(frame(k, stages=True))
        ends[k].record(stream)
    torch.cuda.synchronize(dev)
    clocks.window(w0, time.time())
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = total_ms / (args.steps * world)

    # --- end to end through the public call: camera from the host, image read back to pinned memory ---
    # Frames are enqueued (render_async), so the host builds frame k + 1's
    # camera while the device renders frame k. Two target pairs: the readback
    # of frame k (on a copy stream) overlaps the render of frame k + 1, which
    # waits only for the readback that last used its targets. No L2 flush
    # here: a frame's working set (124 MB of splats, 48 MB of records, 70 MB
    # of pair words, 41 MB of images) is larger than the 126 MB L2.
    host = [(torch.empty((HEIGHT, WIDTH, 4), dtype=torch.float32, pin_memory=True),
             torch.empty((HEIGHT, WIDTH), dtype=torch.float32, pin_memory=True)) for _ in range(2)]
    pair = [targets, L.RenderTargets(WIDTH, HEIGHT, device=dev)]
    copy_stream = torch.cuda.Stream(dev)
    copied = [torch.cuda.Event() for _ in range(2)]
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    settings.time_stages = False

    def e2e_steps(n: int, timed: bool) -> float:
        torch.cuda.synchronize(dev)
        if timed:
            e_start.record(stream)
        for k in range(n):
            t = pair[k % 2]
            if k >= 2:
                stream.wait_event(copied[k % 2])
            raster.render_async(orbit_camera(L, k + rank * 7), instances, settings, t, stream)
            ready = torch.cuda.Event()
            ready.record(stream)
            copy_stream.wait_event(ready)
            with torch.cuda.stream(copy_stream):
                host[k % 2][0].copy_(t.colour, non_blocking=True)
                host[k % 2][1].copy_(t.depth, non_blocking=True)
            copied[k % 2].record(copy_stream)
        if timed:
            stream.wait_stream(copy_stream)
            e_end.record(stream)
        raster.settle()   # raises if an enqueued frame ran out of pair buffer
        torch.cuda.synchronize(dev)
        return e_start.elapsed_time(e_end) if timed else 0.0

    e2e_steps(max(3, args.warmup), timed=False)
    if world > 1:
        dist.barrier()
    w0 = time.time()
    e2e_ms = e2e_steps(args.steps, timed=True)
    clocks.window(w0, time.time())
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = e2e_ms / (args.steps * world)

    # --- forward + backward (the differentiable path, same splats and views) ---
    fwd_bwd = None
    if not args.no_backward:
        raw = L.synthetic_records(SPLATS, SEED)
        keep = raw.shape[0]
        sh = np.zeros((keep, 16, 3), np.float32)
        sh[:, 0, :] = raw[:, 11:14]
        for c in range(3):
            sh[:, 1:, c] = raw[:, 14 + 15 * c:14 + 15 * (c + 1)]
        sh = sh.astype(np.float16).astype(np.float32)
        params = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev).requires_grad_(True) for k, v in (
            ("means", raw[:, 0:3]), ("log_scales", raw[:, 4:7]), ("quats", raw[:, 7:11]), ("logits", raw[:, 3]),
            ("sh", sh))}
        gen = torch.Generator(device=dev).manual_seed(SEED)
        target = torch.rand((HEIGHT, WIDTH, 3), generator=gen, device=dev)
        train_settings = L.RenderSettings(width=WIDTH, height=HEIGHT)
        # The backward writes every gradient into one flat bucket; over
        # several ranks one all-reduce of it per step sums their gradients.
        bucket = GradientBucket(keep, dev)
        ordered = [params[k] for k in ("means", "log_scales", "quats", "logits", "sh")]
        # The fp16 working copy of the SH coefficients the kernels read; a
        # mixed-precision optimizer step refreshes it with the fp32 master.
        sh16 = params["sh"].detach().reshape(keep, 48).half().contiguous()

        def train_step(k: int):
            for v in params.values():
                v.grad = None
            colour, _ = L.rasterize(params["means"], params["log_scales"], params["quats"], params["logits"],
                                    params["sh"], projections[(k + rank * 7) % FRAMES], train_settings, raster,
                                    grad_bucket=bucket, sh_storage=sh16)
            loss = L.l1_loss(colour, target, raster)
            loss.backward()
            bucket.all_reduce(ordered)
            return loss

        for k in range(max(3, args.warmup)):
            train_step(k)
        torch.cuda.synchronize(dev)
        bwd_blend, bwd_proj, fwd_stats = [], [], []
        # Steps run back to back, as a training loop runs them (the host
        # waits only inside each backward, for its forward's counts); each
        # step is timed on the device from after its L2 flush to its end.
        fb_start = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        fb_end = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        torch.cuda.synchronize(dev)
        w0 = time.time()
        for k in range(args.steps):
            flush.fill_(float(k))
            fb_start[k].record(stream)
            train_step(k)
            fb_end[k].record(stream)
        torch.cuda.synchronize(dev)
        clocks.window(w0, time.time())
        fb_ms = [a.elapsed_time(b) for a, b in zip(fb_start, fb_end)]
        # The backward's and the forward's stage breakdowns, from extra steps
        # (not part of the timed steps above).
        for k in range(3):
            train_step(k)
            t_blend, t_proj = L.train.backward_times(raster)
            bwd_blend.append(t_blend)
            bwd_proj.append(t_proj)
        train_settings.time_stages = True
        for k in range(3):
            train_step(k)
            fwd_stats.append(raster.last_train_stats)
        train_settings.time_stages = False
        fb_total = float(sum(fb_ms))
        if world > 1:
            t = torch.tensor([fb_total], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            fb_total = float(t.item())
        fb_value = fb_total / (args.steps * world)
        fwd_bwd = {"ms_per_view": round(fb_value, 4), "ratio_to_plain_forward": round(fb_value / value, 3),
                   "forward_stages_ms": {k: round(float(np.mean([getattr(x, k) for x in fwd_stats])), 4)
                                         for k in ("project_ms", "depth_sort_ms", "emit_ms", "tile_sort_ms",
                                                   "blend_ms")},
                   "backward_blend_ms": round(float(np.mean(bwd_blend)), 4),
                   "backward_reduce_and_projection_ms": round(float(np.mean(bwd_proj)), 4),
                   "loss": "L1 vs a seeded uniform [0,1]^3 target, mean over pixels and channels "
                           "(lucabrtrender_b200.l1_loss: one kernel each way)",
                   "params": "means, log-scales, quaternions, opacity logits, 48 SH (fp16 storage read as it is, "
                             "fp32 master and gradients; the fp16 copy belongs to the optimizer step, not timed)",
                   "gradients": "written into one flat bucket; over N ranks one all-reduce (sum) of it per step, "
                                "inside the timed step"}

    # --- the rows around the hot path ---
    next_rows = None
    if not args.no_next:
        next_rows = run_next_rows(L, torch, dev, raster, packed, cloud, measured_peaks()[0])

    # --- the stand-in for the reference's GPU path, same orbit ---
    standin = None
    if not args.no_standin:
        standin = run_standin(L, torch, dev, raster, cloud, 5)

    # --- the sort-heavy frame ---
    heavy = None
    if not args.no_heavy:
        heavy = run_sort_heavy(L, torch, dev, raster, measured_peaks()[0], clocks, max(3, args.steps // 4),
                               args.heavy_splats)

    # --- many views: one batched call against sequential renders ---
    batch = None
    if not args.no_batch:
        batch = run_batch(L, torch, dev, rank, raster, args, clocks)

    # --- roofline of the dominant kernel, measured live over the timed steps ---
    st = stats_list
    mean = lambda f: float(np.mean([getattr(s, f) for s in st]))  # noqa: E731
    stage = {k: mean(k) for k in ("project_ms", "depth_sort_ms", "emit_ms", "tile_sort_ms", "blend_ms")}
    pairs = float(np.mean([s.pairs for s in st]))
    visible = float(np.mean([s.visible for s in st]))
    tiles = ((WIDTH + 15) // 16) * ((HEIGHT + 15) // 16)
    pixels = WIDTH * HEIGHT
    sort = sort_bytes(SPLATS, pairs, tiles)
    # Algorithmic bytes per launch (per unit x units):
    #   blend:   ranges 8 B/tile + (8 B pair word + 48 B record) per pair + 20 B per pixel written
    #   project: 124 B per splat read (deg 3); 48 + 16 + 4 + 4 B record, rect, count, key
    #            and 8 + 16 B depth and aux words written per slot
    #   emit:    per slot its sorted depth word and count read and its offset written (depth-order
    #            offsets: 8+4+4 B), then its count, rect, aux words and offset read (4+16+16+4 B;
    #            records of large splats not counted), 8 B per pair written
    #   sorts:   see sort_bytes
    bytes_blend = 8 * tiles + 56 * pairs + 20 * pixels
    bytes_project = 124 * SPLATS + 96 * SPLATS
    bytes_emit = 56 * SPLATS + 8 * pairs
    peak, peak_kind = measured_peaks()
    kernels = {
        "blend": (stage["blend_ms"], bytes_blend),
        "tile sort + ranges": (stage["tile_sort_ms"], sort["tile"] + 8 * pairs + 8 * tiles),
        "depth sort": (stage["depth_sort_ms"], sort["depth"]),
        "emit": (stage["emit_ms"], bytes_emit),
        "project + counts": (stage["project_ms"], bytes_project),
    }
    dom_name = max(kernels, key=lambda n: kernels[n][0])
    dom_ms, dom_bytes = kernels[dom_name]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    sort_ms = stage["depth_sort_ms"] + stage["tile_sort_ms"]
    sort_gbs = (sort["depth"] + sort["tile"]) / (sort_ms * 1e-3) / 1e9 if sort_ms > 0 else None
    # project, depth passes, depth-order offsets, pair writes, tile passes,
    # ranges, the tiles' busiest-first order (two kernels), blend, the
    # counters' store into host memory; and one launch that zeroes the
    # counters, the projection's scratch, both sorts' scratch and the ranges
    launches_per_frame = (1 + sort["depth_passes"] + 2 + sort["tile_passes"] + 1 + 2 + 1 + 1) + 1

    clocks.stop()
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            # A bounded sample (about 25 s of CPU work on 16 host threads):
            # the first frames of the same orbit; the --impl reference arm
            # times every frame the GPU arm times.
            threads = os.cpu_count() or 1
            ms, times = cpu_reference_frames(range(args.cpu_frames), threads)
            cpu = {"value": round(ms, 3), "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"frames 0-{args.cpu_frames - 1} of the same orbit on the oracle (C++ restatement "
                             f"of the reference's kernels), {threads} threads"}
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(world),
            "frame": {"pairs": int(pairs), "visible": int(visible), "tiles": tiles, "pixels": pixels},
            "stages_ms": {k: round(v, 4) for k, v in stage.items()},
            "sort_gbs": round(sort_gbs, 1) if sort_gbs else None,
            "roofline": {"kernel": dom_name, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": PROFILED_DRAM_BYTES.get(dom_name),
                         "peak_kind": peak_kind,
                         "secondary": {"bound": "issue", "frac": PROFILED_ISSUE_ACTIVE.get(dom_name),
                                       "source": "ncu issue-active fraction of the profiled launch"}},
            "e2e": {"value": round(e2e_value, 4), "unit": UNIT,
                    "h2d_bytes_per_step": _abi.C.sizeof(_abi.Projection),
                    "d2h_bytes_per_step": pixels * 20},
            "gpu_launches": launches_per_frame * args.steps,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "fwd_bwd": fwd_bwd,
            "batch": batch,
            "sort_heavy": heavy,
            "standin": standin,
            "next_rows": next_rows,
        }
        print(json.dumps(line), flush=True)
    raster.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-frames", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-backward", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-next", action="store_true")
    ap.add_argument("--no-heavy", action="store_true")
    ap.add_argument("--no-standin", action="store_true")
    ap.add_argument("--heavy-only", action="store_true",
                    help="run only the sort-heavy frame (--steps frames after 2 warm-up frames)")
    ap.add_argument("--heavy-splats", type=int, default=HEAVY_SPLATS)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    elif args.heavy_only:
        run_heavy_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
