"""ORACLE -- test infrastructure, not product code.

The benchmark workload built from the oracle alone, for the CPU legs of
``bench.py`` (its ``--impl reference`` arm and its ``cpu_baseline``): the
seeded synthetic records, their packed bytes (the restated loader packing,
R: shaders/lrt/scene/splat_decode.slang:20-91), the orbit's cameras (the
restated camera code, pinned to R: modules/render/src/Camera.cpp:9-48) and
frames rendered by the restated rasteriser. Nothing here imports the
package or loads its library, so the reference arm's numbers do not depend
on the code they are compared with. ``tests/test_bench_workload.py`` checks
that these inputs equal the package's bit for bit.
"""
from __future__ import annotations

import math
import time

import numpy as np

import oracle as ora

# The distributions of the synthetic scenes (splat count, seed and the
# normal parameters per field); the record layout is the PLY one: x y z,
# logit opacity, 3 log scales, rotation w x y z, 3 DC, then the rest
# coefficients all red, then green, then blue.
REST_FOR_DEGREE = {0: 0, 1: 3, 2: 8, 3: 15}


def synthetic_records(count: int, seed: int, *, mean_sigma: float = 1.0, log_scale_mean: float = -4.5,
                      log_scale_sigma: float = 0.5, dc_sigma: float = 0.5, rest_sigma: float = 0.05,
                      degree: int = 3) -> np.ndarray:
    """Raw records: means N(0, mean_sigma), log-scales N(log_scale_mean,
    log_scale_sigma), rotations normalised N(0,1)^4 (uniform on SO(3)),
    opacity logits N(0,1), DC N(0, dc_sigma), rest N(0, rest_sigma); float32
    draws from a Philox generator seeded with `seed`."""
    rest = REST_FOR_DEGREE[degree]
    rng = np.random.Generator(np.random.Philox(seed))
    raw = rng.standard_normal((count, 14 + 3 * rest), dtype=np.float32)
    raw[:, 0:3] *= np.float32(mean_sigma)
    raw[:, 4:7] = raw[:, 4:7] * np.float32(log_scale_sigma) + np.float32(log_scale_mean)
    raw[:, 11:14] *= np.float32(dc_sigma)
    raw[:, 14:] *= np.float32(rest_sigma)
    return raw


def packed_cloud(count: int, seed: int, **dist) -> ora.HostCloud:
    """The packed degree-3 cloud the frames read."""
    return ora.pack(synthetic_records(count, seed, **dist), 15, 15)


def square_pixel_projection(eye, target, width: int, height: int, vertical_fov_deg: float = 60.0,
                            near_z: float = 0.01, up=(0.0, 1.0, 0.0)):
    """A pinhole camera with square pixels and the given vertical field of
    view, in the reference's lens terms (focal_mm = focal_px * haperture / W),
    and its Projection for a width x height target."""
    cam = ora.looking_at(eye, target, up)
    focal_px = (height / 2.0) / math.tan(math.radians(vertical_fov_deg) / 2.0)
    cam.lens.focal = focal_px * cam.lens.haperture / width
    cam.lens.near_z = near_z
    return ora.projection_for(cam, width, height)


def orbit_projection(k: int, frames: int, radius: float, width: int, height: int):
    """Frame k of the orbit: eye at radius * (sin t, 0, cos t), t = 2 pi k / frames, looking at the origin."""
    th = 2.0 * math.pi * (k % frames) / frames
    eye = (radius * math.sin(th), 0.0, radius * math.cos(th))
    return square_pixel_projection(eye, (0.0, 0.0, 0.0), width, height, 60.0, 0.01)


def settings(width: int, height: int):
    """RenderSettings defaults (R: modules/render/include/lrt/render/TileRasterizer.h:105-118):
    antialias on, SH up to degree 3, black transparent background, mean depth,
    threshold 0.5, linearise on."""
    s = ora._abi.RenderSettingsStruct()
    s.width, s.height = width, height
    s.antialias = 1
    s.max_sh_degree = 3
    s.background[:] = [0.0, 0.0, 0.0, 0.0]
    s.depth_mode = 0
    s.depth_threshold = 0.5
    s.linearise = 1
    s.time_stages = 0
    return s


def time_frames(cloud: ora.HostCloud, frame_ids, frames: int, radius: float, width: int, height: int,
                threads: int) -> list[float]:
    """Milliseconds per frame of the restated rasteriser over the given orbit frames."""
    st = settings(width, height)
    out = []
    for k in frame_ids:
        pr = orbit_projection(k, frames, radius, width, height)
        t = time.perf_counter()
        ora.render(pr, [(cloud, np.eye(4), None)], st, threads, want_pairs=False)
        out.append((time.perf_counter() - t) * 1e3)
    return out
