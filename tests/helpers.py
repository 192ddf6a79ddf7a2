"""Shared scene set-ups for the tests: the reference's own render-test scenes
(tests/render/test_splat_render.cpp, tests/render/SplatFixtures.h in the
lucabRTrender tree) and the benchmark's synthetic scenes, built once as packed
bytes and handed to both the oracle (host pointers) and the CUDA path."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

import lucabrtrender_b200 as L
from lucabrtrender_b200 import _abi

import oracle as ora

SH0 = np.float32(0.28209479)


def cloud_record(x, y, z, opacity, sx, sy, sz, wxyz, colour, rest=None) -> np.ndarray:
    """CloudBuilder::add (SplatFixtures.h:30-45): one degree-1 record of 23 floats."""
    f = np.float32
    r = np.zeros(23, np.float32)
    a = f(opacity)
    r[:14] = [x, y, z, np.log(a / (f(1) - a)), np.log(f(sx)), np.log(f(sy)), np.log(f(sz)), *wxyz,
              (f(colour[0]) - f(0.5)) / SH0, (f(colour[1]) - f(0.5)) / SH0, (f(colour[2]) - f(0.5)) / SH0]
    if rest is not None:
        r[14:] = rest
    return r


def packed_from_raw(raw: np.ndarray, file_per_colour: int, max_degree: int = 3) -> L.PackedSplats:
    return L.pack_splats(raw, file_per_colour, max_degree)


def host_cloud(p: L.PackedSplats) -> ora.HostCloud:
    return ora.HostCloud(p.positions, p.shape, p.sh, p.rest_per_colour)


def settings(width=250, height=190, antialias=True, linearise=True, background=(0, 0, 0, 0), depth=0,
             threshold=0.5, max_sh_degree=3) -> L.RenderSettings:
    return L.RenderSettings(width=width, height=height, antialias=antialias, max_sh_degree=max_sh_degree,
                            background=background, depth=L.Depth(depth), depth_threshold=threshold,
                            linearise=linearise)


def camera(eye, target=(0, 0, 0), focal=50.0, orthographic=False, window_translate=(0.0, 0.0),
           window_scale=(1.0, 1.0), roll=0.0, near=0.1) -> L.Camera:
    c = L.Camera.looking_at(eye, target)
    c.lens.focal = focal
    c.lens.orthographic = orthographic
    c.lens.window_translate = tuple(window_translate)
    c.lens.window_scale = tuple(window_scale)
    c.lens.window_roll = roll
    c.lens.near_z = near
    return c


def translation(t) -> np.ndarray:
    m = np.eye(4)
    m[:3, 3] = t
    return m


def rotation_y(deg) -> np.ndarray:
    c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
    return m


def scaling(s) -> np.ndarray:
    return np.diag([s[0], s[1], s[2], 1.0])


def edit_struct(edit: L.SplatEdit | None) -> _abi.SplatEdit | None:
    if edit is None:
        return None
    e = _abi.SplatEdit()
    edit.fill(e)
    return e


@dataclass
class Scene:
    """One frame: packed clouds with transforms and edits, a camera, settings."""
    name: str
    clouds: list            # [(PackedSplats, object_to_world, SplatEdit | None)]
    camera: L.Camera
    settings: L.RenderSettings
    extra: dict = field(default_factory=dict)

    def projection(self) -> L.Projection:
        return L.projection_for(self.camera, self.settings.width, self.settings.height)

    def oracle_instances(self):
        return [(host_cloud(p), m, edit_struct(e)) for p, m, e in self.clouds]

    def oracle_render(self, threads=0, want_pairs=True):
        return ora.render(self.projection().struct(), self.oracle_instances(), self.settings.struct(), threads,
                          want_pairs)

    def oracle_reference(self, threads=0):
        return ora.reference_render(self.projection().struct(), self.oracle_instances(), self.settings.struct(),
                                    threads)

    def gpu_instances(self, device="cuda"):
        out = []
        for p, m, e in self.clouds:
            out.append(L.SplatInstance(L.to_device(p, device), m, e if e is not None else L.SplatEdit()))
        return out


_RANDOM_CACHE = {}


def random_cloud_packed(count=3000, seed=7) -> L.PackedSplats:
    key = (count, seed)
    if key not in _RANDOM_CACHE:
        _RANDOM_CACHE[key] = packed_from_raw(ora.random_cloud(count, seed), 3, 3)
    return _RANDOM_CACHE[key]


def reference_render_scenes() -> list[Scene]:
    """The five sections of "the tile rasteriser renders what the GPU reference
    renders" (test_splat_render.cpp:70-121): a 3000-splat randomCloud(seed 7),
    degree 1, at 250x190 (partial tiles)."""
    cloud = random_cloud_packed(3000, 7)
    I = np.eye(4)
    scenes = [
        Scene("perspective", [(cloud, I, None)], camera((1.5, 1.0, 6.0), focal=30.0), settings()),
        Scene("frustum_edge", [(cloud, I, None)], camera((0.3, -0.2, 2.2), focal=18.0), settings()),
        Scene("orthographic", [(cloud, I, None)], camera((0.0, 3.0, 5.0), focal=5.0, orthographic=True), settings()),
        Scene("no_aa_window_roll", [(cloud, I, None)],
              camera((-2.0, 0.5, 5.0), window_translate=(0.2, 0.0), window_scale=(1.0, 1.3), roll=25.0),
              settings(antialias=False)),
        Scene("two_instances",
              [(cloud, I, None),
               (cloud, translation((0.5, 0.0, -1.5)) @ rotation_y(40.0) @ scaling((1.0, 0.7, 1.3)), None)],
              camera((2.0, 1.5, 7.0), target=(0.0, 0.0, -0.5)), settings()),
    ]
    return scenes


def edit_scenes() -> list[Scene]:
    """"a SplatEdit renders as the GPU reference renders it" (test_splat_render.cpp:231-283)."""
    cloud = random_cloud_packed(3000, 29)
    cam = camera((1.5, 1.0, 6.0), focal=30.0)
    edits = {
        "keep_box": L.SplatEdit(active=True, mode=L.EditMode.KEEP, centre=(0.5, 0.0, 0.0), size=(1.0, 0.8, 1.5)),
        "remove_sphere": L.SplatEdit(active=True, mode=L.EditMode.REMOVE, shape=L.EditShape.SPHERE,
                                     size=(1.2, 0.0, 0.0), tint=(0.2, 1.0, 1.0)),
        "grade_inverted_box": L.SplatEdit(active=True, mode=L.EditMode.GRADE, invert=True, size=(1.0, 1.0, 1.0),
                                          tint=(1.0, 0.6, 0.3), saturation=0.3, brightness=1.4, opacity=0.5),
        "haze_filters": L.SplatEdit(active=True, mode=L.EditMode.GRADE, size=(100.0, 100.0, 100.0), min_opacity=0.4,
                                    max_scale=0.2),
    }
    return [Scene(name, [(cloud, np.eye(4), e)], cam, settings(), extra=dict(edit=e)) for name, e in edits.items()]


def synthetic_scene(count: int, width: int, height: int, seed: int = 1, eye=(0.0, 0.0, 4.0), **dist) -> Scene:
    raw = L.synthetic_records(count, seed, **dist)
    packed = packed_from_raw(raw, 15, 3)
    cam = L.square_pixel_camera(eye, (0.0, 0.0, 0.0), width, height, 60.0, 0.01)
    return Scene(f"synthetic_{count}_{width}x{height}", [(packed, np.eye(4), None)], cam,
                 settings(width=width, height=height))


def pair_words_to_tile_slot(words: np.ndarray, slot_bits: int, depth_bits: int = 24):
    """A sorted pair word is tile << (depth_bits + slot_bits) | depth key <<
    slot_bits | slot: training frames carry the 24-bit depth key, other
    frames (depth_bits 0) only tile << 32 | slot. keys is None without one."""
    w = words.astype(np.uint64)
    slots = (w & np.uint64((1 << slot_bits) - 1)).astype(np.uint32)
    keys = None
    if depth_bits:
        keys = ((w >> np.uint64(slot_bits)) & np.uint64((1 << depth_bits) - 1)).astype(np.uint32)
    tiles = (w >> np.uint64(depth_bits + slot_bits)).astype(np.uint32)
    return tiles, keys, slots


# ------------------------------------------------------------------ points --
def point_style(size_mode: int = 0, size: float = 0.01, constant_colour: bool = False,
                colour=(1.0, 1.0, 1.0)) -> _abi.PointStyleStruct:
    s = _abi.PointStyleStruct()
    s.size_mode = size_mode
    s.size = size
    s.constant_colour = 1 if constant_colour else 0
    s.colour[:] = list(map(float, colour))
    return s


class Lcg:
    """tests/render/test_points.cpp:22-30 in float32 arithmetic."""

    def __init__(self, seed: int = 0):
        self.state = 0x2545F4914F6CDD1D ^ seed

    def next(self) -> np.float32:
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return np.float32((self.state >> 40) & 0xFFFFFF) / np.float32(16777216.0)

    def range(self, lo, hi) -> np.float32:
        lo, hi = np.float32(lo), np.float32(hi)
        return lo + (hi - lo) * self.next()


def fog_records(count: int = 40) -> np.ndarray:
    """The 40 large translucent splats of tests/render/test_points.cpp:164-178,
    the same draws written in the PLY encoding (logit opacity, log scales,
    identity rotation, base colour through the DC term)."""
    rng = Lcg()
    out = []
    for _ in range(count):
        x, y, z = rng.range(-2, 2), rng.range(-1, 1), rng.range(-2, 3)
        opacity = rng.range(0.1, 0.6)
        sx, sy, sz = rng.range(0.1, 0.5), rng.range(0.1, 0.5), rng.range(0.1, 0.5)
        colour = (rng.range(0, 1), rng.range(0, 1), rng.range(0, 1))
        out.append(cloud_record(x, y, z, opacity, sx, sy, sz, (1, 0, 0, 0), colour))
    return np.stack(out)


class FixtureLcg(Lcg):
    """tests/render/SplatFixtures.h:48-55: the same generator from its own state."""

    def __init__(self):
        self.state = 0x853C49E6748FEA9B


def single_splat_cells_records() -> np.ndarray:
    """tests/lod/test_lod.cpp:112-130: six splats, one to a level-1 cell, drawn
    in the order the reference names them (opacity, three sizes, the turn, the
    colour)."""
    rng = FixtureLcg()
    at = [(-2, -2, -2), (2, -2, -2), (-2, 2, -2), (2, 2, 2), (-2, 2, 2), (2, -2, 2)]
    rest = [0.2, -0.1, 0.3, 0.0, 0.1, -0.2, 0.1, 0.0, -0.3]
    out = []
    for p in at:
        opacity = rng.range(0.3, 0.95)
        sx, sy, sz = rng.range(0.1, 0.5), rng.range(0.1, 0.5), rng.range(0.1, 0.5)
        turn = (rng.range(-1, 1), rng.range(-1, 1), rng.range(-1, 1), rng.range(-1, 1))
        colour = (rng.range(0.1, 1.0), rng.range(0.1, 1.0), rng.range(0.1, 1.0))
        out.append(cloud_record(*p, opacity, sx, sy, sz, turn, colour, rest))
    return np.stack(out)


def morton_codes(positions: np.ndarray, lo, extent) -> np.ndarray:
    """morton.slang:23-28 in numpy float32: 10 bits an axis, x highest."""
    unit = (positions[:, :3].astype(np.float32) - np.asarray(lo, np.float32)) / np.float32(max(extent, 1e-20))
    q = np.minimum((np.clip(unit, 0, 1) * np.float32(1024.0)).astype(np.uint32), 1023)
    code = np.zeros(len(positions), np.uint32)
    for b in range(10):
        for axis, shift in ((0, 2), (1, 1), (2, 0)):
            code |= ((q[:, axis] >> b) & 1) << np.uint32(3 * b + shift)
    return code


def cell_axes(cells: np.ndarray, level: int) -> np.ndarray:
    """morton.slang:30-33: per cell its index on x, y, z."""
    out = np.zeros((len(cells), 3), np.uint32)
    for b in range(level):
        for axis, shift in ((0, 2), (1, 1), (2, 0)):
            out[:, axis] |= ((cells >> np.uint32(3 * b + shift)) & 1) << np.uint32(b)
    return out


def projected_edge(cells: np.ndarray, level: int, lo, extent: float, eye, pixels_per_unit: float,
                   orthographic: bool = False) -> np.ndarray:
    """lod_cut.slang:15-26 in numpy float32, one rounding per operation."""
    f = np.float32
    edge = f(extent) / f(1 << level)
    if orthographic:
        return np.full(len(cells), edge * f(pixels_per_unit), np.float32)
    idx = cell_axes(cells, level).astype(np.float32)
    eye = np.asarray(eye, np.float32)
    d = []
    for k in range(3):
        low = f(lo[k]) + idx[:, k] * edge
        nearest = np.minimum(np.maximum(eye[k], low), low + edge)
        d.append(nearest - eye[k])
    dist = np.maximum(np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), f(1e-6))
    return (edge * f(pixels_per_unit)) / dist


def half_sweep() -> np.ndarray:
    """Floats for the float-to-half check: random bit patterns, every exponent,
    the overflow and subnormal edges, and exact ties."""
    rng = np.random.default_rng(5)
    bits = rng.integers(0, 2**32, 400000, dtype=np.uint64).astype(np.uint32)
    edges = np.float32([65504.0, 65519.996, 65520.0, 65536.0, 6.1035156e-05, 6.097555e-05, 5.9604645e-08,
                        2.9802322e-08, 2.9802326e-08, 1e-45, 0.0, np.inf, 1.0 + 2.0**-11, 1.0 + 3 * 2.0**-11])
    ties = ((rng.integers(0x1C400, 0x23C00, 20000, dtype=np.uint32) << np.uint32(13)) | np.uint32(0x1000)).view(np.float32)
    x = np.concatenate([bits.view(np.float32), edges, -edges, ties])
    return x[~np.isnan(x)]
