"""ORACLE -- test infrastructure, not product code.

ctypes wrapper of ``oracle/_build/liblrt_oracle.so``, the CPU restatement of
lucabRTrender's splat tile rasteriser (see ``lrt_oracle.h`` for what it
restates and how it is pinned). Only the tests, the smoke check and the
benchmark's CPU-baseline leg use it, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liblrt_oracle.so"
REF_LIB = HERE / "_ref" / "libref_camera.so"

import sys  # noqa: E402

# The public header's struct layouts (its ctypes mirror beside it); the
# oracle shares them with the package but imports nothing from the package.
if str(HERE.parent / "include") not in sys.path:
    sys.path.insert(0, str(HERE.parent / "include"))
import lrt_raster_ctypes as _abi  # noqa: E402


class FrameOut(C.Structure):
    _fields_ = [
        ("colour", C.c_void_p), ("depth", C.c_void_p), ("proj", C.c_void_p), ("rects", C.c_void_p),
        ("touched", C.c_void_p), ("depth_keys", C.c_void_p), ("pair_tiles", C.c_void_p),
        ("pair_slots", C.c_void_p), ("ranges", C.c_void_p), ("pair_capacity", C.c_uint64),
        ("pairs", C.c_uint64), ("visible", C.c_uint32), ("slots", C.c_uint32), ("stage_ms", C.c_double * 6),
        ("blend_tiles", C.c_void_p),
    ]


def build() -> None:
    """Compile the restatement (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    lib.ora_exp.argtypes = [C.c_float]
    lib.ora_exp.restype = C.c_float
    lib.ora_log.argtypes = [C.c_float]
    lib.ora_log.restype = C.c_float
    lib.ora_math_eval.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32]
    lib.ora_math_eval.restype = None
    lib.ora_camera_looking_at.argtypes = [C.POINTER(C.c_double)] * 3 + [C.POINTER(_abi.CameraStruct)]
    lib.ora_projection_for.argtypes = [C.POINTER(_abi.CameraStruct), C.c_uint32, C.c_uint32,
                                       C.POINTER(_abi.Projection)]
    lib.ora_pack_splats.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    lib.ora_render.argtypes = [C.POINTER(_abi.Projection), C.POINTER(_abi.SplatInstanceStruct), C.c_uint32,
                               C.POINTER(_abi.RenderSettingsStruct), C.POINTER(FrameOut), C.c_uint32]
    lib.ora_reference_render.argtypes = [C.POINTER(_abi.Projection), C.POINTER(_abi.SplatInstanceStruct),
                                         C.c_uint32, C.POINTER(_abi.RenderSettingsStruct), C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_uint32), C.c_uint32]
    lib.ora_render_composite.argtypes = [C.POINTER(_abi.Projection), C.POINTER(_abi.SplatInstanceStruct), C.c_uint32,
                                         C.POINTER(_abi.PointInstanceStruct), C.c_uint32, C.c_void_p, C.c_void_p,
                                         C.POINTER(_abi.RenderSettingsStruct), C.POINTER(FrameOut), C.c_uint32]
    lib.ora_reference_render_composite.argtypes = [
        C.POINTER(_abi.Projection), C.POINTER(_abi.SplatInstanceStruct), C.c_uint32,
        C.POINTER(_abi.PointInstanceStruct), C.c_uint32, C.POINTER(_abi.RenderSettingsStruct), C.c_void_p,
        C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32]
    lib.ora_pack_points.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_uint32)]
    lib.ora_random_points.argtypes = [C.c_uint32, C.c_uint64, C.c_void_p]
    lib.ora_compare_hdr.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                    C.POINTER(C.c_float)]
    lib.ora_count_different.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.ora_count_different.restype = C.c_uint64
    lib.ora_decode_splats.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(_abi.SplatEncoding), C.c_uint32, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    lib.ora_compare_images.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                       C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint64)]
    lib.ora_random_cloud.argtypes = [C.c_uint32, C.c_uint64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]
    lib.ora_f32_to_f16.argtypes = [C.c_float]
    lib.ora_f32_to_f16.restype = C.c_uint16
    lib.ora_f16_to_f32.argtypes = [C.c_uint16]
    lib.ora_f16_to_f32.restype = C.c_float
    lib.ora_lod_build.argtypes = [C.POINTER(_abi.GpuSplatsStruct), C.c_void_p, C.c_float, C.c_uint32,
                                  C.POINTER(C.c_void_p)]
    lib.ora_lod_free.argtypes = [C.c_void_p]
    lib.ora_lod_free.restype = None
    lib.ora_lod_describe.argtypes = [C.c_void_p, C.POINTER(_abi.LodInfo)]
    lib.ora_lod_copy.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    lib.ora_lod_cut.argtypes = [C.c_void_p, C.POINTER(_abi.Projection), C.POINTER(C.c_double), C.c_float, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    _lib = lib
    return lib


def _check(code: int, what: str) -> None:
    if code != 0:
        raise RuntimeError(f"oracle {what} failed with status {code}")


# ---------------------------------------------------------------- camera ----
def looking_at(eye, target, up=(0.0, 1.0, 0.0)) -> _abi.CameraStruct:
    out = _abi.CameraStruct()
    arr = lambda v: (C.c_double * 3)(*map(float, v))  # noqa: E731
    _check(load().ora_camera_looking_at(arr(eye), arr(target), arr(up), C.byref(out)), "looking_at")
    return out


def projection_for(camera: _abi.CameraStruct, width: int, height: int) -> _abi.Projection:
    out = _abi.Projection()
    _check(load().ora_projection_for(C.byref(camera), width, height, C.byref(out)), "projection_for")
    return out


def filter3d(cloud: "HostCloud", views, coefficient: float = 0.2) -> np.ndarray:
    """The 3D filter's variance per splat from (Projection struct, width, height) views."""
    n = len(views)
    cams = (_abi.Projection * max(n, 1))()
    sizes = (C.c_uint32 * max(2 * n, 2))()
    for k, (pr, w, h) in enumerate(views):
        cams[k] = pr
        sizes[2 * k], sizes[2 * k + 1] = int(w), int(h)
    out = np.zeros(cloud.count, np.float32)
    cs = cloud.struct()
    lib = load()
    lib.ora_filter3d.argtypes = [C.POINTER(_abi.GpuSplatsStruct), C.POINTER(_abi.Projection), C.POINTER(C.c_uint32),
                                 C.c_uint32, C.c_float, C.c_void_p]
    _check(lib.ora_filter3d(C.byref(cs), cams, sizes, n, float(coefficient), out.ctypes.data), "filter3d")
    return out


# --------------------------------------------------------------- packing ----
@dataclass
class HostCloud:
    positions: np.ndarray   # [N, 4] float32
    shape: np.ndarray       # [N, 4] uint32
    sh: np.ndarray          # [N, words] uint32
    rest_per_colour: int
    filter3d: np.ndarray | None = None   # [N] float32, the 3D filter's variance

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])

    def struct(self) -> _abi.GpuSplatsStruct:
        s = _abi.GpuSplatsStruct()
        s.count = self.count
        s.rest_per_colour = self.rest_per_colour
        s.sh_words = int(self.sh.shape[1])
        s.positions = self.positions.ctypes.data
        s.shape = self.shape.ctypes.data
        s.sh = self.sh.ctypes.data
        if self.filter3d is not None:
            assert self.filter3d.dtype == np.float32 and self.filter3d.flags["C_CONTIGUOUS"]
            s.filter3d = self.filter3d.ctypes.data
        return s


def pack(raw: np.ndarray, file_per_colour: int, keep: int) -> HostCloud:
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    n, fpr = raw.shape
    words = max((keep * 3 + 1) // 2, 1)
    pos = np.empty((n, 4), np.float32)
    shape = np.empty((n, 4), np.uint32)
    sh = np.empty((n, words), np.uint32)
    kept = C.c_uint32()
    _check(load().ora_pack_splats(raw.ctypes.data, n, fpr, file_per_colour, keep, pos.ctypes.data,
                                  shape.ctypes.data, sh.ctypes.data, C.byref(kept)), "pack")
    k = kept.value
    return HostCloud(pos[:k].copy(), shape[:k].copy(), sh[:k].copy(), keep)


def decode_splats(raw: np.ndarray, encoding: _abi.SplatEncoding, keep: int) -> HostCloud:
    """Raw records of any encoding to the packed layout (the restatement of
    the device decode)."""
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    n = raw.shape[0]
    words = max((keep * 3 + 1) // 2, 1)
    pos = np.empty((n, 4), np.float32)
    shape = np.empty((n, 4), np.uint32)
    sh = np.empty((n, words), np.uint32)
    kept = C.c_uint32()
    _check(load().ora_decode_splats(raw.ctypes.data, n, C.byref(encoding), keep, pos.ctypes.data, shape.ctypes.data,
                                    sh.ctypes.data, C.byref(kept)), "decode_splats")
    k = kept.value
    return HostCloud(pos[:k].copy(), shape[:k].copy(), sh[:k].copy(), keep)


def random_cloud(count: int, seed: int, min_size=0.004, max_size=0.6, min_opacity=0.02,
                 max_opacity=0.99) -> np.ndarray:
    """The reference tests' randomCloud (23-float degree-1 records)."""
    raw = np.empty((count, 23), np.float32)
    _check(load().ora_random_cloud(count, seed, min_size, max_size, min_opacity, max_opacity, raw.ctypes.data),
           "random_cloud")
    return raw


@dataclass
class HostPoints:
    positions: np.ndarray   # [N, 4] float32
    colours: np.ndarray     # [N, 2] uint32 (f16 r|g, b|a)

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])

    def struct(self) -> _abi.GpuPointsStruct:
        s = _abi.GpuPointsStruct()
        s.count = self.count
        s.positions = self.positions.ctypes.data
        s.colours = self.colours.ctypes.data
        return s


def pack_points(raw: np.ndarray, colour_kind: int = 2, detail: float = 1.0) -> HostPoints:
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    n = raw.shape[0]
    pos = np.empty((n, 4), np.float32)
    col = np.empty((n, 2), np.uint32)
    kept = C.c_uint32()
    _check(load().ora_pack_points(raw.ctypes.data, n, colour_kind, detail, pos.ctypes.data, col.ctypes.data,
                                  C.byref(kept)), "pack_points")
    k = kept.value
    return HostPoints(pos[:k].copy(), col[:k].copy())


def random_points(count: int, seed: int) -> np.ndarray:
    """The reference points test's randomPoints (x y z r g b records)."""
    raw = np.empty((count, 6), np.float32)
    _check(load().ora_random_points(count, seed, raw.ctypes.data), "random_points")
    return raw


def _points(points):
    """points: list of (HostPoints, object_to_world 4x4, lrt_point_style)."""
    arr = (_abi.PointInstanceStruct * max(1, len(points)))()
    keep = []
    for k, (cloud, m, style) in enumerate(points):
        cs = cloud.struct()
        keep.append(cs)
        arr[k].points = C.pointer(cs)
        arr[k].object_to_world[:] = [float(v) for v in np.asarray(m, np.float64).reshape(16)]
        arr[k].style = style
    return arr, keep


# ------------------------------------------------------------- rendering ----
def _instances(instances):
    """instances: list of (HostCloud, object_to_world 4x4, edit lrt_splat_edit | None)."""
    arr = (_abi.SplatInstanceStruct * max(1, len(instances)))()
    keep = []
    for k, (cloud, m, edit) in enumerate(instances):
        cs = cloud.struct()
        keep.append(cs)
        arr[k].splats = C.pointer(cs)
        arr[k].object_to_world[:] = [float(v) for v in np.asarray(m, np.float64).reshape(16)]
        if edit is not None:
            arr[k].edit = edit
    return arr, keep


def tile_mask(settings, tiles) -> np.ndarray:
    """One byte per tile of the frame, set for the given tile ids."""
    tiles_x = (settings.width + 15) // 16
    tiles_y = (settings.height + 15) // 16
    m = np.zeros(tiles_x * tiles_y, np.uint8)
    m[np.asarray(list(tiles), np.int64)] = 1
    return m


def render(projection: _abi.Projection, instances, settings: _abi.RenderSettingsStruct, threads: int = 0,
           want_pairs: bool = True, points=(), under=None, blend_tiles=None) -> dict:
    """The restated rasteriser; `points` (HostPoints, matrix, style) are drawn
    as discs after the splats, `under` is an optional (colour [H,W,4], depth
    [H,W]) layer -- either makes the frame a composite one. `blend_tiles`
    (one byte per tile, see tile_mask) blends only the marked tiles; the
    other pixels stay zero."""
    slots = sum(c.count for c, _, _ in instances) + sum(p.count for p, _, _ in points)
    tiles_x = (settings.width + 15) // 16
    tiles_y = (settings.height + 15) // 16
    w, h = settings.width, settings.height
    colour = np.zeros((h, w, 4), np.float32)
    depth = np.zeros((h, w), np.float32)
    proj = np.zeros((slots, 12), np.float32)
    rects = np.zeros((slots, 4), np.uint32)
    touched = np.zeros(slots, np.uint32)
    keys = np.zeros(slots, np.uint32)
    ranges = np.zeros((tiles_x * tiles_y, 2), np.uint32)
    cap = int(touched.size) * 0  # filled on the second call when pairs are wanted
    out = FrameOut()
    out.colour, out.depth = colour.ctypes.data, depth.ctypes.data
    out.proj, out.rects = proj.ctypes.data, rects.ctypes.data
    out.touched, out.depth_keys = touched.ctypes.data, keys.ctypes.data
    out.ranges = ranges.ctypes.data
    out.pair_capacity = cap
    if blend_tiles is not None:
        blend_tiles = np.ascontiguousarray(blend_tiles, np.uint8)
        out.blend_tiles = blend_tiles.ctypes.data
    arr, keep = _instances(instances)
    parr, pkeep = _points(points)
    if under is not None:
        under = (np.ascontiguousarray(under[0], np.float32), np.ascontiguousarray(under[1], np.float32))

    def run(o):
        if not points and under is None:
            return load().ora_render(C.byref(projection), arr, len(instances), C.byref(settings), C.byref(o), threads)
        uc = under[0].ctypes.data if under is not None else None
        ud = under[1].ctypes.data if under is not None else None
        return load().ora_render_composite(C.byref(projection), arr, len(instances), parr, len(points), uc, ud,
                                           C.byref(settings), C.byref(o), threads)

    _check(run(out), "render")
    pairs = int(out.pairs)
    result = dict(colour=colour, depth=depth, proj=proj, rects=rects, touched=touched, depth_keys=keys,
                  ranges=ranges, pairs=pairs, visible=int(out.visible), slots=int(out.slots),
                  stage_ms=list(out.stage_ms))
    if want_pairs:
        # The pair list is only known after the frame: recompute it into buffers of that size
        # (deterministic, so the second run is the same frame).
        pt = np.zeros(pairs, np.uint32)
        ps = np.zeros(pairs, np.uint32)
        out2 = FrameOut()
        out2.pair_tiles, out2.pair_slots, out2.pair_capacity = pt.ctypes.data, ps.ctypes.data, pairs
        no_blend = np.zeros(ranges.shape[0], np.uint8)   # the image is already drawn
        out2.blend_tiles = no_blend.ctypes.data
        _check(run(out2), "render")
        result["pair_tiles"] = pt
        result["pair_slots"] = ps
    return result


def reference_render(projection: _abi.Projection, instances, settings: _abi.RenderSettingsStruct,
                     threads: int = 0, points=()):
    w, h = settings.width, settings.height
    colour = np.zeros((h, w, 4), np.float32)
    depth = np.zeros((h, w), np.float32)
    over = C.c_uint32()
    arr, keep = _instances(instances)
    if points:
        parr, pkeep = _points(points)
        _check(load().ora_reference_render_composite(C.byref(projection), arr, len(instances), parr, len(points),
                                                     C.byref(settings), colour.ctypes.data, depth.ctypes.data,
                                                     C.byref(over), threads), "reference_render")
    else:
        _check(load().ora_reference_render(C.byref(projection), arr, len(instances), C.byref(settings),
                                           colour.ctypes.data, depth.ctypes.data, C.byref(over), threads),
               "reference_render")
    return colour, depth, int(over.value)


@dataclass
class ImageDifference:
    p99: int
    max: int
    over2: int
    pixels: int
    histogram: np.ndarray


def compare_images(a: np.ndarray, b: np.ndarray) -> ImageDifference:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    h, w = a.shape[:2]
    hist = np.zeros(256, np.uint32)
    p99, mx = C.c_uint32(), C.c_uint32()
    over2, pixels = C.c_uint64(), C.c_uint64()
    _check(load().ora_compare_images(a.ctypes.data, b.ctypes.data, w, h, hist.ctypes.data, C.byref(p99),
                                     C.byref(mx), C.byref(over2), C.byref(pixels)), "compare_images")
    return ImageDifference(p99.value, mx.value, over2.value, pixels.value, hist)


def compare_hdr(a: np.ndarray, b: np.ndarray):
    """(histogram [256], summed relative squared error) of compareHdr."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    h, w = a.shape[:2]
    hist = np.zeros(256, np.uint32)
    err = C.c_float()
    _check(load().ora_compare_hdr(a.ctypes.data, b.ctypes.data, w, h, hist.ctypes.data, C.byref(err)), "compare_hdr")
    return hist, err.value


def count_different(a: np.ndarray, b: np.ndarray) -> int:
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    return int(load().ora_count_different(a.ctypes.data, b.ctypes.data, a.size))


def math_eval(fn: int, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    load().ora_math_eval(fn, x.ctypes.data, y.ctypes.data, x.size)
    return y


def threads() -> int:
    return os.cpu_count() or 1


# --------------------------------------------------------- training path ----
@dataclass
class RawCloud:
    """Differentiable parameters on the host (the training path's layout)."""
    means: np.ndarray       # [N, 3] float32
    log_scales: np.ndarray  # [N, 3] float32
    quats: np.ndarray       # [N, 4] float32 (w, x, y, z)
    logits: np.ndarray      # [N] float32
    sh16: np.ndarray        # [N, 16, 3] float16

    @property
    def count(self) -> int:
        return int(self.means.shape[0])

    def struct(self) -> _abi.TrainParams:
        for name in ("means", "log_scales", "quats", "logits", "sh16"):
            a = getattr(self, name)
            assert a.flags["C_CONTIGUOUS"], name
        p = _abi.TrainParams()
        p.count = self.count
        p.means, p.log_scales, p.quats = self.means.ctypes.data, self.log_scales.ctypes.data, self.quats.ctypes.data
        p.opacity_logits, p.sh = self.logits.ctypes.data, self.sh16.ctypes.data
        return p


def train_render(projection: _abi.Projection, cloud: RawCloud, settings: _abi.RenderSettingsStruct,
                 crop=(0, 0, 0, 0), threads: int = 0, crop_only: bool = False) -> dict:
    """The restated training forward; with a crop, each crop pixel's
    contributor list (its slots in blend order). `crop_only` blends only the
    tiles the crop overlaps (the rest of the image stays zero)."""
    lib = load()
    lib.ora_train_render.argtypes = [C.POINTER(_abi.Projection), C.POINTER(_abi.TrainParams),
                                     C.POINTER(_abi.RenderSettingsStruct), C.POINTER(FrameOut), C.c_uint32,
                                     C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                     C.c_uint64, C.POINTER(C.c_uint64)]
    n = cloud.count
    w, h = settings.width, settings.height
    tiles = ((w + 15) // 16) * ((h + 15) // 16)
    colour = np.zeros((h, w, 4), np.float32)
    depth = np.zeros((h, w), np.float32)
    proj = np.zeros((n, 12), np.float32)
    rects = np.zeros((n, 4), np.uint32)
    touched = np.zeros(n, np.uint32)
    keys = np.zeros(n, np.uint32)
    ranges = np.zeros((tiles, 2), np.uint32)
    out = FrameOut()
    out.colour, out.depth, out.proj, out.rects = colour.ctypes.data, depth.ctypes.data, proj.ctypes.data, rects.ctypes.data
    out.touched, out.depth_keys, out.ranges = touched.ctypes.data, keys.ctypes.data, ranges.ctypes.data
    x0, y0, cw, ch = crop
    offsets = np.zeros(cw * ch + 1, np.uint32)
    total = C.c_uint64()
    p = cloud.struct()
    crop_tiles = None
    if cw > 0 and ch > 0:
        tx = range(x0 // 16, (x0 + cw - 1) // 16 + 1)
        ty = range(y0 // 16, (y0 + ch - 1) // 16 + 1)
        crop_tiles = tile_mask(settings, [y * ((w + 15) // 16) + x for y in ty for x in tx])
    if crop_only:
        out.blend_tiles = crop_tiles.ctypes.data if crop_tiles is not None else None
    _check(lib.ora_train_render(C.byref(projection), C.byref(p), C.byref(settings), C.byref(out), threads, x0, y0, cw,
                                ch, offsets.ctypes.data, None, 0, C.byref(total)), "train_render")
    slots = np.zeros(max(1, total.value), np.uint32)
    out2 = FrameOut()
    # The second pass only fills the crop's lists: blend the crop's tiles alone.
    second_mask = crop_tiles if crop_tiles is not None else np.zeros(tiles, np.uint8)
    out2.blend_tiles = second_mask.ctypes.data
    _check(lib.ora_train_render(C.byref(projection), C.byref(p), C.byref(settings), C.byref(out2), threads, x0, y0,
                                cw, ch, offsets.ctypes.data, slots.ctypes.data, total.value, C.byref(total)),
           "train_render")
    return dict(colour=colour, depth=depth, proj=proj, rects=rects, touched=touched, depth_keys=keys, ranges=ranges,
                pairs=int(out.pairs), visible=int(out.visible), list_offsets=offsets, list_slots=slots[:total.value])


# ------------------------------------------------------------------- LOD ----
class OracleLod:
    """The restated levels of detail of one host cloud (ora_lod_build)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self.info = _abi.LodInfo()
        _check(load().ora_lod_describe(handle, C.byref(self.info)), "lod_describe")

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                load().ora_lod_free(self._h)
                self._h = None
        except Exception:   # at interpreter exit the module may be gone
            pass

    def _copy(self, which: int, shape: tuple, dtype) -> np.ndarray:
        out = np.zeros(shape, dtype)
        _check(load().ora_lod_copy(self._h, which, out.ctypes.data), "lod_copy")
        return out

    @property
    def count(self) -> int:
        return int(self.info.count)

    @property
    def level_groups(self) -> list[int]:
        return [int(v) for v in self.info.level_groups[:self.info.levels]]

    @property
    def store(self) -> HostCloud:
        """The splats in Morton order."""
        n, w = self.count, int(self.info.sh_words)
        return HostCloud(self._copy(0, (n, 4), np.float32), self._copy(1, (n, 4), np.uint32),
                         self._copy(2, (n, w), np.uint32), int(self.info.rest_per_colour))

    @property
    def codes(self) -> np.ndarray:
        return self._copy(3, (self.count,), np.uint32)

    @property
    def starts(self) -> np.ndarray:
        return self._copy(4, (self.level_groups[-1],), np.uint32)

    @property
    def merged(self) -> HostCloud:
        """Every stored level's Gaussians, coarsest level first."""
        m, w = int(self.info.merged), int(self.info.sh_words)
        return HostCloud(self._copy(5, (m, 4), np.float32), self._copy(6, (m, 4), np.uint32),
                         self._copy(7, (m, w), np.uint32), int(self.info.rest_per_colour))

    @property
    def cells(self) -> np.ndarray:
        return self._copy(8, (int(self.info.merged),), np.uint32)

    def cut(self, projection: _abi.Projection, object_to_world=None, threshold: float = 0.0):
        """The drawn cloud of one instance and (splats, merged) drawn."""
        n, w = self.count, int(self.info.sh_words)
        pos = np.zeros((n, 4), np.float32)
        shape = np.zeros((n, 4), np.uint32)
        sh = np.zeros((n, w), np.uint32)
        m = np.eye(4) if object_to_world is None else np.asarray(object_to_world, np.float64)
        mat = (C.c_double * 16)(*[float(v) for v in m.reshape(16)])
        splats, merged = C.c_uint32(), C.c_uint32()
        _check(load().ora_lod_cut(self._h, C.byref(projection), mat, float(threshold), pos.ctypes.data,
                                  shape.ctypes.data, sh.ctypes.data, C.byref(splats), C.byref(merged)), "lod_cut")
        k = splats.value + merged.value
        return HostCloud(pos[:k].copy(), shape[:k].copy(), sh[:k].copy(), int(self.info.rest_per_colour)), \
            splats.value, merged.value


def lod_build(cloud: HostCloud, bounds=None, max_group_fraction: float = 0.5, coarsest_level: int = 1) -> OracleLod:
    cs = cloud.struct()
    b = None
    if bounds is not None:
        b = (C.c_float * 6)(*[float(v) for v in np.asarray(bounds, np.float32).reshape(6)])
    h = C.c_void_p()
    _check(load().ora_lod_build(C.byref(cs), b, float(max_group_fraction), int(coarsest_level), C.byref(h)),
           "lod_build")
    return OracleLod(h)
