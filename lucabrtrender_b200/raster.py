"""The tile rasteriser, shaped like the reference's ``lrt::render::TileRasterizer``
(modules/render/include/lrt/render/TileRasterizer.h:26-193): ``create``, then
``render(camera | projection, instances, settings, targets)`` returning
``FrameStats``. Every call goes through the C-ABI of the in-tree CUDA library.
Device memory is torch's; the rasteriser's own scratch is the library's.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _abi
from .camera import Camera, Projection, projection_for
from .scene import GpuPoints, GpuSplats


class EditShape(enum.IntEnum):
    BOX = 0
    SPHERE = 1


class EditMode(enum.IntEnum):
    KEEP = 0
    REMOVE = 1
    GRADE = 2


@dataclass
class SplatEdit:
    """SplatEdit (TileRasterizer.h:29-50)."""
    active: bool = False
    shape: EditShape = EditShape.BOX
    mode: EditMode = EditMode.GRADE
    centre: tuple[float, float, float] = (0.0, 0.0, 0.0)
    size: tuple[float, float, float] = (1.0, 1.0, 1.0)
    tint: tuple[float, float, float] = (1.0, 1.0, 1.0)
    saturation: float = 1.0
    brightness: float = 1.0
    opacity: float = 1.0
    min_opacity: float = 0.0
    max_scale: float = 0.0
    invert: bool = False

    def fill(self, e: _abi.SplatEdit) -> None:
        e.active = 1 if self.active else 0
        e.shape = int(self.shape)
        e.mode = int(self.mode)
        e.invert = 1 if self.invert else 0
        e.centre[:] = list(map(float, self.centre))
        e.size[:] = list(map(float, self.size))
        e.tint[:] = list(map(float, self.tint))
        e.saturation = self.saturation
        e.brightness = self.brightness
        e.opacity = self.opacity
        e.min_opacity = self.min_opacity
        e.max_scale = self.max_scale


@dataclass
class SplatInstance:
    """SplatInstance (TileRasterizer.h:52-67) without relighting."""
    splats: GpuSplats | None
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))
    edit: SplatEdit = field(default_factory=SplatEdit)


@dataclass
class PointStyle:
    """PointStyle (Points.h): what the disc route reads. size_mode 0 world
    units, 1 pixels; size is the diameter."""
    size_mode: int = 0
    size: float = 0.01
    constant_colour: bool = False
    colour: tuple[float, float, float] = (1.0, 1.0, 1.0)

    def fill(self, s: _abi.PointStyleStruct) -> None:
        s.size_mode = int(self.size_mode)
        s.size = float(self.size)
        s.constant_colour = 1 if self.constant_colour else 0
        s.colour[:] = list(map(float, self.colour))


@dataclass
class PointInstance:
    """PointInstance (Points.h): a point cloud drawn as opaque discs."""
    points: GpuPoints | None
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))
    style: PointStyle = field(default_factory=PointStyle)


class Depth(enum.IntEnum):
    MEAN = 0
    THRESHOLD = 1


@dataclass
class RenderSettings:
    """RenderSettings (TileRasterizer.h:105-118), same defaults."""
    width: int = 1920
    height: int = 1080
    antialias: bool = True
    max_sh_degree: int = 3
    background: tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    depth: Depth = Depth.MEAN
    depth_threshold: float = 0.5
    linearise: bool = True
    time_stages: bool = False

    def struct(self) -> _abi.RenderSettingsStruct:
        s = _abi.RenderSettingsStruct()
        s.width, s.height = int(self.width), int(self.height)
        s.antialias = 1 if self.antialias else 0
        s.max_sh_degree = int(self.max_sh_degree)
        s.background[:] = list(map(float, self.background))
        s.depth_mode = int(self.depth)
        s.depth_threshold = float(self.depth_threshold)
        s.linearise = 1 if self.linearise else 0
        s.time_stages = 1 if self.time_stages else 0
        return s


@dataclass
class FrameStats:
    """FrameStats (TileRasterizer.h:120-126)."""
    splats: int = 0
    visible: int = 0
    pairs: int = 0
    project_ms: float = 0.0
    depth_sort_ms: float = 0.0
    counts_ms: float = 0.0
    emit_ms: float = 0.0
    tile_sort_ms: float = 0.0
    blend_ms: float = 0.0
    total_ms: float = 0.0

    @staticmethod
    def from_struct(s: _abi.FrameStatsStruct) -> "FrameStats":
        return FrameStats(s.splats, s.visible, s.pairs, s.project_ms, s.depth_sort_ms, s.counts_ms, s.emit_ms,
                          s.tile_sort_ms, s.blend_ms, s.total_ms)

    def stages_line(self) -> str:
        """The stage breakdown `lrt bench --stages` prints (apps/lrt/src/CmdRender.cpp:412-418)."""
        return (f"project {self.project_ms:.2f}, depth sort {self.depth_sort_ms:.2f}, counts {self.counts_ms:.2f}, "
                f"emit {self.emit_ms:.2f}, tile sort+ranges {self.tile_sort_ms:.2f}, blend {self.blend_ms:.2f}")


@dataclass
class ImageDifference:
    """ImageDifference (ReferenceRenderer.h:50-55), in 8-bit sRGB code values."""
    pixels: int
    p99: int
    max: int
    over2: int


@dataclass
class HdrDifference:
    """HdrDifference (ReferenceRenderer.h:59-64)."""
    pixels: int
    rel_mse: float
    p99_relative: float
    max_relative: float


class RenderTargets:
    """RenderTargets (TileRasterizer.h:128-134): colour float4 premultiplied
    linear [H, W, 4] and depth [H, W], bottom row first, on the device.
    Reallocated by the rasteriser when the frame's size changes."""

    def __init__(self, width: int = 0, height: int = 0, device="cuda"):
        self.width = 0
        self.height = 0
        self.device = device
        self.colour: torch.Tensor | None = None
        self.depth: torch.Tensor | None = None
        if width and height:
            self.reserve(width, height)

    def reserve(self, width: int, height: int) -> None:
        if self.width == width and self.height == height and self.colour is not None:
            return
        self.colour = torch.empty((height, width, 4), dtype=torch.float32, device=self.device)
        self.depth = torch.empty((height, width), dtype=torch.float32, device=self.device)
        self.width, self.height = width, height

    def struct(self) -> _abi.TargetsStruct:
        t = _abi.TargetsStruct()
        t.width, t.height = self.width, self.height
        t.colour = self.colour.data_ptr()
        t.depth = self.depth.data_ptr()
        return t


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


class TileRasterizer:
    """TileRasterizer::create / render over ``lrt_rast_*``."""

    def __init__(self, handle: C.c_void_p, device: int):
        self._handle = handle
        self.device = device

    @staticmethod
    def create(device: int | None = None) -> "TileRasterizer":
        lib = _abi.load()
        if device is None:
            device = torch.cuda.current_device()
        h = C.c_void_p()
        code = lib.lrt_rast_create(C.byref(h), int(device))
        _abi.check(code, f"lrt_rast_create(device {device})")
        return TileRasterizer(h, int(device))

    def close(self) -> None:
        if self._handle:
            _abi.load().lrt_rast_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        return _abi.load().lrt_rast_last_error(self._handle).decode()

    def _check(self, code: int) -> None:
        if code != _abi.OK:
            raise _abi.LrtError(code, self.last_error())

    def render(self, view: Camera | Projection, instances: Sequence[SplatInstance], settings: RenderSettings,
               targets: RenderTargets, stream=None, points: Sequence[PointInstance] = (),
               under: RenderTargets | None = None) -> FrameStats:
        """TileRasterizer::render. `points` are drawn as opaque discs sorted
        with the splats; `under` (the frame's size) is a layer the splats
        composite over (lrt_rast_render_composite)."""
        lib = _abi.load()
        projection = view if isinstance(view, Projection) else projection_for(view, settings.width, settings.height)
        targets.reserve(settings.width, settings.height)
        clouds = []
        arr = (_abi.SplatInstanceStruct * max(1, len(instances)))()
        for k, inst in enumerate(instances):
            if inst.splats is not None and inst.splats.count > 0:
                cs = inst.splats.struct()
                clouds.append(cs)
                arr[k].splats = C.pointer(cs)
            arr[k].object_to_world[:] = [float(v) for v in np.asarray(inst.object_to_world, np.float64).reshape(16)]
            inst.edit.fill(arr[k].edit)
        pr = projection.struct()
        st = settings.struct()
        tg = targets.struct()
        stats = _abi.FrameStatsStruct()
        if points or under is not None:
            parr = (_abi.PointInstanceStruct * max(1, len(points)))()
            for k, inst in enumerate(points):
                if inst.points is not None and inst.points.count > 0:
                    ps = inst.points.struct()
                    clouds.append(ps)
                    parr[k].points = C.pointer(ps)
                parr[k].object_to_world[:] = [float(v) for v in
                                              np.asarray(inst.object_to_world, np.float64).reshape(16)]
                inst.style.fill(parr[k].style)
            ut = under.struct() if under is not None else None
            code = lib.lrt_rast_render_composite(self._handle, C.byref(pr), arr, len(instances), parr, len(points),
                                                 C.byref(ut) if ut is not None else None, C.byref(st), C.byref(tg),
                                                 C.byref(stats), _stream_ptr(stream))
        else:
            code = lib.lrt_rast_render(self._handle, C.byref(pr), arr, len(instances), C.byref(st), C.byref(tg),
                                       C.byref(stats), _stream_ptr(stream))
        self._check(code)
        return FrameStats.from_struct(stats)

    def render_async(self, view: Camera | Projection, instances: Sequence[SplatInstance], settings: RenderSettings,
                     targets: RenderTargets, stream=None) -> None:
        """The frame, returning once it is enqueued (lrt_rast_render_async);
        its counts and status are read by settle()."""
        lib = _abi.load()
        projection = view if isinstance(view, Projection) else projection_for(view, settings.width, settings.height)
        targets.reserve(settings.width, settings.height)
        clouds = []
        arr = (_abi.SplatInstanceStruct * max(1, len(instances)))()
        for k, inst in enumerate(instances):
            if inst.splats is not None and inst.splats.count > 0:
                cs = inst.splats.struct()
                clouds.append(cs)
                arr[k].splats = C.pointer(cs)
            arr[k].object_to_world[:] = [float(v) for v in np.asarray(inst.object_to_world, np.float64).reshape(16)]
            inst.edit.fill(arr[k].edit)
        pr = projection.struct()
        st = settings.struct()
        tg = targets.struct()
        self._check(lib.lrt_rast_render_async(self._handle, C.byref(pr), arr, len(instances), C.byref(st), C.byref(tg),
                                              _stream_ptr(stream)))

    def settle(self) -> FrameStats:
        """Waits for the enqueued frames (lrt_rast_settle); raises LrtError
        with OVERFLOW when one of them ran out of pair buffer."""
        stats = _abi.FrameStatsStruct()
        self._check(_abi.load().lrt_rast_settle(self._handle, C.byref(stats)))
        return FrameStats.from_struct(stats)

    def render_batch(self, views: Sequence[tuple], instances: Sequence[SplatInstance], settings: RenderSettings,
                     targets: Sequence[RenderTargets] | None = None, stream=None):
        """Many views in one call (lrt_rast_render_batch). `views` holds
        (camera | projection, width, height) per view; returns (targets, stats)."""
        lib = _abi.load()
        n = len(views)
        if targets is None:
            targets = [RenderTargets() for _ in range(n)]
        arr_v = (_abi.View * max(1, n))()
        for k, (view, w, h) in enumerate(views):
            projection = view if isinstance(view, Projection) else projection_for(view, w, h)
            targets[k].reserve(w, h)
            arr_v[k].projection = projection.struct()
            arr_v[k].width, arr_v[k].height = w, h
            arr_v[k].colour, arr_v[k].depth = targets[k].colour.data_ptr(), targets[k].depth.data_ptr()
        clouds = []
        arr = (_abi.SplatInstanceStruct * max(1, len(instances)))()
        for k, inst in enumerate(instances):
            if inst.splats is not None and inst.splats.count > 0:
                cs = inst.splats.struct()
                clouds.append(cs)
                arr[k].splats = C.pointer(cs)
            arr[k].object_to_world[:] = [float(v) for v in np.asarray(inst.object_to_world, np.float64).reshape(16)]
            inst.edit.fill(arr[k].edit)
        st = settings.struct()
        stats = _abi.BatchStats()
        self._check(lib.lrt_rast_render_batch(self._handle, arr, len(instances), arr_v, n, C.byref(st),
                                              C.byref(stats), _stream_ptr(stream)))
        return targets, stats

    def decode_splats(self, raw: torch.Tensor, encoding: _abi.SplatEncoding, keep_per_colour: int,
                      stream=None) -> GpuSplats:
        """CloudLoader::upload's decode on the device (lrt_rast_decode_splats):
        raw records [N, floats_per_record] float32 on this device, validated,
        compacted and packed in one kernel."""
        raw = raw.contiguous().float()
        n = raw.shape[0] if raw.dim() > 0 else 0
        dev = raw.device
        words = max((keep_per_colour * 3 + 1) // 2, 1)
        pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
        shape = torch.empty((n, 4), dtype=torch.int32, device=dev)
        sh = torch.empty((n, words), dtype=torch.int32, device=dev)
        kept = C.c_uint32(0)
        self._check(_abi.load().lrt_rast_decode_splats(self._handle, raw.data_ptr() if n else None, n,
                                                       C.byref(encoding), keep_per_colour,
                                                       pos.data_ptr() if n else None, shape.data_ptr() if n else None,
                                                       sh.data_ptr() if n else None, C.byref(kept),
                                                       _stream_ptr(stream)))
        k = kept.value
        return GpuSplats(pos[:k], shape[:k], sh[:k], keep_per_colour)

    def decode_points(self, raw: torch.Tensor, colour_kind: int = 2, detail: float = 1.0, stream=None) -> GpuPoints:
        """Raw x y z r g b point records on this device to a GpuPoints
        (lrt_rast_decode_points)."""
        raw = raw.contiguous().float().reshape(-1, 6)
        n = raw.shape[0]
        dev = raw.device
        pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
        col = torch.empty((n, 2), dtype=torch.int32, device=dev)
        kept = C.c_uint32(0)
        self._check(_abi.load().lrt_rast_decode_points(self._handle, raw.data_ptr() if n else None, n, colour_kind,
                                                       float(detail), pos.data_ptr() if n else None,
                                                       col.data_ptr() if n else None, C.byref(kept),
                                                       _stream_ptr(stream)))
        k = kept.value
        return GpuPoints(pos[:k], col[:k])

    def compare_images(self, a: torch.Tensor, b: torch.Tensor, stream=None):
        """compareImages on the device: (ImageDifference fields, histogram)."""
        h, w = a.shape[:2]
        a, b = a.contiguous(), b.contiguous()
        out = _abi.ImageDifferenceStruct()
        hist = np.zeros(256, np.uint32)
        self._check(_abi.load().lrt_rast_compare_images(self._handle, a.data_ptr(), b.data_ptr(), w, h, C.byref(out),
                                                        hist.ctypes.data, _stream_ptr(stream)))
        return ImageDifference(out.pixels, out.p99, out.max, out.over2), hist

    def compare_hdr(self, a: torch.Tensor, b: torch.Tensor, stream=None) -> "HdrDifference":
        h, w = a.shape[:2]
        a, b = a.contiguous(), b.contiguous()
        out = _abi.HdrDifferenceStruct()
        self._check(_abi.load().lrt_rast_compare_hdr(self._handle, a.data_ptr(), b.data_ptr(), w, h, C.byref(out),
                                                     _stream_ptr(stream)))
        return HdrDifference(out.pixels, out.rel_mse, out.p99_relative, out.max_relative)

    def count_different(self, a: torch.Tensor, b: torch.Tensor, stream=None) -> int:
        a, b = a.contiguous(), b.contiguous()
        n = C.c_uint64()
        self._check(_abi.load().lrt_rast_count_different(self._handle, a.data_ptr(), b.data_ptr(), a.numel(),
                                                         C.byref(n), _stream_ptr(stream)))
        return int(n.value)

    def debug_view(self) -> _abi.DebugView:
        v = _abi.DebugView()
        self._check(_abi.load().lrt_rast_debug_view(self._handle, C.byref(v)))
        return v

    def debug_arrays(self) -> dict[str, torch.Tensor]:
        """Copies of the last frame's intermediate buffers (for parity checks)."""
        v = self.debug_view()
        dev = torch.device("cuda", self.device)

        def grab(ptr, count, dtype, cols=1):
            shape = (count, cols) if cols > 1 else (count,)
            if not count:
                return torch.empty(shape, dtype=dtype, device=dev)
            return device_view(ptr, shape, dtype, self.device).clone()

        return {
            "proj": grab(v.proj, v.slots, torch.float32, 12),
            "rects": grab(v.rects, v.slots, torch.int32, 4),
            "touched": grab(v.touched, v.slots, torch.int32),
            "depth_keys": grab(v.depth_keys, v.slots, torch.int32),
            "pairs": grab(v.pairs, v.pairs_count, torch.int64),
            "ranges": grab(v.ranges, v.tiles, torch.int32, 2),
            "slot_bits": v.slot_bits,
            "depth_bits": v.depth_bits,
            "tile_bits": v.tile_bits,
            "visible": v.visible,
        }

    def filter3d(self, cloud: GpuSplats, views: Sequence[tuple], coefficient: float = 0.2,
                 stream=None) -> torch.Tensor:
        """The Mip-Splatting 3D filter's variance per splat (lrt_rast_filter3d)
        from cameras given as (Camera or Projection, width, height): assign
        the result to ``cloud.filter3d`` to render with the filter."""
        n = len(views)
        cams = (_abi.Projection * max(n, 1))()
        sizes = (C.c_uint32 * max(2 * n, 2))()
        for k, (view, w, h) in enumerate(views):
            cams[k] = (view if isinstance(view, Projection) else projection_for(view, w, h)).struct()
            sizes[2 * k], sizes[2 * k + 1] = int(w), int(h)
        out = torch.empty(cloud.count, dtype=torch.float32, device=cloud.positions.device)
        cs = cloud.struct()
        self._check(_abi.load().lrt_rast_filter3d(self._handle, C.byref(cs), cams, sizes, n, float(coefficient),
                                                  out.data_ptr() if cloud.count else None, _stream_ptr(stream)))
        return out

    def prefix_sum(self, values: torch.Tensor, out: torch.Tensor, total: torch.Tensor, stream=None) -> None:
        """PrefixSum::apply over uint32 bit patterns held in int32 tensors."""
        n = values.numel()
        self._check(_abi.load().lrt_prefix_sum(self._handle, values.data_ptr(), out.data_ptr(), total.data_ptr(), n,
                                              _stream_ptr(stream)))

    def radix_sort(self, keys: torch.Tensor, values: torch.Tensor | None, key_bits: int, stream=None) -> None:
        """RadixSort::sort in place: keys int32 (4-byte) or int64 (8-byte) bit patterns."""
        key_bytes = keys.element_size()
        self._check(_abi.load().lrt_radix_sort(self._handle, keys.data_ptr(),
                                              values.data_ptr() if values is not None else None, keys.numel(),
                                              key_bits, key_bytes, _stream_ptr(stream)))


_TYPESTR = {torch.float32: "<f4", torch.int32: "<i4", torch.int64: "<i8"}


class _DeviceArray:
    """A borrowed device pointer presented through __cuda_array_interface__."""

    def __init__(self, ptr: int, shape: tuple, dtype: torch.dtype):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": _TYPESTR[dtype],
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def device_view(ptr: int, shape: tuple, dtype: torch.dtype, device: int, sync: bool = True) -> torch.Tensor:
    """A tensor viewing library-owned device memory (valid until the next call on the handle).
    `sync`: wait for the device first (callers whose call already waited pass False)."""
    if sync:
        torch.cuda.synchronize(device)
    return torch.as_tensor(_DeviceArray(ptr, shape, dtype), device=torch.device("cuda", device))


def math_eval(fn: int, x: torch.Tensor) -> torch.Tensor:
    """The library's own exp (0), log (1), sRGB-to-linear (2), cut-off power (3), float-to-half
    bits (4) and the half pair (x, -x/2) (5), both as uint32 words in a float tensor, on the device."""
    y = torch.empty_like(x)
    _abi.check(_abi.load().lrt_math_eval(fn, x.data_ptr(), y.data_ptr(), x.numel(),
                                         torch.cuda.current_stream().cuda_stream), "math_eval")
    return y
