"""Levels of detail for splat clouds, built and cut on the device.

Mirrors modules/lod/include/lrt/lod/Lod.h over ``lrt_lod_build`` and
``lrt_lod_select``:

  LodBuilder    once per cloud: Morton order, every level's groups, moments
                from the finest stored level up, one Gaussian per group
  CutSelector   every frame, per instance: which merged Gaussians and which
                splats to draw, gathered into one cloud the rasteriser draws
                like any other

In memory only: every chunk of a cloud's splats is resident (the reference's
``.lrtc`` streaming store is not provided).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _abi
from .camera import Projection
from .raster import SplatEdit, SplatInstance, TileRasterizer, _stream_ptr, device_view
from .scene import GpuSplats

LEVELS = 10   # 30-bit Morton codes (lod_common.slang:36)


@dataclass
class LodBuildSettings:
    """LodBuildSettings (Lod.h:83-93)."""
    max_group_fraction: float = 0.5
    coarsest_level: int = 1
    chunk_splats: int = 1 << 16

    def struct(self) -> _abi.LodBuildSettings:
        s = _abi.LodBuildSettings()
        s.max_group_fraction = float(self.max_group_fraction)
        s.coarsest_level = int(self.coarsest_level)
        s.chunk_splats = int(self.chunk_splats)
        return s


def _view(s: _abi.GpuSplatsStruct, device: int) -> GpuSplats:
    """A GpuSplats whose tensors view library-owned memory (the calls that
    return these clouds have waited for them)."""
    n, words = int(s.count), int(s.sh_words)
    if n == 0:
        dev = torch.device("cuda", device)
        return GpuSplats(torch.empty((0, 4), dtype=torch.float32, device=dev),
                         torch.empty((0, 4), dtype=torch.int32, device=dev),
                         torch.empty((0, words), dtype=torch.int32, device=dev), int(s.rest_per_colour))
    return GpuSplats(device_view(s.positions, (n, 4), torch.float32, device, sync=False),
                     device_view(s.shape, (n, 4), torch.int32, device, sync=False),
                     device_view(s.sh, (n, words), torch.int32, device, sync=False) if words else
                     torch.empty((n, 0), dtype=torch.int32, device=torch.device("cuda", device)),
                     int(s.rest_per_colour))


@dataclass
class LodLevel:
    """LodLevel (Lod.h:34-39): one stored level's merged Gaussians and their cells."""
    level: int
    gaussians: GpuSplats
    cells: torch.Tensor   # int32 bit patterns of each Gaussian's cell code at `level`


class LodCloud:
    """LodCloud (Lod.h:41-80): a cloud with its levels of detail, owned by the
    library (freed by close() or when this object goes)."""

    def __init__(self, handle: C.c_void_p, device: int):
        self._handle = handle
        self.device = device
        info = _abi.LodInfo()
        _abi.check(_abi.load().lrt_lod_get_info(handle, C.byref(info)), "lrt_lod_get_info")
        self.info = info

    def close(self) -> None:
        if self._handle:
            _abi.load().lrt_lod_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def count(self) -> int:
        return int(self.info.count)

    @property
    def chunk_splats(self) -> int:
        return int(self.info.chunk_splats)

    @property
    def bounds_lo(self) -> np.ndarray:
        return np.array(self.info.bounds_lo[:], np.float32)

    @property
    def bounds_hi(self) -> np.ndarray:
        return np.array(self.info.bounds_hi[:], np.float32)

    @property
    def extent(self) -> float:
        return float(self.info.extent)

    def merged_gaussians(self) -> int:
        return int(self.info.merged)

    @property
    def splats(self) -> GpuSplats:
        """The store: the cloud's splats in Morton order."""
        s = _abi.GpuSplatsStruct()
        _abi.check(_abi.load().lrt_lod_splats(self._handle, C.byref(s), None), "lrt_lod_splats")
        return _view(s, self.device)

    @property
    def codes(self) -> torch.Tensor:
        """Each stored splat's 30-bit Morton code (int32 bit patterns)."""
        s = _abi.GpuSplatsStruct()
        ptr = C.c_void_p()
        _abi.check(_abi.load().lrt_lod_splats(self._handle, C.byref(s), C.byref(ptr)), "lrt_lod_splats")
        return device_view(ptr.value, (self.count,), torch.int32, self.device)

    @property
    def starts(self) -> torch.Tensor:
        """The finest stored level's groups' first splats (LodCloud::starts)."""
        ptr, groups = C.c_void_p(), C.c_uint32()
        _abi.check(_abi.load().lrt_lod_starts(self._handle, C.byref(ptr), C.byref(groups)), "lrt_lod_starts")
        return device_view(ptr.value, (groups.value,), torch.int32, self.device)

    @property
    def levels(self) -> list[LodLevel]:
        """Stored levels, coarsest first."""
        out = []
        lib = _abi.load()
        for k in range(int(self.info.levels)):
            level = C.c_uint32()
            s = _abi.GpuSplatsStruct()
            cells = C.c_void_p()
            _abi.check(lib.lrt_lod_level(self._handle, k, C.byref(level), C.byref(s), C.byref(cells)), "lrt_lod_level")
            out.append(LodLevel(int(level.value), _view(s, self.device),
                                device_view(cells.value, (int(s.count),), torch.int32, self.device)))
        return out


class LodBuilder:
    """LodBuilder (Lod.h:95-104)."""

    def __init__(self, raster: TileRasterizer):
        self._raster = raster

    @staticmethod
    def create(raster: TileRasterizer) -> "LodBuilder":
        return LodBuilder(raster)

    def build(self, cloud: GpuSplats, settings: LodBuildSettings | None = None, bounds=None,
              stream=None) -> LodCloud:
        """Levels of detail of `cloud` (its tensors on the raster's device).
        `bounds`: (lo xyz, hi xyz), or None for the positions' own."""
        lib = _abi.load()
        cs = cloud.struct()
        st = (settings or LodBuildSettings()).struct()
        b = None
        if bounds is not None:
            b = (C.c_float * 6)(*[float(v) for v in np.asarray(bounds, np.float32).reshape(6)])
        h = C.c_void_p()
        self._raster._check(lib.lrt_lod_build(self._raster._handle, C.byref(cs), b, C.byref(st), C.byref(h),
                                              _stream_ptr(stream)))
        return LodCloud(h, self._raster.device)


@dataclass
class LodInstance:
    """LodInstance (Lod.h:106-111): threshold None takes the call's."""
    cloud: LodCloud | None
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))
    edit: SplatEdit = field(default_factory=SplatEdit)
    threshold: float | None = None


@dataclass
class CutStats:
    """CutStats (Lod.h:113-124) without the streaming needs."""
    splats: int = 0      # the cloud's own splats drawn
    merged: int = 0      # merged Gaussians drawn
    available: int = 0   # splats in the cloud


class CutSelector:
    """CutSelector (Lod.h:126-152). The clouds a select returns belong to the
    rasteriser handle and are rewritten by its next select."""

    def __init__(self, raster: TileRasterizer):
        self._raster = raster

    @staticmethod
    def create(raster: TileRasterizer) -> "CutSelector":
        return CutSelector(raster)

    def select(self, projection: Projection, instances: Sequence[LodInstance], threshold: float,
               stats: list | None = None, stream=None) -> list[SplatInstance]:
        """Each instance's cut for this view. A cell is drawn merged when it
        projects to at most `threshold` pixels; 0 draws every splat."""
        lib = _abi.load()
        n = len(instances)
        arr = (_abi.LodInstanceStruct * max(1, n))()
        for k, inst in enumerate(instances):
            arr[k].cloud = inst.cloud._handle if inst.cloud is not None else None
            arr[k].object_to_world[:] = [float(v) for v in np.asarray(inst.object_to_world, np.float64).reshape(16)]
            inst.edit.fill(arr[k].edit)
            arr[k].threshold = -1.0 if inst.threshold is None else float(inst.threshold)
        out = (_abi.SplatInstanceStruct * max(1, n))()
        st = (_abi.CutStatsStruct * max(1, n))()
        written = C.c_uint32()
        pr = projection.struct()
        self._raster._check(lib.lrt_lod_select(self._raster._handle, C.byref(pr), arr, n, float(threshold), out,
                                               C.byref(written), st, _stream_ptr(stream)))
        if stats is not None:
            stats.clear()
            stats.extend(CutStats(int(s.splats), int(s.merged), int(s.available)) for s in st[:n])
        # out holds, in order, the instances that draw anything.
        result = []
        k = 0
        for inst, s in zip(instances, st[:n]):
            if s.splats + s.merged == 0:
                continue
            o = out[k]
            k += 1
            result.append(SplatInstance(_view(o.splats.contents, self._raster.device),
                                        np.array(o.object_to_world[:], np.float64).reshape(4, 4), inst.edit))
        assert k == written.value
        return result
