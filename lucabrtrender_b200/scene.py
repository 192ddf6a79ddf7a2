"""Splat clouds on the device (the reference's scene::GpuSplats,
modules/scene/include/lrt/scene/GpuClouds.h:41-76) and seeded synthetic scenes.

Raw records use the 3DGS PLY encoding: x y z, logit opacity, three log
scales, rotation w x y z, three SH DC coefficients, then the rest
coefficients all red, then all green, then all blue. ``CloudLoader.upload``
packs them on the host (``lrt_pack_splats``: the reference's validate +
compact + decode, shaders/lrt/scene/splat_decode.slang:20-91) and copies the
packed buffers to the device.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi

REST_FOR_DEGREE = {0: 0, 1: 3, 2: 8, 3: 15}


def sh_words_for(rest_per_colour: int) -> int:
    """Words of f16 pairs a splat's rest coefficients take (packing.slang:117-118); at least one."""
    return max((rest_per_colour * 3 + 1) // 2, 1)


def record_floats(file_per_colour: int) -> int:
    return 14 + 3 * file_per_colour


@dataclass
class PackedSplats:
    """Host copy of the packed layout."""
    positions: np.ndarray   # [N, 4] float32
    shape: np.ndarray       # [N, 4] uint32
    sh: np.ndarray          # [N, sh_words] uint32
    rest_per_colour: int

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])

    @property
    def sh_words(self) -> int:
        return int(self.sh.shape[1])


@dataclass
class GpuSplats:
    """A packed cloud on the device. The tensors own the memory. `filter3d`
    (optional, [N] float32): the Mip-Splatting 3D filter's variance per splat
    (TileRasterizer.filter3d computes it); None leaves the filter off."""
    positions: torch.Tensor   # [N, 4] float32
    shape: torch.Tensor       # [N, 4] int32 (bit patterns)
    sh: torch.Tensor          # [N, sh_words] int32 (bit patterns)
    rest_per_colour: int
    filter3d: torch.Tensor | None = None

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])

    @property
    def sh_words(self) -> int:
        return int(self.sh.shape[1])

    @property
    def degree(self) -> int:
        r = self.rest_per_colour
        return 3 if r >= 15 else 2 if r >= 8 else 1 if r >= 3 else 0

    def struct(self) -> _abi.GpuSplatsStruct:
        s = _abi.GpuSplatsStruct()
        s.count = self.count
        s.rest_per_colour = self.rest_per_colour
        s.sh_words = self.sh_words
        s.positions = self.positions.data_ptr() if self.count else None
        s.shape = self.shape.data_ptr() if self.count else None
        s.sh = self.sh.data_ptr() if self.count else None
        if self.filter3d is not None and self.count:
            if self.filter3d.dtype != torch.float32 or self.filter3d.numel() != self.count or \
                    not self.filter3d.is_contiguous():
                raise ValueError("filter3d must be a contiguous float32 tensor with one value per splat")
            s.filter3d = self.filter3d.data_ptr()
        return s

    @property
    def bytes(self) -> int:
        return self.count * (16 + 16 + 4 * self.sh_words)


def ply_encoding(rest_per_colour: int) -> _abi.SplatEncoding:
    """The 3DGS PLY record layout (lrt_splat_encoding_ply)."""
    e = _abi.SplatEncoding()
    _abi.check(_abi.load().lrt_splat_encoding_ply(rest_per_colour, C.byref(e)), "ply_encoding")
    return e


def pack_splats(raw: np.ndarray, file_per_colour: int, max_degree: int = 3) -> PackedSplats:
    """Validate, compact and pack raw records on the host (lrt_pack_splats)."""
    lib = _abi.load()
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    n, fpr = raw.shape
    if fpr < record_floats(file_per_colour):
        raise ValueError("records are shorter than their harmonics layout")
    keep = min(file_per_colour, REST_FOR_DEGREE[max(0, min(3, max_degree))])
    words = sh_words_for(keep)
    positions = np.empty((n, 4), np.float32)
    shape = np.empty((n, 4), np.uint32)
    sh = np.empty((n, words), np.uint32)
    kept = C.c_uint32(0)
    _abi.check(lib.lrt_pack_splats(raw.ctypes.data, n, fpr, file_per_colour, keep, positions.ctypes.data,
                                   shape.ctypes.data, sh.ctypes.data, C.byref(kept)), "pack_splats")
    k = kept.value
    return PackedSplats(positions[:k].copy(), shape[:k].copy(), sh[:k].copy(), keep)


def to_device(packed: PackedSplats, device="cuda") -> GpuSplats:
    pos = torch.from_numpy(packed.positions).to(device)
    shape = torch.from_numpy(packed.shape.view(np.int32)).to(device)
    sh = torch.from_numpy(packed.sh.view(np.int32)).to(device)
    return GpuSplats(pos, shape, sh, packed.rest_per_colour)


@dataclass
class PackedPoints:
    """Host copy of a point cloud's layout: positions (x, y, z, 1) and two
    words of fp16 halves per point (r | g, b | a), linear."""
    positions: np.ndarray   # [N, 4] float32
    colours: np.ndarray     # [N, 2] uint32

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])


@dataclass
class GpuPoints:
    """scene::GpuPoints (GpuClouds.h:78-85) on the device."""
    positions: torch.Tensor   # [N, 4] float32
    colours: torch.Tensor     # [N, 2] int32 (bit patterns)

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])

    def struct(self) -> _abi.GpuPointsStruct:
        s = _abi.GpuPointsStruct()
        s.count = self.count
        s.positions = self.positions.data_ptr() if self.count else None
        s.colours = self.colours.data_ptr() if self.count else None
        return s


def pack_points(raw: np.ndarray, colour_kind: int = 2, detail: float = 1.0) -> PackedPoints:
    """Raw (x y z r g b) records to the point layout on the host
    (lrt_pack_points). colour_kind: 0 none, 1 sRGB bytes, 2 linear floats."""
    raw = np.ascontiguousarray(raw, dtype=np.float32).reshape(-1, 6)
    n = raw.shape[0]
    positions = np.empty((n, 4), np.float32)
    colours = np.empty((n, 2), np.uint32)
    kept = C.c_uint32(0)
    _abi.check(_abi.load().lrt_pack_points(raw.ctypes.data, n, colour_kind, float(detail), positions.ctypes.data,
                                           colours.ctypes.data, C.byref(kept)), "pack_points")
    k = kept.value
    return PackedPoints(positions[:k].copy(), colours[:k].copy())


def points_to_device(packed: PackedPoints, device="cuda") -> GpuPoints:
    return GpuPoints(torch.from_numpy(packed.positions).to(device),
                     torch.from_numpy(packed.colours.view(np.int32)).to(device))


class CloudLoader:
    """CloudLoader (GpuClouds.h:126-175): raw records in, a GpuSplats (or,
    for points, a GpuPoints) out."""

    def __init__(self, device="cuda"):
        self.device = device

    def upload(self, raw: np.ndarray, file_per_colour: int, max_degree: int = 3) -> GpuSplats:
        return to_device(pack_splats(raw, file_per_colour, max_degree), self.device)

    def upload_points(self, raw: np.ndarray, colour_kind: int = 2, detail: float = 1.0) -> GpuPoints:
        return points_to_device(pack_points(raw, colour_kind, detail), self.device)


def synthetic_records(count: int, seed: int, *, mean_sigma: float = 1.0, log_scale_mean: float = -4.5,
                      log_scale_sigma: float = 0.5, dc_sigma: float = 0.5, rest_sigma: float = 0.05,
                      degree: int = 3) -> np.ndarray:
    """Seeded raw 3DGS records with the benchmark's distributions: means
    N(0, mean_sigma) per axis, log-scales N(log_scale_mean, log_scale_sigma),
    rotations uniform on SO(3) (normalised N(0,1)^4), opacity sigmoid(N(0,1))
    (the record holds the logit), DC N(0, dc_sigma), rest N(0, rest_sigma).
    Counter-based Philox generator, so a seed names one scene everywhere."""
    rest = REST_FOR_DEGREE[degree]
    rng = np.random.Generator(np.random.Philox(seed))
    raw = rng.standard_normal((count, record_floats(rest)), dtype=np.float32)
    raw[:, 0:3] *= np.float32(mean_sigma)
    raw[:, 4:7] = raw[:, 4:7] * np.float32(log_scale_sigma) + np.float32(log_scale_mean)
    raw[:, 11:14] *= np.float32(dc_sigma)
    raw[:, 14:] *= np.float32(rest_sigma)
    return raw
