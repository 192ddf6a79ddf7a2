"""B200-native splat tile rasteriser with lucabRTrender's TileRasterizer interface.

The compute path is the in-tree CUDA library ``lib/liblrt_raster.so`` (sm_100a
kernels behind the C-ABI of ``include/lrt_raster.h``); this package is the
Python host mirror of the reference's C++ interface over that ABI.
"""
from ._abi import LrtError
from .camera import Camera, Lens, Projection, projection_for, square_pixel_camera
from .raster import (Depth, EditMode, EditShape, FrameStats, PointInstance, PointStyle, RenderSettings, RenderTargets,
                     SplatEdit, SplatInstance, TileRasterizer, math_eval)
from ._abi import SplatEncoding
from .scene import (CloudLoader, GpuPoints, GpuSplats, PackedPoints, PackedSplats, pack_points, pack_splats,
                    ply_encoding, points_to_device, synthetic_records, to_device)
from .train import l1_loss, rasterize, train_batch
from .lod import CutSelector, CutStats, LodBuildSettings, LodBuilder, LodCloud, LodInstance, LodLevel

__all__ = [
    "LrtError", "Camera", "Lens", "Projection", "projection_for", "square_pixel_camera", "Depth", "EditMode", "EditShape",
    "FrameStats", "RenderSettings", "RenderTargets", "SplatEdit", "SplatInstance", "TileRasterizer", "math_eval",
    "CloudLoader", "GpuSplats", "PackedSplats", "pack_splats", "synthetic_records", "to_device", "rasterize",
    "PointInstance", "PointStyle", "GpuPoints", "PackedPoints", "pack_points", "points_to_device",
    "SplatEncoding", "ply_encoding", "l1_loss", "CutSelector", "CutStats", "LodBuildSettings", "LodBuilder",
    "LodCloud", "LodInstance", "LodLevel", "train_batch",
]
