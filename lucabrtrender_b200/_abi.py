"""The loader of the in-tree library, with the ctypes mirror of
``include/lrt_raster.h`` (``include/lrt_raster_ctypes.py``) re-exported.

The library is loaded from ``lucabrtrender_b200/lib/liblrt_raster.so``; there
is no fallback of any kind: if it is missing or does not load, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import sys as _sys
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "lib" / "liblrt_raster.so"

_INCLUDE = str(Path(__file__).resolve().parents[1] / "include")
if _INCLUDE not in _sys.path:
    _sys.path.insert(0, _INCLUDE)
from lrt_raster_ctypes import *  # noqa: E402,F401,F403  (the header's constants and structs)
from lrt_raster_ctypes import STATUS_NAMES, OK, ABI_VERSION  # noqa: E402

_lib = None


def load() -> C.CDLL:
    """The loaded library; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise RuntimeError(
            f"the CUDA library {LIBRARY_PATH} is not built: run `python -m lucabrtrender_b200.build` "
            "(or __graft_entry__.build())")
    lib = C.CDLL(str(LIBRARY_PATH))
    lib.lrt_abi_version.restype = C.c_uint32
    lib.lrt_rast_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
    lib.lrt_rast_destroy.argtypes = [C.c_void_p]
    lib.lrt_rast_destroy.restype = None
    lib.lrt_rast_last_error.argtypes = [C.c_void_p]
    lib.lrt_rast_last_error.restype = C.c_char_p
    lib.lrt_rast_render.argtypes = [C.c_void_p, C.POINTER(Projection), C.POINTER(SplatInstanceStruct), C.c_uint32,
                                    C.POINTER(RenderSettingsStruct), C.POINTER(TargetsStruct),
                                    C.POINTER(FrameStatsStruct), C.c_void_p]
    lib.lrt_rast_render_async.argtypes = [C.c_void_p, C.POINTER(Projection), C.POINTER(SplatInstanceStruct),
                                          C.c_uint32, C.POINTER(RenderSettingsStruct), C.POINTER(TargetsStruct),
                                          C.c_void_p]
    lib.lrt_rast_settle.argtypes = [C.c_void_p, C.POINTER(FrameStatsStruct)]
    lib.lrt_rast_render_composite.argtypes = [C.c_void_p, C.POINTER(Projection), C.POINTER(SplatInstanceStruct),
                                              C.c_uint32, C.POINTER(PointInstanceStruct), C.c_uint32,
                                              C.POINTER(TargetsStruct), C.POINTER(RenderSettingsStruct),
                                              C.POINTER(TargetsStruct), C.POINTER(FrameStatsStruct), C.c_void_p]
    lib.lrt_pack_points.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_uint32)]
    lib.lrt_splat_encoding_ply.argtypes = [C.c_uint32, C.POINTER(SplatEncoding)]
    lib.lrt_rast_l1_loss.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    lib.lrt_l1_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.lrt_rast_compare_images.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                            C.POINTER(ImageDifferenceStruct), C.c_void_p, C.c_void_p]
    lib.lrt_rast_compare_hdr.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                         C.POINTER(HdrDifferenceStruct), C.c_void_p]
    lib.lrt_rast_count_different.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                             C.POINTER(C.c_uint64), C.c_void_p]
    lib.lrt_rast_decode_splats.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(SplatEncoding), C.c_uint32,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p]
    lib.lrt_rast_decode_points.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_void_p,
                                           C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p]
    lib.lrt_rast_debug_view.argtypes = [C.c_void_p, C.POINTER(DebugView)]
    lib.lrt_camera_looking_at.argtypes = [C.POINTER(C.c_double)] * 3 + [C.POINTER(CameraStruct)]
    lib.lrt_projection_for.argtypes = [C.POINTER(CameraStruct), C.c_uint32, C.c_uint32, C.POINTER(Projection)]
    lib.lrt_prefix_sum.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.lrt_radix_sort.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                   C.c_void_p]
    lib.lrt_rast_debug_sort.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32]
    lib.lrt_rast_debug_train_chunking.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
    lib.lrt_rast_filter3d.argtypes = [C.c_void_p, C.POINTER(GpuSplatsStruct), C.POINTER(Projection),
                                      C.POINTER(C.c_uint32), C.c_uint32, C.c_float, C.c_void_p, C.c_void_p]
    lib.lrt_pack_splats.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    lib.lrt_math_eval.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.lrt_prefix_sum_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.lrt_rast_train_forward.argtypes = [C.c_void_p, C.POINTER(Projection), C.POINTER(TrainParams),
                                           C.POINTER(RenderSettingsStruct), C.POINTER(TargetsStruct),
                                           C.POINTER(FrameStatsStruct), C.c_void_p]
    lib.lrt_rast_train_backward.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(TrainGrads), C.c_void_p]
    lib.lrt_rast_render_batch.argtypes = [C.c_void_p, C.POINTER(SplatInstanceStruct), C.c_uint32, C.POINTER(View),
                                          C.c_uint32, C.POINTER(RenderSettingsStruct), C.POINTER(BatchStats),
                                          C.c_void_p]
    lib.lrt_rast_backward_times.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.lrt_rast_train_batch.argtypes = [C.c_void_p, C.POINTER(TrainParams), C.POINTER(TrainViewStruct), C.c_uint32,
                                         C.POINTER(RenderSettingsStruct), C.POINTER(TrainGrads),
                                         C.POINTER(BatchStats), C.c_void_p]
    lib.lrt_lod_build_settings_default.argtypes = [C.POINTER(LodBuildSettings)]
    lib.lrt_lod_build.argtypes = [C.c_void_p, C.POINTER(GpuSplatsStruct), C.c_void_p, C.POINTER(LodBuildSettings),
                                  C.POINTER(C.c_void_p), C.c_void_p]
    lib.lrt_lod_destroy.argtypes = [C.c_void_p]
    lib.lrt_lod_destroy.restype = None
    lib.lrt_lod_get_info.argtypes = [C.c_void_p, C.POINTER(LodInfo)]
    lib.lrt_lod_splats.argtypes = [C.c_void_p, C.POINTER(GpuSplatsStruct), C.POINTER(C.c_void_p)]
    lib.lrt_lod_level.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(GpuSplatsStruct),
                                  C.POINTER(C.c_void_p)]
    lib.lrt_lod_starts.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint32)]
    lib.lrt_lod_select.argtypes = [C.c_void_p, C.POINTER(Projection), C.POINTER(LodInstanceStruct), C.c_uint32,
                                   C.c_float, C.POINTER(SplatInstanceStruct), C.POINTER(C.c_uint32),
                                   C.POINTER(CutStatsStruct), C.c_void_p]
    if lib.lrt_abi_version() != ABI_VERSION:
        raise RuntimeError(f"ABI version mismatch: library {lib.lrt_abi_version()}, bindings {ABI_VERSION}")
    _lib = lib
    return lib


class LrtError(RuntimeError):
    """A failed call: ``code`` is the lrt_status (the reference's ErrorCode)."""

    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")


def check(code: int, message: str = "") -> None:
    if code != OK:
        raise LrtError(code, message)
