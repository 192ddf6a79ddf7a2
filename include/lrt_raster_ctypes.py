"""ctypes mirror of ``include/lrt_raster.h``: its status codes, constants and
struct layouts, nothing else. It loads no library; the package's loader
(``lucabrtrender_b200/_abi.py``) and the oracle's test harness
(``oracle/oracle.py``) both take their struct types from here, so a struct
made by one is accepted by the other, and the oracle never imports the
package."""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 1
TILE = 16

# lrt_status
OK = 0
UNKNOWN = 1
NOT_FOUND = 2
INVALID_ARGUMENT = 3
UNSUPPORTED = 4
IO_FAILURE = 5
DEVICE_FAILURE = 6
OUT_OF_MEMORY = 8
INTERNAL_ERROR = 10
OVERFLOW = 11
TRAIN_SORT_VALUES = 1   # lrt_train_params.flags
TIMEOUT = 12

STATUS_NAMES = {
    OK: "Ok", UNKNOWN: "Unknown", NOT_FOUND: "NotFound", INVALID_ARGUMENT: "InvalidArgument",
    UNSUPPORTED: "Unsupported", IO_FAILURE: "IoFailure", DEVICE_FAILURE: "DeviceFailure",
    OUT_OF_MEMORY: "OutOfMemory", INTERNAL_ERROR: "InternalError", OVERFLOW: "Overflow", TIMEOUT: "Timeout",
}

# Every symbol include/lrt_raster.h declares.
EXPORTS = (
    "lrt_abi_version", "lrt_rast_create", "lrt_rast_destroy", "lrt_rast_last_error", "lrt_rast_render",
    "lrt_rast_debug_view", "lrt_camera_looking_at", "lrt_projection_for", "lrt_prefix_sum", "lrt_radix_sort",
    "lrt_pack_splats", "lrt_math_eval", "lrt_prefix_sum_noalloc", "lrt_rast_train_forward",
    "lrt_rast_train_backward", "lrt_rast_backward_times", "lrt_rast_render_batch", "lrt_rast_render_async",
    "lrt_rast_settle", "lrt_rast_render_composite", "lrt_pack_points", "lrt_splat_encoding_ply",
    "lrt_rast_decode_splats", "lrt_rast_decode_points", "lrt_rast_compare_images", "lrt_rast_compare_hdr",
    "lrt_rast_count_different", "lrt_rast_l1_loss", "lrt_l1_loss_grad", "lrt_lod_build_settings_default",
    "lrt_lod_build", "lrt_lod_destroy", "lrt_lod_get_info", "lrt_lod_splats", "lrt_lod_level", "lrt_lod_starts",
    "lrt_lod_select", "lrt_rast_train_batch", "lrt_rast_debug_sort", "lrt_rast_filter3d", "lrt_rast_debug_train_chunking",
)
PREFIX_SUM_NOALLOC_MAX = 1 << 26


class Projection(C.Structure):
    _fields_ = [
        ("world_to_view", C.c_double * 16),
        ("focal_x", C.c_double), ("focal_y", C.c_double),
        ("centre_x", C.c_double), ("centre_y", C.c_double),
        ("near_z", C.c_double), ("far_z", C.c_double),
        ("eye_world", C.c_double * 3),
        ("orthographic", C.c_uint32), ("reserved", C.c_uint32),
    ]


class Lens(C.Structure):
    _fields_ = [
        ("orthographic", C.c_uint32), ("reserved", C.c_uint32),
        ("focal", C.c_double), ("haperture", C.c_double), ("vaperture", C.c_double),
        ("near_z", C.c_double), ("far_z", C.c_double),
        ("window_translate", C.c_double * 2), ("window_scale", C.c_double * 2),
        ("window_roll", C.c_double),
    ]


class CameraStruct(C.Structure):
    _fields_ = [("camera_to_world", C.c_double * 16), ("lens", Lens)]


class SplatEdit(C.Structure):
    _fields_ = [
        ("active", C.c_uint32), ("shape", C.c_uint32), ("mode", C.c_uint32), ("invert", C.c_uint32),
        ("centre", C.c_float * 3), ("size", C.c_float * 3), ("tint", C.c_float * 3),
        ("saturation", C.c_float), ("brightness", C.c_float), ("opacity", C.c_float),
        ("min_opacity", C.c_float), ("max_scale", C.c_float),
    ]


class GpuSplatsStruct(C.Structure):
    _fields_ = [
        ("count", C.c_uint32), ("rest_per_colour", C.c_uint32), ("sh_words", C.c_uint32),
        ("reserved", C.c_uint32),
        ("positions", C.c_void_p), ("shape", C.c_void_p), ("sh", C.c_void_p), ("filter3d", C.c_void_p),
    ]


class SplatInstanceStruct(C.Structure):
    _fields_ = [
        ("splats", C.POINTER(GpuSplatsStruct)),
        ("object_to_world", C.c_double * 16),
        ("edit", SplatEdit),
    ]


class GpuPointsStruct(C.Structure):
    _fields_ = [("count", C.c_uint32), ("reserved", C.c_uint32), ("positions", C.c_void_p), ("colours", C.c_void_p)]


class PointStyleStruct(C.Structure):
    _fields_ = [("size_mode", C.c_uint32), ("size", C.c_float), ("constant_colour", C.c_uint32),
                ("colour", C.c_float * 3)]


class PointInstanceStruct(C.Structure):
    _fields_ = [
        ("points", C.POINTER(GpuPointsStruct)),
        ("object_to_world", C.c_double * 16),
        ("style", PointStyleStruct),
    ]


class SplatEncoding(C.Structure):
    """lrt_splat_encoding (io::SplatEncoding): field offsets and modes."""
    _fields_ = [(n, C.c_uint32) for n in (
        "floats_per_record", "x", "y", "z", "opacity", "scale0", "scale1", "scale2", "rot_w", "rot_x", "rot_y",
        "rot_z", "dc0", "dc1", "dc2", "rest_base", "rest_per_colour", "rest_colour_outer", "opacity_mode",
        "scale_mode", "colour_mode", "rotation_mode", "rest_mode")] + [("position_scale", C.c_float),
                                                                        ("flip_yz", C.c_uint32)]


class ImageDifferenceStruct(C.Structure):
    _fields_ = [("pixels", C.c_uint64), ("p99", C.c_uint32), ("max", C.c_uint32), ("over2", C.c_uint64)]


class HdrDifferenceStruct(C.Structure):
    _fields_ = [("pixels", C.c_uint64), ("rel_mse", C.c_double), ("p99_relative", C.c_double),
                ("max_relative", C.c_double)]


class RenderSettingsStruct(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("antialias", C.c_uint32),
        ("max_sh_degree", C.c_uint32), ("background", C.c_float * 4), ("depth_mode", C.c_uint32),
        ("depth_threshold", C.c_float), ("linearise", C.c_uint32), ("time_stages", C.c_uint32),
    ]


class FrameStatsStruct(C.Structure):
    _fields_ = [
        ("splats", C.c_uint32), ("visible", C.c_uint32), ("pairs", C.c_uint32), ("reserved", C.c_uint32),
        ("project_ms", C.c_double), ("depth_sort_ms", C.c_double), ("counts_ms", C.c_double),
        ("emit_ms", C.c_double), ("tile_sort_ms", C.c_double), ("blend_ms", C.c_double),
        ("total_ms", C.c_double),
    ]


class TargetsStruct(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("colour", C.c_void_p), ("depth", C.c_void_p)]


class DebugView(C.Structure):
    _fields_ = [
        ("proj", C.c_void_p), ("rects", C.c_void_p), ("touched", C.c_void_p), ("depth_keys", C.c_void_p),
        ("pairs", C.c_void_p), ("ranges", C.c_void_p),
        ("slots", C.c_uint32), ("pairs_count", C.c_uint32), ("tiles", C.c_uint32), ("slot_bits", C.c_uint32),
        ("depth_bits", C.c_uint32), ("tile_bits", C.c_uint32), ("visible", C.c_uint32), ("reserved", C.c_uint32),
    ]


class View(C.Structure):
    _fields_ = [("projection", Projection), ("width", C.c_uint32), ("height", C.c_uint32),
                ("colour", C.c_void_p), ("depth", C.c_void_p)]


class BatchStats(C.Structure):
    _fields_ = [
        ("views", C.c_uint32), ("splats", C.c_uint32), ("pairs", C.c_uint32), ("chunks", C.c_uint32),
        ("views_per_chunk", C.c_uint32), ("blend_blocks_per_sm", C.c_uint32), ("graph_replayed", C.c_uint32),
        ("reserved", C.c_uint32), ("device_ms", C.c_double), ("total_ms", C.c_double),
    ]


class TrainParams(C.Structure):
    _fields_ = [
        ("count", C.c_uint32), ("flags", C.c_uint32),
        ("means", C.c_void_p), ("log_scales", C.c_void_p), ("quats", C.c_void_p),
        ("opacity_logits", C.c_void_p), ("sh", C.c_void_p),
    ]


class TrainGrads(C.Structure):
    _fields_ = [
        ("means", C.c_void_p), ("log_scales", C.c_void_p), ("quats", C.c_void_p),
        ("opacity_logits", C.c_void_p), ("sh", C.c_void_p),
    ]


class TrainViewStruct(C.Structure):
    _fields_ = [("projection", Projection), ("width", C.c_uint32), ("height", C.c_uint32), ("colour", C.c_void_p),
                ("depth", C.c_void_p), ("target", C.c_void_p), ("loss", C.c_void_p)]


class LodBuildSettings(C.Structure):
    _fields_ = [("max_group_fraction", C.c_float), ("coarsest_level", C.c_uint32), ("chunk_splats", C.c_uint32),
                ("reserved", C.c_uint32)]


class LodInfo(C.Structure):
    _fields_ = [("count", C.c_uint32), ("rest_per_colour", C.c_uint32), ("sh_words", C.c_uint32),
                ("levels", C.c_uint32), ("coarsest", C.c_uint32), ("finest", C.c_uint32), ("merged", C.c_uint32),
                ("chunk_splats", C.c_uint32), ("bounds_lo", C.c_float * 3), ("bounds_hi", C.c_float * 3),
                ("extent", C.c_float), ("level_groups", C.c_uint32 * 10)]


class LodInstanceStruct(C.Structure):
    _fields_ = [("cloud", C.c_void_p), ("object_to_world", C.c_double * 16), ("edit", SplatEdit),
                ("threshold", C.c_float), ("reserved", C.c_uint32)]


class CutStatsStruct(C.Structure):
    _fields_ = [("splats", C.c_uint32), ("merged", C.c_uint32), ("available", C.c_uint32), ("reserved", C.c_uint32)]
