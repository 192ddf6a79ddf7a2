"""Camera, Lens and Projection: the reference's camera model
(modules/render/include/lrt/render/Camera.h:23-85), with ``looking_at`` and
``projection_for`` computed by the library's C++ host code
(``lrt_camera_looking_at`` / ``lrt_projection_for``)."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi


@dataclass
class Lens:
    """Lens (Camera.h:23-44): a focal length and a horizontal aperture in mm."""
    orthographic: bool = False
    focal: float = 50.0
    haperture: float = 24.576
    vaperture: float = 18.672
    near_z: float = 0.1
    far_z: float = 10000.0
    window_translate: tuple[float, float] = (0.0, 0.0)
    window_scale: tuple[float, float] = (1.0, 1.0)
    window_roll: float = 0.0


@dataclass
class Camera:
    """Camera (Camera.h:46-53): camera-to-world (row-major 4x4, looks down its -Z) and a lens."""
    camera_to_world: np.ndarray = field(default_factory=lambda: np.eye(4))
    lens: Lens = field(default_factory=Lens)

    @staticmethod
    def looking_at(eye, target, up=(0.0, 1.0, 0.0)) -> "Camera":
        lib = _abi.load()
        out = _abi.CameraStruct()
        arr = lambda v: (C.c_double * 3)(*map(float, v))  # noqa: E731
        _abi.check(lib.lrt_camera_looking_at(arr(eye), arr(target), arr(up), C.byref(out)), "looking_at")
        return Camera(np.array(out.camera_to_world[:], dtype=np.float64).reshape(4, 4), Lens())

    def struct(self) -> _abi.CameraStruct:
        s = _abi.CameraStruct()
        s.camera_to_world[:] = [float(v) for v in np.asarray(self.camera_to_world, dtype=np.float64).reshape(16)]
        L = self.lens
        s.lens.orthographic = 1 if L.orthographic else 0
        s.lens.focal = L.focal
        s.lens.haperture = L.haperture
        s.lens.vaperture = L.vaperture
        s.lens.near_z = L.near_z
        s.lens.far_z = L.far_z
        s.lens.window_translate[:] = list(L.window_translate)
        s.lens.window_scale[:] = list(L.window_scale)
        s.lens.window_roll = L.window_roll
        return s


@dataclass
class Projection:
    """Projection (Camera.h:56-82), the part the rasteriser reads."""
    world_to_view: np.ndarray
    focal_x: float
    focal_y: float
    centre_x: float
    centre_y: float
    near_z: float
    far_z: float
    orthographic: bool
    eye_world: np.ndarray

    def struct(self) -> _abi.Projection:
        p = _abi.Projection()
        p.world_to_view[:] = [float(v) for v in np.asarray(self.world_to_view, dtype=np.float64).reshape(16)]
        p.focal_x, p.focal_y = self.focal_x, self.focal_y
        p.centre_x, p.centre_y = self.centre_x, self.centre_y
        p.near_z, p.far_z = self.near_z, self.far_z
        p.eye_world[:] = [float(v) for v in self.eye_world]
        p.orthographic = 1 if self.orthographic else 0
        return p

    @staticmethod
    def from_struct(p: _abi.Projection) -> "Projection":
        return Projection(np.array(p.world_to_view[:], dtype=np.float64).reshape(4, 4), p.focal_x, p.focal_y,
                          p.centre_x, p.centre_y, p.near_z, p.far_z, bool(p.orthographic),
                          np.array(p.eye_world[:], dtype=np.float64))


def projection_for(camera: Camera, width: int, height: int) -> Projection:
    """projectionFor (modules/render/src/Camera.cpp:15-48)."""
    lib = _abi.load()
    out = _abi.Projection()
    cs = camera.struct()
    _abi.check(lib.lrt_projection_for(C.byref(cs), int(width), int(height), C.byref(out)), "projection_for")
    return Projection.from_struct(out)


def square_pixel_camera(eye, target, width: int, height: int, vertical_fov_deg: float = 60.0,
                        near_z: float = 0.01, up=(0.0, 1.0, 0.0)) -> Camera:
    """A pinhole camera with the given vertical field of view, expressed in the
    reference's lens terms: focal_px = (H/2) / tan(fov/2), focal_mm = focal_px * haperture / W."""
    cam = Camera.looking_at(eye, target, up)
    focal_px = (height / 2.0) / math.tan(math.radians(vertical_fov_deg) / 2.0)
    cam.lens.focal = focal_px * cam.lens.haperture / width
    cam.lens.near_z = near_z
    return cam
