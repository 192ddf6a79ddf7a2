"""ctypes wrapper of baseline/standin/libstandin.so: the reference's GPU path
as a labelled stand-in (see standin.cu). Comparison only; the package never
loads it."""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "libstandin.so"
sys.path.insert(0, str(HERE.parents[1] / "include"))
import lrt_raster_ctypes as abi  # noqa: E402

STAGES = ("project", "counts", "depth_sort", "emit", "tile_sort", "blend")


def build() -> Path:
    import subprocess
    root = HERE.parents[1]
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
           "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr", "-I", str(root / "include"), "-shared", "-o",
           str(LIB), str(HERE / "standin.cu")]
    subprocess.run(cmd, check=True)
    return LIB


class Standin:
    def __init__(self, device: int = 0):
        self.lib = C.CDLL(str(LIB))
        self.lib.standin_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
        self.lib.standin_destroy.argtypes = [C.c_void_p]
        self.lib.standin_destroy.restype = None
        self.lib.standin_render.argtypes = [C.c_void_p, C.POINTER(abi.Projection), C.POINTER(abi.GpuSplatsStruct),
                                            C.POINTER(abi.RenderSettingsStruct), C.POINTER(abi.TargetsStruct),
                                            C.POINTER(C.c_double), C.c_void_p]
        self.handle = C.c_void_p()
        code = self.lib.standin_create(C.byref(self.handle), device)
        if code != 0:
            raise RuntimeError(f"standin_create failed: {code}")

    def render(self, projection, cloud, settings, targets, stream=None) -> dict:
        """projection/cloud/settings/targets: the ctypes structs of the public header."""
        ms = (C.c_double * 6)()
        code = self.lib.standin_render(self.handle, C.byref(projection), C.byref(cloud), C.byref(settings),
                                       C.byref(targets), ms, stream)
        if code != 0:
            raise RuntimeError(f"standin_render failed: {code}")
        return dict(zip(STAGES, list(ms)))

    def close(self) -> None:
        if self.handle:
            self.lib.standin_destroy(self.handle)
            self.handle = C.c_void_p()
